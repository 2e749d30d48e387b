// Typed neighbour list (cell binning + per-centre scan), sm_100a.
//
// Semantics (bit-exact target): the reference canonicalises coordinates as
// (coord % box) * (ref/box) * (1 - 5e-7) in float32 and sorts atoms by type
// (deepmd_jax/md_utils.py:364-373); jax_md's dense neighbour list keeps j != i
// with float32 d2 < cutoff^2 where d = mod(Ri - Rj + L/2, L) - L/2; get_nm
// (md_utils.py:431-459) then keeps per neighbour type the sel_j smallest
// indices in ascending order, type-local, padded with N, and flags overflow
// when more than sel_j exist.
//
// Layout: cells are binned per frame and each cell slot also holds its
// atom's canonical position and index as one float4 (cell order), so a
// candidate is one coalesced 16-byte load.  A warp owns one centre atom,
// centres taken in cell order so that the warps of a block share their
// neighbourhood in L1; it walks the 27 (or fewer, for 2-cell or 1-cell axes)
// neighbouring cells, appends hits per type into shared memory with ballots,
// then ranks the hits (indices are distinct, so rank = number of smaller
// hits) and writes the sorted prefix into the centre's own row.
#include "dpb_common.cuh"
#include <algorithm>
#include <climits>
#include <cmath>

namespace dpb {

struct NlGrid {
  int nc[3];
  int ncell;      // per frame
  int image_mode; // 1: explicit images (min(L) < 2 rc)
  int nimg[3];    // image range per axis in image mode
};

static NlGrid make_grid(const float box[3], float rc) {
  NlGrid g;
  g.image_mode = 0;
  for (int d = 0; d < 3; ++d) {
    int n = (int)floorf(box[d] / rc);
    g.nc[d] = std::max(1, std::min(n, 512));
    if (box[d] < 2.f * rc) g.image_mode = 1;
    g.nimg[d] = (int)floorf(rc / box[d] + 0.5f);  // images with |minimg + m L| < rc
  }
  if (g.image_mode) {
    g.nc[0] = g.nc[1] = g.nc[2] = 1;
  }
  g.ncell = g.nc[0] * g.nc[1] * g.nc[2];
  return g;
}

// A non-null gate makes every kernel of the build a no-op unless *gate != 0,
// so the rebuild can sit inside a captured MD step and run only when the
// drift test asks for it.
__global__ void nl_zero_kernel(int *__restrict__ a, int na, int *__restrict__ b, int nb,
                               const unsigned *__restrict__ gate) {
  if (gate && *gate == 0u) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < na) a[i] = 0;
  if (i < nb) b[i] = 0;
}

// dbox (device, (F,3)) replaces L and scale = RB / L when the box changes on
// the device (NPT): the reference's canonicalize(coord, box) with the current
// box (md_utils.py:364-373).
__global__ void nl_canon_kernel(const float *__restrict__ pos, const int32_t *__restrict__ perm,
                                int N, int F, float3 L, float3 scale, float3 RB, int3 nc,
                                float *__restrict__ canon, int *__restrict__ atom_cell,
                                int *__restrict__ cell_count, const unsigned *__restrict__ gate,
                                const float *__restrict__ dbox) {
  if (gate && *gate == 0u) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N * F) return;
  int f = g / N, k = g - f * N;
  if (dbox) {
    L = make_float3(dbox[f * 3], dbox[f * 3 + 1], dbox[f * 3 + 2]);
    scale = make_float3(__fdiv_rn(RB.x, L.x), __fdiv_rn(RB.y, L.y), __fdiv_rn(RB.z, L.z));
  }
  int src = perm ? perm[k] : k;
  const float *p = pos + ((size_t)f * N + src) * 3;
  const float shrink = 0.9999995f;  // float32(1 - 5e-7)
  float c0 = __fmul_rn(__fmul_rn(jmod(p[0], L.x), scale.x), shrink);
  float c1 = __fmul_rn(__fmul_rn(jmod(p[1], L.y), scale.y), shrink);
  float c2 = __fmul_rn(__fmul_rn(jmod(p[2], L.z), scale.z), shrink);
  canon[(size_t)g * 3 + 0] = c0;
  canon[(size_t)g * 3 + 1] = c1;
  canon[(size_t)g * 3 + 2] = c2;
  // cell bins of the reference box (canonical coordinates live in [0, ref))
  int ix = min(max((int)(c0 / RB.x * nc.x), 0), nc.x - 1);
  int iy = min(max((int)(c1 / RB.y * nc.y), 0), nc.y - 1);
  int iz = min(max((int)(c2 / RB.z * nc.z), 0), nc.z - 1);
  int cell = (ix * nc.y + iy) * nc.z + iz;
  atom_cell[g] = cell;
  atomicAdd(&cell_count[f * (nc.x * nc.y * nc.z) + cell], 1);
}

// Exclusive scan of n ints with one block (n up to a few million).
__global__ void nl_scan_kernel(const int *__restrict__ in, int *__restrict__ out, int n,
                               const unsigned *__restrict__ gate) {
  if (gate && *gate == 0u) return;
  __shared__ int part[1024];
  int t = threadIdx.x;
  int per = (n + blockDim.x - 1) / blockDim.x;
  int b = t * per, e = min(b + per, n);
  int s = 0;
  for (int i = b; i < e; ++i) s += in[i];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = t ? part[t - 1] : 0;
  for (int i = b; i < e; ++i) {
    out[i] = run;
    run += in[i];
  }
  if (t == blockDim.x - 1) out[n] = part[t];
}

__global__ void nl_scatter_kernel(const int *__restrict__ atom_cell, const int *__restrict__ cell_start,
                                  int *__restrict__ cursor, int *__restrict__ cell_atoms,
                                  const float *__restrict__ canon, float4 *__restrict__ cell_pos, int N, int F,
                                  int ncell, const unsigned *__restrict__ gate) {
  if (gate && *gate == 0u) return;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N * F) return;
  int f = g / N;
  int c = f * ncell + atom_cell[g];
  int slot = atomicAdd(&cursor[c], 1);
  const int q = cell_start[c] + slot;
  cell_atoms[q] = g - f * N;  // frame-local sorted index
  cell_pos[q] = make_float4(canon[(size_t)g * 3], canon[(size_t)g * 3 + 1], canon[(size_t)g * 3 + 2],
                            __int_as_float(g - f * N));
}

struct NlParams {
  int N, F, ntypes, cap;
  int offs[kMaxTypes + 1];
  int sel[kMaxTypes];
  int col[kMaxTypes + 1];
  float3 L;      // reference box (canonical frame)
  float rc2;
  int3 nc;
  int image_mode;
  int3 nimg;
};

// Append the hits of one 32-candidate round into the per-type lists; the
// per-type counts are warp-uniform registers.  Hits past cap are dropped
// (that count is flagged as an overflow), in traversal order.
__device__ __forceinline__ void append_hits(bool hit, int t, int key, int ntypes, int cap, int (&cnt)[kMaxTypes],
                                            int *lists) {
  const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
#pragma unroll
  for (int tt = 0; tt < kMaxTypes; ++tt) {
    if (tt >= ntypes) break;
    const bool mine = hit && t == tt;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (mine) {
      const int p = cnt[tt] + __popc(m & lt);
      if (p < cap) lists[tt * cap + p] = key;
    }
    cnt[tt] += __popc(m);
  }
}

// Rank of each of a lane's KPL keys (lane, lane + 32, ...) among the nn
// distinct keys of a hit list padded with INT_MAX to nn4 (a multiple of 4),
// read four at a time; the keys with rank < sel go to out[rank] - off.
template <int KPL>
__device__ __forceinline__ void rank_write(const int *__restrict__ L_, int nn, int nn4, int sel, int off,
                                           int32_t *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  int key[KPL], rank[KPL];
#pragma unroll
  for (int k = 0; k < KPL; ++k) {
    key[k] = lane + 32 * k < nn ? L_[lane + 32 * k] : INT_MAX;
    rank[k] = 0;
  }
  for (int e2 = 0; e2 < nn4; e2 += 4) {
    const int4 v = *reinterpret_cast<const int4 *>(L_ + e2);
#pragma unroll
    for (int k = 0; k < KPL; ++k)
      rank[k] += (v.x < key[k]) + (v.y < key[k]) + (v.z < key[k]) + (v.w < key[k]);
  }
#pragma unroll
  for (int k = 0; k < KPL; ++k)
    if (lane + 32 * k < nn && rank[k] < sel) out[rank[k]] = key[k] - off;
}

__device__ __forceinline__ bool pair_hit(float3 ci, float3 cj, float3 L, float rc2) {
  // jax_md.space.periodic displacement, centre minus neighbour, float32
  float hx = 0.5f * L.x, hy = 0.5f * L.y, hz = 0.5f * L.z;
  float dx = __fsub_rn(jmod(__fadd_rn(__fsub_rn(ci.x, cj.x), hx), L.x), hx);
  float dy = __fsub_rn(jmod(__fadd_rn(__fsub_rn(ci.y, cj.y), hy), L.y), hy);
  float dz = __fsub_rn(jmod(__fadd_rn(__fsub_rn(ci.z, cj.z), hz), L.z), hz);
  float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  return d2 < rc2;
}

// 40 registers: 48 resident warps per SM at every launch shape (128-512
// threads), with nothing spilled.
__global__ void __maxnreg__(40) nl_search_kernel(NlParams P, const float *__restrict__ canon,
                                                 const int *__restrict__ cell_start,
                                                 const int *__restrict__ cell_atoms,
                                                 const float4 *__restrict__ cell_pos,
                                                 int32_t *__restrict__ nbrs,
                                                 int32_t *__restrict__ counts,
                                                 uint32_t *__restrict__ status,
                                                 const unsigned *__restrict__ gate) {
  if (gate && *gate == 0u) return;
  extern __shared__ __align__(16) int smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  int *lists = smem + warp * P.ntypes * P.cap;
  const int gc = blockIdx.x * wpb + warp;  // position in cell order
  if (gc >= P.N * P.F) return;
  const int f = gc / P.N, i = cell_atoms[gc];  // frame-local sorted index of the centre
  const int g = f * P.N + i;
  const float *cf = canon + (size_t)f * P.N * 3;
  float3 ci = make_float3(cf[i * 3], cf[i * 3 + 1], cf[i * 3 + 2]);
  int cnt[kMaxTypes] = {0, 0, 0, 0};

  if (!P.image_mode) {
    const int ncell = P.nc.x * P.nc.y * P.nc.z;
    const int *cs = cell_start + f * ncell;
    int ix = min(max((int)(ci.x / P.L.x * P.nc.x), 0), P.nc.x - 1);
    int iy = min(max((int)(ci.y / P.L.y * P.nc.y), 0), P.nc.y - 1);
    int iz = min(max((int)(ci.z / P.L.z * P.nc.z), 0), P.nc.z - 1);
    int lox = P.nc.x >= 3 ? -1 : 0, hix = P.nc.x >= 2 ? 1 : 0;
    int loy = P.nc.y >= 3 ? -1 : 0, hiy = P.nc.y >= 2 ? 1 : 0;
    int loz = P.nc.z >= 3 ? -1 : 0, hiz = P.nc.z >= 2 ? 1 : 0;
    // candidates of [b, e) of cell order, 32 per round
    auto scan = [&](int b, int e) {
      for (int base = b; base < e; base += 32) {
        const int q = base + lane;
        bool hit = false;
        int j = 0, t = 0;
        if (q < e) {
          const float4 v = cell_pos[q];
          j = __float_as_int(v.w);
          hit = (j != i) && pair_hit(ci, make_float3(v.x, v.y, v.z), P.L, P.rc2);
          t = type_of(j, P.offs, P.ntypes);
        }
        append_hits(hit, t, j, P.ntypes, P.cap, cnt, lists);
      }
    };
    // ix + o lies in [-1, nc], so one conditional add or subtract is the
    // periodic wrap.  With three or more cells along z the cells iz-1..iz+1
    // of a row are one range of cell order, or two where the row wraps, so
    // a round takes 32 candidates of the row rather than of one cell (the
    // visiting order only matters past cap hits, already an overflow).
    for (int ox = lox; ox <= hix; ++ox) {
      int cx = ix + ox;
      cx += cx < 0 ? P.nc.x : 0;
      cx -= cx >= P.nc.x ? P.nc.x : 0;
      for (int oy = loy; oy <= hiy; ++oy) {
        int cy = iy + oy;
        cy += cy < 0 ? P.nc.y : 0;
        cy -= cy >= P.nc.y ? P.nc.y : 0;
        const int cxy = (cx * P.nc.y + cy) * P.nc.z, nz = P.nc.z;
        if (nz >= 3) {
          if (iz >= 1 && iz <= nz - 2) {
            scan(cs[cxy + iz - 1], cs[cxy + iz + 2]);
          } else if (iz == 0) {
            scan(cs[cxy], cs[cxy + 2]);
            scan(cs[cxy + nz - 1], cs[cxy + nz]);
          } else {
            scan(cs[cxy + nz - 2], cs[cxy + nz]);
            scan(cs[cxy], cs[cxy + 1]);
          }
        } else {
          for (int oz = loz; oz <= hiz; ++oz) {
            int cz = iz + oz;
            cz -= cz >= nz ? nz : 0;
            scan(cs[cxy + cz], cs[cxy + cz + 1]);
          }
        }
      }
    }
  } else {
    // small box: j is listed once if any periodic image lies within rc
    const int nx = 2 * P.nimg.x + 1, ny = 2 * P.nimg.y + 1, nz = 2 * P.nimg.z + 1;
    const int nim = nx * ny * nz;
    for (int base = 0; base < P.N; base += 32) {
      const int j = base + lane;
      bool hit = false;
      int t = 0;
      if (j < P.N) {
        const float3 cj = make_float3(cf[j * 3], cf[j * 3 + 1], cf[j * 3 + 2]);
        const float3 d0 = make_float3(shift_ortho(cj.x - ci.x, P.L.x), shift_ortho(cj.y - ci.y, P.L.y),
                                      shift_ortho(cj.z - ci.z, P.L.z));
        for (int m = 0; m < nim && !hit; ++m) {
          const int a = m / (ny * nz) - P.nimg.x, bb = (m / nz) % ny - P.nimg.y, cc = m % nz - P.nimg.z;
          if (j == i && a == 0 && bb == 0 && cc == 0) continue;
          const float x = d0.x + a * P.L.x, y = d0.y + bb * P.L.y, z = d0.z + cc * P.L.z;
          hit = x * x + y * y + z * z < P.rc2;
        }
        t = type_of(j, P.offs, P.ntypes);
      }
      append_hits(hit, t, j, P.ntypes, P.cap, cnt, lists);
    }
  }
  // rank-sort each type's hits and write the sel_t smallest
  const int S = P.col[P.ntypes];
  int32_t *out = nbrs + (size_t)g * S;
  bool ovf = false;
#pragma unroll 1
  for (int t = 0; t < P.ntypes; ++t) {
    const int n = t == 0 ? cnt[0] : t == 1 ? cnt[1] : t == 2 ? cnt[2] : cnt[3];
    if (counts && lane == 0) counts[(size_t)g * P.ntypes + t] = n;
    ovf |= (n > P.sel[t]) || (n > P.cap);
    const int nn = min(n, P.cap), nn4 = (nn + 3) & ~3;  // cap is a multiple of 4
    int *L_ = lists + t * P.cap;
    if (lane < nn4 - nn) L_[nn + lane] = INT_MAX;
    __syncwarp();
    int32_t *o = out + P.col[t];
    const int sel = P.sel[t], off = P.offs[t];
    if (nn <= 32) rank_write<1>(L_, nn, nn4, sel, off, o);
    else if (nn <= 64) rank_write<2>(L_, nn, nn4, sel, off, o);
    else if (nn <= 96) rank_write<3>(L_, nn, nn4, sel, off, o);
    else if (nn <= 128) rank_write<4>(L_, nn, nn4, sel, off, o);
    else  // long lists (large sel): one key per lane at a time, few registers
      for (int e = lane; e < nn; e += 32) {
        const int key = L_[e];
        int rank = 0;
        for (int e2 = 0; e2 < nn; ++e2) rank += (L_[e2] < key);
        if (rank < sel) o[rank] = key - off;
      }
    for (int e = nn + lane; e < sel; e += 32) o[e] = P.N;
  }
  if (ovf && lane == 0) atomicOr(status, DPB_ST_NLIST_OVERFLOW);
}

}  // namespace dpb

using namespace dpb;

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int dpb_nlist_workspace_bytes(int natoms, int nframes, const float box[3], float rc,
                                         size_t *bytes) {
  if (!bytes || natoms <= 0 || nframes <= 0 || !box || rc <= 0) return DPB_ERR_INVALID_ARG;
  NlGrid g = make_grid(box, rc);
  size_t NF = (size_t)natoms * nframes, C = (size_t)g.ncell * nframes;
  *bytes = align_up(C * 4) * 2 + align_up((C + 1) * 4) + align_up(NF * 4) * 2 + align_up(NF * 16) +
           align_up(NF * 12);
  return DPB_OK;
}

namespace dpb {
int nlist_build_impl(const float *pos, const int32_t *perm, int natoms, int nframes, int ntypes,
                     const int *type_count, const int *sel, const float box[3], const float *ref_box, float rc,
                     int32_t *nbrs, float *ref_pos, int32_t *counts, uint32_t *status, void *workspace,
                     size_t ws_bytes, const unsigned *gate, cudaStream_t stream, const float *dbox,
                     int nl_warps) {
  if (!pos || natoms <= 0 || nframes <= 0 || ntypes < 1 || ntypes > kMaxTypes || !type_count || !sel ||
      !box || !nbrs || !status || rc <= 0)
    return DPB_ERR_INVALID_ARG;
  if (natoms >= (1 << 24)) return DPB_ERR_UNSUPPORTED;
  float rb[3] = {box[0], box[1], box[2]};
  if (ref_box) { rb[0] = ref_box[0]; rb[1] = ref_box[1]; rb[2] = ref_box[2]; }
  // jax_md receives rcut * max(ref/box) as float32 and squares it in float32
  float smax = std::max(rb[0] / box[0], std::max(rb[1] / box[1], rb[2] / box[2]));
  float rc_eff = rc * smax;
  NlGrid g = make_grid(rb, rc_eff);
  if (g.image_mode && (g.nimg[0] > 4 || g.nimg[1] > 4 || g.nimg[2] > 4)) return DPB_ERR_UNSUPPORTED;
  size_t need = 0;
  dpb_nlist_workspace_bytes(natoms, nframes, rb, rc_eff, &need);
  if (!workspace || ws_bytes < need) return DPB_ERR_WORKSPACE;
  NlParams P;
  P.N = natoms; P.F = nframes; P.ntypes = ntypes;
  int smax_sel = 0, off = 0, col = 0;
  for (int t = 0; t < ntypes; ++t) {
    if (type_count[t] < 0 || sel[t] < 0) return DPB_ERR_INVALID_ARG;
    P.offs[t] = off; off += type_count[t];
    P.sel[t] = sel[t]; P.col[t] = col; col += sel[t];
    smax_sel = std::max(smax_sel, sel[t]);
  }
  if (off != natoms) return DPB_ERR_INVALID_ARG;
  for (int t = ntypes; t <= kMaxTypes; ++t) P.offs[t] = natoms;
  P.col[ntypes] = col;
  // hit buffer per type: the sorted prefix is exact whenever a type's count
  // fits (counts above cap only occur with overflow already flagged)
  int cap = 256;
  while (cap < smax_sel + 1) cap <<= 1;
  if (cap > 1024) return DPB_ERR_UNSUPPORTED;
  P.cap = cap;
  P.L = make_float3(rb[0], rb[1], rb[2]);
  P.rc2 = rc_eff * rc_eff;
  P.nc = make_int3(g.nc[0], g.nc[1], g.nc[2]);
  P.image_mode = g.image_mode;
  P.nimg = make_int3(g.nimg[0], g.nimg[1], g.nimg[2]);

  size_t NF = (size_t)natoms * nframes, C = (size_t)g.ncell * nframes;
  char *w = (char *)workspace;
  int *cell_count = (int *)w; w += align_up(C * 4);
  int *cursor = (int *)w; w += align_up(C * 4);
  int *cell_start = (int *)w; w += align_up((C + 1) * 4);
  int *atom_cell = (int *)w; w += align_up(NF * 4);
  int *cell_atoms = (int *)w; w += align_up(NF * 4);
  float4 *cell_pos = (float4 *)w; w += align_up(NF * 16);
  float *canon = ref_pos ? ref_pos : (float *)w;

  nl_zero_kernel<<<(int)((C + 255) / 256), 256, 0, stream>>>(cell_count, (int)C, cursor, (int)C, gate);
  float3 L = make_float3(box[0], box[1], box[2]);
  float3 scale = make_float3(rb[0] / box[0], rb[1] / box[1], rb[2] / box[2]);
  int nb = (int)((NF + 255) / 256);
  nl_canon_kernel<<<nb, 256, 0, stream>>>(pos, perm, natoms, nframes, L, scale, P.L, P.nc, canon, atom_cell,
                                          cell_count, gate, dbox);
  nl_scan_kernel<<<1, 1024, 0, stream>>>(cell_count, cell_start, (int)C, gate);
  nl_scatter_kernel<<<nb, 256, 0, stream>>>(atom_cell, cell_start, cursor, cell_atoms, canon, cell_pos, natoms,
                                            nframes, g.ncell, gate);
  if (nl_warps != 4 && nl_warps != 8 && nl_warps != 16) return DPB_ERR_INVALID_ARG;
  const int wpb = nl_warps, threads = 32 * wpb;  // centres (warps) per block
  size_t smem = (size_t)wpb * ntypes * cap * 4;
  if (smem > 200 * 1024) return DPB_ERR_UNSUPPORTED;  // hit lists of this many warps do not fit
  if (smem > 48 * 1024) {
    DPB_CUDA_TRY(cudaFuncSetAttribute(nl_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  nl_search_kernel<<<(int)((NF + wpb - 1) / wpb), threads, smem, stream>>>(P, canon, cell_start, cell_atoms,
                                                                           cell_pos, nbrs, counts, status, gate);
  count_launch(5);
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}
}  // namespace dpb

extern "C" int dpb_nlist_build(const float *pos, const int32_t *perm, int natoms, int nframes, int ntypes,
                               const int *type_count, const int *sel, const float box[3],
                               const float *ref_box, float rc, int32_t *nbrs, float *ref_pos,
                               int32_t *counts, uint32_t *status, void *workspace, size_t ws_bytes,
                               void *stream) {
  return dpb::nlist_build_impl(pos, perm, natoms, nframes, ntypes, type_count, sel, box, ref_box, rc, nbrs,
                               ref_pos, counts, status, workspace, ws_bytes, nullptr, (cudaStream_t)stream,
                               nullptr, 8);
}

// ---------------------------------------------------------------- packed batches
namespace dpb {
// Where the frames of one request land in a packed batch: frame f's type-t
// atoms are packed rows row0[t] + f * stride[t] + m (m < count of type t), and
// its type-t atom m is type-local index base0[t] + f * stride[t] + m of the
// packed type block.
struct PackMap {
  int ntypes, S, Ns, nframes, Np;
  int soffs[kMaxTypes + 1];
  int col[kMaxTypes + 1];
  int row0[kMaxTypes], base0[kMaxTypes], stride[kMaxTypes];
};

__global__ void nl_pack_kernel(const int32_t *__restrict__ src, PackMap m, int32_t *__restrict__ dst) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per_frame = (size_t)m.Ns * m.S;
  if (e >= per_frame * m.nframes) return;
  const int f = (int)(e / per_frame);
  const size_t rc = e - (size_t)f * per_frame;
  const int r = (int)(rc / m.S), c = (int)(rc - (size_t)r * m.S);
  int i = 0, j = 0;
  while (i + 1 < m.ntypes && r >= m.soffs[i + 1]) ++i;
  while (j + 1 < m.ntypes && c >= m.col[j + 1]) ++j;
  const int v = src[e] & DPB_NBR_INDEX_MASK;
  const int cnt_j = m.soffs[j + 1] - m.soffs[j];
  const int out = v < cnt_j ? m.base0[j] + f * m.stride[j] + v : m.Np;
  const size_t row = (size_t)m.row0[i] + (size_t)f * m.stride[i] + (r - m.soffs[i]);
  dst[row * m.S + c] = out;
}
}  // namespace dpb

extern "C" int dpb_nlist_pack(const int32_t *src, int natoms, int nframes, int ntypes, const int *type_count,
                              const int *sel, const int *row0, const int *base0, const int *stride,
                              int packed_natoms, int32_t *dst, void *stream) {
  if (!src || !dst || !type_count || !sel || !row0 || !base0 || !stride || natoms <= 0 || nframes <= 0 ||
      ntypes < 1 || ntypes > dpb::kMaxTypes || packed_natoms <= 0)
    return DPB_ERR_INVALID_ARG;
  dpb::PackMap m;
  m.ntypes = ntypes; m.Ns = natoms; m.nframes = nframes; m.Np = packed_natoms;
  int off = 0, col = 0;
  for (int t = 0; t < ntypes; ++t) {
    if (type_count[t] < 0 || sel[t] < 0 || stride[t] < type_count[t]) return DPB_ERR_INVALID_ARG;
    m.soffs[t] = off; off += type_count[t];
    m.col[t] = col; col += sel[t];
    m.row0[t] = row0[t]; m.base0[t] = base0[t]; m.stride[t] = stride[t];
    if (row0[t] < 0 || base0[t] < 0 || (long long)row0[t] + (long long)stride[t] * nframes > packed_natoms)
      return DPB_ERR_INVALID_ARG;
  }
  if (off != natoms) return DPB_ERR_INVALID_ARG;
  m.soffs[ntypes] = off; m.col[ntypes] = col; m.S = col;
  const size_t n = (size_t)natoms * col * nframes;
  if (n == 0) return DPB_OK;
  dpb::nl_pack_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, m, dst);
  dpb::count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}
