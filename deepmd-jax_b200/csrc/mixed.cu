// Mixed-precision (BF16 tensor-core) evaluation path.
#include "internal.cuh"
#include "tc.cuh"

namespace dpb {

// ---------------------------------------------------------------- self-test
// Known-answer test of the tcgen05 path: D(128x64) = A(128x32) B(32x64) with
// A[m][k] = ((m*3 + k*5) % 17 - 8) / 8, B[k][n] = ((k*7 + n*11) % 13 - 6) / 4
// (all exact in bf16).  variant 0: A and B K-major; 1: A and B MN-major.
// Writes D row-major to out; err gets 1 on an mbarrier timeout.
__global__ void __launch_bounds__(128) k_selftest_umma(int variant, float *out, int *err) {
  constexpr int M = 128, N = 64, K = 32;
  __shared__ __align__(128) __nv_bfloat16 As[M * K];
  __shared__ __align__(128) __nv_bfloat16 Bs[N * K];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x;
  char *Ab = reinterpret_cast<char *>(As), *Bb = reinterpret_cast<char *>(Bs);
  for (int e = tid; e < M * K; e += 128) {
    const int m = e / K, k = e % K;
    const float v = (float)((m * 3 + k * 5) % 17 - 8) / 8.f;
    const uint32_t off = variant == 0 ? tc::kmajor_off(m, k, K) : tc::mnmajor_off(k, m, M);
    *reinterpret_cast<__nv_bfloat16 *>(Ab + off) = __float2bfloat16_rn(v);
  }
  for (int e = tid; e < N * K; e += 128) {
    const int k = e / N, n = e % N;
    const float v = (float)((k * 7 + n * 11) % 13 - 6) / 4.f;
    const uint32_t off = variant == 0 ? tc::kmajor_off(n, k, K) : tc::mnmajor_off(k, n, N);
    *reinterpret_cast<__nv_bfloat16 *>(Bb + off) = __float2bfloat16_rn(v);
  }
  if (tid == 0) tc::mbar_init(&mbar, 1);
  if (tid < 32) tc::tmem_alloc(&tbase, 64);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t d = tbase;
  if (tid == 0) {
    const uint32_t idesc = tc::idesc_bf16(M, N, variant, variant);
    const uint32_t a0 = tc::smem_u32(As), b0 = tc::smem_u32(Bs);
    for (int ks = 0; ks < K / 16; ++ks) {
      uint64_t ad, bd;
      if (variant == 0) {
        ad = tc::make_desc(a0 + tc::kmajor_off(0, ks * 16, K), 128, (K / 8) * 128);
        bd = tc::make_desc(b0 + tc::kmajor_off(0, ks * 16, K), 128, (K / 8) * 128);
      } else {
        ad = tc::make_desc(a0 + tc::mnmajor_off(ks * 16, 0, M), (M / 8) * 128, 128);
        bd = tc::make_desc(b0 + tc::mnmajor_off(ks * 16, 0, N), (N / 8) * 128, 128);
      }
      tc::mma_bf16(d, ad, bd, idesc, ks > 0);
    }
    tc::commit(&mbar);
  }
  if (!tc::mbar_wait(&mbar, 0)) atomicOr(err, 1);
  tc::fence_after_sync();
  const int warp = tid >> 5;
  for (int c = 0; c < N; c += 16) {
    float v[16];
    tc::tmem_ld16(d + ((uint32_t)(warp * 32) << 16) + c, v);
    for (int i = 0; i < 16; ++i) out[tid * N + c + i] = v[i];
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) tc::tmem_dealloc(d, 64);
}

// ---------------------------------------------------------------- shared pieces
template <int E0, int E1, int E2>
struct MixDims {
  static constexpr int K1 = (E0 + 15) / 16 * 16;
  static constexpr int N1 = (E1 + 15) / 16 * 16;
  static constexpr int K2 = N1;
  static constexpr int N2 = (E2 + 15) / 16 * 16;
  static constexpr int W1B = N1 * K1 * 2;  // bytes of the layer-1 B tile (K-major)
  static constexpr int W2B = N2 * K2 * 2;  // bytes of the layer-2 B tile (K-major)
  static constexpr int NETB = W1B + W2B;
  static constexpr int NSMALL = 2 * E0 + E1 + E2;  // w0, b0, b1, b2 (fp32)
  static constexpr int OPA_A0 = 128 * K1 * 2, OPA_A1 = 128 * K2 * 2, OPA_H2 = 128 * N2 * 2;
  static constexpr int OPA = OPA_A0 > OPA_A1 ? (OPA_A0 > OPA_H2 ? OPA_A0 : OPA_H2) : (OPA_A1 > OPA_H2 ? OPA_A1 : OPA_H2);
  static constexpr int Z1 = E1 / E0, Z2 = E2 / E1;
};

constexpr int kBlkAtoms = 8;    // centre atoms per block (T accumulators: 8 slots x 16 channels = 128 lanes)
constexpr int kRowCap = 256;    // compacted-row buffer (one tile + the carry of the next compaction round)
constexpr int kRblkBytes = 128 * 128 * 2;

// Bounded wait on the block's MMA barrier, made uniform across the block.
#define MIX_WAIT()                                  \
  do {                                              \
    const bool w_ = tc::mbar_wait(&mbar, ph);       \
    ph ^= 1;                                        \
    ok = __syncthreads_and(w_ && ok) != 0;          \
    tc::fence_after_sync();                         \
  } while (0)

// Weights of nets (ti, tj), tj < ntypes, as BF16 B tiles (K-major, zero
// padded) plus the FP32 first layer and biases.
template <int E0, int E1, int E2>
__device__ void mix_load_nets(const DevModel &M, int ti, char *netb, float *small) {
  using D = MixDims<E0, E1, E2>;
  for (int tj = 0; tj < M.ntypes; ++tj) {
    const int k = ti * M.ntypes + tj;
    char *w1 = netb + tj * D::NETB, *w2 = w1 + D::W1B;
    const float *W1 = M.ew[k][1], *W2 = M.ew[k][2];
    for (int e = threadIdx.x; e < D::N1 * D::K1; e += blockDim.x) {
      const int n = e / D::K1, kk = e - n * D::K1;
      const float v = (n < E1 && kk < E0) ? W1[kk * E1 + n] : 0.f;
      *reinterpret_cast<__nv_bfloat16 *>(w1 + tc::kmajor_off(n, kk, D::K1)) = __float2bfloat16_rn(v);
    }
    for (int e = threadIdx.x; e < D::N2 * D::K2; e += blockDim.x) {
      const int n = e / D::K2, kk = e - n * D::K2;
      const float v = (n < E2 && kk < E1) ? W2[kk * E2 + n] : 0.f;
      *reinterpret_cast<__nv_bfloat16 *>(w2 + tc::kmajor_off(n, kk, D::K2)) = __float2bfloat16_rn(v);
    }
    float *sm = small + tj * D::NSMALL;
    for (int e = threadIdx.x; e < E0; e += blockDim.x) {
      sm[e] = M.ew[k][0][e];
      sm[E0 + e] = M.eb[k][0][e];
    }
    for (int e = threadIdx.x; e < E1; e += blockDim.x) sm[2 * E0 + e] = M.eb[k][1][e];
    for (int e = threadIdx.x; e < E2; e += blockDim.x) sm[2 * E0 + E1 + e] = M.eb[k][2][e];
  }
}

// Block-wide stream compaction of one 128-candidate round: returns this
// thread's slot among the kept candidates; *total gets the round's count.
__device__ __forceinline__ int block_compact(bool keep, int *wcnt, int *total) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) wcnt[warp] = __popc(m);
  __syncthreads();
  int off = 0, tot = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    if (w < warp) off += wcnt[w];
    tot += wcnt[w];
  }
  __syncthreads();
  *total = tot;
  return off + __popc(m & ((1u << lane) - 1u));
}

// Geometry of a compacted row and the 10-channel env row (FP32).
__device__ __forceinline__ void mix_row_env(float4 rb, float rcut, float inv_std, float mean, RowGeom &gm,
                                            float &st, float R[10]) {
  row_geom(make_float3(rb.x, rb.y, rb.z), rcut, gm);
  const float sn = gm.s * inv_std;
  st = (gm.s - mean) * inv_std;
  const float inv_rp = 1.f / (gm.r + 1e-16f);
  const float xh[3] = {gm.x[0] * inv_rp, gm.x[1] * inv_rp, gm.x[2] * inv_rp};
  env_row(sn, xh, R);
}

// ---------------------------------------------------------------- embedding forward (BF16 tcgen05)
// Per block of 8 centre atoms of type ti: neighbour rows with s(r) != 0 are
// compacted block-wide into 128-row tiles.  Per tile (thread = row = TMEM lane):
//   layer 0 (1 -> E0) FP32 on CUDA cores, h0 -> A0 (bf16)
//   D  = A0 . W1   (tcgen05, 128 x N1)   -> h1 = tanh(D + b1) + rep(h0) -> A1
//   D  = A1 . W2   (tcgen05, 128 x N2)   -> h2 = tanh(D + b2) + rep(h1) -> H2
//   D3 += Rblk . H2 (tcgen05, M = 8 slots x 16 channels, K = 128 rows)
// where Rblk holds each row's env row R~ in its atom's 16-lane slot (zero
// elsewhere), so D3 accumulates T_a = sum_rows R~^T h2 for the 8 atoms in
// TMEM across all tiles of both neighbour types.  The block epilogue writes
// T / Nnbrs (FP32) and the descriptor G (dpmodel.py:74-78).
template <int E0, int E1, int E2>
__global__ void __launch_bounds__(128) k_mix_embed_fwd(DevModel M, SysDesc D, int ti, const float *__restrict__ pos,
                                                       const int32_t *__restrict__ perm,
                                                       const float *__restrict__ box, const int32_t *__restrict__ nbrs,
                                                       float *__restrict__ Tout, float *__restrict__ Gout,
                                                       int *__restrict__ err) {
  using MD = MixDims<E0, E1, E2>;
  extern __shared__ __align__(1024) char smem[];
  char *netb = smem;
  float *small = reinterpret_cast<float *>(netb + M.ntypes * MD::NETB);
  char *opa = reinterpret_cast<char *>(small) + ((M.ntypes * MD::NSMALL * 4 + 1023) / 1024) * 1024;
  char *rblk = opa + ((MD::OPA + 1023) / 1024) * 1024;
  float4 *rowbuf = reinterpret_cast<float4 *>(rblk + kRblkBytes);
  __shared__ int wcnt[4];
  __shared__ float3 ri_s[kBlkAtoms];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase_s;
  const int tid = threadIdx.x, warp = tid >> 5;

  mix_load_nets<E0, E1, E2>(M, ti, netb, small);
  for (int e = tid; e < kRblkBytes / 16; e += 128) reinterpret_cast<uint4 *>(rblk)[e] = make_uint4(0, 0, 0, 0);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  if (warp == 0) tc::tmem_alloc(&tbase_s, 256);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tbase_s;
  const uint32_t tD = tbase, tD3 = tbase + 128, lane_off = (uint32_t)(warp * 32) << 16;
  uint32_t ph = 0;
  bool ok = true;

  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  const int nbpf = (cnt_i + kBlkAtoms - 1) / kBlkAtoms;
  const int nblk = nbpf * D.F;
  const float inv_std = M.inv_std[ti], mean = M.mean[ti];
  const uint32_t idesc1 = tc::idesc_bf16(128, MD::N1, 0, 0);
  const uint32_t idesc2 = tc::idesc_bf16(128, MD::N2, 0, 0);
  const uint32_t idesc3 = tc::idesc_bf16(128, MD::N2, 1, 1);
  const uint32_t opa_u = tc::smem_u32(opa), rblk_u = tc::smem_u32(rblk), net_u = tc::smem_u32(netb);

  for (int blk = blockIdx.x; blk < nblk && ok; blk += gridDim.x) {
    const int f = blk / nbpf, a0 = (blk - f * nbpf) * kBlkAtoms;
    const int nb = min(kBlkAtoms, cnt_i - a0);
    const size_t g0 = (size_t)f * D.N + D.offs[ti] + a0;
    const float3 L = make_float3(box[f * 3], box[f * 3 + 1], box[f * 3 + 2]);
    const int3 ni = image_range(L, M.rcut);
    const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
    if (tid < nb) {
      const int src = perm ? perm[D.offs[ti] + a0 + tid] : D.offs[ti] + a0 + tid;
      const float *p = pos + ((size_t)f * D.N + src) * 3;
      ri_s[tid] = make_float3(p[0], p[1], p[2]);
    }
    __syncthreads();
    int ntile = 0;           // tiles issued for this block
    bool pending = false;    // an MMA3 in flight
    int my_slot = -1;        // Rblk slot written by this thread's row in the pending tile
    int rowcount = 0;
    for (int tj = 0; tj < D.ntypes && ok; ++tj) {
      const int sel = D.sel[tj], cnt_j = D.offs[tj + 1] - D.offs[tj];
      const int per_atom = sel * nim, total = nb * per_atom;
      const char *w1t = netb + tj * MD::NETB;
      const uint32_t w1_u = net_u + tj * MD::NETB, w2_u = w1_u + MD::W1B;
      const float *sm = small + tj * MD::NSMALL;
      for (int base = 0; base < total + 128 && ok; base += 128) {
        // ---- compaction round (the extra round flushes the tail of this type)
        const bool flush = base >= total;
        if (!flush) {
          const int p = base + tid;
          bool keep = false;
          float4 rv = make_float4(0.f, 0.f, 0.f, 0.f);
          if (p < total) {
            const int slot = p / per_atom, rem = p - slot * per_atom;
            const int sidx = nim == 1 ? rem : rem / nim, mimg = rem - sidx * nim;
            const int idx = nbrs[(g0 + slot) * D.S + D.col[tj] + sidx] & DPB_NBR_INDEX_MASK;
            if (idx < cnt_j) {
              const int js = D.offs[tj] + idx;
              const int src = perm ? perm[js] : js;
              const float *pj = pos + ((size_t)f * D.N + src) * 3;
              const float3 x = rel_coord(ri_s[slot], make_float3(pj[0], pj[1], pj[2]), L, ni, mimg);
              RowGeom gm;
              row_geom(x, M.rcut, gm);
              if (gm.s != 0.f) {
                keep = true;
                rv = make_float4(x.x, x.y, x.z, __int_as_float(slot));
              }
            }
          }
          int tot;
          const int pos_ = block_compact(keep, wcnt, &tot);
          if (keep) rowbuf[rowcount + pos_] = rv;
          rowcount += tot;
          __syncthreads();
        }
        while (rowcount >= 128 || (flush && rowcount > 0)) {
          const int nrows = min(rowcount, 128);
          // ---- wait for the previous contraction, clear its Rblk entries
          if (pending) {
            MIX_WAIT();
            if (!ok) break;
            if (my_slot >= 0) {
              const uint32_t o = tc::mnmajor_off(tid, 16 * my_slot, 128);
              *reinterpret_cast<uint4 *>(rblk + o) = make_uint4(0, 0, 0, 0);
              *reinterpret_cast<uint4 *>(rblk + o + 128) = make_uint4(0, 0, 0, 0);
            }
            pending = false;
          }
          // ---- row data, layer 0 (FP32), A0 and Rblk
          const bool act = tid < nrows;
          const float4 rv = act ? rowbuf[tid] : make_float4(100.f, 100.f, 100.f, 0.f);
          const int slot = act ? __float_as_int(rv.w) : -1;
          RowGeom gm;
          float st, R[10];
          mix_row_env(rv, M.rcut, inv_std, mean, gm, st, R);
          float h0[E0];
#pragma unroll
          for (int k = 0; k < E0; ++k) h0[k] = tanhf(fmaf(st, sm[k], sm[E0 + k]));
#pragma unroll
          for (int k8 = 0; k8 < MD::K1; k8 += 8) {
            uint4 q;
            q.x = tc::pack_bf16(k8 + 0 < E0 ? h0[min(k8 + 0, E0 - 1)] : 0.f, k8 + 1 < E0 ? h0[min(k8 + 1, E0 - 1)] : 0.f);
            q.y = tc::pack_bf16(k8 + 2 < E0 ? h0[min(k8 + 2, E0 - 1)] : 0.f, k8 + 3 < E0 ? h0[min(k8 + 3, E0 - 1)] : 0.f);
            q.z = tc::pack_bf16(k8 + 4 < E0 ? h0[min(k8 + 4, E0 - 1)] : 0.f, k8 + 5 < E0 ? h0[min(k8 + 5, E0 - 1)] : 0.f);
            q.w = tc::pack_bf16(k8 + 6 < E0 ? h0[min(k8 + 6, E0 - 1)] : 0.f, k8 + 7 < E0 ? h0[min(k8 + 7, E0 - 1)] : 0.f);
            *reinterpret_cast<uint4 *>(opa + tc::kmajor_off(tid, k8, MD::K1)) = q;
          }
          my_slot = slot;
          if (act) {
            const uint32_t o = tc::mnmajor_off(tid, 16 * slot, 128);
            *reinterpret_cast<uint4 *>(rblk + o) =
                make_uint4(tc::pack_bf16(R[0], R[1]), tc::pack_bf16(R[2], R[3]), tc::pack_bf16(R[4], R[5]),
                           tc::pack_bf16(R[6], R[7]));
            *reinterpret_cast<uint4 *>(rblk + o + 128) = make_uint4(tc::pack_bf16(R[8], R[9]), 0u, 0u, 0u);
          }
          tc::fence_proxy_async();
          tc::fence_before_sync();
          __syncthreads();
          if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int ks = 0; ks < MD::K1 / 16; ++ks)
              tc::mma_bf16(tD, tc::make_desc(opa_u + tc::kmajor_off(0, 16 * ks, MD::K1), 128, (MD::K1 / 8) * 128),
                           tc::make_desc(w1_u + tc::kmajor_off(0, 16 * ks, MD::K1), 128, (MD::K1 / 8) * 128),
                           idesc1, ks > 0);
            tc::commit(&mbar);
          }
          MIX_WAIT();
          if (!ok) break;
          // ---- layer 1 epilogue: h1 = tanh(z + b1) + rep(h0) -> A1
          float h1[E1];
#pragma unroll
          for (int c0 = 0; c0 < MD::N1; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tD + lane_off + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
              if (c0 + i < E1) h1[c0 + i] = tc::tanh_fast(v[i] + sm[2 * E0 + c0 + i]) + h0[(c0 + i) / MD::Z1];
          }
#pragma unroll
          for (int k8 = 0; k8 < MD::K2; k8 += 8) {
            float t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t[u] = (k8 + u < E1) ? h1[min(k8 + u, E1 - 1)] : 0.f;
            *reinterpret_cast<uint4 *>(opa + tc::kmajor_off(tid, k8, MD::K2)) =
                make_uint4(tc::pack_bf16(t[0], t[1]), tc::pack_bf16(t[2], t[3]), tc::pack_bf16(t[4], t[5]),
                           tc::pack_bf16(t[6], t[7]));
          }
          tc::fence_proxy_async();
          tc::fence_before_sync();
          __syncthreads();
          if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int ks = 0; ks < MD::K2 / 16; ++ks)
              tc::mma_bf16(tD, tc::make_desc(opa_u + tc::kmajor_off(0, 16 * ks, MD::K2), 128, (MD::K2 / 8) * 128),
                           tc::make_desc(w2_u + tc::kmajor_off(0, 16 * ks, MD::K2), 128, (MD::K2 / 8) * 128),
                           idesc2, ks > 0);
            tc::commit(&mbar);
          }
          MIX_WAIT();
          if (!ok) break;
          // ---- layer 2 epilogue: h2 = tanh(z + b2) + rep(h1) -> H2 (MN-major B of the contraction)
#pragma unroll
          for (int c0 = 0; c0 < MD::N2; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tD + lane_off + c0, v);
            float h2[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)
              h2[i] = (c0 + i < E2) ? tc::tanh_fast(v[i] + sm[2 * E0 + E1 + min(c0 + i, E2 - 1)]) +
                                          h1[min((c0 + i) / MD::Z2, E1 - 1)]
                                    : 0.f;
#pragma unroll
            for (int h = 0; h < 16; h += 8)
              *reinterpret_cast<uint4 *>(opa + tc::mnmajor_off(tid, c0 + h, MD::N2)) =
                  make_uint4(tc::pack_bf16(h2[h], h2[h + 1]), tc::pack_bf16(h2[h + 2], h2[h + 3]),
                             tc::pack_bf16(h2[h + 4], h2[h + 5]), tc::pack_bf16(h2[h + 6], h2[h + 7]));
          }
          tc::fence_proxy_async();
          tc::fence_before_sync();
          __syncthreads();
          if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int ks = 0; ks < 8; ++ks)
              tc::mma_bf16(tD3, tc::make_desc(rblk_u + tc::mnmajor_off(16 * ks, 0, 128), (128 / 8) * 128, 128),
                           tc::make_desc(opa_u + tc::mnmajor_off(16 * ks, 0, MD::N2), (MD::N2 / 8) * 128, 128),
                           idesc3, (ntile > 0 || ks > 0) ? 1u : 0u);
            tc::commit(&mbar);
          }
          pending = true;
          ++ntile;
          // ---- drop the processed rows, keep the carry
          const int rem = rowcount - nrows;
          float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
          if (tid < rem) carry = rowbuf[nrows + tid];
          __syncthreads();
          if (tid < rem) rowbuf[tid] = carry;
          rowcount = rem;
          __syncthreads();
        }
      }
    }
    // ---- block epilogue: T (FP32) and G from the TMEM accumulators
    if (!ok) break;
    if (pending) {
      MIX_WAIT();
      pending = false;
      if (!ok) break;
      if (my_slot >= 0) {
        const uint32_t o = tc::mnmajor_off(tid, 16 * my_slot, 128);
        *reinterpret_cast<uint4 *>(rblk + o) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(rblk + o + 128) = make_uint4(0, 0, 0, 0);
      }
    }
    float *Xs = reinterpret_cast<float *>(rblk);  // staging [slot][c][w], 8 x 10 x E2 floats
    {
      const int slot = tid >> 4, c = tid & 15;
#pragma unroll
      for (int c0 = 0; c0 < MD::N2; c0 += 16) {
        float v[16];
        if (ntile > 0) {
          tc::tmem_ld16(tD3 + lane_off + c0, v);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] = 0.f;
        }
        if (slot < nb && c < 10) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int w = c0 + i;
            if (w < E2) {
              const float t = v[i] * M.inv_nnbrs;
              Tout[(g0 + slot) * 10 * E2 + c * E2 + w] = t;
              Xs[(slot * 10 + c) * E2 + w] = t + (c == 0 ? M.tbias[w] : 0.f);
            }
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    const int A = M.A;
    for (int idx = tid; idx < nb * A * E2; idx += 128) {
      const int slot = idx / (A * E2), rem = idx - slot * A * E2, aa = rem / E2, w = rem - aa * E2;
      const float *X = Xs + slot * 10 * E2;
      const float y1 = X[1 * E2 + A + aa], y2 = X[2 * E2 + A + aa], y3 = X[3 * E2 + A + aa];
      float v = X[aa] * X[w] + X[E2 + aa] * X[E2 + w] + X[2 * E2 + aa] * X[2 * E2 + w] + X[3 * E2 + aa] * X[3 * E2 + w];
      v = fmaf(y1 * y1 + X[4 * E2 + A + aa], X[4 * E2 + w], v);
      v = fmaf(y2 * y2 + X[5 * E2 + A + aa], X[5 * E2 + w], v);
      v = fmaf(y3 * y3 + X[6 * E2 + A + aa], X[6 * E2 + w], v);
      v = fmaf(kSqrt2 * y1 * y3 + X[7 * E2 + A + aa], X[7 * E2 + w], v);
      v = fmaf(kSqrt2 * y2 * y1 + X[8 * E2 + A + aa], X[8 * E2 + w], v);
      v = fmaf(kSqrt2 * y3 * y2 + X[9 * E2 + A + aa], X[9 * E2 + w], v);
      Gout[(g0 + slot) * (size_t)A * E2 + aa * E2 + w] = v;
    }
    __syncthreads();
    for (int e = tid; e < kRblkBytes / 16; e += 128) reinterpret_cast<uint4 *>(rblk)[e] = make_uint4(0, 0, 0, 0);
    __syncthreads();
  }
  if (!ok) {
    // a wait gave up: flag it, give in-flight MMAs one more bounded wait, release TMEM
    if (tid == 0) atomicOr(err, 1);
    tc::mbar_wait(&mbar, ph);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

template <int E0, int E1, int E2>
size_t mix_fwd_smem(int ntypes) {
  using MD = MixDims<E0, E1, E2>;
  return (size_t)ntypes * MD::NETB + ((ntypes * MD::NSMALL * 4 + 1023) / 1024) * 1024 +
         ((MD::OPA + 1023) / 1024) * 1024 + kRblkBytes + kRowCap * 16 + 1024;
}

template <int E0, int E1, int E2>
int launch_mix_embed_fwd(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                         const float *box, const int32_t *nbrs, float *T, float *G, int *err, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  const int nblk = (cnt + kBlkAtoms - 1) / kBlkAtoms * D.F;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = mix_fwd_smem<E0, E1, E2>(M.ntypes);
  DPB_CUDA_TRY(cudaFuncSetAttribute(k_mix_embed_fwd<E0, E1, E2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  const int grid = nblk < 2 * nsm ? nblk : 2 * nsm;
  k_mix_embed_fwd<E0, E1, E2><<<grid, 128, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, G, err);
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

// ---------------------------------------------------------------- embedding adjoint (BF16 tcgen05)
// Per block of 8 centre atoms: dE/dT of each atom (adjoint of
// dpmodel.py:74-78, FP32) is written, scaled by 1/Nnbrs, into the B tile DTB
// (N = 8 slots x 16 channels, K = W).  The rows are recomputed with their
// tangent along s~ (forward mode): [h0, dh0] -> tcgen05 -> [h1, dh1] ->
// tcgen05 -> [h2, dh2], then U = H2 . DTB and V = dH2 . DTB on the tensor
// cores; a row reads its atom's slot: u = dE/dR~, dE/ds~ = R~ . v.  The FP32
// row adjoint gives dE/dx, scattered as forces and reduced into the virial.
template <int E0, int E1, int E2>
__global__ void __launch_bounds__(128, 1) k_mix_embed_bwd(DevModel M, SysDesc D, int ti,
                                                          const float *__restrict__ pos,
                                                          const int32_t *__restrict__ perm,
                                                          const float *__restrict__ box,
                                                          const int32_t *__restrict__ nbrs,
                                                          const float *__restrict__ Tin, const float *__restrict__ dG,
                                                          float4 *__restrict__ F4, double *__restrict__ virial,
                                                          int *__restrict__ err) {
  using MD = MixDims<E0, E1, E2>;
  constexpr int DTB_BYTES = 128 * MD::N2 * 2;
  constexpr int OPB = 2 * MD::OPA_H2;  // H2 + dH2 (largest pair)
  extern __shared__ __align__(1024) char smem[];
  char *netb = smem;
  float *small = reinterpret_cast<float *>(netb + M.ntypes * MD::NETB);
  char *dtb = reinterpret_cast<char *>(small) + ((M.ntypes * MD::NSMALL * 4 + 1023) / 1024) * 1024;
  char *opb = dtb + ((DTB_BYTES + 1023) / 1024) * 1024;
  float4 *rowbuf = reinterpret_cast<float4 *>(opb + ((OPB + 1023) / 1024) * 1024);
  __shared__ int wcnt[4];
  __shared__ float3 ri_s[kBlkAtoms];
  __shared__ float fi_s[kBlkAtoms * 3];
  __shared__ double vir_s[9];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase_s;
  const int tid = threadIdx.x, warp = tid >> 5;

  mix_load_nets<E0, E1, E2>(M, ti, netb, small);
  if (tid < 9) vir_s[tid] = 0.0;
  if (tid == 0) tc::mbar_init(&mbar, 1);
  if (warp == 0) tc::tmem_alloc(&tbase_s, 256);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tbase_s, lane_off = (uint32_t)(warp * 32) << 16;
  uint32_t ph = 0;
  bool ok = true;
  float vir[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vir[k] = 0.f;

  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  const int nbpf = (cnt_i + kBlkAtoms - 1) / kBlkAtoms;
  const int nblk = nbpf * D.F;
  const float inv_std = M.inv_std[ti], mean = M.mean[ti];
  const int A = M.A;
  const uint32_t idesc1 = tc::idesc_bf16(128, MD::N1, 0, 0);
  const uint32_t idesc2 = tc::idesc_bf16(128, MD::N2, 0, 0);
  const uint32_t idesc3 = tc::idesc_bf16(128, 128, 0, 0);
  const uint32_t opb_u = tc::smem_u32(opb), dtb_u = tc::smem_u32(dtb), net_u = tc::smem_u32(netb);
  // operand placements inside opb (byte offsets)
  const uint32_t oA0 = 0, oA0t = MD::OPA_A0, oA1 = 0, oA1t = MD::OPA_A1, oH2 = 0, oH2t = MD::OPA_H2;

  for (int blk = blockIdx.x; blk < nblk && ok; blk += gridDim.x) {
    const int f = blk / nbpf, a0 = (blk - f * nbpf) * kBlkAtoms;
    const int nb = min(kBlkAtoms, cnt_i - a0);
    const size_t g0 = (size_t)f * D.N + D.offs[ti] + a0;
    const size_t frame_base = (size_t)f * D.N;
    const float3 L = make_float3(box[f * 3], box[f * 3 + 1], box[f * 3 + 2]);
    const int3 ni = image_range(L, M.rcut);
    const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
    if (tid < nb) {
      const int src = perm ? perm[D.offs[ti] + a0 + tid] : D.offs[ti] + a0 + tid;
      const float *p = pos + (frame_base + src) * 3;
      ri_s[tid] = make_float3(p[0], p[1], p[2]);
    }
    if (tid < kBlkAtoms * 3) fi_s[tid] = 0.f;
    // ---- dE/dT per atom -> DTB (bf16, K-major [n = 16 slot + c][k = w])
    for (int e = tid; e < DTB_BYTES / 16; e += 128) reinterpret_cast<uint4 *>(dtb)[e] = make_uint4(0, 0, 0, 0);
    float *Xs = reinterpret_cast<float *>(opb);      // 10 x E2
    float *dGs = Xs + 10 * E2;                       // A x E2
    float *Qs = dGs + A * E2;                        // 10 x A
    float *dQs = Qs + 10 * A;                        // 10 x A
    float *dXs = dQs + 10 * A;                       // 10 x E2
    __syncthreads();
    for (int a = 0; a < nb; ++a) {
      const size_t g = g0 + a;
      for (int e = tid; e < 10 * E2; e += 128) Xs[e] = Tin[g * 10 * E2 + e] + (e < E2 ? M.tbias[e] : 0.f);
      for (int e = tid; e < A * E2; e += 128) dGs[e] = dG[g * (size_t)A * E2 + e];
      __syncthreads();
      for (int e = tid; e < 10 * A; e += 128) {
        const int c = e / A, aa = e - c * A;
        float qv;
        if (c < 4) {
          qv = Xs[c * E2 + aa];
        } else {
          const float y1 = Xs[E2 + A + aa], y2 = Xs[2 * E2 + A + aa], y3 = Xs[3 * E2 + A + aa];
          const int m = c - 4;
          const float b6[6] = {y1 * y1, y2 * y2, y3 * y3, kSqrt2 * y1 * y3, kSqrt2 * y2 * y1, kSqrt2 * y3 * y2};
          qv = b6[m] + Xs[c * E2 + A + aa];
        }
        Qs[e] = qv;
        float dq = 0.f;
        for (int w = 0; w < E2; ++w) dq = fmaf(dGs[aa * E2 + w], Xs[c * E2 + w], dq);
        dQs[e] = dq;
      }
      __syncthreads();
      for (int e = tid; e < 10 * E2; e += 128) {
        const int c = e / E2, w = e - c * E2;
        float v = 0.f;
        for (int aa = 0; aa < A; ++aa) v = fmaf(dGs[aa * E2 + w], Qs[c * A + aa], v);
        if (w < A && c < 4) v += dQs[c * A + w];
        if (w >= A && w < 2 * A) {
          const int aa = w - A;
          if (c >= 4) {
            v += dQs[c * A + aa];
          } else if (c >= 1) {
            const float y1 = Xs[E2 + w], y2 = Xs[2 * E2 + w], y3 = Xs[3 * E2 + w];
            const float d0 = dQs[4 * A + aa], d1 = dQs[5 * A + aa], d2 = dQs[6 * A + aa], d3 = dQs[7 * A + aa],
                        d4 = dQs[8 * A + aa], d5 = dQs[9 * A + aa];
            if (c == 1) v += 2.f * y1 * d0 + kSqrt2 * y3 * d3 + kSqrt2 * y2 * d4;
            if (c == 2) v += 2.f * y2 * d1 + kSqrt2 * y1 * d4 + kSqrt2 * y3 * d5;
            if (c == 3) v += 2.f * y3 * d2 + kSqrt2 * y1 * d3 + kSqrt2 * y2 * d5;
          }
        }
        dXs[e] = v * M.inv_nnbrs;
      }
      __syncthreads();
      for (int e = tid; e < 10 * MD::N2; e += 128) {
        const int c = e / MD::N2, w = e - c * MD::N2;
        const float v = w < E2 ? dXs[c * E2 + w] : 0.f;
        *reinterpret_cast<__nv_bfloat16 *>(dtb + tc::kmajor_off(16 * a + c, w, MD::N2)) = __float2bfloat16_rn(v);
      }
      __syncthreads();
    }
    // ---- rows
    int rowcount = 0;
    for (int tj = 0; tj < D.ntypes && ok; ++tj) {
      const int sel = D.sel[tj], cnt_j = D.offs[tj + 1] - D.offs[tj];
      const int per_atom = sel * nim, total = nb * per_atom;
      const uint32_t w1_u = net_u + tj * MD::NETB, w2_u = w1_u + MD::W1B;
      const float *sm = small + tj * MD::NSMALL;
      for (int base = 0; base < total + 128 && ok; base += 128) {
        const bool flush = base >= total;
        if (!flush) {
          const int p = base + tid;
          bool keep = false;
          float4 rv = make_float4(0.f, 0.f, 0.f, 0.f);
          if (p < total) {
            const int slot = p / per_atom, rem = p - slot * per_atom;
            const int sidx = nim == 1 ? rem : rem / nim, mimg = rem - sidx * nim;
            const int idx = nbrs[(g0 + slot) * D.S + D.col[tj] + sidx] & DPB_NBR_INDEX_MASK;
            if (idx < cnt_j) {
              const int js = D.offs[tj] + idx;
              const int src = perm ? perm[js] : js;
              const float *pj = pos + (frame_base + src) * 3;
              const float3 x = rel_coord(ri_s[slot], make_float3(pj[0], pj[1], pj[2]), L, ni, mimg);
              RowGeom gm;
              row_geom(x, M.rcut, gm);
              if (gm.s != 0.f) {
                keep = true;
                rv = make_float4(x.x, x.y, x.z, __int_as_float((src << 3) | slot));
              }
            }
          }
          int tot;
          const int pos_ = block_compact(keep, wcnt, &tot);
          if (keep) rowbuf[rowcount + pos_] = rv;
          rowcount += tot;
          __syncthreads();
        }
        while (rowcount >= 128 || (flush && rowcount > 0)) {
          const int nrows = min(rowcount, 128);
          const bool act = tid < nrows;
          const float4 rv = act ? rowbuf[tid] : make_float4(100.f, 100.f, 100.f, 0.f);
          const int packed = act ? __float_as_int(rv.w) : 0;
          const int slot = packed & 7, jsrc = packed >> 3;
          RowGeom gm;
          float st, R[10];
          mix_row_env(rv, M.rcut, inv_std, mean, gm, st, R);
          // ---- layer 0 with tangent: h0, d0 = dh0/ds~ -> A0, A0t
          float h1[E1], d1[E1];
          {
            float h0[E0], d0[E0];
#pragma unroll
            for (int k = 0; k < E0; ++k) {
              const float t = tanhf(fmaf(st, sm[k], sm[E0 + k]));
              h0[k] = t;
              d0[k] = (1.f - t * t) * sm[k];
            }
#pragma unroll
            for (int k8 = 0; k8 < MD::K1; k8 += 8) {
              float a_[8], b_[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                a_[u] = (k8 + u < E0) ? h0[min(k8 + u, E0 - 1)] : 0.f;
                b_[u] = (k8 + u < E0) ? d0[min(k8 + u, E0 - 1)] : 0.f;
              }
              *reinterpret_cast<uint4 *>(opb + oA0 + tc::kmajor_off(tid, k8, MD::K1)) =
                  make_uint4(tc::pack_bf16(a_[0], a_[1]), tc::pack_bf16(a_[2], a_[3]), tc::pack_bf16(a_[4], a_[5]),
                             tc::pack_bf16(a_[6], a_[7]));
              *reinterpret_cast<uint4 *>(opb + oA0t + tc::kmajor_off(tid, k8, MD::K1)) =
                  make_uint4(tc::pack_bf16(b_[0], b_[1]), tc::pack_bf16(b_[2], b_[3]), tc::pack_bf16(b_[4], b_[5]),
                             tc::pack_bf16(b_[6], b_[7]));
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
              tc::fence_after_sync();
#pragma unroll
              for (int ks = 0; ks < MD::K1 / 16; ++ks) {
                const uint64_t bd = tc::make_desc(w1_u + tc::kmajor_off(0, 16 * ks, MD::K1), 128, (MD::K1 / 8) * 128);
                tc::mma_bf16(tbase, tc::make_desc(opb_u + oA0 + tc::kmajor_off(0, 16 * ks, MD::K1), 128,
                                                  (MD::K1 / 8) * 128), bd, idesc1, ks > 0);
                tc::mma_bf16(tbase + 64, tc::make_desc(opb_u + oA0t + tc::kmajor_off(0, 16 * ks, MD::K1), 128,
                                                       (MD::K1 / 8) * 128), bd, idesc1, ks > 0);
              }
              tc::commit(&mbar);
            }
            MIX_WAIT();
            if (!ok) break;
            // ---- layer 1 epilogue with tangent -> A1, A1t
#pragma unroll
            for (int c0 = 0; c0 < MD::N1; c0 += 16) {
              float z[16], dz[16];
              tc::tmem_ld16(tbase + lane_off + c0, z);
              tc::tmem_ld16(tbase + 64 + lane_off + c0, dz);
#pragma unroll
              for (int i = 0; i < 16; ++i)
                if (c0 + i < E1) {
                  const float t = tc::tanh_fast(z[i] + sm[2 * E0 + c0 + i]);
                  h1[c0 + i] = t + h0[(c0 + i) / MD::Z1];
                  d1[c0 + i] = (1.f - t * t) * dz[i] + d0[(c0 + i) / MD::Z1];
                }
            }
          }
#pragma unroll
          for (int k8 = 0; k8 < MD::K2; k8 += 8) {
            float a_[8], b_[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              a_[u] = (k8 + u < E1) ? h1[min(k8 + u, E1 - 1)] : 0.f;
              b_[u] = (k8 + u < E1) ? d1[min(k8 + u, E1 - 1)] : 0.f;
            }
            *reinterpret_cast<uint4 *>(opb + oA1 + tc::kmajor_off(tid, k8, MD::K2)) =
                make_uint4(tc::pack_bf16(a_[0], a_[1]), tc::pack_bf16(a_[2], a_[3]), tc::pack_bf16(a_[4], a_[5]),
                           tc::pack_bf16(a_[6], a_[7]));
            *reinterpret_cast<uint4 *>(opb + oA1t + tc::kmajor_off(tid, k8, MD::K2)) =
                make_uint4(tc::pack_bf16(b_[0], b_[1]), tc::pack_bf16(b_[2], b_[3]), tc::pack_bf16(b_[4], b_[5]),
                           tc::pack_bf16(b_[6], b_[7]));
          }
          tc::fence_proxy_async();
          tc::fence_before_sync();
          __syncthreads();
          if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int ks = 0; ks < MD::K2 / 16; ++ks) {
              const uint64_t bd = tc::make_desc(w2_u + tc::kmajor_off(0, 16 * ks, MD::K2), 128, (MD::K2 / 8) * 128);
              tc::mma_bf16(tbase, tc::make_desc(opb_u + oA1 + tc::kmajor_off(0, 16 * ks, MD::K2), 128,
                                                (MD::K2 / 8) * 128), bd, idesc2, ks > 0);
              tc::mma_bf16(tbase + 128, tc::make_desc(opb_u + oA1t + tc::kmajor_off(0, 16 * ks, MD::K2), 128,
                                                      (MD::K2 / 8) * 128), bd, idesc2, ks > 0);
            }
            tc::commit(&mbar);
          }
          MIX_WAIT();
          if (!ok) break;
          // ---- layer 2 epilogue with tangent -> H2, H2t (K-major A of U / V)
#pragma unroll
          for (int c0 = 0; c0 < MD::N2; c0 += 16) {
            float z[16], dz[16];
            tc::tmem_ld16(tbase + lane_off + c0, z);
            tc::tmem_ld16(tbase + 128 + lane_off + c0, dz);
            float hh[16], dd[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              if (c0 + i < E2) {
                const float t = tc::tanh_fast(z[i] + sm[2 * E0 + E1 + min(c0 + i, E2 - 1)]);
                hh[i] = t + h1[min((c0 + i) / MD::Z2, E1 - 1)];
                dd[i] = (1.f - t * t) * dz[i] + d1[min((c0 + i) / MD::Z2, E1 - 1)];
              } else {
                hh[i] = 0.f;
                dd[i] = 0.f;
              }
            }
#pragma unroll
            for (int h = 0; h < 16; h += 8) {
              *reinterpret_cast<uint4 *>(opb + oH2 + tc::kmajor_off(tid, c0 + h, MD::N2)) =
                  make_uint4(tc::pack_bf16(hh[h], hh[h + 1]), tc::pack_bf16(hh[h + 2], hh[h + 3]),
                             tc::pack_bf16(hh[h + 4], hh[h + 5]), tc::pack_bf16(hh[h + 6], hh[h + 7]));
              *reinterpret_cast<uint4 *>(opb + oH2t + tc::kmajor_off(tid, c0 + h, MD::N2)) =
                  make_uint4(tc::pack_bf16(dd[h], dd[h + 1]), tc::pack_bf16(dd[h + 2], dd[h + 3]),
                             tc::pack_bf16(dd[h + 4], dd[h + 5]), tc::pack_bf16(dd[h + 6], dd[h + 7]));
            }
          }
          tc::fence_proxy_async();
          tc::fence_before_sync();
          __syncthreads();
          if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int ks = 0; ks < MD::N2 / 16; ++ks) {
              const uint64_t bd = tc::make_desc(dtb_u + tc::kmajor_off(0, 16 * ks, MD::N2), 128, (MD::N2 / 8) * 128);
              tc::mma_bf16(tbase, tc::make_desc(opb_u + oH2 + tc::kmajor_off(0, 16 * ks, MD::N2), 128,
                                                (MD::N2 / 8) * 128), bd, idesc3, ks > 0);
              tc::mma_bf16(tbase + 128, tc::make_desc(opb_u + oH2t + tc::kmajor_off(0, 16 * ks, MD::N2), 128,
                                                      (MD::N2 / 8) * 128), bd, idesc3, ks > 0);
            }
            tc::commit(&mbar);
          }
          MIX_WAIT();
          if (!ok) break;
          // ---- u, v of this row's atom slot; FP32 row adjoint
          float u[10], v[10];
#pragma unroll
          for (int c = 0; c < 10; ++c) u[c] = v[c] = 0.f;
#pragma unroll
          for (int q = 0; q < kBlkAtoms; ++q) {
            float uu[16], vv[16];
            tc::tmem_ld16(tbase + lane_off + 16 * q, uu);
            tc::tmem_ld16(tbase + 128 + lane_off + 16 * q, vv);
            if (q == slot) {
#pragma unroll
              for (int c = 0; c < 10; ++c) {
                u[c] = uu[c];
                v[c] = vv[c];
              }
            }
          }
          tc::fence_before_sync();
          float gst = 0.f;
#pragma unroll
          for (int c = 0; c < 10; ++c) gst = fmaf(R[c], v[c], gst);
          float gx[3];
          row_adjoint(gm, inv_std, u, gst, gx);
          if (act) {
            atomicAdd(&F4[frame_base + jsrc], make_float4(-gx[0], -gx[1], -gx[2], 0.f));
            atomicAdd(&fi_s[slot * 3 + 0], gx[0]);
            atomicAdd(&fi_s[slot * 3 + 1], gx[1]);
            atomicAdd(&fi_s[slot * 3 + 2], gx[2]);
#pragma unroll
            for (int p3 = 0; p3 < 3; ++p3)
#pragma unroll
              for (int q3 = 0; q3 < 3; ++q3) vir[p3 * 3 + q3] -= gm.x[p3] * gx[q3];
          }
          // ---- drop the processed rows, keep the carry
          const int rem = rowcount - nrows;
          float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
          if (tid < rem) carry = rowbuf[nrows + tid];
          __syncthreads();
          if (tid < rem) rowbuf[tid] = carry;
          rowcount = rem;
          __syncthreads();
        }
      }
    }
    if (!ok) break;
    __syncthreads();
    if (tid < nb * 3) {
      const int a = tid / 3, k = tid - a * 3;
      const int src = perm ? perm[D.offs[ti] + a0 + a] : D.offs[ti] + a0 + a;
      atomicAdd(reinterpret_cast<float *>(&F4[frame_base + src]) + k, fi_s[tid]);
    }
    __syncthreads();
  }
  // virial: per thread -> block (FP64) -> one atomic per component (frames
  // of a block share f; blocks may span frames, so use the last frame only
  // when F == 1 and the per-frame path otherwise)
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const float s = warp_sum(vir[k]);
    if ((tid & 31) == 0 && s != 0.f) atomicAdd(&vir_s[k], (double)s);
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1);
    tc::mbar_wait(&mbar, ph);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 9 && D.F == 1) atomicAdd(&virial[tid], vir_s[tid]);
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

template <int E0, int E1, int E2>
size_t mix_bwd_smem(int ntypes) {
  using MD = MixDims<E0, E1, E2>;
  return (size_t)ntypes * MD::NETB + ((ntypes * MD::NSMALL * 4 + 1023) / 1024) * 1024 +
         ((128 * MD::N2 * 2 + 1023) / 1024) * 1024 + ((2 * MD::OPA_H2 + 1023) / 1024) * 1024 + kRowCap * 16 + 1024;
}

template <int E0, int E1, int E2>
int launch_mix_embed_bwd(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                         const float *box, const int32_t *nbrs, const float *T, const float *dG, float4 *F4,
                         double *virial, int *err, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  const int nblk = (cnt + kBlkAtoms - 1) / kBlkAtoms * D.F;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = mix_bwd_smem<E0, E1, E2>(M.ntypes);
  DPB_CUDA_TRY(cudaFuncSetAttribute(k_mix_embed_bwd<E0, E1, E2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  // frames are separate grid slices when F > 1 so that each block's virial
  // belongs to one frame
  if (D.F == 1) {
    const int grid = nblk < nsm ? nblk : nsm;
    k_mix_embed_bwd<E0, E1, E2><<<grid, 128, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, dG, F4, virial, err);
    count_launch();
  } else {
    for (int f = 0; f < D.F; ++f) {
      SysDesc Df = D;
      Df.F = 1;
      const int nb1 = (cnt + kBlkAtoms - 1) / kBlkAtoms;
      const int grid = nb1 < nsm ? nb1 : nsm;
      const size_t off = (size_t)f * D.N;
      k_mix_embed_bwd<E0, E1, E2><<<grid, 128, smem, st>>>(M, Df, ti, pos + off * 3, perm, box + f * 3,
                                                            nbrs + off * D.S, T + off * 10 * M.E2,
                                                            dG + off * M.A * M.E2, F4 + off, virial + f * 9, err);
      count_launch();
    }
  }
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

// ---------------------------------------------------------------- fitting chain (BF16 tcgen05)
// One CTA per 128 atoms of one centre type (thread = atom = TMEM lane).  The
// forward layers and the adjoint down to dE/dG are GEMMs of M = 128 on the
// tensor cores with the B operand (weights, BF16, K contiguous) streamed from
// global memory through two shared-memory buffers, accumulating in TMEM
// (two 256-column regions used alternately).  Epilogues run in FP32 on the
// CUDA cores: tanh, dt-residuals, the energy dot product (FP64 frame sums) and
// the adjoint gates; tanh values and residual sources go to a per-atom FP32
// scratch, the BF16 activation for the next GEMM stays in shared memory.
constexpr int kFitKC = 48;                 // K per streamed chunk (multiple of 16)
constexpr int kFitMaxN = 256;              // N per GEMM pass (TMEM region)

struct FitStream {
  char *buf[2];
  uint64_t *bar;      // [2]
  uint32_t uses[2];
};

// B tile chunk: rows n in [n0, n0 + N) of a BF16 matrix with row stride ldb
// (K contiguous), columns [k0, k0 + KC) -> K-major tile (N x KC) in dst.
__device__ __forceinline__ void fit_load_b(char *dst, const __nv_bfloat16 *__restrict__ B, int ldb, int n0, int nvalid,
                                           int N, int k0, int kvalid) {
  const int nchunk8 = kFitKC / 8;
  for (int e = threadIdx.x; e < N * nchunk8; e += blockDim.x) {
    const int n = e / nchunk8, k8 = (e - n * nchunk8) * 8;
    uint4 q = make_uint4(0, 0, 0, 0);
    if (n < nvalid && k8 < kvalid) {
      const __nv_bfloat16 *src = B + (size_t)(n0 + n) * ldb + k0 + k8;
      if (k8 + 8 <= kvalid && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
        q = *reinterpret_cast<const uint4 *>(src);
      } else {
        __nv_bfloat16 t[8];
        for (int u = 0; u < 8; ++u) t[u] = (k8 + u < kvalid) ? src[u] : __float2bfloat16_rn(0.f);
        q = *reinterpret_cast<uint4 *>(t);
      }
    }
    *reinterpret_cast<uint4 *>(dst + tc::kmajor_off(n, k8, kFitKC)) = q;
  }
}

// A chunk from FP32 global rows (the descriptor G): 128 x KC -> K-major BF16.
__device__ __forceinline__ void fit_load_a(char *dst, const float *__restrict__ Gm, const size_t *atom_of_row,
                                           int nrows, int ld, int k0, int kvalid) {
  const int nchunk8 = kFitKC / 8;
  for (int e = threadIdx.x; e < 128 * nchunk8; e += blockDim.x) {
    const int r = e / nchunk8, k8 = (e - r * nchunk8) * 8;
    float t[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (r < nrows && k8 < kvalid) {
      const float *src = Gm + atom_of_row[r] * ld + k0 + k8;
      if (k8 + 8 <= kvalid) {
        const float4 a = *reinterpret_cast<const float4 *>(src), b = *reinterpret_cast<const float4 *>(src + 4);
        t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = a.w; t[4] = b.x; t[5] = b.y; t[6] = b.z; t[7] = b.w;
      } else {
        for (int u = 0; u < 8 && k8 + u < kvalid; ++u) t[u] = src[u];
      }
    }
    *reinterpret_cast<uint4 *>(dst + tc::kmajor_off(r, k8, kFitKC)) =
        make_uint4(tc::pack_bf16(t[0], t[1]), tc::pack_bf16(t[2], t[3]), tc::pack_bf16(t[4], t[5]),
                   tc::pack_bf16(t[6], t[7]));
  }
}

// D[128 x N] = A[128 x K] . B^T-rows[n0 : n0 + N][k] (B row stride ldb).  A is
// either resident (K-major tile with row length Kres) or streamed from G.
// Returns false when a barrier wait gave up.
__device__ bool fit_gemm(FitStream &S, uint32_t tmem_d, int N, int nvalid, int K, const __nv_bfloat16 *B, int ldb,
                         int n0, const char *A_res, int Kres, const float *Gm, const size_t *atom_of_row, int nrows,
                         int ldg) {
  const int nch = (K + kFitKC - 1) / kFitKC;
  const uint32_t idesc = tc::idesc_bf16(128, N, 0, 0);
  const int a_bytes = A_res ? 0 : 128 * kFitKC * 2;
  bool ok = true;
  for (int c = 0; c < nch; ++c) {
    const int b = c & 1;
    if (S.uses[b] > 0) {
      const bool w = tc::mbar_wait(&S.bar[b], (S.uses[b] - 1) & 1);
      ok = __syncthreads_and(w && ok) != 0;
      if (!ok) return false;
    }
    const int k0 = c * kFitKC, kv = min(kFitKC, K - k0);
    char *bufb = S.buf[b];
    if (!A_res) fit_load_a(bufb, Gm, atom_of_row, nrows, ldg, k0, kv);
    fit_load_b(bufb + a_bytes, B, ldb, n0, nvalid, N, k0, kv);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      const uint32_t bu = tc::smem_u32(bufb);
      for (int ks = 0; ks < kFitKC / 16; ++ks) {
        uint64_t ad;
        if (A_res)
          ad = tc::make_desc(tc::smem_u32(A_res) + tc::kmajor_off(0, k0 + 16 * ks, Kres), 128, (Kres / 8) * 128);
        else
          ad = tc::make_desc(bu + tc::kmajor_off(0, 16 * ks, kFitKC), 128, (kFitKC / 8) * 128);
        const uint64_t bd = tc::make_desc(bu + a_bytes + tc::kmajor_off(0, 16 * ks, kFitKC), 128, (kFitKC / 8) * 128);
        tc::mma_bf16(tmem_d, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
      }
      tc::commit(&S.bar[b]);
    }
    S.uses[b]++;
  }
  // the accumulator is complete when the last chunk's MMAs are
  const int bl = (nch - 1) & 1;
  const bool w = tc::mbar_wait(&S.bar[bl], (S.uses[bl] - 1) & 1);
  ok = __syncthreads_and(w && ok) != 0;
  tc::fence_after_sync();
  return ok;
}

// Store a row of FW FP32 values into the K-major BF16 activation tile.
__device__ __forceinline__ void fit_store_act(char *HA, int row, int k8, const float (&v)[8], int FWp) {
  *reinterpret_cast<uint4 *>(HA + tc::kmajor_off(row, k8, FWp)) =
      make_uint4(tc::pack_bf16(v[0], v[1]), tc::pack_bf16(v[2], v[3]), tc::pack_bf16(v[4], v[5]),
                 tc::pack_bf16(v[6], v[7]));
}

template <int FW>
__global__ void __launch_bounds__(128, 1) k_mix_fit(DevModel M, int ti, int Mrows, RowMap rm, const float *__restrict__ Gin,
                                                   float *__restrict__ dGout, float *__restrict__ scratch,
                                                   float *__restrict__ Eatom, double *__restrict__ energy, int N,
                                                   int *__restrict__ err) {
  static_assert(FW % 16 == 0 && FW <= kFitMaxN, "fit width");
  constexpr int BUFB = 128 * kFitKC * 2 + kFitMaxN * kFitKC * 2;
  extern __shared__ __align__(1024) char smem[];
  char *HA = smem;                                  // 128 x FW bf16 (K-major)
  char *bufs = HA + ((128 * FW * 2 + 1023) / 1024) * 1024;
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tbase_s;
  __shared__ size_t atom_s[128];
  __shared__ double es[128];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int L = M.nfit, K0 = M.A * M.E2;
  if (tid < 2) tc::mbar_init(&bars[tid], 1);
  if (warp == 0) tc::tmem_alloc(&tbase_s, 512);
  FitStream S;
  S.buf[0] = bufs;
  S.buf[1] = bufs + BUFB;
  S.bar = bars;
  S.uses[0] = S.uses[1] = 0;
  const int r0 = blockIdx.x * 128, nrows = min(128, Mrows - r0);
  const bool act = tid < nrows;
  atom_s[tid] = act ? rm.atom(r0 + tid) : rm.atom(r0);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tb = tbase_s, lane_off = (uint32_t)(warp * 32) << 16;
  const size_t me = atom_s[tid];
  // per-atom scratch: t_l (L x FW), H_l (L x FW), gH (FW)
  float *tl = scratch + me * (size_t)(2 * L + 1) * FW;
  float *hl = tl + (size_t)L * FW;
  float *gh = hl + (size_t)L * FW;
  bool ok = true;
  uint32_t region = 0;
  // ---- forward
  for (int l = 0; l < L && ok; ++l) {
    const uint32_t td = tb + region * 256;
    if (l == 0)
      ok = fit_gemm(S, td, FW, FW, K0, M.fwT_bf[ti][0], K0, 0, nullptr, 0, Gin, atom_s, nrows, K0);
    else
      ok = fit_gemm(S, td, FW, FW, FW, M.fwT_bf[ti][l], FW, 0, HA, FW, nullptr, nullptr, 0, 0);
    if (!ok) break;
    const float *bias = M.fb[ti][l], *dt = M.fdt[ti][l];
    for (int c0 = 0; c0 < FW; c0 += 16) {
      float v[16];
      tc::tmem_ld16(td + lane_off + c0, v);
      float hv[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = c0 + i;
        const float t = tc::tanh_fast(v[i] + bias[n]);
        float h = t;
        if (dt) h = t * dt[n] + hl[(size_t)(l - 1) * FW + n];
        hv[i] = h;
        if (act) {
          tl[(size_t)l * FW + n] = t;
          hl[(size_t)l * FW + n] = h;
        }
      }
      tc::fence_before_sync();
      __syncthreads();  // every thread has read this chunk; HA may be overwritten after the GEMM
      fit_store_act(HA, tid, c0, *reinterpret_cast<float(*)[8]>(hv), FW);
      fit_store_act(HA, tid, c0 + 8, *reinterpret_cast<float(*)[8]>(hv + 8), FW);
    }
    region ^= 1;
  }
  // ---- energy and the first adjoint gate
  double e_me = 0.0;
  if (ok) {
    const float *wf = M.fw[ti][L], *dtL = M.fdt[ti][L - 1];
    float s = 0.f;
    for (int c0 = 0; c0 < FW; c0 += 8) {
      float g[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int n = c0 + i;
        s = fmaf(hl[(size_t)(L - 1) * FW + n], wf[n], s);
        const float t = tl[(size_t)(L - 1) * FW + n];
        g[i] = wf[n] * (dtL ? dtL[n] : 1.f) * (1.f - t * t);
      }
      fit_store_act(HA, tid, c0, g, FW);
    }
    s += M.fb[ti][L][0];
    if (act) Eatom[me] = s;
    e_me = act ? (double)s : 0.0;
  }
  es[tid] = e_me;
  __syncthreads();
  if (tid == 0 && ok) {
    double run = 0.0;
    int cf = (int)(atom_s[0] / N);
    for (int k = 0; k < nrows; ++k) {
      const int fk = (int)(atom_s[k] / N);
      if (fk != cf) {
        atomicAdd(&energy[cf], run);
        run = 0.0;
        cf = fk;
      }
      run += es[k];
    }
    atomicAdd(&energy[cf], run);
  }
  // ---- adjoint: layers L-1 .. 1, gH_{l-1} = gZ_l W_l^T (+ gH_l if residual)
  for (int l = L - 1; l >= 1 && ok; --l) {
    const uint32_t td = tb + region * 256;
    ok = fit_gemm(S, td, FW, FW, FW, M.fw_bf[ti][l], FW, 0, HA, FW, nullptr, nullptr, 0, 0);
    if (!ok) break;
    const bool res_l = M.fdt[ti][l] != nullptr, res_lm1 = (l - 1 > 0) && M.fdt[ti][l - 1] != nullptr;
    const float *dtm1 = M.fdt[ti][l - 1], *wf = M.fw[ti][L];
    for (int c0 = 0; c0 < FW; c0 += 16) {
      float v[16];
      tc::tmem_ld16(td + lane_off + c0, v);
      float gz[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = c0 + i;
        float g = v[i];
        if (res_l) g += (l == L - 1) ? wf[n] : gh[n];
        const float t = tl[(size_t)(l - 1) * FW + n];
        gz[i] = g * (res_lm1 ? dtm1[n] : 1.f) * (1.f - t * t);
        if (act && res_lm1) gh[n] = g;  // read by the next layer's epilogue (same thread)
      }
      tc::fence_before_sync();
      __syncthreads();
      fit_store_act(HA, tid, c0, *reinterpret_cast<float(*)[8]>(gz), FW);
      fit_store_act(HA, tid, c0 + 8, *reinterpret_cast<float(*)[8]>(gz + 8), FW);
    }
    region ^= 1;
  }
  // ---- dE/dG = gZ_0 W_0^T in column passes of 256
  for (int n0 = 0; n0 < K0 && ok; n0 += kFitMaxN) {
    const int nv = min(kFitMaxN, K0 - n0), Np = (nv + 15) / 16 * 16;
    const uint32_t td = tb + region * 256;
    ok = fit_gemm(S, td, Np, nv, FW, M.fw_bf[ti][0], FW, n0, HA, FW, nullptr, nullptr, 0, 0);
    if (!ok) break;
    for (int c0 = 0; c0 < Np; c0 += 16) {
      float v[16];
      tc::tmem_ld16(td + lane_off + c0, v);
      if (act) {
#pragma unroll
        for (int i = 0; i < 16; i += 4)
          if (c0 + i < nv)
            *reinterpret_cast<float4 *>(dGout + me * K0 + n0 + c0 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
    }
    tc::fence_before_sync();
    region ^= 1;
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1);
    tc::mbar_wait(&bars[0], 0);
    tc::mbar_wait(&bars[1], 0);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tb, 512);
}

template <int FW>
int launch_mix_fit(const DevModel &M, const SysDesc &D, float *G, float *dG, float *scratch, float *Eatom,
                   double *energy, int *err, cudaStream_t st) {
  constexpr int BUFB = 128 * kFitKC * 2 + kFitMaxN * kFitKC * 2;
  const size_t smem = ((128 * FW * 2 + 1023) / 1024) * 1024 + 2 * BUFB;
  DPB_CUDA_TRY(cudaFuncSetAttribute(k_mix_fit<FW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int ti = 0; ti < M.ntypes; ++ti) {
    const int cnt = D.offs[ti + 1] - D.offs[ti];
    if (!cnt) continue;
    const RowMap rm{cnt, D.N, D.offs[ti]};
    const int Mrows = cnt * D.F;
    k_mix_fit<FW><<<(Mrows + 127) / 128, 128, smem, st>>>(M, ti, Mrows, rm, G, dG, scratch, Eatom, energy, D.N, err);
    count_launch();
    DPB_LAUNCH_CHECK();
  }
  return DPB_OK;
}

// ---------------------------------------------------------------- dispatch
template <int E0, int E1, int E2>
int launch_embed_bwd(const DevModel &, const SysDesc &, int, const float *, const int32_t *, const float *,
                     const int32_t *, const float *, const float *, float4 *, double *, cudaStream_t);
int launch_sgemm(int, int, int, const float *, int, RowMap, const float *, const Epi &, cudaStream_t);
int launch_fit_energy(int, RowMap, int, const float *, const float *, const float *, const float *, const float *,
                      float *, float *, double *, int, cudaStream_t);
int fit_fp32_chain(const DevModel &M, const SysDesc &D, float *G, float *Eatom, double *energy, char *w,
                   cudaStream_t st);

int mixed_supported(const DevModel &M) {
  return (M.E0 == 25 && M.E1 == 50 && M.E2 == 100) || (M.E0 == 32 && M.E1 == 32 && M.E2 == 64);
}

size_t mixed_workspace_per_atom(const DevModel &M) {
  const int FW = M.FW[0];
  return (size_t)(10 * M.E2 + M.A * M.E2 + 2 * M.nfit * FW + 4 * FW + 1) * 4 + 16 + 64;
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int mixed_descriptors(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm, const float *box,
                      const int32_t *nbrs, float *T, float *G, int *err, cudaStream_t st) {
  prof_begin(PROF_MIXED_EMBED_FWD, st);
  for (int ti = 0; ti < M.ntypes; ++ti) {
    int rc = (M.E2 == 100) ? launch_mix_embed_fwd<25, 50, 100>(M, D, ti, pos, perm, box, nbrs, T, G, err, st)
                           : launch_mix_embed_fwd<32, 32, 64>(M, D, ti, pos, perm, box, nbrs, T, G, err, st);
    if (rc) return rc;
  }
  prof_end(PROF_MIXED_EMBED_FWD, st);
  return DPB_OK;
}

int mixed_eval(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm, const float *box,
               const int32_t *nbrs, double *energy, float *Eatom, float4 *F4, double *virial, void *ws,
               cudaStream_t st) {
  const size_t NF = (size_t)D.N * D.F;
  char *w = (char *)ws;
  int *err = (int *)w; w += 256;
  float *T = (float *)w; w += al256(NF * 10 * M.E2 * 4);
  float *G = (float *)w; w += al256(NF * M.A * M.E2 * 4);
  DPB_CUDA_TRY(cudaMemsetAsync(err, 0, 4, st));
  int rc = mixed_descriptors(M, D, pos, perm, box, nbrs, T, G, err, st);
  if (rc) return rc;
  prof_begin(PROF_MIXED_FIT, st);
  if (M.FW[0] == 240) {
    rc = launch_mix_fit<240>(M, D, G, G, reinterpret_cast<float *>(w), Eatom, energy, err, st);
  } else if (M.FW[0] == 128) {
    rc = launch_mix_fit<128>(M, D, G, G, reinterpret_cast<float *>(w), Eatom, energy, err, st);
  } else {
    rc = fit_fp32_chain(M, D, G, Eatom, energy, w, st);
  }
  prof_end(PROF_MIXED_FIT, st);
  if (rc) return rc;
  prof_begin(PROF_MIXED_EMBED_BWD, st);
  for (int ti = 0; ti < M.ntypes; ++ti) {
    rc = (M.E2 == 100)
             ? launch_mix_embed_bwd<25, 50, 100>(M, D, ti, pos, perm, box, nbrs, T, G, F4, virial, err, st)
             : launch_mix_embed_bwd<32, 32, 64>(M, D, ti, pos, perm, box, nbrs, T, G, F4, virial, err, st);
    if (rc) return rc;
  }
  prof_end(PROF_MIXED_EMBED_BWD, st);
  return DPB_OK;
}

}  // namespace dpb

extern "C" int dpb_selftest_tcgen05(int variant, float *out, int *err, void *stream) {
  if (!out || !err || variant < 0 || variant > 1) return DPB_ERR_INVALID_ARG;
  dpb::k_selftest_umma<<<1, 128, 0, (cudaStream_t)stream>>>(variant, out, err);
  dpb::count_launch();
  return cudaGetLastError() == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
}
