// Plain FP32 evaluation path: energy, forces and virial of the se_a model.
//
// Three stages per centre type (reference model: deepmd_jax/dpmodel.py:30-100,
// embedding/fitting nets deepmd_jax/utils.py:100-166):
//   1. k_embed_fwd   warp per centre atom: neighbour rows with s(r) != 0 are
//                    compacted, pushed through the per-type-pair embedding MLP,
//                    contracted with the 10-channel env rows into T (10 x W);
//                    the epilogue forms the descriptor G (A x W).
//   2. fitting       tiled SGEMM chain over the atoms of one centre type, fused
//                    tanh / dt-residual epilogues, per-atom energy, and the
//                    adjoint chain down to dE/dG.
//   3. k_embed_bwd   warp per centre atom: dE/dT from dE/dG, then the rows are
//                    recomputed with forward-mode tangents (h, dh/ds~) so
//                    dE/ds~ and dE/dR~ come out of one sweep; the row adjoint
//                    gives dE/dx, scattered as forces (float4 atomics) and
//                    reduced into the virial.
// Rows with s(r) = 0 contribute exactly zero in the reference (R~ = 0) and are
// skipped here.
#include "eval_common.cuh"

namespace dpb {

__device__ __forceinline__ float3 load_pos(const float *__restrict__ pos, const int32_t *__restrict__ perm,
                                           int f, int k, int N) {
  int src = perm ? perm[k] : k;
  const float *p = pos + ((size_t)f * N + src) * 3;
  return make_float3(p[0], p[1], p[2]);
}

template <int E0, int E1, int E2>
struct EmbedDims {
  static constexpr int NW = 2 * E0 + E0 * E1 + E1 + E1 * E2 + E2;  // floats per net
  static constexpr int NQ = (E2 + 31) / 32;
  static constexpr int Z1 = E1 / E0;
  static constexpr int Z2 = E2 / E1;
};

// Load the weights of nets (ti, tj), tj < ntypes, into shared memory.
template <int E0, int E1, int E2>
__device__ void load_nets(const DevModel &M, int ti, float *wsm) {
  using D = EmbedDims<E0, E1, E2>;
  for (int tj = 0; tj < M.ntypes; ++tj) {
    int k = ti * M.ntypes + tj;
    float *w = wsm + tj * D::NW;
    const float *src[6] = {M.ew[k][0], M.eb[k][0], M.ew[k][1], M.eb[k][1], M.ew[k][2], M.eb[k][2]};
    const int len[6] = {E0, E0, E0 * E1, E1, E1 * E2, E2};
    int o = 0;
    for (int s = 0; s < 6; ++s) {
      for (int e = threadIdx.x; e < len[s]; e += blockDim.x) w[o + e] = src[s][e];
      o += len[s];
    }
  }
}

// ---------------------------------------------------------------- forward
// One round of up to 32 compacted rows (row = lane).  Every layer runs
// input-outer from activations staged per lane in shared memory
// (h0s/h1s[k][lane]), so residual sources h[col / Z] are read with runtime
// columns and no register array is indexed dynamically.  The contraction
// T += R~^T h2 is accumulated per 32-column chunk in registers and added into
// the warp's shared T (Ts[c][col]) once per round.
template <int E0, int E1, int E2>
__device__ __forceinline__ void embed_rows_fwd(const float *__restrict__ W, int n,
                                               const float *__restrict__ rowbuf, float *__restrict__ h0s,
                                               float *__restrict__ h1s, float *__restrict__ h2s,
                                               float *__restrict__ Ts, int lane) {
  using D = EmbedDims<E0, E1, E2>;
  const float *w0 = W, *b0 = W + E0, *w1 = W + 2 * E0, *b1 = w1 + E0 * E1, *w2 = b1 + E1,
              *b2 = w2 + E1 * E2;
  const float st = lane < n ? rowbuf[lane * 12] : 0.f;
#pragma unroll
  for (int k = 0; k < E0; ++k) h0s[k * 32 + lane] = tanhf(fmaf(st, w0[k], b0[k]));
#pragma unroll 1
  for (int q = 0; q < (E1 + 31) / 32; ++q) {
    float acc[32];
#pragma unroll
    for (int o = 0; o < 32; ++o) acc[o] = (q * 32 + o < E1) ? b1[q * 32 + o] : 0.f;
#pragma unroll 2
    for (int k = 0; k < E0; ++k) {
      const float hv = h0s[k * 32 + lane];
      const float *wr = w1 + k * E1 + q * 32;
#pragma unroll
      for (int o = 0; o < 32; ++o)
        if (q * 32 + o < E1) acc[o] = fmaf(hv, wr[o], acc[o]);
    }
#pragma unroll
    for (int o = 0; o < 32; ++o) {
      const int col = q * 32 + o;
      if (col < E1) h1s[col * 32 + lane] = tanhf(acc[o]) + h0s[(col / D::Z1) * 32 + lane];
    }
  }
  __syncwarp();  // h2s aliases h0s
#pragma unroll 1
  for (int q = 0; q < D::NQ; ++q) {
    float acc[32];
#pragma unroll
    for (int o = 0; o < 32; ++o) acc[o] = (q * 32 + o < E2) ? b2[q * 32 + o] : 0.f;
#pragma unroll 2
    for (int k = 0; k < E1; ++k) {
      const float hv = h1s[k * 32 + lane];
      const float *wr = w2 + k * E2 + q * 32;
#pragma unroll
      for (int o = 0; o < 32; ++o)
        if (q * 32 + o < E2) acc[o] = fmaf(hv, wr[o], acc[o]);
    }
#pragma unroll
    for (int o = 0; o < 32; ++o) {
      const int col = q * 32 + o;
      if (col < E2) h2s[lane * 33 + o] = tanhf(acc[o]) + h1s[(col / D::Z2) * 32 + lane];
    }
    __syncwarp();
    const int col = q * 32 + lane;
    if (col < E2) {
      float Tq[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) Tq[c] = 0.f;
      for (int r = 0; r < n; ++r) {
        const float hv = h2s[r * 33 + lane];
        const float *R = rowbuf + r * 12 + 1;
#pragma unroll
        for (int c = 0; c < 10; ++c) Tq[c] = fmaf(R[c], hv, Tq[c]);
      }
#pragma unroll
      for (int c = 0; c < 10; ++c) Ts[c * E2 + col] += Tq[c];
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- compressed embedding
// The table lookup of the compressed embedding net (deepmd_jax/utils.py:126-151):
// x = s~ - srmin; idx = trunc(x / delta); x0 = x - idx * delta; the gather
// clamps idx into [0, Ngrids) while x0 keeps the unclamped idx; h[w] =
// sum_i c[idx][i][w] x0^(5-i), evaluated here by Horner's rule.
__device__ __forceinline__ void cmp_locate(float st, float srmin, float delta, int ng, int &idx, float &x0) {
  const float x = __fsub_rn(st, srmin);
  const int k = (int)__fdiv_rn(x, delta);  // truncation toward zero, like astype(int)
  x0 = __fsub_rn(x, __fmul_rn((float)k, delta));
  idx = k < 0 ? 0 : (k >= ng ? ng - 1 : k);
}

// One round of up to 32 compacted rows, column-parallel: lane owns columns
// q*32 + lane; the rows' (idx, x0) and env rows are read from the row buffer
// (st slot overwritten by x0, slot 11 by idx) and each table row is read with
// coalesced loads.  T += R~^T h accumulates into the warp's shared T.
template <int E2>
__device__ __forceinline__ void embed_rows_fwd_cmp(const float *__restrict__ coeff, float srmin, float delta,
                                                   int ng, int n, float *__restrict__ rowbuf,
                                                   float *__restrict__ Ts, int lane) {
  if (lane < n) {
    int idx;
    float x0;
    cmp_locate(rowbuf[lane * 12], srmin, delta, ng, idx, x0);
    rowbuf[lane * 12] = x0;
    rowbuf[lane * 12 + 11] = __int_as_float(idx);
  }
  __syncwarp();
#pragma unroll 1
  for (int q = 0; q < (E2 + 31) / 32; ++q) {
    const int col = q * 32 + lane;
    if (col < E2) {
      float Tq[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) Tq[c] = 0.f;
      for (int r = 0; r < n; ++r) {
        const float *rb = rowbuf + r * 12;
        const float x0 = rb[0];
        const float *cr = coeff + (size_t)__float_as_int(rb[11]) * 6 * E2 + col;
        float h = __ldg(cr);
#pragma unroll
        for (int i = 1; i < 6; ++i) h = fmaf(h, x0, __ldg(cr + i * E2));
#pragma unroll
        for (int c = 0; c < 10; ++c) Tq[c] = fmaf(rb[1 + c], h, Tq[c]);
      }
#pragma unroll
      for (int c = 0; c < 10; ++c) Ts[c * E2 + col] += Tq[c];
    }
  }
  __syncwarp();
}

template <int E0, int E1, int E2>
__host__ __device__ constexpr int embed_fwd_warp_floats() {
  return 64 * 12 + (32 * 33 > E0 * 32 ? 32 * 33 : E0 * 32) + E1 * 32 + 10 * E2;
}

template <int E0, int E1, int E2, bool CMP>
__global__ void __launch_bounds__(256) k_embed_fwd(DevModel M, SysDesc D, int ti, const float *__restrict__ pos,
                                                   const int32_t *__restrict__ perm, const float *__restrict__ box,
                                                   const int32_t *__restrict__ nbrs, float *__restrict__ Tout,
                                                   float *__restrict__ Gout) {
  using ED = EmbedDims<E0, E1, E2>;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  float *wsm = smem;
  float *rowbuf = smem + (CMP ? 0 : M.ntypes * ED::NW) + warp * embed_fwd_warp_floats<E0, E1, E2>();
  float *h2s = rowbuf + 64 * 12;  // aliases h0s
  float *h0s = h2s;
  float *h1s = h2s + (32 * 33 > E0 * 32 ? 32 * 33 : E0 * 32);
  float *Ts = h1s + E1 * 32;
  if (!CMP) load_nets<E0, E1, E2>(M, ti, wsm);
  __syncthreads();
  const int f = blockIdx.y;
  const int a = blockIdx.x * wpb + warp;
  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  if (a >= cnt_i) return;
  const int i = D.offs[ti] + a;
  const size_t g = (size_t)f * D.N + i;
  const float3 ri = load_pos(pos, perm, f, i, D.N);
  const int bs = box_slot(D, g, f);
  const float3 L = make_float3(box[bs * 3], box[bs * 3 + 1], box[bs * 3 + 2]);
  const int3 ni = image_range(L, M.rcut);
  const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
  const float inv_std = M.inv_std[ti], mean = M.mean[ti];
  const unsigned lt = (1u << lane) - 1u;
  for (int e = lane; e < 10 * E2; e += 32) Ts[e] = 0.f;
  __syncwarp();

  for (int tj = 0; tj < D.ntypes; ++tj) {
    const float *W = wsm + tj * ED::NW;
    const int32_t *nb = nbrs + g * D.S + D.col[tj];
    const int sel = D.sel[tj], cnt_j = D.offs[tj + 1] - D.offs[tj];
    int nbuf = 0;
    const int total = sel * nim;
    for (int base = 0; base < total; base += 32) {
      const int p = base + lane;
      bool keep = false;
      float st = 0.f, R[10];
      if (p < total) {
        const int slot = nim == 1 ? p : p / nim, mimg = p - slot * nim;
        const int idx = nb[slot] & DPB_NBR_INDEX_MASK;
        if (idx < cnt_j) {
          const float3 rj = load_pos(pos, perm, f, D.offs[tj] + idx, D.N);
          RowGeom gm;
          row_geom(rel_coord(ri, rj, L, ni, mimg), M.rcut, gm);
          if (gm.s != 0.f) {
            keep = true;
            const float sn = gm.s * inv_std;
            st = (gm.s - mean) * inv_std;
            const float inv_rp = 1.f / (gm.r + 1e-16f);
            const float xh[3] = {gm.x[0] * inv_rp, gm.x[1] * inv_rp, gm.x[2] * inv_rp};
            env_row(sn, xh, R);
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        float *dst = rowbuf + (nbuf + __popc(m & lt)) * 12;
        dst[0] = st;
#pragma unroll
        for (int c = 0; c < 10; ++c) dst[1 + c] = R[c];
      }
      nbuf += __popc(m);
      __syncwarp();
      if (nbuf >= 32) {
        if constexpr (CMP)
          embed_rows_fwd_cmp<E2>(M.cmp_coeff[ti * M.ntypes + tj], M.cmp_srmin[ti * M.ntypes + tj],
                                 M.cmp_delta[ti * M.ntypes + tj], M.ngrids, 32, rowbuf, Ts, lane);
        else
          embed_rows_fwd<E0, E1, E2>(W, 32, rowbuf, h0s, h1s, h2s, Ts, lane);
        const int rem = nbuf - 32;
        if (lane < rem)
          for (int c = 0; c < 12; ++c) rowbuf[lane * 12 + c] = rowbuf[(32 + lane) * 12 + c];
        __syncwarp();
        nbuf = rem;
      }
    }
    if (nbuf > 0) {
      if constexpr (CMP)
        embed_rows_fwd_cmp<E2>(M.cmp_coeff[ti * M.ntypes + tj], M.cmp_srmin[ti * M.ntypes + tj],
                               M.cmp_delta[ti * M.ntypes + tj], M.ngrids, nbuf, rowbuf, Ts, lane);
      else
        embed_rows_fwd<E0, E1, E2>(W, nbuf, rowbuf, h0s, h1s, h2s, Ts, lane);
    }
    __syncwarp();
  }

  // T = sum / Nnbrs (written out); Ts becomes X = T with Tbias on channel 0
  for (int e = lane; e < 10 * E2; e += 32) {
    const float t = Ts[e] * M.inv_nnbrs;
    Tout[g * 10 * E2 + e] = t;
    Ts[e] = t + (e < E2 ? M.tbias[e] : 0.f);
  }
  __syncwarp();
  // G[a][w] = sum_c Q[c][a] X[c][w] (dpmodel.py:74-78), Q[c<4][a] = X[c][a],
  // Q[4+m][a] = tensor_3to6(X[1:4][A+a])[m] + X[4+m][A+a]
  const int A = M.A;
  float *Gg = Gout + g * (size_t)A * E2;
  for (int aa = 0; aa < A; ++aa) {
    float Q[10];
#pragma unroll
    for (int c = 0; c < 4; ++c) Q[c] = Ts[c * E2 + aa];
    const float y1 = Ts[1 * E2 + A + aa], y2 = Ts[2 * E2 + A + aa], y3 = Ts[3 * E2 + A + aa];
    Q[4] = y1 * y1 + Ts[4 * E2 + A + aa];
    Q[5] = y2 * y2 + Ts[5 * E2 + A + aa];
    Q[6] = y3 * y3 + Ts[6 * E2 + A + aa];
    Q[7] = kSqrt2 * y1 * y3 + Ts[7 * E2 + A + aa];
    Q[8] = kSqrt2 * y2 * y1 + Ts[8 * E2 + A + aa];
    Q[9] = kSqrt2 * y3 * y2 + Ts[9 * E2 + A + aa];
    for (int col = lane; col < E2; col += 32) {
      float v = 0.f;
#pragma unroll
      for (int c = 0; c < 10; ++c) v = fmaf(Q[c], Ts[c * E2 + col], v);
      Gg[aa * E2 + col] = v;
    }
  }
}

// ---------------------------------------------------------------- adjoint
// Adjoint of one round of rows.  The row's embedding is recomputed with its
// tangent along s~ (forward mode): h2 and dh2/ds~ give, against dE/dT,
// u = dT.h2 = dE/dR~ and v = dT.dh2, so dE/ds~ = R~.v — no reverse sweep.
template <int E0, int E1, int E2>
__device__ __forceinline__ void embed_rows_bwd(const float *__restrict__ W, int n,
                                               const float *__restrict__ rowbuf, const float *__restrict__ dT,
                                               float *__restrict__ h1s, float *__restrict__ d1s,
                                               float inv_std, float mean, int lane, float &fi0, float &fi1,
                                               float &fi2, float (&vir)[9], float4 *__restrict__ F4,
                                               size_t frame_base) {
  using D = EmbedDims<E0, E1, E2>;
  const float *w0 = W, *b0 = W + E0, *w1 = W + 2 * E0, *b1 = w1 + E0 * E1, *w2 = b1 + E1,
              *b2 = w2 + E1 * E2;
  const bool act = lane < n;
  RowGeom gm;
  int jj = 0;
  if (act) {
    const float *rb = rowbuf + lane * 8;
    gm.x[0] = rb[0]; gm.x[1] = rb[1]; gm.x[2] = rb[2];
    gm.r = rb[3]; gm.s = rb[4]; gm.dsdr = rb[5];
    jj = __float_as_int(rb[6]);
  } else {
    gm.x[0] = gm.x[1] = gm.x[2] = 0.f; gm.r = 1.f; gm.s = 0.f; gm.dsdr = 0.f;
  }
  const float sn = gm.s * inv_std, st = (gm.s - mean) * inv_std;
  const float inv_rp = 1.f / (gm.r + 1e-16f);
  const float xh[3] = {gm.x[0] * inv_rp, gm.x[1] * inv_rp, gm.x[2] * inv_rp};
  {
    float h0[E0], d0[E0];
#pragma unroll
    for (int k = 0; k < E0; ++k) {
      const float t = tanhf(fmaf(st, w0[k], b0[k]));
      h0[k] = t;
      d0[k] = (1.f - t * t) * w0[k];
    }
#pragma unroll
    for (int o = 0; o < E1; ++o) {
      float z = b1[o], dz = 0.f;
#pragma unroll
      for (int k = 0; k < E0; ++k) {
        z = fmaf(h0[k], w1[k * E1 + o], z);
        dz = fmaf(d0[k], w1[k * E1 + o], dz);
      }
      const float t = tanhf(z);
      h1s[o * 32 + lane] = t + h0[o / D::Z1];
      d1s[o * 32 + lane] = (1.f - t * t) * dz + d0[o / D::Z1];
    }
  }
  __syncwarp();
  float u[10], v[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) u[c] = v[c] = 0.f;
  constexpr int NQ16 = (E2 + 15) / 16;
#pragma unroll 1
  for (int q = 0; q < NQ16; ++q) {
    float z[16], dz[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      z[o] = (q * 16 + o < E2) ? b2[q * 16 + o] : 0.f;
      dz[o] = 0.f;
    }
#pragma unroll 2
    for (int k = 0; k < E1; ++k) {
      const float hv = h1s[k * 32 + lane], dv = d1s[k * 32 + lane];
      const float *wr = w2 + k * E2 + q * 16;
#pragma unroll
      for (int o = 0; o < 16; ++o)
        if (q * 16 + o < E2) {
          const float wv = wr[o];
          z[o] = fmaf(hv, wv, z[o]);
          dz[o] = fmaf(dv, wv, dz[o]);
        }
    }
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      const int col = q * 16 + o;
      if (col < E2) {
        const float t = tanhf(z[o]);
        const int src = (col / D::Z2) * 32 + lane;
        const float h2 = t + h1s[src];
        const float dh2 = (1.f - t * t) * dz[o] + d1s[src];
#pragma unroll
        for (int c = 0; c < 10; ++c) {
          const float dtc = dT[c * E2 + col];
          u[c] = fmaf(dtc, h2, u[c]);
          v[c] = fmaf(dtc, dh2, v[c]);
        }
      }
    }
  }
  __syncwarp();
  float R[10];
  env_row(sn, xh, R);
  float gst = 0.f;
#pragma unroll
  for (int c = 0; c < 10; ++c) gst = fmaf(R[c], v[c], gst);
  float gx[3];
  row_adjoint(gm, inv_std, u, gst, gx);
  if (act) {
    atomicAdd(&F4[frame_base + jj], make_float4(-gx[0], -gx[1], -gx[2], 0.f));
    fi0 += gx[0]; fi1 += gx[1]; fi2 += gx[2];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int qq = 0; qq < 3; ++qq) vir[p * 3 + qq] -= gm.x[p] * gx[qq];
  }
}

// Adjoint of one round of rows of a compressed net (row = lane): h and
// dh/ds~ = dh/dx0 from the row's table entry (float4 loads along w), u =
// dT.h, v = dT.dh, then the same env-row adjoint as the MLP path.
template <int E2>
__device__ __forceinline__ void embed_rows_bwd_cmp(const float *__restrict__ coeff, float srmin, float delta,
                                                   int ng, int n, const float *__restrict__ rowbuf,
                                                   const float *__restrict__ dT, float inv_std, float mean,
                                                   int lane, float &fi0, float &fi1, float &fi2, float (&vir)[9],
                                                   float4 *__restrict__ F4, size_t frame_base) {
  static_assert(E2 % 4 == 0, "table width");
  const bool act = lane < n;
  RowGeom gm;
  int jj = 0;
  if (act) {
    const float *rb = rowbuf + lane * 8;
    gm.x[0] = rb[0]; gm.x[1] = rb[1]; gm.x[2] = rb[2];
    gm.r = rb[3]; gm.s = rb[4]; gm.dsdr = rb[5];
    jj = __float_as_int(rb[6]);
  } else {
    gm.x[0] = gm.x[1] = gm.x[2] = 0.f; gm.r = 1.f; gm.s = 0.f; gm.dsdr = 0.f;
  }
  const float sn = gm.s * inv_std, st = (gm.s - mean) * inv_std;
  int idx;
  float x0;
  cmp_locate(st, srmin, delta, ng, idx, x0);
  float u[10], v[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) u[c] = v[c] = 0.f;
  const float4 *cr = reinterpret_cast<const float4 *>(coeff + (size_t)idx * 6 * E2);
#pragma unroll 1
  for (int w4 = 0; w4 < E2 / 4; ++w4) {
    float4 c[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) c[i] = __ldg(cr + i * (E2 / 4) + w4);
    const float cc[6][4] = {{c[0].x, c[0].y, c[0].z, c[0].w}, {c[1].x, c[1].y, c[1].z, c[1].w},
                            {c[2].x, c[2].y, c[2].z, c[2].w}, {c[3].x, c[3].y, c[3].z, c[3].w},
                            {c[4].x, c[4].y, c[4].z, c[4].w}, {c[5].x, c[5].y, c[5].z, c[5].w}};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float h = cc[0][e], dh = 5.f * cc[0][e];
#pragma unroll
      for (int i = 1; i < 5; ++i) {
        h = fmaf(h, x0, cc[i][e]);
        dh = fmaf(dh, x0, (float)(5 - i) * cc[i][e]);
      }
      h = fmaf(h, x0, cc[5][e]);
      const int col = w4 * 4 + e;
#pragma unroll
      for (int ch = 0; ch < 10; ++ch) {
        const float dtc = dT[ch * E2 + col];
        u[ch] = fmaf(dtc, h, u[ch]);
        v[ch] = fmaf(dtc, dh, v[ch]);
      }
    }
  }
  const float inv_rp = 1.f / (gm.r + 1e-16f);
  const float xh[3] = {gm.x[0] * inv_rp, gm.x[1] * inv_rp, gm.x[2] * inv_rp};
  float R[10];
  env_row(sn, xh, R);
  float gst = 0.f;
#pragma unroll
  for (int c = 0; c < 10; ++c) gst = fmaf(R[c], v[c], gst);
  float gx[3];
  row_adjoint(gm, inv_std, u, gst, gx);
  if (act) {
    atomicAdd(&F4[frame_base + jj], make_float4(-gx[0], -gx[1], -gx[2], 0.f));
    fi0 += gx[0]; fi1 += gx[1]; fi2 += gx[2];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int qq = 0; qq < 3; ++qq) vir[p * 3 + qq] -= gm.x[p] * gx[qq];
  }
}

template <int E0, int E1, int E2, bool CMP>
__global__ void __launch_bounds__(256) k_embed_bwd(DevModel M, SysDesc D, int ti, const float *__restrict__ pos,
                                                   const int32_t *__restrict__ perm, const float *__restrict__ box,
                                                   const int32_t *__restrict__ nbrs, const float *__restrict__ Tin,
                                                   const float *__restrict__ dG, float4 *__restrict__ F4,
                                                   double *__restrict__ virial) {
  using ED = EmbedDims<E0, E1, E2>;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int A = M.A;
  float *wsm = smem;
  const int r1 = (A * E2 > 64 * 8 + 2 * E1 * 32) ? A * E2 : 64 * 8 + 2 * E1 * 32;
  const int per_warp = r1 + 10 * E2 + 20 * A;
  float *bufA = smem + (CMP ? 0 : M.ntypes * ED::NW) + warp * per_warp;  // dG, later rows + h1/dh1 staging
  float *bufB = bufA + r1;                                   // X, later dT
  float *Qs = bufB + 10 * E2;                                // 10 x A
  float *dQs = Qs + 10 * A;                                  // 10 x A
  __shared__ double vsm[9];
  if (threadIdx.x < 9) vsm[threadIdx.x] = 0.0;
  if (!CMP) load_nets<E0, E1, E2>(M, ti, wsm);
  __syncthreads();
  const int f = blockIdx.y;
  const int a = blockIdx.x * wpb + warp;
  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  float vir[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vir[k] = 0.f;
  if (a < cnt_i) {
    const int i = D.offs[ti] + a;
    const size_t g = (size_t)f * D.N + i;
    // ---- dE/dT from dE/dG (adjoint of dpmodel.py:74-78)
    for (int e = lane; e < 10 * E2; e += 32) {
      const int c = e / E2, w = e - c * E2;
      bufB[e] = Tin[g * 10 * E2 + e] + (c == 0 ? M.tbias[w] : 0.f);
    }
    for (int e = lane; e < A * E2; e += 32) bufA[e] = dG[g * (size_t)A * E2 + e];
    __syncwarp();
    for (int e = lane; e < 10 * A; e += 32) {
      const int c = e / A, aa = e - c * A;
      float qv;
      if (c < 4) {
        qv = bufB[c * E2 + aa];
      } else {
        const float y1 = bufB[1 * E2 + A + aa], y2 = bufB[2 * E2 + A + aa], y3 = bufB[3 * E2 + A + aa];
        const int m = c - 4;
        const float base[6] = {y1 * y1, y2 * y2, y3 * y3, kSqrt2 * y1 * y3, kSqrt2 * y2 * y1, kSqrt2 * y3 * y2};
        qv = base[m] + bufB[c * E2 + A + aa];
      }
      Qs[e] = qv;
      float dq = 0.f;
      for (int w = 0; w < E2; ++w) dq = fmaf(bufA[aa * E2 + w], bufB[c * E2 + w], dq);
      dQs[e] = dq;
    }
    __syncwarp();
    float dX[ED::NQ][10];
#pragma unroll
    for (int q = 0; q < ED::NQ; ++q) {
      const int col = q * 32 + lane;
#pragma unroll
      for (int c = 0; c < 10; ++c) dX[q][c] = 0.f;
      if (col < E2) {
        for (int aa = 0; aa < A; ++aa) {
          const float dg = bufA[aa * E2 + col];
#pragma unroll
          for (int c = 0; c < 10; ++c) dX[q][c] = fmaf(dg, Qs[c * A + aa], dX[q][c]);
        }
      }
    }
    // row contributions through Q: channels 0..3 at w = a, G2 terms at w = A + a
    if (lane < A) {
#pragma unroll
      for (int c = 0; c < 4; ++c) dX[0][c] += dQs[c * A + lane];
    } else if (lane < 2 * A) {
      const int aa = lane - A;
      float d2[6];
#pragma unroll
      for (int m = 0; m < 6; ++m) d2[m] = dQs[(4 + m) * A + aa];
      const float y1 = bufB[1 * E2 + lane], y2 = bufB[2 * E2 + lane], y3 = bufB[3 * E2 + lane];
#pragma unroll
      for (int m = 0; m < 6; ++m) dX[0][4 + m] += d2[m];
      dX[0][1] += 2.f * y1 * d2[0] + kSqrt2 * y3 * d2[3] + kSqrt2 * y2 * d2[4];
      dX[0][2] += 2.f * y2 * d2[1] + kSqrt2 * y1 * d2[4] + kSqrt2 * y3 * d2[5];
      dX[0][3] += 2.f * y3 * d2[2] + kSqrt2 * y1 * d2[3] + kSqrt2 * y2 * d2[5];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < ED::NQ; ++q) {
      const int col = q * 32 + lane;
      if (col < E2)
#pragma unroll
        for (int c = 0; c < 10; ++c) bufB[c * E2 + col] = dX[q][c] * M.inv_nnbrs;
    }
    __syncwarp();
    // ---- rows: recompute with tangents, scatter forces
    const float3 ri = load_pos(pos, perm, f, i, D.N);
    const int bs = box_slot(D, g, f);
    const float3 L = make_float3(box[bs * 3], box[bs * 3 + 1], box[bs * 3 + 2]);
    const int3 ni = image_range(L, M.rcut);
    const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
    const float inv_std = M.inv_std[ti], mean = M.mean[ti];
    const unsigned lt = (1u << lane) - 1u;
    float *rowbuf = bufA;  // 64 rows x 8 floats
    float *h1s = bufA + 64 * 8, *d1s = h1s + E1 * 32;
    float fi0 = 0.f, fi1 = 0.f, fi2 = 0.f;
    const size_t frame_base = (size_t)f * D.N;
    for (int tj = 0; tj < D.ntypes; ++tj) {
      const float *W = wsm + tj * ED::NW;
      const int32_t *nb = nbrs + g * D.S + D.col[tj];
      const int sel = D.sel[tj], cnt_j = D.offs[tj + 1] - D.offs[tj];
      int nbuf = 0;
      const int total = sel * nim;
      for (int base = 0; base < total; base += 32) {
        const int p = base + lane;
        bool keep = false;
        RowGeom gm;
        int jj = 0;
        if (p < total) {
          const int slot = nim == 1 ? p : p / nim, mimg = p - slot * nim;
          const int idx = nb[slot] & DPB_NBR_INDEX_MASK;
          if (idx < cnt_j) {
            jj = D.offs[tj] + idx;
            const float3 rj = load_pos(pos, perm, f, jj, D.N);
            row_geom(rel_coord(ri, rj, L, ni, mimg), M.rcut, gm);
            keep = gm.s != 0.f;
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          float *dst = rowbuf + (nbuf + __popc(m & lt)) * 8;
          dst[0] = gm.x[0]; dst[1] = gm.x[1]; dst[2] = gm.x[2];
          dst[3] = gm.r; dst[4] = gm.s; dst[5] = gm.dsdr;
          dst[6] = __int_as_float(perm ? perm[jj] : jj);
        }
        nbuf += __popc(m);
        __syncwarp();
        if (nbuf >= 32) {
          if constexpr (CMP)
            embed_rows_bwd_cmp<E2>(M.cmp_coeff[ti * M.ntypes + tj], M.cmp_srmin[ti * M.ntypes + tj],
                                   M.cmp_delta[ti * M.ntypes + tj], M.ngrids, 32, rowbuf, bufB, inv_std, mean,
                                   lane, fi0, fi1, fi2, vir, F4, frame_base);
          else
            embed_rows_bwd<E0, E1, E2>(W, 32, rowbuf, bufB, h1s, d1s, inv_std, mean, lane, fi0, fi1, fi2,
                                       vir, F4, frame_base);
          const int rem = nbuf - 32;
          if (lane < rem)
            for (int c = 0; c < 8; ++c) rowbuf[lane * 8 + c] = rowbuf[(32 + lane) * 8 + c];
          __syncwarp();
          nbuf = rem;
        }
      }
      if (nbuf > 0) {
        if constexpr (CMP)
          embed_rows_bwd_cmp<E2>(M.cmp_coeff[ti * M.ntypes + tj], M.cmp_srmin[ti * M.ntypes + tj],
                                 M.cmp_delta[ti * M.ntypes + tj], M.ngrids, nbuf, rowbuf, bufB, inv_std, mean,
                                 lane, fi0, fi1, fi2, vir, F4, frame_base);
        else
          embed_rows_bwd<E0, E1, E2>(W, nbuf, rowbuf, bufB, h1s, d1s, inv_std, mean, lane, fi0, fi1, fi2,
                                     vir, F4, frame_base);
      }
      __syncwarp();
    }
    fi0 = warp_sum(fi0); fi1 = warp_sum(fi1); fi2 = warp_sum(fi2);
    if (lane == 0) atomicAdd(&F4[frame_base + (perm ? perm[i] : i)], make_float4(fi0, fi1, fi2, 0.f));
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    float s = warp_sum(vir[k]);
    if (lane == 0 && s != 0.f) atomicAdd(&vsm[k], (double)s);
  }
  __syncthreads();
  // the block's 8 atoms share one frame (segment-aligned in packed batches)
  if (threadIdx.x < 9) {
    const int vs = box_slot(D, (size_t)f * D.N + D.offs[ti] + blockIdx.x * wpb, f);
    atomicAdd(&virial[vs * 9 + threadIdx.x], vsm[threadIdx.x]);
  }
}

// ---------------------------------------------------------------- fitting (SGEMM chain)
constexpr int GB_M = 64, GB_N = 64, GB_K = 16;

__global__ void __launch_bounds__(256) k_sgemm(int Mrows, int Nc, int K, const float *__restrict__ A, int lda,
                                               RowMap rm, const float *__restrict__ B, Epi ep) {
  __shared__ float As[GB_K][GB_M + 4];
  __shared__ __align__(16) float Bs[GB_K][GB_N];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
  float acc[4][4] = {};
  // A tile loader: 64 rows x 16 k, one float4 (4 k) per thread
  const int la_r = tid >> 2, la_k = (tid & 3) * 4;
  const int ar = m0 + la_r;
  const float *Arow = ar < Mrows ? A + rm.atom(ar) * (size_t)lda : nullptr;
  // B tile loader: 16 k x 64 n, one float4 (4 n) per thread
  const int lb_k = tid >> 4, lb_n = (tid & 15) * 4;
  for (int k0 = 0; k0 < K; k0 += GB_K) {
    float4 av = make_float4(0.f, 0.f, 0.f, 0.f);
    if (Arow) {
      const int kk = k0 + la_k;
      if (kk + 3 < K) av = *reinterpret_cast<const float4 *>(Arow + kk);
      else {
        float t[4] = {0.f, 0.f, 0.f, 0.f};
        for (int u = 0; u < 4; ++u) if (kk + u < K) t[u] = Arow[kk + u];
        av = make_float4(t[0], t[1], t[2], t[3]);
      }
    }
    As[la_k + 0][la_r] = av.x; As[la_k + 1][la_r] = av.y;
    As[la_k + 2][la_r] = av.z; As[la_k + 3][la_r] = av.w;
    {
      const int kk = k0 + lb_k, nn = n0 + lb_n;
      float t[4] = {0.f, 0.f, 0.f, 0.f};
      if (kk < K) {
        if (nn + 3 < Nc && ((Nc & 3) == 0)) {
          float4 bv = *reinterpret_cast<const float4 *>(B + (size_t)kk * Nc + nn);
          t[0] = bv.x; t[1] = bv.y; t[2] = bv.z; t[3] = bv.w;
        } else {
          for (int u = 0; u < 4; ++u) if (nn + u < Nc) t[u] = B[(size_t)kk * Nc + nn + u];
        }
      }
      *reinterpret_cast<float4 *>(&Bs[lb_k][lb_n]) = make_float4(t[0], t[1], t[2], t[3]);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GB_K; ++k) {
      float a4[4], b4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a4[u] = As[k][ty * 4 + u];
      const float4 bv = *reinterpret_cast<const float4 *>(&Bs[k][tx * 4]);
      b4[0] = bv.x; b4[1] = bv.y; b4[2] = bv.z; b4[3] = bv.w;
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a4[u], b4[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int r = m0 + ty * 4 + u;
    if (r >= Mrows) continue;
    const size_t at = rm.atom(r) * (size_t)ep.ld;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int n = n0 + tx * 4 + v;
      if (n >= Nc) continue;
      const float x = acc[u][v];
      switch (ep.mode) {
        case EPI_STORE: ep.out1[at + n] = x; break;
        case EPI_TANH: {
          const float t = tanhf(x + ep.bias[n]);
          ep.out1[at + n] = t;
          if (ep.out2) ep.out2[at + n] = t;
          break;
        }
        case EPI_TANH_RES: {
          const float t = tanhf(x + ep.bias[n]);
          ep.out1[at + n] = t;
          ep.out2[at + n] = t * ep.dt[n] + ep.hprev[at + n];
          break;
        }
        case EPI_GRAD_RES: {
          const float gh = x + (ep.gvec ? ep.gvec[n] : ep.gmat[at + n]);
          const float t = ep.tin[at + n];
          ep.out2[at + n] = gh;
          ep.out1[at + n] = gh * ep.dt[n] * (1.f - t * t);
          break;
        }
        case EPI_GRAD: {
          const float gh = x + (ep.gvec ? ep.gvec[n] : (ep.gmat ? ep.gmat[at + n] : 0.f));
          const float t = ep.tin[at + n];
          ep.out1[at + n] = gh * (1.f - t * t);
          break;
        }
      }
    }
  }
}

// Per-atom energy E = H . w + b' and the first adjoint gZ of the last hidden
// layer (64 atoms per block); per-frame energies reduced in FP64, one atomic
// per (block, frame).
__global__ void __launch_bounds__(256) k_fit_energy(int Mrows, RowMap rm, int FWl, const float *__restrict__ H,
                                                    const float *__restrict__ tl, const float *__restrict__ wfin,
                                                    const float *__restrict__ bfin, const float *__restrict__ dtl,
                                                    float *__restrict__ Eatom, float *__restrict__ gZ,
                                                    double *__restrict__ energy, int N,
                                                    const int32_t *__restrict__ seg) {
  __shared__ double es[64];
  __shared__ int fs[64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = 0; k < 8; ++k) {
    const int slot = warp * 8 + k;
    const int r = blockIdx.x * 64 + slot;
    if (r >= Mrows) {
      if (lane == 0) { es[slot] = 0.0; fs[slot] = -1; }
      continue;
    }
    const size_t at = rm.atom(r);
    float s = 0.f;
    for (int n = lane; n < FWl; n += 32) {
      s = fmaf(H[at * FWl + n], wfin[n], s);
      const float t = tl[at * FWl + n];
      gZ[at * FWl + n] = wfin[n] * (dtl ? dtl[n] : 1.f) * (1.f - t * t);
    }
    s = warp_sum(s) + bfin[0];
    if (lane == 0) {
      Eatom[at] = s;
      es[slot] = (double)s;
      fs[slot] = energy_slot(seg, at, N);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0.0;
    int cf = fs[0];
    for (int k = 0; k < 64; ++k) {
      if (fs[k] != cf) {
        if (cf >= 0) atomicAdd(&energy[cf], run);
        run = 0.0;
        cf = fs[k];
      }
      run += es[k];
    }
    if (cf >= 0) atomicAdd(&energy[cf], run);
  }
}

// Forces (float4 accumulator) and per-atom energies to the caller's layout;
// non-finite positions or results raise status bit 16 and, as NaN inputs do
// in the reference's float arithmetic, make the frame's energy NaN.
__global__ void k_finalize(int NF, int N, const float4 *__restrict__ F4, float *__restrict__ force,
                           const float *__restrict__ Eatom_sorted, const int32_t *__restrict__ perm,
                           float *__restrict__ atom_energy, double *__restrict__ energy, int nE,
                           const float *__restrict__ pos, const int32_t *__restrict__ seg,
                           uint32_t *__restrict__ status) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < NF) {
    const float4 v = F4[g];
    force[(size_t)g * 3 + 0] = v.x;
    force[(size_t)g * 3 + 1] = v.y;
    force[(size_t)g * 3 + 2] = v.z;
    const int f = g / N, k = g - f * N;
    const int dst = perm ? perm[k] : k;
    if (atom_energy) atom_energy[(size_t)f * N + dst] = Eatom_sorted[g];
    const float *p = pos + ((size_t)f * N + dst) * 3;  // position of sorted atom g
    const bool bad_in = !isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]);
    if (bad_in || !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) atomicOr(status, DPB_ST_NONFINITE);
    const int e = energy_slot(seg, g, N);
    if (bad_in && e >= 0) energy[e] = __longlong_as_double(0x7ff8000000000000LL);
  }
  if (g < nE && !isfinite(energy[g])) atomicOr(status, DPB_ST_NONFINITE);
}

// Explicit instantiation helpers used by the C ABI dispatch.
template <int E0, int E1, int E2>
size_t embed_fwd_smem(int ntypes) {
  return (size_t)(ntypes * EmbedDims<E0, E1, E2>::NW + 8 * embed_fwd_warp_floats<E0, E1, E2>()) * sizeof(float);
}
template <int E0, int E1, int E2>
size_t embed_bwd_smem(int ntypes, int A) {
  const int r1 = (A * E2 > 64 * 8 + 2 * E1 * 32) ? A * E2 : 64 * 8 + 2 * E1 * 32;
  return (size_t)(ntypes * EmbedDims<E0, E1, E2>::NW + 8 * (r1 + 10 * E2 + 20 * A)) * sizeof(float);
}

template <int E0, int E1, int E2>
int launch_embed_fwd(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                     const float *box, const int32_t *nbrs, float *T, float *G, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  dim3 grid((cnt + 7) / 8, D.F);
  if (M.ngrids > 0) {
    size_t smem = embed_fwd_smem<E0, E1, E2>(0);
    cudaFuncSetAttribute(k_embed_fwd<E0, E1, E2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_embed_fwd<E0, E1, E2, true><<<grid, 256, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, G);
  } else {
    size_t smem = embed_fwd_smem<E0, E1, E2>(M.ntypes);
    cudaFuncSetAttribute(k_embed_fwd<E0, E1, E2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_embed_fwd<E0, E1, E2, false><<<grid, 256, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, G);
  }
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

template <int E0, int E1, int E2>
int launch_embed_bwd(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                     const float *box, const int32_t *nbrs, const float *T, const float *dG, float4 *F4,
                     double *virial, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  dim3 grid((cnt + 7) / 8, D.F);
  if (M.ngrids > 0) {
    size_t smem = embed_bwd_smem<E0, E1, E2>(0, M.A);
    cudaFuncSetAttribute(k_embed_bwd<E0, E1, E2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_embed_bwd<E0, E1, E2, true><<<grid, 256, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, dG, F4, virial);
  } else {
    size_t smem = embed_bwd_smem<E0, E1, E2>(M.ntypes, M.A);
    cudaFuncSetAttribute(k_embed_bwd<E0, E1, E2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_embed_bwd<E0, E1, E2, false><<<grid, 256, smem, st>>>(M, D, ti, pos, perm, box, nbrs, T, dG, F4, virial);
  }
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

template int launch_embed_fwd<25, 50, 100>(const DevModel &, const SysDesc &, int, const float *, const int32_t *,
                                           const float *, const int32_t *, float *, float *, cudaStream_t);
template int launch_embed_bwd<25, 50, 100>(const DevModel &, const SysDesc &, int, const float *, const int32_t *,
                                           const float *, const int32_t *, const float *, const float *, float4 *,
                                           double *, cudaStream_t);
template int launch_embed_fwd<32, 32, 64>(const DevModel &, const SysDesc &, int, const float *, const int32_t *,
                                          const float *, const int32_t *, float *, float *, cudaStream_t);
template int launch_embed_bwd<32, 32, 64>(const DevModel &, const SysDesc &, int, const float *, const int32_t *,
                                          const float *, const int32_t *, const float *, const float *, float4 *,
                                          double *, cudaStream_t);

int launch_sgemm(int Mrows, int Nc, int K, const float *A, int lda, RowMap rm, const float *B, const Epi &ep,
                 cudaStream_t st) {
  if (Mrows == 0) return DPB_OK;
  dim3 grid((Nc + GB_N - 1) / GB_N, (Mrows + GB_M - 1) / GB_M);
  k_sgemm<<<grid, 256, 0, st>>>(Mrows, Nc, K, A, lda, rm, B, ep);
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

int launch_fit_energy(int Mrows, RowMap rm, int FWl, const float *H, const float *tl, const float *wfin,
                      const float *bfin, const float *dtl, float *Eatom, float *gZ, double *energy, int N,
                      const int32_t *seg, cudaStream_t st) {
  if (Mrows == 0) return DPB_OK;
  k_fit_energy<<<(Mrows + 63) / 64, 256, 0, st>>>(Mrows, rm, FWl, H, tl, wfin, bfin, dtl, Eatom, gZ, energy, N,
                                                  seg);
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

int launch_finalize(int NF, int N, const float4 *F4, float *force, const float *Eatom, const int32_t *perm,
                    float *atom_energy, double *energy, int nE, const float *pos, const int32_t *seg,
                    uint32_t *status, cudaStream_t st) {
  int n = NF > nE ? NF : nE;
  k_finalize<<<(n + 255) / 256, 256, 0, st>>>(NF, N, F4, force, Eatom, perm, atom_energy, energy, nE, pos, seg,
                                              status);
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

}  // namespace dpb
