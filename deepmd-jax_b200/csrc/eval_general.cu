// FP32 embedding kernels for any embedding-net shape the reference builds
// (deepmd_jax/utils.py:100-151): 1 to 4 layers of any widths whose ratios
// are integers either way (a wider layer adds repeat(x, Z), a narrower one
// the mean over the Z groups of its input, utils.py:116-124), compressed
// tables of any width.  Shapes with a tuned instantiation (25-50-100,
// 32-32-64) take eval_fp32.cu; every other shape takes these kernels.
//
// Same structure as eval_fp32.cu (warp per centre atom, rows compacted 32 at a
// time, row = lane): here every layer width is a runtime value, hidden-layer
// activations are staged per lane in shared memory ([column][lane]) and each
// layer is computed 32 (forward) or 16 (adjoint) output columns at a time, so
// no register array is indexed by a runtime value.  The adjoint recomputes
// the rows with their tangent along s~ (forward mode), as the tuned kernels do.
#include "eval_common.cuh"
#include "internal.cuh"

namespace dpb {

// Layout of one net's weights in shared memory: layer l's kernel (in x out,
// in = 1 for layer 0) at ow[l], its bias at ob[l].
struct GenNet {
  int L;
  int w[kMaxEmbedLayers];
  int E;   // output width
  int HM;  // widest hidden layer (layers 0 .. L-2), 0 for one layer
  int NW;  // floats per net
  int ow[kMaxEmbedLayers], ob[kMaxEmbedLayers];
};

GenNet gen_net(const DevModel &M) {
  GenNet G{};
  G.L = M.nemb;
  int o = 0, in = 1;
  for (int l = 0; l < G.L; ++l) {
    G.w[l] = M.EW[l];
    G.ow[l] = o;
    o += in * G.w[l];
    G.ob[l] = o;
    o += G.w[l];
    in = G.w[l];
    if (l < G.L - 1 && G.w[l] > G.HM) G.HM = G.w[l];
  }
  G.E = G.w[G.L - 1];
  G.NW = o;
  return G;
}

__device__ __forceinline__ float3 gen_load_pos(const float *__restrict__ pos, const int32_t *__restrict__ perm, int f,
                                               int k, int N) {
  const int src = perm ? perm[k] : k;
  const float *p = pos + ((size_t)f * N + src) * 3;
  return make_float3(p[0], p[1], p[2]);
}

// Residual source of output column col of a layer in -> out, from the input
// staged as hin[k * 32 + lane]: repeat(x, out / in) when the layer widens,
// the mean over the in / out groups x[g * out + col] when it narrows.
__device__ __forceinline__ float gen_res(const float *__restrict__ hin, int in, int out, int col, int lane) {
  if (out >= in) return hin[(col / (out / in)) * 32 + lane];
  const int ng = in / out;
  float s = 0.f;
  for (int g = 0; g < ng; ++g) s += hin[(g * out + col) * 32 + lane];
  return s / (float)ng;
}

__device__ void gen_load_nets(const DevModel &M, const GenNet &G, int ti, float *wsm) {
  for (int tj = 0; tj < M.ntypes; ++tj) {
    const int k = ti * M.ntypes + tj;
    float *w = wsm + tj * G.NW;
    int in = 1;
    for (int l = 0; l < G.L; ++l) {
      for (int e = threadIdx.x; e < in * G.w[l]; e += blockDim.x) w[G.ow[l] + e] = M.ew[k][l][e];
      for (int e = threadIdx.x; e < G.w[l]; e += blockDim.x) w[G.ob[l] + e] = M.eb[k][l][e];
      in = G.w[l];
    }
  }
}

// layer 0 and the hidden layers 1 .. L-2 of the forward for the round's rows;
// returns the buffer that holds layer L-2
__device__ float *gen_hidden_fwd(const GenNet &G, const float *__restrict__ W, float st, float *hA, float *hB,
                                 int lane) {
  const float *w0 = W + G.ow[0], *b0 = W + G.ob[0];
  for (int k = 0; k < G.w[0]; ++k) hA[k * 32 + lane] = tanhf(fmaf(st, w0[k], b0[k]));
  float *cur = hA, *nxt = hB;
  for (int l = 1; l < G.L - 1; ++l) {
    const int in = G.w[l - 1], out = G.w[l];
    const float *wl = W + G.ow[l], *bl = W + G.ob[l];
    for (int q = 0; q < (out + 31) / 32; ++q) {
      float acc[32];
#pragma unroll
      for (int o = 0; o < 32; ++o) acc[o] = (q * 32 + o < out) ? bl[q * 32 + o] : 0.f;
      for (int k = 0; k < in; ++k) {
        const float hv = cur[k * 32 + lane];
        const float *wr = wl + k * out + q * 32;
#pragma unroll
        for (int o = 0; o < 32; ++o)
          if (q * 32 + o < out) acc[o] = fmaf(hv, wr[o], acc[o]);
      }
#pragma unroll
      for (int o = 0; o < 32; ++o) {
        const int col = q * 32 + o;
        if (col < out) nxt[col * 32 + lane] = tanhf(acc[o]) + gen_res(cur, in, out, col, lane);
      }
    }
    float *t = cur;
    cur = nxt;
    nxt = t;
  }
  return cur;
}

// One round of up to 32 compacted rows: the net, then T += R~^T h.
__device__ void gen_rows_fwd(const GenNet &G, const float *__restrict__ W, int n, const float *__restrict__ rowbuf,
                             float *hA, float *hB, float *h2s, float *Ts, int lane) {
  const float st = lane < n ? rowbuf[lane * 12] : 0.f;
  const float *cur = G.L > 1 ? gen_hidden_fwd(G, W, st, hA, hB, lane) : nullptr;
  const int E = G.E, in = G.L > 1 ? G.w[G.L - 2] : 1;
  const float *wl = W + G.ow[G.L - 1], *bl = W + G.ob[G.L - 1];
  __syncwarp();
  for (int q = 0; q < (E + 31) / 32; ++q) {
    if (G.L == 1) {
#pragma unroll
      for (int o = 0; o < 32; ++o) {
        const int col = q * 32 + o;
        if (col < E) h2s[lane * 33 + o] = tanhf(fmaf(st, wl[col], bl[col]));
      }
    } else {
      float acc[32];
#pragma unroll
      for (int o = 0; o < 32; ++o) acc[o] = (q * 32 + o < E) ? bl[q * 32 + o] : 0.f;
      for (int k = 0; k < in; ++k) {
        const float hv = cur[k * 32 + lane];
        const float *wr = wl + k * E + q * 32;
#pragma unroll
        for (int o = 0; o < 32; ++o)
          if (q * 32 + o < E) acc[o] = fmaf(hv, wr[o], acc[o]);
      }
#pragma unroll
      for (int o = 0; o < 32; ++o) {
        const int col = q * 32 + o;
        if (col < E) h2s[lane * 33 + o] = tanhf(acc[o]) + gen_res(cur, in, E, col, lane);
      }
    }
    __syncwarp();
    const int col = q * 32 + lane;
    if (col < E) {
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
      for (int c = 0; c < 10; ++c) Ts[c * E + col] += Tq[c];
    }
    __syncwarp();
  }
}

// The compressed net's table lookup (deepmd_jax/utils.py:126-151) for a round
// of rows, lane = column, any width E.
__device__ __forceinline__ void gen_locate(float st, float srmin, float delta, int ng, int &idx, float &x0) {
  const float x = __fsub_rn(st, srmin);
  const int k = (int)__fdiv_rn(x, delta);
  x0 = __fsub_rn(x, __fmul_rn((float)k, delta));
  idx = k < 0 ? 0 : (k >= ng ? ng - 1 : k);
}

__device__ void gen_rows_fwd_cmp(const float *__restrict__ coeff, float srmin, float delta, int ng, int E, int n,
                                 float *__restrict__ rowbuf, float *__restrict__ Ts, int lane) {
  if (lane < n) {
    int idx;
    float x0;
    gen_locate(rowbuf[lane * 12], srmin, delta, ng, idx, x0);
    rowbuf[lane * 12] = x0;
    rowbuf[lane * 12 + 11] = __int_as_float(idx);
  }
  __syncwarp();
  for (int q = 0; q < (E + 31) / 32; ++q) {
    const int col = q * 32 + lane;
    if (col < E) {
      float Tq[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) Tq[c] = 0.f;
      for (int r = 0; r < n; ++r) {
        const float *rb = rowbuf + r * 12;
        const float x0 = rb[0];
        const float *cr = coeff + (size_t)__float_as_int(rb[11]) * 6 * E + col;
        float h = __ldg(cr);
#pragma unroll
        for (int i = 1; i < 6; ++i) h = fmaf(h, x0, __ldg(cr + i * E));
#pragma unroll
        for (int c = 0; c < 10; ++c) Tq[c] = fmaf(rb[1 + c], h, Tq[c]);
      }
#pragma unroll
      for (int c = 0; c < 10; ++c) Ts[c * E + col] += Tq[c];
    }
  }
  __syncwarp();
}

// per-warp shared floats of the forward kernel
__host__ __device__ inline int gen_fwd_warp_floats(const GenNet &G) { return 64 * 12 + 2 * G.HM * 32 + 32 * 33 + 10 * G.E; }

template <bool CMP>
__global__ void __launch_bounds__(256) k_embed_fwd_gen(DevModel M, GenNet G, SysDesc D, int ti,
                                                       const float *__restrict__ pos, const int32_t *__restrict__ perm,
                                                       const float *__restrict__ box, const int32_t *__restrict__ nbrs,
                                                       float *__restrict__ Tout, float *__restrict__ Gout) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  float *wsm = smem;
  float *rowbuf = smem + (CMP ? 0 : M.ntypes * G.NW) + warp * gen_fwd_warp_floats(G);
  float *hA = rowbuf + 64 * 12, *hB = hA + G.HM * 32, *h2s = hB + G.HM * 32, *Ts = h2s + 32 * 33;
  const int E = G.E;
  if (!CMP) gen_load_nets(M, G, ti, wsm);
  __syncthreads();
  const int f = blockIdx.y;
  const int a = blockIdx.x * wpb + warp;
  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  if (a >= cnt_i) return;
  const int i = D.offs[ti] + a;
  const size_t g = (size_t)f * D.N + i;
  const float3 ri = gen_load_pos(pos, perm, f, i, D.N);
  const int bs = box_slot(D, g, f);
  const float3 L = make_float3(box[bs * 3], box[bs * 3 + 1], box[bs * 3 + 2]);
  const int3 ni = image_range(L, M.rcut);
  const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
  const float inv_std = M.inv_std[ti], mean = M.mean[ti];
  const unsigned lt = (1u << lane) - 1u;
  for (int e = lane; e < 10 * E; e += 32) Ts[e] = 0.f;
  __syncwarp();
  for (int tj = 0; tj < D.ntypes; ++tj) {
    const float *W = wsm + tj * G.NW;
    const int knet = ti * M.ntypes + tj;
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
          const float3 rj = gen_load_pos(pos, perm, f, D.offs[tj] + idx, D.N);
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
        if (CMP)
          gen_rows_fwd_cmp(M.cmp_coeff[knet], M.cmp_srmin[knet], M.cmp_delta[knet], M.ngrids, E, 32, rowbuf, Ts,
                           lane);
        else
          gen_rows_fwd(G, W, 32, rowbuf, hA, hB, h2s, Ts, lane);
        const int rem = nbuf - 32;
        if (lane < rem)
          for (int c = 0; c < 12; ++c) rowbuf[lane * 12 + c] = rowbuf[(32 + lane) * 12 + c];
        __syncwarp();
        nbuf = rem;
      }
    }
    if (nbuf > 0) {
      if (CMP)
        gen_rows_fwd_cmp(M.cmp_coeff[knet], M.cmp_srmin[knet], M.cmp_delta[knet], M.ngrids, E, nbuf, rowbuf, Ts,
                         lane);
      else
        gen_rows_fwd(G, W, nbuf, rowbuf, hA, hB, h2s, Ts, lane);
    }
    __syncwarp();
  }
  // T = sum / Nnbrs (written out); Ts becomes X = T with Tbias on channel 0
  for (int e = lane; e < 10 * E; e += 32) {
    const float t = Ts[e] * M.inv_nnbrs;
    Tout[g * 10 * E + e] = t;
    Ts[e] = t + (e < E ? M.tbias[e] : 0.f);
  }
  __syncwarp();
  // G[a][w] = sum_c Q[c][a] X[c][w] (dpmodel.py:74-78)
  const int A = M.A;
  float *Gg = Gout + g * (size_t)A * E;
  for (int aa = 0; aa < A; ++aa) {
    float Q[10];
#pragma unroll
    for (int c = 0; c < 4; ++c) Q[c] = Ts[c * E + aa];
    const float y1 = Ts[1 * E + A + aa], y2 = Ts[2 * E + A + aa], y3 = Ts[3 * E + A + aa];
    Q[4] = y1 * y1 + Ts[4 * E + A + aa];
    Q[5] = y2 * y2 + Ts[5 * E + A + aa];
    Q[6] = y3 * y3 + Ts[6 * E + A + aa];
    Q[7] = kSqrt2 * y1 * y3 + Ts[7 * E + A + aa];
    Q[8] = kSqrt2 * y2 * y1 + Ts[8 * E + A + aa];
    Q[9] = kSqrt2 * y3 * y2 + Ts[9 * E + A + aa];
    for (int col = lane; col < E; col += 32) {
      float v = 0.f;
#pragma unroll
      for (int c = 0; c < 10; ++c) v = fmaf(Q[c], Ts[c * E + col], v);
      Gg[aa * E + col] = v;
    }
  }
}

// ---------------------------------------------------------------- adjoint
struct RowOut {
  float fi0, fi1, fi2;
  float vir[9];
};

__device__ __forceinline__ void gen_row_finish(const RowGeom &gm, bool act, int jj, float inv_std, const float u[10],
                                               const float v[10], RowOut &ro, float4 *__restrict__ F4,
                                               size_t frame_base) {
  const float sn = gm.s * inv_std;
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
    ro.fi0 += gx[0];
    ro.fi1 += gx[1];
    ro.fi2 += gx[2];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int qq = 0; qq < 3; ++qq) ro.vir[p * 3 + qq] -= gm.x[p] * gx[qq];
  }
}

__device__ __forceinline__ void gen_row_geom(const float *rowbuf, bool act, int lane, RowGeom &gm, int &jj) {
  jj = 0;
  if (act) {
    const float *rb = rowbuf + lane * 8;
    gm.x[0] = rb[0]; gm.x[1] = rb[1]; gm.x[2] = rb[2];
    gm.r = rb[3]; gm.s = rb[4]; gm.dsdr = rb[5];
    jj = __float_as_int(rb[6]);
  } else {
    gm.x[0] = gm.x[1] = gm.x[2] = 0.f; gm.r = 1.f; gm.s = 0.f; gm.dsdr = 0.f;
  }
}

// Adjoint of one round of rows: the net recomputed with tangents along s~,
// u = dT.h, v = dT.dh at the output, then the row adjoint.
__device__ void gen_rows_bwd(const GenNet &G, const float *__restrict__ W, int n, const float *__restrict__ rowbuf,
                             const float *__restrict__ dT, float *hA, float *dA, float *hB, float *dB, float inv_std,
                             float mean, int lane, RowOut &ro, float4 *__restrict__ F4, size_t frame_base) {
  const bool act = lane < n;
  RowGeom gm;
  int jj;
  gen_row_geom(rowbuf, act, lane, gm, jj);
  const float st = (gm.s - mean) * inv_std;
  const float *w0 = W + G.ow[0], *b0 = W + G.ob[0];
  float *hc = hA, *dc = dA, *hn = hB, *dn = dB;
  if (G.L > 1) {
    for (int k = 0; k < G.w[0]; ++k) {
      const float t = tanhf(fmaf(st, w0[k], b0[k]));
      hc[k * 32 + lane] = t;
      dc[k * 32 + lane] = (1.f - t * t) * w0[k];
    }
  }
  for (int l = 1; l < G.L - 1; ++l) {
    const int in = G.w[l - 1], out = G.w[l];
    const float *wl = W + G.ow[l], *bl = W + G.ob[l];
    for (int q = 0; q < (out + 15) / 16; ++q) {
      float z[16], dz[16];
#pragma unroll
      for (int o = 0; o < 16; ++o) {
        z[o] = (q * 16 + o < out) ? bl[q * 16 + o] : 0.f;
        dz[o] = 0.f;
      }
      for (int k = 0; k < in; ++k) {
        const float hv = hc[k * 32 + lane], dv = dc[k * 32 + lane];
        const float *wr = wl + k * out + q * 16;
#pragma unroll
        for (int o = 0; o < 16; ++o)
          if (q * 16 + o < out) {
            z[o] = fmaf(hv, wr[o], z[o]);
            dz[o] = fmaf(dv, wr[o], dz[o]);
          }
      }
#pragma unroll
      for (int o = 0; o < 16; ++o) {
        const int col = q * 16 + o;
        if (col < out) {
          const float t = tanhf(z[o]);
          hn[col * 32 + lane] = t + gen_res(hc, in, out, col, lane);
          dn[col * 32 + lane] = (1.f - t * t) * dz[o] + gen_res(dc, in, out, col, lane);
        }
      }
    }
    float *t = hc; hc = hn; hn = t;
    t = dc; dc = dn; dn = t;
  }
  __syncwarp();
  float u[10], v[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) u[c] = v[c] = 0.f;
  const int E = G.E, in = G.L > 1 ? G.w[G.L - 2] : 1;
  const float *wl = W + G.ow[G.L - 1], *bl = W + G.ob[G.L - 1];
  for (int q = 0; q < (E + 15) / 16; ++q) {
    float z[16], dz[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      const int col = q * 16 + o;
      z[o] = (col < E) ? (G.L == 1 ? fmaf(st, wl[col], bl[col]) : bl[col]) : 0.f;
      dz[o] = (col < E && G.L == 1) ? wl[col] : 0.f;
    }
    if (G.L > 1) {
      for (int k = 0; k < in; ++k) {
        const float hv = hc[k * 32 + lane], dv = dc[k * 32 + lane];
        const float *wr = wl + k * E + q * 16;
#pragma unroll
        for (int o = 0; o < 16; ++o)
          if (q * 16 + o < E) {
            z[o] = fmaf(hv, wr[o], z[o]);
            dz[o] = fmaf(dv, wr[o], dz[o]);
          }
      }
    }
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      const int col = q * 16 + o;
      if (col < E) {
        const float t = tanhf(z[o]);
        const float h = t + (G.L > 1 ? gen_res(hc, in, E, col, lane) : 0.f);
        const float dh = (1.f - t * t) * dz[o] + (G.L > 1 ? gen_res(dc, in, E, col, lane) : 0.f);
#pragma unroll
        for (int c = 0; c < 10; ++c) {
          const float dtc = dT[c * E + col];
          u[c] = fmaf(dtc, h, u[c]);
          v[c] = fmaf(dtc, dh, v[c]);
        }
      }
    }
  }
  __syncwarp();
  gen_row_finish(gm, act, jj, inv_std, u, v, ro, F4, frame_base);
}

__device__ void gen_rows_bwd_cmp(const float *__restrict__ coeff, float srmin, float delta, int ng, int E, int n,
                                 const float *__restrict__ rowbuf, const float *__restrict__ dT, float inv_std,
                                 float mean, int lane, RowOut &ro, float4 *__restrict__ F4, size_t frame_base) {
  const bool act = lane < n;
  RowGeom gm;
  int jj;
  gen_row_geom(rowbuf, act, lane, gm, jj);
  const float st = (gm.s - mean) * inv_std;
  int idx;
  float x0;
  gen_locate(st, srmin, delta, ng, idx, x0);
  float u[10], v[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) u[c] = v[c] = 0.f;
  const float *cr = coeff + (size_t)idx * 6 * E;
  for (int col = 0; col < E; ++col) {
    float cc[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) cc[i] = __ldg(cr + i * E + col);
    float h = cc[0], dh = 5.f * cc[0];
#pragma unroll
    for (int i = 1; i < 5; ++i) {
      h = fmaf(h, x0, cc[i]);
      dh = fmaf(dh, x0, (float)(5 - i) * cc[i]);
    }
    h = fmaf(h, x0, cc[5]);
#pragma unroll
    for (int c = 0; c < 10; ++c) {
      const float dtc = dT[c * E + col];
      u[c] = fmaf(dtc, h, u[c]);
      v[c] = fmaf(dtc, dh, v[c]);
    }
  }
  gen_row_finish(gm, act, jj, inv_std, u, v, ro, F4, frame_base);
}

// per-warp shared floats of the adjoint kernel: r1 holds dE/dG, later the row
// buffer and the four staging buffers; then X (later dE/dT), Q and dQ
__host__ __device__ inline int gen_bwd_r1(const GenNet &G, int A) {
  const int rows = 64 * 8 + 4 * G.HM * 32;
  return A * G.E > rows ? A * G.E : rows;
}
__host__ __device__ inline int gen_bwd_warp_floats(const GenNet &G, int A) {
  return gen_bwd_r1(G, A) + 10 * G.E + 20 * A;
}

template <bool CMP>
__global__ void __launch_bounds__(256) k_embed_bwd_gen(DevModel M, GenNet G, SysDesc D, int ti,
                                                       const float *__restrict__ pos, const int32_t *__restrict__ perm,
                                                       const float *__restrict__ box, const int32_t *__restrict__ nbrs,
                                                       const float *__restrict__ Tin, const float *__restrict__ dG,
                                                       float4 *__restrict__ F4, double *__restrict__ virial) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int A = M.A, E = G.E;
  float *wsm = smem;
  float *bufA = smem + (CMP ? 0 : M.ntypes * G.NW) + warp * gen_bwd_warp_floats(G, A);
  float *bufB = bufA + gen_bwd_r1(G, A);  // X, later dE/dT
  float *Qs = bufB + 10 * E, *dQs = Qs + 10 * A;
  __shared__ double vsm[9];
  if (threadIdx.x < 9) vsm[threadIdx.x] = 0.0;
  if (!CMP) gen_load_nets(M, G, ti, wsm);
  __syncthreads();
  const int f = blockIdx.y;
  const int a = blockIdx.x * wpb + warp;
  const int cnt_i = D.offs[ti + 1] - D.offs[ti];
  RowOut ro{};
  if (a < cnt_i) {
    const int i = D.offs[ti] + a;
    const size_t g = (size_t)f * D.N + i;
    // ---- dE/dT from dE/dG (adjoint of dpmodel.py:74-78)
    for (int e = lane; e < 10 * E; e += 32) {
      const int c = e / E, w = e - c * E;
      bufB[e] = Tin[g * 10 * E + e] + (c == 0 ? M.tbias[w] : 0.f);
    }
    for (int e = lane; e < A * E; e += 32) bufA[e] = dG[g * (size_t)A * E + e];
    __syncwarp();
    for (int e = lane; e < 10 * A; e += 32) {
      const int c = e / A, aa = e - c * A;
      float qv;
      if (c < 4) {
        qv = bufB[c * E + aa];
      } else {
        const float y1 = bufB[1 * E + A + aa], y2 = bufB[2 * E + A + aa], y3 = bufB[3 * E + A + aa];
        const float base[6] = {y1 * y1, y2 * y2, y3 * y3, kSqrt2 * y1 * y3, kSqrt2 * y2 * y1, kSqrt2 * y3 * y2};
        qv = base[c - 4] + bufB[c * E + A + aa];
      }
      Qs[e] = qv;
      float dq = 0.f;
      for (int w = 0; w < E; ++w) dq = fmaf(bufA[aa * E + w], bufB[c * E + w], dq);
      dQs[e] = dq;
    }
    __syncwarp();
    // dX for columns q*32 + lane; the Q -> X terms live at columns < 2A <= 32
    // (chunk 0), read before the lane overwrites its own X column
    for (int q = 0; q < (E + 31) / 32; ++q) {
      const int col = q * 32 + lane;
      float dX[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) dX[c] = 0.f;
      if (col < E)
        for (int aa = 0; aa < A; ++aa) {
          const float dg = bufA[aa * E + col];
#pragma unroll
          for (int c = 0; c < 10; ++c) dX[c] = fmaf(dg, Qs[c * A + aa], dX[c]);
        }
      if (q == 0) {
        if (lane < A) {
#pragma unroll
          for (int c = 0; c < 4; ++c) dX[c] += dQs[c * A + lane];
        } else if (lane < 2 * A) {
          const int aa = lane - A;
          float d2[6];
#pragma unroll
          for (int m = 0; m < 6; ++m) d2[m] = dQs[(4 + m) * A + aa];
          const float y1 = bufB[1 * E + lane], y2 = bufB[2 * E + lane], y3 = bufB[3 * E + lane];
#pragma unroll
          for (int m = 0; m < 6; ++m) dX[4 + m] += d2[m];
          dX[1] += 2.f * y1 * d2[0] + kSqrt2 * y3 * d2[3] + kSqrt2 * y2 * d2[4];
          dX[2] += 2.f * y2 * d2[1] + kSqrt2 * y1 * d2[4] + kSqrt2 * y3 * d2[5];
          dX[3] += 2.f * y3 * d2[2] + kSqrt2 * y1 * d2[3] + kSqrt2 * y2 * d2[5];
        }
      }
      __syncwarp();
      if (col < E)
#pragma unroll
        for (int c = 0; c < 10; ++c) bufB[c * E + col] = dX[c] * M.inv_nnbrs;
      __syncwarp();
    }
    // ---- rows: recompute with tangents, scatter forces
    const float3 ri = gen_load_pos(pos, perm, f, i, D.N);
    const int bs = box_slot(D, g, f);
    const float3 L = make_float3(box[bs * 3], box[bs * 3 + 1], box[bs * 3 + 2]);
    const int3 ni = image_range(L, M.rcut);
    const int nim = (2 * ni.x + 1) * (2 * ni.y + 1) * (2 * ni.z + 1);
    const float inv_std = M.inv_std[ti], mean = M.mean[ti];
    const unsigned lt = (1u << lane) - 1u;
    float *rowbuf = bufA;  // 64 rows x 8 floats
    float *hA = bufA + 64 * 8, *dA = hA + G.HM * 32, *hB = dA + G.HM * 32, *dB = hB + G.HM * 32;
    const size_t frame_base = (size_t)f * D.N;
    for (int tj = 0; tj < D.ntypes; ++tj) {
      const float *W = wsm + tj * G.NW;
      const int knet = ti * M.ntypes + tj;
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
            const float3 rj = gen_load_pos(pos, perm, f, jj, D.N);
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
          if (CMP)
            gen_rows_bwd_cmp(M.cmp_coeff[knet], M.cmp_srmin[knet], M.cmp_delta[knet], M.ngrids, E, 32, rowbuf, bufB,
                             inv_std, mean, lane, ro, F4, frame_base);
          else
            gen_rows_bwd(G, W, 32, rowbuf, bufB, hA, dA, hB, dB, inv_std, mean, lane, ro, F4, frame_base);
          const int rem = nbuf - 32;
          if (lane < rem)
            for (int c = 0; c < 8; ++c) rowbuf[lane * 8 + c] = rowbuf[(32 + lane) * 8 + c];
          __syncwarp();
          nbuf = rem;
        }
      }
      if (nbuf > 0) {
        if (CMP)
          gen_rows_bwd_cmp(M.cmp_coeff[knet], M.cmp_srmin[knet], M.cmp_delta[knet], M.ngrids, E, nbuf, rowbuf, bufB,
                           inv_std, mean, lane, ro, F4, frame_base);
        else
          gen_rows_bwd(G, W, nbuf, rowbuf, bufB, hA, dA, hB, dB, inv_std, mean, lane, ro, F4, frame_base);
      }
      __syncwarp();
    }
    const float f0 = warp_sum(ro.fi0), f1 = warp_sum(ro.fi1), f2 = warp_sum(ro.fi2);
    if (lane == 0) atomicAdd(&F4[frame_base + (perm ? perm[i] : i)], make_float4(f0, f1, f2, 0.f));
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const float s = warp_sum(ro.vir[k]);
    if (lane == 0 && s != 0.f) atomicAdd(&vsm[k], (double)s);
  }
  __syncthreads();
  // the block's atoms share one frame (segment-aligned in packed batches)
  if (threadIdx.x < 9) {
    const int vs = box_slot(D, (size_t)f * D.N + D.offs[ti] + blockIdx.x * wpb, f);
    atomicAdd(&virial[vs * 9 + threadIdx.x], vsm[threadIdx.x]);
  }
}

// Warps per block from the shared memory the shape needs (at most 8, at
// least 1; a block's warps are consecutive atoms of one frame, and a packed
// batch's segments start at multiples of 8 atoms, so any power of two up to 8
// keeps a block inside one segment).
static int gen_warps(size_t fixed_floats, size_t per_warp_floats, size_t *smem) {
  int dev = 0, cap = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int w = 8;
  while (w > 1 && (fixed_floats + w * per_warp_floats) * 4 > (size_t)cap) w >>= 1;
  *smem = (fixed_floats + w * per_warp_floats) * 4;
  return (*smem <= (size_t)cap) ? w : 0;
}

int launch_embed_fwd_gen(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                         const float *box, const int32_t *nbrs, float *T, float *G, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  const GenNet net = gen_net(M);
  const bool cmp = M.ngrids > 0;
  size_t smem = 0;
  const int wpb = gen_warps(cmp ? 0 : (size_t)M.ntypes * net.NW, gen_fwd_warp_floats(net), &smem);
  if (wpb == 0) return DPB_ERR_UNSUPPORTED;
  dim3 grid((cnt + wpb - 1) / wpb, D.F);
  if (cmp) {
    DPB_CUDA_TRY(cudaFuncSetAttribute(k_embed_fwd_gen<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_embed_fwd_gen<true><<<grid, 32 * wpb, smem, st>>>(M, net, D, ti, pos, perm, box, nbrs, T, G);
  } else {
    DPB_CUDA_TRY(cudaFuncSetAttribute(k_embed_fwd_gen<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_embed_fwd_gen<false><<<grid, 32 * wpb, smem, st>>>(M, net, D, ti, pos, perm, box, nbrs, T, G);
  }
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

int launch_embed_bwd_gen(const DevModel &M, const SysDesc &D, int ti, const float *pos, const int32_t *perm,
                         const float *box, const int32_t *nbrs, const float *T, const float *dG, float4 *F4,
                         double *virial, cudaStream_t st) {
  const int cnt = D.offs[ti + 1] - D.offs[ti];
  if (cnt == 0) return DPB_OK;
  const GenNet net = gen_net(M);
  const bool cmp = M.ngrids > 0;
  size_t smem = 0;
  const int wpb = gen_warps(cmp ? 0 : (size_t)M.ntypes * net.NW, gen_bwd_warp_floats(net, M.A), &smem);
  if (wpb == 0) return DPB_ERR_UNSUPPORTED;
  dim3 grid((cnt + wpb - 1) / wpb, D.F);
  if (cmp) {
    DPB_CUDA_TRY(cudaFuncSetAttribute(k_embed_bwd_gen<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_embed_bwd_gen<true><<<grid, 32 * wpb, smem, st>>>(M, net, D, ti, pos, perm, box, nbrs, T, dG, F4, virial);
  } else {
    DPB_CUDA_TRY(cudaFuncSetAttribute(k_embed_bwd_gen<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_embed_bwd_gen<false><<<grid, 32 * wpb, smem, st>>>(M, net, D, ti, pos, perm, box, nbrs, T, dG, F4, virial);
  }
  count_launch();
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

// Whether the shared-memory budget admits the shape (host check at model creation).
bool embed_general_fits(const DevModel &M) {
  const GenNet net = gen_net(M);
  size_t smem = 0;
  const bool cmp = M.ngrids > 0;
  return gen_warps(cmp ? 0 : (size_t)M.ntypes * net.NW, gen_fwd_warp_floats(net), &smem) > 0 &&
         gen_warps(cmp ? 0 : (size_t)M.ntypes * net.NW, gen_bwd_warp_floats(net, M.A), &smem) > 0;
}

}  // namespace dpb
