// C ABI of libdpb200: model upload, workspace sizing and evaluation dispatch.
#include "internal.cuh"
#include "tc.cuh"
#include <cuda_bf16.h>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace dpb {
std::atomic<uint64_t> g_launches{0};

// ---- per-kernel event timing (dpb_profile_*)
static bool g_prof_on = false;
static std::vector<cudaEvent_t> g_prof_pool;
static size_t g_prof_next = 0;
struct ProfRec { int id; cudaEvent_t a, b; };
static std::vector<ProfRec> g_prof_open, g_prof_done;
static double g_prof_ms[PROF_COUNT];
static uint64_t g_prof_n[PROF_COUNT];

static cudaEvent_t prof_event() {
  if (g_prof_next == g_prof_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    g_prof_pool.push_back(e);
  }
  return g_prof_pool[g_prof_next++];
}
void prof_begin(int id, cudaStream_t st) {
  if (!g_prof_on) return;
  ProfRec r{id, prof_event(), nullptr};
  cudaEventRecord(r.a, st);
  g_prof_open.push_back(r);
}
void prof_end(int id, cudaStream_t st) {
  if (!g_prof_on) return;
  for (size_t k = g_prof_open.size(); k-- > 0;)
    if (g_prof_open[k].id == id) {
      ProfRec r = g_prof_open[k];
      g_prof_open.erase(g_prof_open.begin() + k);
      r.b = prof_event();
      cudaEventRecord(r.b, st);
      g_prof_done.push_back(r);
      return;
    }
}
static void prof_collect() {
  for (auto &r : g_prof_done) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    g_prof_ms[r.id] += ms;
    g_prof_n[r.id] += 1;
  }
  g_prof_done.clear();
  g_prof_next = 0;
}

// fp32 path (eval_fp32.cu)
template <int E0, int E1, int E2>
int launch_embed_fwd(const DevModel &, const SysDesc &, int, const float *, const int32_t *, const float *,
                     const int32_t *, float *, float *, cudaStream_t);
template <int E0, int E1, int E2>
int launch_embed_bwd(const DevModel &, const SysDesc &, int, const float *, const int32_t *, const float *,
                     const int32_t *, const float *, const float *, float4 *, double *, cudaStream_t);
int launch_sgemm(int, int, int, const float *, int, RowMap, const float *, const Epi &, cudaStream_t);
// any embedding shape (eval_general.cu)
int launch_embed_fwd_gen(const DevModel &, const SysDesc &, int, const float *, const int32_t *, const float *,
                         const int32_t *, float *, float *, cudaStream_t);
int launch_embed_bwd_gen(const DevModel &, const SysDesc &, int, const float *, const int32_t *, const float *,
                         const int32_t *, const float *, const float *, float4 *, double *, cudaStream_t);
int launch_fit_energy(int, RowMap, int, const float *, const float *, const float *, const float *,
                      const float *, float *, float *, double *, int, const int32_t *, cudaStream_t);
int launch_finalize(int, int, const float4 *, float *, const float *, const int32_t *, float *, double *, int,
                    const float *, const int32_t *, uint32_t *, cudaStream_t);
// mixed path (mixed.cu)
int mixed_supported(const DevModel &M);
int mixed_fit_width(const DevModel &M);
size_t mixed_workspace_per_atom(const DevModel &M);
size_t mixed_workspace_fixed(const DevModel &M);
int mixed_eval(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm, const float *box,
               const int32_t *nbrs, double *energy, float *Eatom, float4 *F4, double *virial, void *ws,
               cudaStream_t st, int dT_warps, bool fit_deep);
int mixed_descriptors_f32(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm,
                          const float *box, const int32_t *nbrs, float *T, float *G, int *err, void *ws,
                          cudaStream_t st);
int fit_fp32_chain(const DevModel &M, const SysDesc &D, float *G, float *Eatom, double *energy, char *w,
                   cudaStream_t st);
}  // namespace dpb

using namespace dpb;



static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

template <class T>
static int upload(dpb_model *m, const T *host, size_t n, const T **dev) {
  void *p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return DPB_ERR_CUDA;
  m->allocs.push_back(p);
  if (cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return DPB_ERR_CUDA;
  *dev = (const T *)p;
  return DPB_OK;
}

// B operand chunks of the mixed fitting kernel from a row-major matrix
// (rows x K) times `scale`: for pass p of br rows and K chunk k (16 wide), the
// chunk is [half (2)][row (br)][8] FP16, rows past `rows` zero (mixed.cu,
// k_mix_fit).
static int upload_fit_tiles(dpb_model *m, const std::vector<float> &a, int rows, int K, int br, float scale,
                            const __half **dev) {
  const int nk = K / 16, npass = (rows + br - 1) / br;
  std::vector<float> t((size_t)npass * nk * 2 * br * 8, 0.f);
  for (int p = 0; p < npass; ++p)
    for (int k = 0; k < nk; ++k)
      for (int h = 0; h < 2; ++h)
        for (int r = 0; r < br; ++r) {
          const int row = p * br + r;
          if (row >= rows) continue;
          for (int e = 0; e < 8; ++e)
            t[((((size_t)p * nk + k) * 2 + h) * br + r) * 8 + e] = a[(size_t)row * K + k * 16 + h * 8 + e];
        }
  std::vector<__half> b(t.size());
  for (size_t i = 0; i < t.size(); ++i) b[i] = __float2half_rn(t[i] * scale);
  return upload(m, b.data(), b.size(), dev);
}

// 2^k with x 2^k in (2^13, 2^14] (x > 0; 1 for x = 0 or non-finite), k
// clamped to [-40, 40].
static float pow2_scale_to_2p14(double x) {
  if (!(x > 0.0) || !std::isfinite(x)) return 1.f;
  int k = 14 - (int)std::ceil(std::log2(x));
  k = std::max(-40, std::min(40, k));
  return std::ldexp(1.f, k);
}

// The tuned three-layer embedding instantiations (FP32 and tensor-core kernels).
static bool embed_tuned(const DevModel &M) {
  return M.nemb == 3 && ((M.E0 == 25 && M.E1 == 50 && M.E2 == 100) || (M.E0 == 32 && M.E1 == 32 && M.E2 == 64));
}

// Shapes the reference's embedding_net builds (utils.py:110-124): widths whose
// consecutive ratio is an integer one way or the other.
static bool embed_shape_ok(const dpb_model_desc *d) {
  if (d->n_embed < 1 || d->n_embed > kMaxEmbedLayers) return false;
  for (int l = 0; l < d->n_embed; ++l) {
    const int w = d->embed_widths[l];
    if (w < 1 || w > 256) return false;
    if (l > 0) {
      const int p = d->embed_widths[l - 1];
      if (w % p != 0 && p % w != 0) return false;
    }
  }
  return true;
}

namespace dpb {
bool embed_general_fits(const DevModel &M);
}

extern "C" int dpb_model_create(const dpb_model_desc *d, dpb_model **out) {
  if (!d || !out) return DPB_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DPB_ERR_NO_DEVICE;
  const int nt = d->ntypes;
  if (nt < 1 || nt > kMaxTypes || !embed_shape_ok(d) || d->n_fit < 1 || d->n_fit > kMaxFitLayers)
    return DPB_ERR_UNSUPPORTED;
  for (int l = 0; l < d->n_fit; ++l)
    if (d->fit_widths[l] < 1 || d->fit_widths[l] > 1024) return DPB_ERR_UNSUPPORTED;
  dpb_model *m = new dpb_model();
  cudaGetDevice(&m->device);
  DevModel &M = m->dm;
  std::memset(&M, 0, sizeof(M));
  M.ntypes = nt;
  M.nemb = d->n_embed;
  for (int l = 0; l < d->n_embed; ++l) M.EW[l] = d->embed_widths[l];
  // E2 is the output width everywhere; E0 / E1 name the tuned kernels' layers
  M.E2 = d->embed_widths[d->n_embed - 1];
  M.E0 = d->n_embed == 3 ? d->embed_widths[0] : 0;
  M.E1 = d->n_embed == 3 ? d->embed_widths[1] : 0;
  M.emb_tuned = embed_tuned(M) ? 1 : 0;
  M.A = d->axis;
  M.nfit = d->n_fit;
  for (int l = 0; l < d->n_fit; ++l) M.FW[l] = d->fit_widths[l];
  M.rcut = (float)d->rcut;
  M.inv_nnbrs = (float)(1.0 / d->nnbrs);
  if (M.A < 1 || 2 * M.A > 32 || 2 * M.A > M.E2) {
    delete m;
    return DPB_ERR_UNSUPPORTED;
  }
  for (int t = 0; t < nt; ++t) {
    M.mean[t] = (float)d->sr_mean[t];
    M.inv_std[t] = (float)(1.0 / d->sr_std[t]);
  }
  int ew_in[kMaxEmbedLayers], ew_out[kMaxEmbedLayers];
  for (int l = 0; l < M.nemb; ++l) {
    ew_in[l] = l == 0 ? 1 : M.EW[l - 1];
    ew_out[l] = M.EW[l];
  }
  int rc = DPB_OK;
  const bool have_mlp = d->embed_kernel != nullptr && d->embed_bias != nullptr;
  if (d->n_grids < 0 || (d->n_grids == 0 && !have_mlp) ||
      (d->n_grids > 0 && (!d->cmp_coeff || !d->cmp_srmin || !d->cmp_srmax))) {
    delete m;
    return DPB_ERR_INVALID_ARG;
  }
  // compressed tables: the reference's lookup runs in float32 (srmin, srmax
  // and delta = (srmax - srmin) / Ngrids as float32 arrays, utils.py:131-134)
  M.ngrids = d->n_grids;
  for (int k = 0; k < nt * nt && rc == DPB_OK && M.ngrids > 0; ++k) {
    if (!d->cmp_coeff[k]) rc = DPB_ERR_INVALID_ARG;
    if (rc == DPB_OK) rc = upload(m, d->cmp_coeff[k], (size_t)M.ngrids * 6 * M.E2, &M.cmp_coeff[k]);
    const float lo = (float)d->cmp_srmin[k], hi = (float)d->cmp_srmax[k];
    volatile float span = hi - lo;  // float32 rounding, as in the reference
    M.cmp_srmin[k] = lo;
    M.cmp_delta[k] = span / (float)M.ngrids;
  }
  const int ne = M.nemb;
  for (int k = 0; k < nt * nt && rc == DPB_OK && have_mlp; ++k)
    for (int l = 0; l < ne && rc == DPB_OK; ++l) {
      rc = upload(m, d->embed_kernel[k * ne + l], (size_t)ew_in[l] * ew_out[l], &M.ew[k][l]);
      if (rc == DPB_OK) rc = upload(m, d->embed_bias[k * ne + l], (size_t)ew_out[l], &M.eb[k][l]);
    }
  // shared-memory images of the embedding nets for the tensor-core kernels:
  // FP16 B tiles (K-major) of layers 1 and 2 with the layer's bias as one
  // more K row (the A operands carry a ones column there), and the FP32 first
  // layer (w0, b0 in FP32) (mixed.cu, MixDims)
  {
    const int K1 = (M.E0 + 1 + 15) / 16 * 16, N1 = (M.E1 + 15) / 16 * 16;
    const int K2 = (M.E1 + 1 + 15) / 16 * 16, N2 = (M.E2 + 15) / 16 * 16;
    const int W1B = N1 * K1 * 2, W2B = N2 * K2 * 2;
    M.net_img_bytes = W1B + W2B;
    M.net_small_floats = (2 * M.E0 + 3) / 4 * 4;
    for (int k = 0; k < nt * nt && rc == DPB_OK && have_mlp && M.emb_tuned; ++k) {
      std::vector<uint8_t> img(M.net_img_bytes, 0);
      const float *W1 = d->embed_kernel[k * 3 + 1], *W2 = d->embed_kernel[k * 3 + 2];
      const float *b1 = d->embed_bias[k * 3 + 1], *b2 = d->embed_bias[k * 3 + 2];
      for (int n = 0; n < N1; ++n)
        for (int kk = 0; kk < K1; ++kk) {
          float v = 0.f;
          if (n < M.E1 && kk < M.E0) v = W1[kk * M.E1 + n];
          if (n < M.E1 && kk == M.E0) v = b1[n];
          *reinterpret_cast<__half *>(img.data() + dpb::tc::kmajor_off(n, kk, K1)) = __float2half_rn(v);
        }
      for (int n = 0; n < N2; ++n)
        for (int kk = 0; kk < K2; ++kk) {
          float v = 0.f;
          if (n < M.E2 && kk < M.E1) v = W2[kk * M.E2 + n];
          if (n < M.E2 && kk == M.E1) v = b2[n];
          *reinterpret_cast<__half *>(img.data() + W1B + dpb::tc::kmajor_off(n, kk, K2)) = __float2half_rn(v);
        }
      const char *dimg = nullptr;
      rc = upload(m, reinterpret_cast<const char *>(img.data()), img.size(), &dimg);
      M.net_img[k] = dimg;
      std::vector<float> sm(M.net_small_floats, 0.f);
      const float *w0 = d->embed_kernel[k * 3 + 0], *b0 = d->embed_bias[k * 3 + 0];
      for (int e = 0; e < M.E0; ++e) {
        sm[e] = w0[e];
        sm[M.E0 + e] = b0[e];
      }
      if (rc == DPB_OK) rc = upload(m, sm.data(), sm.size(), &M.net_small[k]);
    }
  }
  if (rc == DPB_OK) rc = upload(m, d->tbias, (size_t)M.E2, &M.tbias);
  const int K0 = M.A * M.E2;
  M.mfw = dpb::mixed_fit_width(M);
  double dg_bound = 0.0;  // largest bound on |dE/dG| over the types
  for (int t = 0; t < nt && rc == DPB_OK; ++t) {
    // per layer: max over inputs i of sum_o |W[i][o]|, max |dt| (1 without
    // residual), and max |w_out|: the bounds behind fit_gsc
    std::vector<double> rowsum(M.nfit + 1, 0.0), maxdt(M.nfit + 1, 1.0);
    double wout_max = 0.0;
    for (int l = 0; l <= M.nfit && rc == DPB_OK; ++l) {
      const int in = l == 0 ? K0 : M.FW[l - 1];
      const int outw = l == M.nfit ? 1 : M.FW[l];
      const float *kh = d->fit_kernel[t * (M.nfit + 1) + l];
      const float *bh = d->fit_bias[t * (M.nfit + 1) + l];
      std::vector<float> kv(kh, kh + (size_t)in * outw), bv(bh, bh + outw);
      if (l == M.nfit) {  // fold out_norm and Ebias into the output layer
        for (auto &x : kv) x = (float)(x * d->out_norm);
        for (auto &x : bv) x = (float)((x + d->ebias[t]) * d->out_norm);
      }
      rc = upload(m, kv.data(), kv.size(), &M.fw[t][l]);
      if (rc == DPB_OK) rc = upload(m, bv.data(), bv.size(), &M.fb[t][l]);
      std::vector<float> kt((size_t)in * outw);
      for (int i = 0; i < in; ++i)
        for (int o = 0; o < outw; ++o) kt[(size_t)o * in + i] = kv[(size_t)i * outw + o];
      if (rc == DPB_OK) rc = upload(m, kt.data(), kt.size(), &M.fwT[t][l]);
      const float *dt = (l < M.nfit && d->fit_dt) ? d->fit_dt[t * M.nfit + l] : nullptr;
      if (rc == DPB_OK && dt) rc = upload(m, dt, (size_t)outw, &M.fdt[t][l]);
      double wmax = 0.0;
      for (int i = 0; i < in; ++i) {
        double rs = 0.0;
        for (int o = 0; o < outw; ++o) {
          rs += std::fabs((double)kv[(size_t)i * outw + o]);
          wmax = std::max(wmax, std::fabs((double)kv[(size_t)i * outw + o]));
        }
        rowsum[l] = std::max(rowsum[l], rs);
      }
      if (dt)  // the kernel multiplies by dt or by 1: bound by both
        for (int o = 0; o < outw; ++o) maxdt[l] = std::max(maxdt[l], std::fabs((double)dt[o]));
      if (l == M.nfit) wout_max = wmax;
      else M.fit_wsc[t][l] = pow2_scale_to_2p14(wmax);
      if (rc == DPB_OK && M.mfw > 0) {
        // the tensor-core fitting's copy: every hidden width padded to mfw with zeros
        const int P = M.mfw, inp = l == 0 ? K0 : P, outp = l == M.nfit ? 1 : P;
        std::vector<float> kp((size_t)inp * outp, 0.f), ktp((size_t)outp * inp, 0.f);
        for (int i = 0; i < in; ++i)
          for (int o = 0; o < outw; ++o) {
            kp[(size_t)i * outp + o] = kv[(size_t)i * outw + o];
            ktp[(size_t)o * inp + i] = kv[(size_t)i * outw + o];
          }
        if (l < M.nfit) {
          std::vector<float> bp(P, 0.f), dp(P, 0.f);
          for (int o = 0; o < outw; ++o) {
            bp[o] = bv[o];
            if (dt) dp[o] = dt[o];
          }
          rc = upload(m, bp.data(), bp.size(), &M.mfb[t][l]);
          if (rc == DPB_OK && dt) rc = upload(m, dp.data(), dp.size(), &M.mfdt[t][l]);
          const float ws = M.fit_wsc[t][l];
          if (rc == DPB_OK) rc = upload_fit_tiles(m, ktp, outp, inp, outp, ws, &M.fit_bt[t][kFitBtFwd + l]);
          if (rc == DPB_OK && l >= 1) rc = upload_fit_tiles(m, kp, inp, outp, inp, ws, &M.fit_bt[t][kFitBtAdj + l]);
          if (rc == DPB_OK && l == 0) rc = upload_fit_tiles(m, kp, K0, outp, 128, ws, &M.fit_bt[t][kFitBtDg]);
        } else {
          rc = upload(m, kp.data(), kp.size(), &M.mfwout[t]);
        }
      }
    }
    // bound on the adjoint gate g_l of every layer (what the kernel packs as
    // layer l's A operand): g_{L-1} = w_out dt (1 - t^2); the accumulator
    // g_l W_l^T of row i is at most G_l rowsum_l, plus the residual's
    // dE/dh term where layer l has one
    const int L = M.nfit;
    std::vector<double> G(L, 0.0);
    double Hb = wout_max;  // bound on dE/dh_{L-1}
    G[L - 1] = Hb * maxdt[L - 1];
    for (int l = L - 1; l >= 1; --l) {
      const bool res_l = d->fit_dt && d->fit_dt[t * M.nfit + l];
      Hb = G[l] * rowsum[l] + (res_l ? Hb : 0.0);
      G[l - 1] = Hb * maxdt[l - 1];
    }
    for (int l = 0; l < L; ++l) M.fit_gsc[t][l] = pow2_scale_to_2p14(G[l]);
    dg_bound = std::max(dg_bound, G[0] * rowsum[0]);
  }
  M.fit_dgsc = pow2_scale_to_2p14(dg_bound);
  if (rc == DPB_OK && !M.emb_tuned && !dpb::embed_general_fits(M)) rc = DPB_ERR_UNSUPPORTED;
  // the uploads are blocking copies from pageable memory, whose DMA may land
  // after they return and which order themselves only against the legacy
  // stream: the weights are in place before any stream's kernel reads them
  if (rc == DPB_OK && cudaDeviceSynchronize() != cudaSuccess) rc = DPB_ERR_CUDA;
  if (rc != DPB_OK) {
    dpb_model_destroy(m);
    return rc;
  }
  *out = m;
  return DPB_OK;
}

extern "C" int dpb_model_destroy(dpb_model *m) {
  if (!m) return DPB_ERR_INVALID_ARG;
  for (void *p : m->allocs) cudaFree(p);
  delete m;
  return DPB_OK;
}

static int fit_width_max(const DevModel &M) {
  int w = 0;
  for (int l = 0; l < M.nfit; ++l) w = std::max(w, M.FW[l]);
  return w;
}

static size_t fp32_ws_per_atom(const DevModel &M) {
  int hid = 0;
  for (int l = 0; l < M.nfit; ++l) hid += M.FW[l];
  return (size_t)(10 * M.E2 + M.A * M.E2 + 2 * hid + 4 * fit_width_max(M) + 1) * 4 + 16;
}

// Workspace of NF atoms with nE energy / virial rows.
static size_t eval_ws_bytes(const DevModel &M, size_t NF, size_t nE) {
  size_t a = al(NF * fp32_ws_per_atom(M)) + 16 * 256 + al(nE * 9 * 8);
  size_t b = al(NF * mixed_workspace_per_atom(M)) + mixed_workspace_fixed(M) + al(NF * 16) + al(NF * 4) +
             al(nE * 9 * 8) + 16 * 256;
  return std::max(a, b);
}

extern "C" int dpb_eval_workspace_bytes(const dpb_model *m, int natoms, int nframes, size_t *bytes) {
  if (!m || !bytes || natoms <= 0 || nframes <= 0) return DPB_ERR_INVALID_ARG;
  *bytes = eval_ws_bytes(m->dm, (size_t)natoms * nframes, (size_t)nframes);
  return DPB_OK;
}

extern "C" int dpb_eval_packed_workspace_bytes(const dpb_model *m, int natoms, int nseg, size_t *bytes) {
  if (!m || !bytes || natoms <= 0 || nseg <= 0) return DPB_ERR_INVALID_ARG;
  *bytes = eval_ws_bytes(m->dm, (size_t)natoms, (size_t)nseg);
  return DPB_OK;
}

static int fill_sys(const dpb_model *m, int natoms, int nframes, const int *type_count, const int *sel,
                    SysDesc &D) {
  const int nt = m->dm.ntypes;
  D.N = natoms; D.F = nframes; D.ntypes = nt;
  D.seg = nullptr;
  int off = 0, col = 0;
  for (int t = 0; t < nt; ++t) {
    if (type_count[t] < 0 || sel[t] < 0) return DPB_ERR_INVALID_ARG;
    D.offs[t] = off; off += type_count[t];
    D.sel[t] = sel[t]; D.col[t] = col; col += sel[t];
  }
  if (off != natoms) return DPB_ERR_INVALID_ARG;
  for (int t = nt; t <= kMaxTypes; ++t) D.offs[t] = natoms;
  D.col[nt] = col;
  D.S = col;
  return DPB_OK;
}

// FP32 fitting chain (tiled SGEMMs with fused epilogues) for every centre
// type: G -> per-atom energies (FP64 frame sums) and dE/dG written over G.
// Hidden layer l has width FW[l]; a dt residual (utils.py:158-163) exists
// only where FW[l] == FW[l-1], so every residual pairs equal widths.
// w: scratch for the per-layer activations and adjoints.
int dpb::fit_fp32_chain(const DevModel &M, const SysDesc &D, float *G, float *Eatom, double *energy, char *w,
                        cudaStream_t st) {
  const size_t NF = (size_t)D.N * D.F;
  const int E2 = M.E2, A = M.A, K0 = A * E2, L = M.nfit, FWM = fit_width_max(M);
  float *tb[kMaxFitLayers], *hb[kMaxFitLayers];
  for (int l = 0; l < L; ++l) { tb[l] = (float *)w; w += al(NF * M.FW[l] * 4); }
  for (int l = 0; l < L; ++l) { hb[l] = (float *)w; w += al(NF * M.FW[l] * 4); }
  float *gz[2], *gh[2];
  gz[0] = (float *)w; w += al(NF * FWM * 4);
  gz[1] = (float *)w; w += al(NF * FWM * 4);
  gh[0] = (float *)w; w += al(NF * FWM * 4);
  gh[1] = (float *)w; w += al(NF * FWM * 4);
  int rc;
  for (int ti = 0; ti < M.ntypes; ++ti) {
    const int cnt = D.offs[ti + 1] - D.offs[ti];
    if (!cnt) continue;
    const RowMap rm{cnt, D.N, D.offs[ti]};
    const int Mrows = cnt * D.F;
    for (int l = 0; l < L; ++l) {
      const int out = M.FW[l], in = l == 0 ? K0 : M.FW[l - 1];
      Epi ep{};
      ep.bias = M.fb[ti][l];
      ep.out1 = tb[l];
      ep.out2 = hb[l];
      ep.ld = out;
      if (l > 0 && M.fdt[ti][l]) {
        ep.mode = EPI_TANH_RES;
        ep.dt = M.fdt[ti][l];
        ep.hprev = hb[l - 1];
      } else {
        ep.mode = EPI_TANH;
      }
      if (l == 0) rc = launch_sgemm(Mrows, out, in, G, K0, rm, M.fw[ti][0], ep, st);
      else rc = launch_sgemm(Mrows, out, in, hb[l - 1], in, rm, M.fw[ti][l], ep, st);
      if (rc) return rc;
    }
    int cur = 0;
    rc = launch_fit_energy(Mrows, rm, M.FW[L - 1], hb[L - 1], tb[L - 1], M.fw[ti][L], M.fb[ti][L],
                           M.fdt[ti][L - 1], Eatom, gz[cur], energy, D.N, D.seg, st);
    if (rc) return rc;
    for (int l = L - 1; l >= 1; --l) {
      // gH_{l-1} = gZ_l W_l^T (+ gH_l through layer l's residual)
      const int out = M.FW[l - 1], in = M.FW[l];
      Epi ep{};
      ep.ld = out;
      ep.tin = tb[l - 1];
      if (M.fdt[ti][l]) {
        if (l == L - 1) ep.gvec = M.fw[ti][L];
        else ep.gmat = gh[cur];
      }
      ep.out1 = gz[cur ^ 1];
      if (l - 1 > 0 && M.fdt[ti][l - 1]) {
        ep.mode = EPI_GRAD_RES;
        ep.dt = M.fdt[ti][l - 1];
        ep.out2 = gh[cur ^ 1];
      } else {
        ep.mode = EPI_GRAD;
      }
      rc = launch_sgemm(Mrows, out, in, gz[cur], in, rm, M.fwT[ti][l], ep, st);
      if (rc) return rc;
      cur ^= 1;
    }
    Epi ep{};
    ep.mode = EPI_STORE;
    ep.out1 = G;
    ep.ld = K0;
    rc = launch_sgemm(Mrows, K0, M.FW[0], gz[cur], M.FW[0], rm, M.fwT[ti][0], ep, st);
    if (rc) return rc;
  }
  return DPB_OK;
}

static int eval_fp32(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm,
                     const float *box, const int32_t *nbrs, double *energy, float4 *F4, float *Eatom,
                     double *virial, char *w, cudaStream_t st) {
  const size_t NF = (size_t)D.N * D.F;
  const int E2 = M.E2, A = M.A, K0 = A * E2;
  float *T = (float *)w; w += al(NF * 10 * E2 * 4);
  float *G = (float *)w; w += al(NF * K0 * 4);  // G, later dE/dG
  int rc;
  prof_begin(PROF_EMBED_FWD, st);
  for (int ti = 0; ti < M.ntypes; ++ti) {
    if (!M.emb_tuned) rc = launch_embed_fwd_gen(M, D, ti, pos, perm, box, nbrs, T, G, st);
    else if (M.E2 == 100) rc = launch_embed_fwd<25, 50, 100>(M, D, ti, pos, perm, box, nbrs, T, G, st);
    else rc = launch_embed_fwd<32, 32, 64>(M, D, ti, pos, perm, box, nbrs, T, G, st);
    if (rc) return rc;
  }
  prof_end(PROF_EMBED_FWD, st);
  prof_begin(PROF_FIT, st);
  rc = fit_fp32_chain(M, D, G, Eatom, energy, w, st);
  if (rc) return rc;
  prof_end(PROF_FIT, st);
  prof_begin(PROF_EMBED_BWD, st);
  for (int ti = 0; ti < M.ntypes; ++ti) {
    if (!M.emb_tuned) rc = launch_embed_bwd_gen(M, D, ti, pos, perm, box, nbrs, T, G, F4, virial, st);
    else if (M.E2 == 100) rc = launch_embed_bwd<25, 50, 100>(M, D, ti, pos, perm, box, nbrs, T, G, F4, virial, st);
    else rc = launch_embed_bwd<32, 32, 64>(M, D, ti, pos, perm, box, nbrs, T, G, F4, virial, st);
    if (rc) return rc;
  }
  prof_end(PROF_EMBED_BWD, st);
  return DPB_OK;
}

int dpb::eval_impl(const dpb_model *m, int precision, const float *pos, const int32_t *perm, int natoms,
                   int nframes, const int *type_count, const float *box, const int32_t *nbrs, const int *sel,
                   double *energy, float *atom_energy, float *force, double *virial, uint32_t *status,
                   void *workspace, size_t ws_bytes, cudaStream_t st, const int32_t *seg, int nseg) {
  if (!m || !pos || !box || !nbrs || !energy || !force || !status || !type_count || !sel || natoms <= 0 ||
      nframes <= 0)
    return DPB_ERR_INVALID_ARG;
  if (precision != DPB_PREC_FP32 && precision != DPB_PREC_MIXED) return DPB_ERR_INVALID_ARG;
  if (natoms >= (1 << 24)) return DPB_ERR_UNSUPPORTED;
  if (seg && (nframes != 1 || nseg <= 0)) return DPB_ERR_INVALID_ARG;
  const size_t nE = seg ? (size_t)nseg : (size_t)nframes;
  if (!workspace || ws_bytes < eval_ws_bytes(m->dm, (size_t)natoms * nframes, nE)) return DPB_ERR_WORKSPACE;
  SysDesc D;
  int rc = fill_sys(m, natoms, nframes, type_count, sel, D);
  if (rc) return rc;
  D.seg = seg;
  const DevModel &M = m->dm;
  const size_t NF = (size_t)natoms * nframes;
  char *w = (char *)workspace;
  float4 *F4 = (float4 *)w; w += al(NF * 16);
  float *Eatom = (float *)w; w += al(NF * 4);
  double *vir = virial;
  double *vscratch = (double *)w; w += al(nE * 9 * 8);
  if (!vir) vir = vscratch;
  DPB_CUDA_TRY(cudaMemsetAsync(F4, 0, NF * 16, st));
  DPB_CUDA_TRY(cudaMemsetAsync(energy, 0, nE * 8, st));
  DPB_CUDA_TRY(cudaMemsetAsync(vir, 0, nE * 72, st));
  if (precision == DPB_PREC_FP32) {
    rc = eval_fp32(M, D, pos, perm, box, nbrs, energy, F4, Eatom, vir, w, st);
  } else {
    if (!mixed_supported(M)) return DPB_ERR_UNSUPPORTED;
    rc = mixed_eval(M, D, pos, perm, box, nbrs, energy, Eatom, F4, vir, w, st, m->dT_warps, m->fit_deep != 0);
  }
  if (rc) return rc;
  return launch_finalize((int)NF, natoms, F4, force, Eatom, perm, atom_energy, energy, (int)nE, pos, seg, status,
                         st);
}

namespace dpb {
// The dE/dT part of the mixed evaluation's workspace sits after the pieces
// eval_impl carves first (forces, atom energies, virial rows).
int eval_tune_dT(const dpb_model *m, int natoms, int nframes, void *workspace, cudaStream_t st, int *best) {
  const size_t NF = (size_t)natoms * nframes;
  char *w = (char *)workspace;
  w += al(NF * 16);
  w += al(NF * 4);
  w += al((size_t)nframes * 9 * 8);
  return mixed_tune_dT(m->dm, NF, w, st, best);
}
}  // namespace dpb

extern "C" int dpb_eval_packed(const dpb_model *m, int precision, const float *pos, const int32_t *perm,
                               int natoms, const int *type_count, const int32_t *seg, int nseg, const float *box,
                               const int32_t *nbrs, const int *sel, double *energy, float *atom_energy,
                               float *force, double *virial, uint32_t *status, void *workspace, size_t ws_bytes,
                               void *stream) {
  if (!seg) return DPB_ERR_INVALID_ARG;
  return dpb::eval_impl(m, precision, pos, perm, natoms, 1, type_count, box, nbrs, sel, energy, atom_energy, force,
                        virial, status, workspace, ws_bytes, (cudaStream_t)stream, seg, nseg);
}

extern "C" int dpb_eval(const dpb_model *m, int precision, const float *pos, const int32_t *perm, int natoms,
                        int nframes, const int *type_count, const float *box, const int32_t *nbrs, const int *sel,
                        double *energy, float *atom_energy, float *force, double *virial, uint32_t *status,
                        void *workspace, size_t ws_bytes, void *stream) {
  return dpb::eval_impl(m, precision, pos, perm, natoms, nframes, type_count, box, nbrs, sel, energy, atom_energy,
                        force, virial, status, workspace, ws_bytes, (cudaStream_t)stream);
}

extern "C" int dpb_profile_enable(int on) {
  dpb::prof_collect();
  for (int k = 0; k < dpb::PROF_COUNT; ++k) { dpb::g_prof_ms[k] = 0.0; dpb::g_prof_n[k] = 0; }
  dpb::g_prof_on = on != 0;
  return DPB_OK;
}

extern "C" int dpb_profile_read(int id, double *ms, uint64_t *count) {
  if (id < 0 || id >= dpb::PROF_COUNT || !ms || !count) return DPB_ERR_INVALID_ARG;
  dpb::prof_collect();
  *ms = dpb::g_prof_ms[id];
  *count = dpb::g_prof_n[id];
  return DPB_OK;
}

// fp32 descriptor stage (eval_fp32.cu kernels), T and G of every atom
static int descriptors_fp32(const DevModel &M, const SysDesc &D, const float *pos, const int32_t *perm,
                            const float *box, const int32_t *nbrs, float *T, float *G, cudaStream_t st) {
  for (int ti = 0; ti < M.ntypes; ++ti) {
    int rc = !M.emb_tuned   ? launch_embed_fwd_gen(M, D, ti, pos, perm, box, nbrs, T, G, st)
             : M.E2 == 100 ? launch_embed_fwd<25, 50, 100>(M, D, ti, pos, perm, box, nbrs, T, G, st)
                           : launch_embed_fwd<32, 32, 64>(M, D, ti, pos, perm, box, nbrs, T, G, st);
    if (rc) return rc;
  }
  return DPB_OK;
}

extern "C" int dpb_eval_descriptors(const dpb_model *m, int precision, const float *pos, const int32_t *perm,
                                    int natoms, int nframes, const int *type_count, const float *box,
                                    const int32_t *nbrs, const int *sel, float *T, float *G, int *err,
                                    void *workspace, size_t ws_bytes, void *stream) {
  if (!m || !pos || !box || !nbrs || !T || !G || !err || !type_count || !sel || natoms <= 0 || nframes <= 0)
    return DPB_ERR_INVALID_ARG;
  size_t need = 0;
  dpb_eval_workspace_bytes(m, natoms, nframes, &need);
  if (!workspace || ws_bytes < need) return DPB_ERR_WORKSPACE;
  SysDesc D;
  int rc = fill_sys(m, natoms, nframes, type_count, sel, D);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == DPB_PREC_FP32) return descriptors_fp32(m->dm, D, pos, perm, box, nbrs, T, G, st);
  if (precision == DPB_PREC_MIXED) {
    if (!mixed_supported(m->dm)) return DPB_ERR_UNSUPPORTED;
    // the mixed form's embedding runs in the FP32 kernels for tables and untuned shapes
    if (m->dm.ngrids > 0 || !m->dm.emb_tuned) return descriptors_fp32(m->dm, D, pos, perm, box, nbrs, T, G, st);
    return mixed_descriptors_f32(m->dm, D, pos, perm, box, nbrs, T, G, err, workspace, st);
  }
  return DPB_ERR_INVALID_ARG;
}

extern "C" uint64_t dpb_kernel_launch_count(void) { return g_launches.load(); }

extern "C" const char *dpb_version(void) { return "dpb200 0.1 (sm_100a)"; }
