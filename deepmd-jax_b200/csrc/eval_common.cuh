// Device-side model description shared by the FP32 and mixed evaluation paths.
#pragma once
#include "dpb_common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace dpb {

constexpr int kMaxEmbedLayers = 4;
constexpr int kMaxFitLayers = 4;  // hidden layers

struct DevModel {
  int ntypes;
  int E0, E1, E2;      // embedding widths of the tuned three-layer kernels
  int nemb;            // embedding layers (1 .. kMaxEmbedLayers) and their widths
  int EW[kMaxEmbedLayers];
  int emb_tuned;       // 1: a tuned instantiation (25-50-100 or 32-32-64) serves the shape
  int A;               // axis neurons
  int nfit;            // hidden fitting layers
  int FW[kMaxFitLayers];
  float rcut;
  float inv_nnbrs;
  float mean[kMaxTypes];
  float inv_std[kMaxTypes];
  // FP32 weights (device), per embedding net k = i*ntypes + j
  const float *ew[kMaxTypes * kMaxTypes][kMaxEmbedLayers];
  const float *eb[kMaxTypes * kMaxTypes][kMaxEmbedLayers];
  const float *tbias;
  // fitting per centre type: kernels (in,out), biases, dt (NULL if none);
  // the final layer (index nfit) has out_norm folded into kernel and
  // out_norm * (bias + Ebias) as its bias.
  const float *fw[kMaxTypes][kMaxFitLayers + 1];
  const float *fb[kMaxTypes][kMaxFitLayers + 1];
  const float *fdt[kMaxTypes][kMaxFitLayers];
  // transposed fitting kernels (out,in) for the adjoint GEMMs
  const float *fwT[kMaxTypes][kMaxFitLayers + 1];
  // per embedding net: the shared-memory image of its FP16 B tiles (layer 1
  // and layer 2, K-major, the layer's bias as the K row after the inputs,
  // zero padded to multiples of 16) and of its first layer (w0, b0 in FP32),
  // copied verbatim by the mixed kernels
  const char *net_img[kMaxTypes * kMaxTypes];
  const float *net_small[kMaxTypes * kMaxTypes];
  int net_img_bytes, net_small_floats;
  // compressed embedding (ngrids > 0): per net, poly_coeff (ngrids, 6, E2)
  // and the float32 srmin / interval width of the reference's table lookup
  int ngrids;
  const float *cmp_coeff[kMaxTypes * kMaxTypes];
  float cmp_srmin[kMaxTypes * kMaxTypes], cmp_delta[kMaxTypes * kMaxTypes];
  // FP16 fitting weights pre-tiled as the B operand chunks of the mixed
  // fitting kernel (K = 16 per chunk, [chunk][k8 (2)][row][8]): forward layer l
  // at kFitBtFwd + l (W_l^T), adjoint layer l >= 1 at kFitBtAdj + l (W_l), and
  // W_0 in passes of 128 rows at kFitBtDg; null when the mixed form is unsupported.
  // Layer l's weights are stored times fit_wsc[t][l] = 2^k (largest magnitude
  // in (2^13, 2^14]), and the adjoint's A operand of layer l (the gate g of
  // dE/dz_l) times fit_gsc[t][l] = 2^k' with k' from a bound on |g| that
  // propagates max |w_out|, max |dt| and the row sums of |W| down the chain;
  // the kernel divides each accumulator by its two powers of two (exact).
  const __half *fit_bt[kMaxTypes][2 * kMaxFitLayers + 1];
  float fit_wsc[kMaxTypes][kMaxFitLayers], fit_gsc[kMaxTypes][kMaxFitLayers];
  // dE/dG leaves the fitting kernel as FP16 times fit_dgsc = 2^k, k from the
  // gate bound of layer 0 times the row sums of |W_0| (largest over
  // the types), and k_mix_dT divides it out
  float fit_dgsc;
  // the tensor-core fitting runs every hidden layer at one width mfw (a
  // multiple of 16 with a kernel instantiation, >= every FW[l]; 0: no
  // tensor-core fitting for this shape); the padding columns carry zero
  // weights, biases and dt, which keeps them exactly zero through the chain.
  // Padded FP32 biases, dt and output weights (out_norm folded) of that path:
  int mfw;
  const float *mfb[kMaxTypes][kMaxFitLayers];
  const float *mfdt[kMaxTypes][kMaxFitLayers];
  const float *mfwout[kMaxTypes];
};

constexpr int kFitBtFwd = 0, kFitBtAdj = kMaxFitLayers, kFitBtDg = 2 * kMaxFitLayers;

// Frame/type geometry of one evaluation call.
// Packed (ragged) batches run as one frame (F = 1) whose atoms come from many
// request frames: seg[k] is the request frame ("segment") of sorted atom k,
// i.e. the row of its box and of its energy / virial; padding atoms carry
// -(s + 1) (box of segment s, no energy).  Each segment's run of atoms of one
// type starts at a multiple of 8 of the type block, so every 8-atom block of
// the embedding kernels lies in one segment.  seg == NULL: ordinary frames.
struct SysDesc {
  int N, F, ntypes, S;
  int offs[kMaxTypes + 1];
  int sel[kMaxTypes];
  int col[kMaxTypes + 1];
  const int32_t *seg;
};

// Box row of sorted atom g (global index f * N + k) of frame f.
__device__ __forceinline__ int box_slot(const SysDesc &D, size_t g, int f) {
  if (!D.seg) return f;
  const int s = D.seg[g];
  return s >= 0 ? s : -s - 1;
}

// Energy row of sorted atom g, or -1 for a padding atom.
__device__ __forceinline__ int energy_slot(const int32_t *seg, size_t g, int N) {
  if (!seg) return (int)(g / N);
  const int s = seg[g];
  return s >= 0 ? s : -1;
}

// Rows of the fitting GEMMs are the atoms of one centre type across frames:
// row r -> atom (r / cnt) * N + off + r % cnt.
struct RowMap {
  int cnt, N, off;
  __host__ __device__ __forceinline__ size_t atom(int r) const {
    int f = r / cnt;
    return (size_t)f * N + off + (r - f * cnt);
  }
};

enum EpiMode : int {
  EPI_STORE = 0,      // out1 = acc
  EPI_TANH = 1,       // t = tanh(acc + b); out1 = t; out2 = t (H = t)
  EPI_TANH_RES = 2,   // t = tanh(acc + b); out1 = t; out2 = t * dt + Hprev
  EPI_GRAD_RES = 3,   // gH = acc + gadd; out2 = gH; out1 = gZ = gH * dt * (1 - t^2)
  EPI_GRAD = 4,       // gH = acc + gadd; out1 = gZ = gH * (1 - t^2)
};

// Fused epilogue of one fitting-layer GEMM (forward or adjoint).
struct Epi {
  int mode;
  const float *bias;    // [Nc]
  const float *dt;      // [Nc]
  const float *hprev;   // per atom, ld
  const float *tin;     // per atom tanh values of the layer below, ld
  const float *gvec;    // [Nc] broadcast addend (or NULL)
  const float *gmat;    // per atom addend (or NULL)
  float *out1, *out2;   // per atom, ld
  int ld;
};

}  // namespace dpb
