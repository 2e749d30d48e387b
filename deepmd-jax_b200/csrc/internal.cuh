// Internal interfaces shared between the translation units of libdpb200.
#pragma once
#include "eval_common.cuh"
#include <vector>

struct dpb_model {
  dpb::DevModel dm;
  std::vector<void *> allocs;
  int device;
  // launch shapes chosen by dpb_md_autotune (they never change results):
  // atoms (warps) per block of the mixed dE/dT kernel, and the mixed fitting
  // kernel's deep weight ring (1 CTA per SM) instead of the shallow one (2
  // CTAs per SM)
  mutable int dT_warps = 4;
  mutable int fit_deep = 0;
};

namespace dpb {
int eval_impl(const dpb_model *m, int precision, const float *pos, const int32_t *perm, int natoms, int nframes,
              const int *type_count, const float *box, const int32_t *nbrs, const int *sel, double *energy,
              float *atom_energy, float *force, double *virial, uint32_t *status, void *workspace,
              size_t ws_bytes, cudaStream_t st, const int32_t *seg = nullptr, int nseg = 0);
int nlist_build_impl(const float *pos, const int32_t *perm, int natoms, int nframes, int ntypes,
                     const int *type_count, const int *sel, const float box[3], const float *ref_box, float rc,
                     int32_t *nbrs, float *ref_pos, int32_t *counts, uint32_t *status, void *workspace,
                     size_t ws_bytes, const unsigned *gate, cudaStream_t stream, const float *dbox = nullptr,
                     int nl_warps = 8);
// Times the mixed dE/dT kernel at 2, 4 and 8 atoms per block on the
// workspace of the last mixed evaluation of NF atoms; *best gets the fastest.
int mixed_tune_dT(const DevModel &M, size_t NF, void *ws, cudaStream_t st, int *best);
// The same on the workspace of the last eval_impl call (F = nframes frames).
int eval_tune_dT(const dpb_model *m, int natoms, int nframes, void *workspace, cudaStream_t st, int *best);
}  // namespace dpb
