// Internal interfaces shared between the translation units of libdpb200.
#pragma once
#include "eval_common.cuh"
#include <vector>

struct dpb_model {
  dpb::DevModel dm;
  std::vector<void *> allocs;
  int device;
};

namespace dpb {
int eval_impl(const dpb_model *m, int precision, const float *pos, const int32_t *perm, int natoms, int nframes,
              const int *type_count, const float *box, const int32_t *nbrs, const int *sel, double *energy,
              float *atom_energy, float *force, double *virial, uint32_t *status, void *workspace,
              size_t ws_bytes, cudaStream_t st, const int32_t *seg = nullptr, int nseg = 0);
int nlist_build_impl(const float *pos, const int32_t *perm, int natoms, int nframes, int ntypes,
                     const int *type_count, const int *sel, const float box[3], const float *ref_box, float rc,
                     int32_t *nbrs, float *ref_pos, int32_t *counts, uint32_t *status, void *workspace,
                     size_t ws_bytes, const unsigned *gate, cudaStream_t stream, const float *dbox = nullptr);
}  // namespace dpb
