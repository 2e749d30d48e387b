// XLA FFI handlers over the libdpb200 C ABI, for registration as jax.ffi
// custom calls (jax.ffi.register_ffi_target(..., platform="CUDA")).
//
// They are the binding a deepmd-jax maintainer adds so that the reference's
// JAX code calls the sm_100a kernels without leaving XLA:
//   dpb_eval_ffi        replaces DPModel.energy_and_force inside the force
//                       function of deepmd_jax/md.py:292 (dpmodel.py:106-108)
//   dpb_nlist_build_ffi replaces typed_neighbor_list(...).allocate/update
//                       (deepmd_jax/md_utils.py:376-429) for one frame layout
// Buffers are XLA's (device pointers on XLA's stream); the model handle and
// the per-type counts / capacities are attributes.  Built against jaxlib's
// xla/ffi/api/ffi.h (Makefile in this directory; skipped without jaxlib).
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "xla/ffi/api/ffi.h"
#include "dpb200.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status_error(int rc, const char *what) {
  if (rc == DPB_OK) return ffi::Error::Success();
  return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + " failed with code " + std::to_string(rc));
}

bool copy_counts(ffi::Span<const int64_t> a, ffi::Span<const int64_t> b, int *ia, int *ib, int cap) {
  if (a.size() != b.size() || a.size() == 0 || (int)a.size() > cap) return false;
  for (size_t i = 0; i < a.size(); ++i) {
    ia[i] = (int)a[i];
    ib[i] = (int)b[i];
  }
  return true;
}

// pos (F,N,3) f32, perm (N) s32, box (F,3) f32, nbrs (F,N,S) s32 ->
// energy (F) f64, force (F,N,3) f32, virial (F,9) f64, status (1) u32,
// workspace (bytes) u8.  The kernels OR bits into the status word, and XLA
// does not zero result buffers, so the handler clears it first.
ffi::Error DpbEval(cudaStream_t st, ffi::Buffer<ffi::F32> pos, ffi::Buffer<ffi::S32> perm,
                   ffi::Buffer<ffi::F32> box, ffi::Buffer<ffi::S32> nbrs, ffi::ResultBuffer<ffi::F64> energy,
                   ffi::ResultBuffer<ffi::F32> force, ffi::ResultBuffer<ffi::F64> virial,
                   ffi::ResultBuffer<ffi::U32> status, ffi::ResultBuffer<ffi::U8> workspace, int64_t model,
                   int64_t precision, ffi::Span<const int64_t> type_count, ffi::Span<const int64_t> sel) {
  int tc[8], sl[8];
  if (!copy_counts(type_count, sel, tc, sl, 8))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "type_count and sel: one entry per type");
  const auto d = pos.dimensions();
  if (d.size() != 3 || d[2] != 3)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "pos must be (frames, atoms, 3)");
  if (cudaMemsetAsync(status->typed_data(), 0, sizeof(uint32_t), st) != cudaSuccess)
    return ffi::Error(ffi::ErrorCode::kInternal, "clearing the status word failed");
  const int rc = dpb_eval(reinterpret_cast<const dpb_model *>(model), (int)precision, pos.typed_data(),
                          perm.typed_data(), (int)d[1], (int)d[0], tc, box.typed_data(), nbrs.typed_data(), sl,
                          energy->typed_data(), nullptr, force->typed_data(), virial->typed_data(),
                          status->typed_data(), workspace->typed_data(), workspace->element_count(), st);
  return status_error(rc, "dpb_eval");
}

// pos (F,N,3) f32, perm (N) s32 -> nbrs (F,N,S) s32, ref_pos (F,N,3) f32,
// status (1) u32 (cleared here), workspace (bytes) u8; the box and the
// reference box are attributes (host values, as the C entry point takes them).
ffi::Error DpbNlistBuild(cudaStream_t st, ffi::Buffer<ffi::F32> pos, ffi::Buffer<ffi::S32> perm,
                         ffi::ResultBuffer<ffi::S32> nbrs, ffi::ResultBuffer<ffi::F32> ref_pos,
                         ffi::ResultBuffer<ffi::U32> status, ffi::ResultBuffer<ffi::U8> workspace,
                         ffi::Span<const int64_t> type_count, ffi::Span<const int64_t> sel,
                         ffi::Span<const float> box, ffi::Span<const float> ref_box, float rcut_plus_skin) {
  int tc[8], sl[8];
  if (!copy_counts(type_count, sel, tc, sl, 8))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "type_count and sel: one entry per type");
  if (box.size() != 3 || (ref_box.size() != 0 && ref_box.size() != 3))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "box (3,) and ref_box (3,) or empty");
  const auto d = pos.dimensions();
  if (d.size() != 3 || d[2] != 3)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "pos must be (frames, atoms, 3)");
  float b[3], rb[3];
  std::memcpy(b, box.begin(), sizeof b);
  if (ref_box.size() == 3) std::memcpy(rb, ref_box.begin(), sizeof rb);
  if (cudaMemsetAsync(status->typed_data(), 0, sizeof(uint32_t), st) != cudaSuccess)
    return ffi::Error(ffi::ErrorCode::kInternal, "clearing the status word failed");
  const int rc = dpb_nlist_build(pos.typed_data(), perm.typed_data(), (int)d[1], (int)d[0], (int)type_count.size(),
                                 tc, sl, b, ref_box.size() == 3 ? rb : nullptr, rcut_plus_skin,
                                 nbrs->typed_data(), ref_pos->typed_data(), nullptr, status->typed_data(),
                                 workspace->typed_data(), workspace->element_count(), st);
  return status_error(rc, "dpb_nlist_build");
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(dpb_eval_ffi, DpbEval,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F32>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Arg<ffi::Buffer<ffi::F32>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F32>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::U32>>()
                                  .Ret<ffi::Buffer<ffi::U8>>()
                                  .Attr<int64_t>("model")
                                  .Attr<int64_t>("precision")
                                  .Attr<ffi::Span<const int64_t>>("type_count")
                                  .Attr<ffi::Span<const int64_t>>("sel"));

XLA_FFI_DEFINE_HANDLER_SYMBOL(dpb_nlist_build_ffi, DpbNlistBuild,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F32>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::F32>>()
                                  .Ret<ffi::Buffer<ffi::U32>>()
                                  .Ret<ffi::Buffer<ffi::U8>>()
                                  .Attr<ffi::Span<const int64_t>>("type_count")
                                  .Attr<ffi::Span<const int64_t>>("sel")
                                  .Attr<ffi::Span<const float>>("box")
                                  .Attr<ffi::Span<const float>>("ref_box")
                                  .Attr<float>("rcut_plus_skin"));
