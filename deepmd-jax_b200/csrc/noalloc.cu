// Allocation-free evaluation entry point.
//
// dpb_eval needs a scratch workspace (per-atom descriptors, fitting-layer
// activations, force accumulators) that its caller allocates.  Some callers
// cannot allocate device memory at all: a host code that embeds the force
// field inside its own fixed memory pool, a plugin loaded into a process
// whose allocator forbids foreign cudaMalloc calls, or code running between
// steps where an allocation could fail or synchronise the device.  For them
// dpb_eval_noalloc evaluates with its scratch in a fixed-size array that is
// part of the library image on the device.
//
// Limits and behaviour:
//   * the scratch is kNoAllocScratchBytes (64 MiB); systems whose workspace
//     (dpb_eval_workspace_bytes) exceeds it are rejected with
//     DPB_ERR_SCRATCH_LIMIT before any device work;
//   * every GPU that loads the library holds this array until the process
//     exits;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress with that device current) and caches it, keyed
//     on the unique id of the CUDA context current at the time; make that
//     first call before capturing a stream into a CUDA graph.  A device reset
//     (cudaDeviceReset) or a re-created primary context gives a new context
//     id, so the next call looks the address up again instead of using a
//     stale one (the first call after a reset is then again a set-up call);
//   * all calls share the one array and the array keeps the last call's
//     contents: the evaluation zeroes every accumulator it needs, but two
//     calls that overlap on the GPU (different streams, or different host
//     threads) race on the scratch and corrupt each other — serialise them;
//   * no cudaMalloc, cudaFree or other allocating routine is called.
#include "internal.cuh"
#include <cuda.h>
#include <mutex>

namespace {
constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct ScratchEntry {
  unsigned long long ctx_id;  // unique id of the context the address belongs to
  void *ptr;
};
std::mutex g_noalloc_mu;
ScratchEntry g_noalloc[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context (0 when there is none
// yet).  The two driver calls are reached through the runtime's entry-point
// lookup, so the library needs no link against the driver library.
bool current_ctx_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || !a)
      return false;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qb != cudaDriverEntryPointSuccess || !b)
      return false;
    get_current = reinterpret_cast<CtxGetCurrentFn>(a);
    get_id = reinterpret_cast<CtxGetIdFn>(b);
  }
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS) return false;
  *id = 0;
  return !c || get_id(c, id) == CUDA_SUCCESS;
}
}  // namespace

extern "C" int dpb_eval_noalloc(const dpb_model *m, int precision, const float *pos, const int32_t *perm,
                                int natoms, int nframes, const int *type_count, const float *box,
                                const int32_t *nbrs, const int *sel, double *energy, float *atom_energy,
                                float *force, double *virial, uint32_t *status, void *stream) {
  if (!m || !pos || !box || !nbrs || !energy || !force || !status || !type_count || !sel || natoms <= 0 ||
      nframes <= 0)
    return DPB_ERR_INVALID_ARG;
  size_t need = 0;
  int rc = dpb_eval_workspace_bytes(m, natoms, nframes, &need);
  if (rc) return rc;
  if (need > kNoAllocScratchBytes) return DPB_ERR_SCRATCH_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DPB_ERR_CUDA;
  void *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned long long ctx = 0;
    if (!current_ctx_id(&ctx)) return DPB_ERR_CUDA;
    ScratchEntry &e = g_noalloc[dev];
    if (ctx == 0 || e.ptr == nullptr || e.ctx_id != ctx) {
      // The host-side symbol is a stand-in, not a device address: resolve the
      // device address of the array in the current context (this creates the
      // device's primary context if there is none yet), then key it on that
      // context.
      if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch) return DPB_ERR_CUDA;
      if (!current_ctx_id(&ctx) || ctx == 0) return DPB_ERR_CUDA;
      e.ptr = scratch;
      e.ctx_id = ctx;
    }
    scratch = e.ptr;
  }
  return dpb::eval_impl(m, precision, pos, perm, natoms, nframes, type_count, box, nbrs, sel, energy, atom_energy,
                        force, virial, status, scratch, kNoAllocScratchBytes, (cudaStream_t)stream);
}
