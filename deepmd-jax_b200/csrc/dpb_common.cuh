// Shared device helpers for libdpb200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include "../../include/dpb200.h"

namespace dpb {

constexpr int kMaxTypes = 4;
constexpr float kSqrt2 = 1.41421356237309515f;
constexpr float kSqrt3 = 1.73205080756887719f;

extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Optional per-kernel timing with CUDA events on the launching stream
// (diagnostics; off by default and never used inside graph capture).
enum ProfId : int {
  PROF_NLIST = 0,
  PROF_EMBED_FWD = 1,
  PROF_FIT = 2,
  PROF_EMBED_BWD = 3,
  PROF_INTEGRATE = 4,
  PROF_MIXED_EMBED_FWD = 5,
  PROF_MIXED_FIT = 6,
  PROF_MIXED_EMBED_BWD = 7,
  PROF_MIXED_DT = 8,
  PROF_COUNT = 9
};
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st);

#define DPB_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return DPB_ERR_CUDA;              \
  } while (0)

#define DPB_LAUNCH_CHECK()                                   \
  do {                                                       \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return DPB_ERR_CUDA;              \
  } while (0)

// jnp.mod / jnp.remainder: fmod, then add y where the remainder's sign differs
// from y's (y > 0 here).  fmod itself is only evaluated outside (-y, 2y):
// inside, fmod(x, y) is x for |x| < y and x - y for y <= x < 2y (an exact
// difference, Sterbenz), so the result is bit-identical for every x.
__device__ __forceinline__ float jmod(float x, float y) {
  float r;
  if (x > -y && x < y) r = x;
  else if (x >= y && x < 2.f * y) r = x - y;
  else r = fmodf(x, y);
  return (r != 0.f && r < 0.f) ? r + y : r;
}

// Minimum-image displacement of the reference's model path
// (deepmd_jax/utils.py:24-26): (d - L/2) mod L - L/2.
__device__ __forceinline__ float shift_ortho(float d, float L) {
  return jmod(d - 0.5f * L, L) - 0.5f * L;
}

// Periodic images that can lie within rc of a centre, per axis: the
// minimum-image displacement has |d| <= L/2, so |d + m L| < rc needs
// |m| <= floor(rc / L + 1/2).  Zero for boxes with L > 2 rc (minimum image
// only), as in the reference's lattice path (deepmd_jax/utils.py:66-78).
__device__ __forceinline__ int3 image_range(float3 L, float rc) {
  return make_int3((int)floorf(rc / L.x + 0.5f), (int)floorf(rc / L.y + 0.5f), (int)floorf(rc / L.z + 0.5f));
}

// Relative coordinate of neighbour j seen from centre i, the reference's
// neighbour-list branch (utils.py:79-82), plus the m-th lattice translation
// of the image box given by ni (m = 0 .. (2ni.x+1)(2ni.y+1)(2ni.z+1) - 1).
__device__ __forceinline__ float3 rel_coord(float3 ri, float3 rj, float3 L, int3 ni, int m) {
  float3 x;
  x.x = shift_ortho(rj.x - ri.x, L.x);
  x.y = shift_ortho(rj.y - ri.y, L.y);
  x.z = shift_ortho(rj.z - ri.z, L.z);
  if (ni.x | ni.y | ni.z) {
    const int ny = 2 * ni.y + 1, nz = 2 * ni.z + 1;
    const int a = m / (ny * nz) - ni.x, b = (m / nz) % ny - ni.y, c = m % nz - ni.z;
    x.x += (float)a * L.x;
    x.y += (float)b * L.y;
    x.z += (float)c * L.z;
  }
  return x;
}

// Per-row geometry of one (centre, neighbour) pair: the reference's guarded
// norm, smooth 1/r switch (utils.py:29-32) and its radial derivative.
struct RowGeom {
  float x[3];
  float r;      // guarded norm
  float s;      // s(r)
  float dsdr;   // ds/dr
};

__device__ __forceinline__ void row_geom(float3 x, float rcut, RowGeom &g) {
  g.x[0] = x.x; g.x[1] = x.y; g.x[2] = x.z;
  float gx = fabsf(x.x) > 1e-15f ? x.x : 1e-15f;
  float gy = fabsf(x.y) > 1e-15f ? x.y : 1e-15f;
  float gz = fabsf(x.z) > 1e-15f ? x.z : 1e-15f;
  float r = sqrtf(gx * gx + gy * gy + gz * gz);
  g.r = r;
  float t = r / rcut;
  float poly = 1.f - 3.f * t * t + 2.f * t * t * t;
  float den = r + 1e-15f;
  bool in = (r > 1e-14f) && (t < 1.f);
  g.s = in ? poly / den : 0.f;
  float dpoly = (-6.f * t + 6.f * t * t) / rcut;
  g.dsdr = in ? (dpoly * den - poly) / (den * den) : 0.f;
}

// 10-channel environment row (dpmodel.py:41-47) from s/std and x/(r+1e-16).
__device__ __forceinline__ void env_row(float sn, const float xh[3], float R[10]) {
  R[0] = sn;
  R[1] = kSqrt3 * sn * xh[0];
  R[2] = kSqrt3 * sn * xh[1];
  R[3] = kSqrt3 * sn * xh[2];
  R[4] = 3.f * sn * (xh[0] * xh[0] - (1.f / 3.f));
  R[5] = 3.f * sn * (xh[1] * xh[1] - (1.f / 3.f));
  R[6] = 3.f * sn * (xh[2] * xh[2] - (1.f / 3.f));
  R[7] = 3.f * kSqrt2 * sn * xh[0] * xh[2];
  R[8] = 3.f * kSqrt2 * sn * xh[1] * xh[0];
  R[9] = 3.f * kSqrt2 * sn * xh[2] * xh[1];
}

// Adjoint of the row: from dE/dR (10), dE/ds_tilde, produce dE/dx (3).
__device__ __forceinline__ void row_adjoint(const RowGeom &g, float inv_std, const float gR[10],
                                            float gst, float gx[3]) {
  float rp = g.r + 1e-16f;
  float inv_rp = 1.f / rp;
  float xh0 = g.x[0] * inv_rp, xh1 = g.x[1] * inv_rp, xh2 = g.x[2] * inv_rp;
  float sn = g.s * inv_std;
  float g_sn = gR[0] + kSqrt3 * (gR[1] * xh0 + gR[2] * xh1 + gR[3] * xh2) +
               3.f * (gR[4] * (xh0 * xh0 - (1.f / 3.f)) + gR[5] * (xh1 * xh1 - (1.f / 3.f)) +
                      gR[6] * (xh2 * xh2 - (1.f / 3.f))) +
               3.f * kSqrt2 * (gR[7] * xh0 * xh2 + gR[8] * xh1 * xh0 + gR[9] * xh2 * xh1);
  float gh0 = sn * (kSqrt3 * gR[1] + 6.f * gR[4] * xh0 + 3.f * kSqrt2 * (gR[7] * xh2 + gR[8] * xh1));
  float gh1 = sn * (kSqrt3 * gR[2] + 6.f * gR[5] * xh1 + 3.f * kSqrt2 * (gR[8] * xh0 + gR[9] * xh2));
  float gh2 = sn * (kSqrt3 * gR[3] + 6.f * gR[6] * xh2 + 3.f * kSqrt2 * (gR[7] * xh0 + gR[9] * xh1));
  float g_s = (g_sn + gst) * inv_std;
  float g_r = g_s * g.dsdr - (gh0 * g.x[0] + gh1 * g.x[1] + gh2 * g.x[2]) * inv_rp * inv_rp;
  float inv_r = 1.f / g.r;
  float d0 = fabsf(g.x[0]) > 1e-15f ? g.x[0] * inv_r : 0.f;
  float d1 = fabsf(g.x[1]) > 1e-15f ? g.x[1] * inv_r : 0.f;
  float d2 = fabsf(g.x[2]) > 1e-15f ? g.x[2] * inv_r : 0.f;
  gx[0] = gh0 * inv_rp + g_r * d0;
  gx[1] = gh1 * inv_rp + g_r * d1;
  gx[2] = gh2 * inv_rp + g_r * d2;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int type_of(int i, const int *offs, int ntypes) {
  int t = 0;
#pragma unroll
  for (int k = 1; k < kMaxTypes; ++k)
    if (k < ntypes && i >= offs[k]) t = k;
  return t;
}

}  // namespace dpb
