// Device-resident MD engine: velocity Verlet (NVE), Nose-Hoover chain (NVT),
// ring-polymer BAOAB with the PILE-L thermostat (PIMD NVT) and the MTK
// barostat with Nose-Hoover chains (NPT, orthorhombic, coupled axis groups).
//
// One step (the reference's scan body, deepmd_jax/md.py:763-795):
//   1. soft neighbour update: max drift of the canonical positions since the
//      last rebuild (md.py:697-739); the gated rebuild kernels run only when
//      it exceeds ((rcut + skin) - rcut) / 2 - 1e-6 * min(L);
//   2. status: NaN/Inf of positions or velocities (bit 16), list overflow
//      (bit 2) from the rebuild (md.py:618-641);
//   3. the integrator with one force evaluation;
//   4. optional trajectory frame.
// Every kernel of a step is enqueued on the caller's stream with no host
// synchronisation, so a chunk of steps can be captured into a CUDA graph.
// State lives in type-sorted order; positions are kept unwrapped (the
// reference's shift + min_image_unwrap, md.py:785-786, is the identity on a
// displacement of one step).
#include "internal.cuh"
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <numeric>

namespace dpb {

constexpr int kMaxChain = 8;
constexpr int kMaxBeads = 64;
constexpr int kBoxHist = 1024;  // steps of box history kept per dpb_md_run call (NPT)

struct MdScalars {
  unsigned drift_bits;
  unsigned rebuild;
  unsigned pad0, pad1;
  unsigned long long nrebuild;
  unsigned long long step;
  double ke;         // kinetic energy of the current momenta (FP64 reduction)
  double twork;      // cumulative thermostat work (PILE-L)
  double scale;      // momentum scale of the last Nose-Hoover substep
  double profile;    // EMA of rebuilds per step (md.py:733)
  double chain_ke;   // Nose-Hoover chain kinetic_energy field
  double dof;
  double xi[kMaxChain], pxi[kMaxChain], Q[kMaxChain];
  double com[4];     // centre-of-mass removal: sum of momenta (3), total mass
};

// ---------------------------------------------------------------- kernels
__global__ void k_md_begin(MdScalars *sc) {
  sc->drift_bits = 0u;
  sc->ke = 0.0;
  sc->com[0] = sc->com[1] = sc->com[2] = sc->com[3] = 0.0;
}

// Centre-of-mass removal (md.py:793-796): V = sum(mob m v) / sum(mob m) over
// the mobile atoms, v <- v - V for every atom (md.py:788-789), after the
// fixed atoms' momenta were masked (routine.py:130-134); mobile == NULL:
// every atom mobile.  k_com_sum: FP64 block sums of the mobile momenta and
// masses.
__global__ void k_com_sum(const float *__restrict__ mom, const float *__restrict__ mass,
                          const float *__restrict__ mobile, int N, MdScalars *sc) {
  __shared__ double part[4][8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < N && (!mobile || mobile[i] != 0.f)) {
    v[0] = mom[i * 3];
    v[1] = mom[i * 3 + 1];
    v[2] = mom[i * 3 + 2];
    v[3] = mass[i];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 4; ++k) part[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 4; ++k) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[k][w];
      atomicAdd(&sc->com[k], t);
    }
    if (blockIdx.x == 0) sc->ke = 0.0;  // recomputed from the new momenta by k_com_sub
  }
}

// k_com_sub: the subtraction and the kinetic energy of the new momenta.
// mask_fixed: the NVE / NVT wrapper zeroes the fixed atoms' momenta after the
// step (routine.py:130-134); the Langevin step keeps them (routine.py:46-107).
__global__ void k_com_sub(float *__restrict__ mom, const float *__restrict__ mass, const float *__restrict__ inv_mass,
                          const float *__restrict__ mobile, int mask_fixed, int N, MdScalars *sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float ke = 0.f;
  if (i < N) {
    const double f = (double)mass[i] / sc->com[3];
    const bool mob = !mobile || !mask_fixed || mobile[i] != 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float p = (float)((mob ? (double)mom[i * 3 + k] : 0.0) - f * sc->com[k]);
      mom[i * 3 + k] = p;
      ke += 0.5f * p * p * inv_mass[i];
    }
  }
  ke = warp_sum(ke);
  if ((threadIdx.x & 31) == 0 && ke != 0.f) atomicAdd(&sc->ke, (double)ke);
}

// Fixed atoms: zero force rows, the gradient that the stop_gradient on their
// coordinates removes (md.py:428-430); the mobile atoms' forces keep every
// term, including those through fixed neighbours.
__global__ void k_mask_rows(float *__restrict__ force, const float *__restrict__ mobile, int N) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < N * 3 && mobile[e / 3] == 0.f) force[e] = 0.f;
}

// Drift of canonical positions since the last rebuild, reference
// _drift_per_bead: (pos % box) * ref/box against reference_position, minimum
// image in the reference box (utils.py:11-18); also the NaN/Inf check of the
// pre-step state (md.py:638-640).
__global__ void k_md_drift(const float *__restrict__ pos, const float *__restrict__ mom,
                           const float *__restrict__ ref_pos, int NF, float3 L, float3 scale, float3 RB,
                           MdScalars *sc, uint32_t *status, const float *__restrict__ dbox) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (dbox) {  // NPT: the current box lives on the device (single frame)
    L = make_float3(dbox[0], dbox[1], dbox[2]);
    scale = make_float3(__fdiv_rn(RB.x, L.x), __fdiv_rn(RB.y, L.y), __fdiv_rn(RB.z, L.z));
  }
  float dn = 0.f;
  bool bad = false;
  if (g < NF) {
    const float *p = pos + (size_t)g * 3, *q = ref_pos + (size_t)g * 3, *v = mom + (size_t)g * 3;
    float d[3];
    const float Lv[3] = {L.x, L.y, L.z}, sv[3] = {scale.x, scale.y, scale.z}, rv[3] = {RB.x, RB.y, RB.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float c = jmod(p[k], Lv[k]) * sv[k];
      d[k] = jmod(c - q[k] - 0.5f * rv[k], rv[k]) - 0.5f * rv[k];
      bad |= !isfinite(p[k]) || !isfinite(v[k]);
    }
    dn = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(dn >= 0.f)) dn = 3.0e38f;  // NaN drift forces a rebuild (status bit 16 is set anyway)
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dn = fmaxf(dn, __shfl_xor_sync(0xffffffffu, dn, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&sc->drift_bits, __float_as_uint(dn));
  if (bad) atomicOr(status, DPB_ST_NONFINITE);
}

// NPT (dbox != NULL): the allowed drift shrinks with the box, safe scale
// 1.02 max(ref / box) (md.py:727-731), and status bit 1 flags a box that
// shrank past the skin or below 2 (rcut + skin) (md.py:630-634).
__global__ void k_md_decide(MdScalars *sc, float threshold, const float *__restrict__ dbox, float3 RB, float rc,
                            float skin, uint32_t *status) {
  if (dbox) {
    const float L[3] = {dbox[0], dbox[1], dbox[2]}, R[3] = {RB.x, RB.y, RB.z};
    float smax = 0.f, shrink = -1e30f, lmin = 1e30f, rmin = 1e30f;
    for (int a = 0; a < 3; ++a) {
      smax = fmaxf(smax, R[a] / L[a]);
      shrink = fmaxf(shrink, 1.f - L[a] / R[a]);
      lmin = fminf(lmin, L[a]);
      rmin = fminf(rmin, R[a]);
    }
    threshold = ((rc + skin) - rc * (smax * 1.02f)) / 2.f - rmin * 1e-6f;
    if (shrink > 0.8f * skin / (rc + skin) || lmin < 2.f * (rc + skin) * 1.02f) atomicOr(status, DPB_ST_BOX_SHRUNK);
  }
  const unsigned r = __uint_as_float(sc->drift_bits) > threshold ? 1u : 0u;
  sc->rebuild = r;
  sc->nrebuild += r;
  sc->profile = sc->profile * (1.0 - 1.0 / 100.0) + (1.0 / 100.0) * r;
  sc->step += 1ull;
}

// B + A of velocity Verlet: p = s p + dt/2 F ; r += dt p / m   (s: Nose-Hoover
// momentum scale of the first chain half step, 1 for NVE).
__global__ void k_vv_kick_drift(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                                const float *__restrict__ inv_mass, int N, int NF, float dt,
                                const MdScalars *__restrict__ sc, int use_scale) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NF * 3) return;
  const int atom = (e / 3) % N;
  const float s = use_scale ? (float)sc->scale : 1.f;
  const float p = mom[e] * s + 0.5f * dt * force[e];
  mom[e] = p;
  pos[e] = pos[e] + dt * p * inv_mass[atom];
}

// B of velocity Verlet and the kinetic-energy reduction; optional frame.
__global__ void k_vv_kick(float *__restrict__ mom, const float *__restrict__ force, const float *__restrict__ inv_mass,
                          int N, int NF, float dt, MdScalars *sc) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  float ke = 0.f;
  if (e < NF * 3) {
    const int atom = (e / 3) % N;
    const float p = mom[e] + 0.5f * dt * force[e];
    mom[e] = p;
    ke = 0.5f * p * p * inv_mass[atom];
  }
  ke = warp_sum(ke);
  __shared__ float part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = ke;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
    atomicAdd(&sc->ke, s);
  }
}

// One MTK Nose-Hoover chain substep of length delta/2 (jax_md
// nose_hoover_chain, wrapped by deepmd_jax/routine.py:147-158), FP64, on a
// chain (xi, p, Q) of L links over `dof` degrees of freedom with kinetic
// energy ke (updated); returns the momentum scale.
__device__ double nhc_half(double *xi, double *p, double *Q, double &ke, double dof, int L, double kT, double tau,
                           double delta) {
  // update_mass (kT fixed): Q = kT tau^2, Q0 *= DOF
  for (int m = 0; m < L; ++m) Q[m] = kT * tau * tau;
  Q[0] *= dof;
  const double d2 = delta / 2, d4 = d2 / 2, d8 = d4 / 2;
  const int M = L - 1;
  double G = p[M - 1] * p[M - 1] / Q[M - 1] - kT;
  p[M] += d4 * G;
  for (int m = M - 1; m > 0; --m) {
    G = p[m - 1] * p[m - 1] / Q[m - 1] - kT;
    const double sc_ = exp(-d8 * p[m + 1] / Q[m + 1]);
    p[m] = sc_ * (sc_ * p[m] + d4 * G);
  }
  G = 2.0 * ke - dof * kT;
  double s1 = exp(-d8 * p[1] / Q[1]);
  p[0] = s1 * (s1 * p[0] + d4 * G);
  const double scale = exp(-d2 * p[0] / Q[0]);
  ke *= scale * scale;
  for (int m = 0; m < L; ++m) xi[m] += d2 * p[m] / Q[m];
  G = 2.0 * ke - dof * kT;
  for (int m = 0; m < M; ++m) {
    const double sm = exp(-d8 * p[m + 1] / Q[m + 1]);
    p[m] = sm * (sm * p[m] + d4 * G);
    G = p[m] * p[m] / Q[m] - kT;
  }
  p[M] += d4 * G;
  return scale;
}

// which == 1: first half step, uses chain_ke; which == 2: second half step,
// chain_ke := KE of the current momenta first.
__global__ void k_nhc_substep(MdScalars *sc, int L, double kT, double tau, double delta, int which) {
  if (which == 2) sc->chain_ke = sc->ke;
  sc->scale = nhc_half(sc->xi, sc->pxi, sc->Q, sc->chain_ke, sc->dof, L, kT, tau, delta);
  if (which == 2) sc->ke = sc->chain_ke;  // the kinetic energy of the scaled momenta
}

__global__ void k_scale_mom(float *__restrict__ mom, int n, const MdScalars *__restrict__ sc) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) mom[e] = (float)(mom[e] * sc->scale);
}

__global__ void k_copy_frame(const float *__restrict__ src, float *__restrict__ dst, int n) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dst[e] = src[e];
}

// ---------------------------------------------------------------- NPT (MTK barostat)
// State of the barostat (deepmd_jax/routine.py:161-456): per coupled group g
// the log box scale Rb, its momentum Pb and mass Mb; the per-group dU/d(eps)
// of the last force evaluation (the reference caches it between steps); the
// per-axis sum of p^2/m and the per-axis factors of the two propagators.
struct NptScalars {
  int G;
  int ngrp[3];          // axes in group g
  int gid[3];           // group of axis a, -1 for a fixed axis
  double ref[3];        // the integrator's reference box
  double Rb[3], Pb[3], Mb[3];
  double dUde[3];
  double ke2[3];
  double a2[3], b2[3];  // exp_iL2: p <- p a2 + F b2
  double a1[3], b1[3];  // exp_iL1: r <- r a1 + (p / m) b1
  double pressure;
  double bxi[kMaxChain], bp[kMaxChain], bQ[kMaxChain];
  double bke, bdof;
  // NPT-PIMD: centroid drift e^y - 1 per axis, the internal-mode virial
  // sum(r - r_centroid) . f per axis of the last evaluation, barostat work
  double e1m1[3];
  double intvir[3];
  double btwork;
};

// sinh(x)/x by the series the reference uses (routine.py:290-292)
__device__ __forceinline__ double sinhx_x(double x) {
  const double x2 = x * x;
  return 1.0 + x2 / 6.0 + x2 * x2 / 120.0 + x2 * x2 * x2 / 5040.0 + x2 * x2 * x2 * x2 / 362880.0 +
         x2 * x2 * x2 * x2 * x2 / 39916800.0;
}

__device__ double npt_volume(const NptScalars *np) {
  double V = 1.0;
  for (int a = 0; a < 3; ++a) V *= np->ref[a] * (np->gid[a] >= 0 ? exp(np->Rb[np->gid[a]]) : 1.0);
  return V;
}

// G_g = KE2_g + (n_g / N_f) KE2_total - dU/deps_g - P V n_g   (routine.py:279-286)
__device__ void npt_box_force(const NptScalars *np, double V, double Nf, double *Gout) {
  const double tot = np->ke2[0] + np->ke2[1] + np->ke2[2];
  for (int g = 0; g < np->G; ++g) {
    double k = 0.0;
    for (int a = 0; a < 3; ++a)
      if (np->gid[a] == g) k += np->ke2[a];
    Gout[g] = k + (np->ngrp[g] / Nf) * tot - np->dUde[g] - np->pressure * V * np->ngrp[g];
  }
}

// Start of a step: box masses, barostat and thermostat half steps
// (routine.py:415-426); the thermostat scale is applied by k_npt_scale_ke2.
__global__ void k_npt_begin(MdScalars *sc, NptScalars *np, int Lt, int Lb, double kT, double tau_t, double tau_p,
                            double dt, int N) {
  for (int g = 0; g < np->G; ++g) np->Mb[g] = np->ngrp[g] * (N + 1.0) * kT * tau_p * tau_p;
  const double bs = nhc_half(np->bxi, np->bp, np->bQ, np->bke, np->bdof, Lb, kT, tau_p, dt);
  for (int g = 0; g < np->G; ++g) np->Pb[g] *= bs;
  sc->scale = nhc_half(sc->xi, sc->pxi, sc->Q, sc->chain_ke, sc->dof, Lt, kT, tau_t, dt);
  np->ke2[0] = np->ke2[1] = np->ke2[2] = 0.0;
}

// Per-axis sum of p^2 / m over the atoms (FP64 block sums), optionally after
// scaling the momenta; with ke != NULL also the kinetic energy.
__device__ void npt_reduce3(float v0, float v1, float v2, double *out, double *ke) {
  __shared__ float part[3][8];
  float v[3] = {v0, v1, v2};
#pragma unroll
  for (int a = 0; a < 3; ++a) v[a] = warp_sum(v[a]);
  if ((threadIdx.x & 31) == 0)
    for (int a = 0; a < 3; ++a) part[a][threadIdx.x >> 5] = v[a];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[3] = {0.0, 0.0, 0.0};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      for (int a = 0; a < 3; ++a) t[a] += part[a][w];
    for (int a = 0; a < 3; ++a) atomicAdd(&out[a], t[a]);
    if (ke) atomicAdd(ke, 0.5 * (t[0] + t[1] + t[2]));
  }
}

// Thermostat scale of the first half step, then the per-axis sums.
__global__ void k_npt_scale_ke2(float *__restrict__ mom, const float *__restrict__ inv_mass, int N,
                                const MdScalars *__restrict__ sc, NptScalars *np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float k[3] = {0.f, 0.f, 0.f};
  if (i < N) {
    const float s = (float)sc->scale, im = inv_mass[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float p = mom[i * 3 + a] * s;
      mom[i * 3 + a] = p;
      k[a] = p * p * im;
    }
  }
  npt_reduce3(k[0], k[1], k[2], np->ke2, nullptr);
}

// First barostat kick with the cached dU/deps, the box update and the
// propagator factors (routine.py:383-396, 294-311).
__global__ void k_npt_box1(NptScalars *np, float *boxd, double dt, int N) {
  const double Nf = 3.0 * N;
  double Ge[3];
  npt_box_force(np, npt_volume(np), Nf, Ge);
  double Vb[3] = {0.0, 0.0, 0.0}, tr = 0.0;
  for (int g = 0; g < np->G; ++g) {
    np->Pb[g] += 0.5 * dt * Ge[g];
    Vb[g] = np->Pb[g] / np->Mb[g];
    tr += np->ngrp[g] * Vb[g];
  }
  for (int a = 0; a < 3; ++a) {
    const double va = np->gid[a] >= 0 ? Vb[np->gid[a]] : 0.0;
    const double x = (va + tr / Nf) * (0.5 * dt), x2 = x / 2;
    np->a2[a] = exp(-x);
    np->b2[a] = 0.5 * dt * sinhx_x(x2) * exp(-x2);
    const double y = va * dt, y2 = y / 2;
    np->a1[a] = exp(y);
    np->b1[a] = dt * exp(y2) * sinhx_x(y2);
  }
  for (int g = 0; g < np->G; ++g) np->Rb[g] += Vb[g] * dt;
  for (int a = 0; a < 3; ++a)
    boxd[a] = (float)(np->ref[a] * (np->gid[a] >= 0 ? exp(np->Rb[np->gid[a]]) : 1.0));
  np->ke2[0] = np->ke2[1] = np->ke2[2] = 0.0;
}

// p <- exp_iL2(p, F); r <- exp_iL1(r, p / m)
__global__ void k_npt_move(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                           const float *__restrict__ inv_mass, int N3, const NptScalars *__restrict__ np) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N3) return;
  const int a = e % 3;
  const float p = mom[e] * (float)np->a2[a] + force[e] * (float)np->b2[a];
  mom[e] = p;
  pos[e] = pos[e] * (float)np->a1[a] + p * inv_mass[e / 3] * (float)np->b1[a];
}

// p <- exp_iL2(p, F) with the new forces; per-axis sums and the kinetic energy.
__global__ void k_npt_kick2(float *__restrict__ mom, const float *__restrict__ force,
                            const float *__restrict__ inv_mass, int N, MdScalars *sc, NptScalars *np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float k[3] = {0.f, 0.f, 0.f};
  if (i < N) {
    const float im = inv_mass[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float p = mom[i * 3 + a] * (float)np->a2[a] + force[i * 3 + a] * (float)np->b2[a];
      mom[i * 3 + a] = p;
      k[a] = p * p * im;
    }
  }
  npt_reduce3(k[0], k[1], k[2], np->ke2, &sc->ke);
}

// Second barostat kick with the new dU/deps, then the thermostat and
// barostat half steps (routine.py:398-436); the thermostat scale is applied
// by k_scale_mom.
__global__ void k_npt_end(MdScalars *sc, NptScalars *np, const double *__restrict__ virial, int Lt, int Lb,
                          double kT, double tau_t, double tau_p, double dt, int N) {
  for (int g = 0; g < np->G; ++g) np->dUde[g] = 0.0;
  for (int a = 0; a < 3; ++a)
    if (np->gid[a] >= 0) np->dUde[np->gid[a]] -= virial[a * 3 + a];  // dU/deps_a = -W_aa
  double Ge[3];
  npt_box_force(np, npt_volume(np), 3.0 * N, Ge);
  double kb = 0.0;
  for (int g = 0; g < np->G; ++g) {
    np->Pb[g] += 0.5 * dt * Ge[g];
    kb += 0.5 * np->Pb[g] * np->Pb[g] / np->Mb[g];
  }
  np->bke = kb;
  sc->chain_ke = sc->ke;
  sc->scale = nhc_half(sc->xi, sc->pxi, sc->Q, sc->chain_ke, sc->dof, Lt, kT, tau_t, dt);
  sc->ke = sc->chain_ke;  // the kinetic energy of the momenta after k_scale_mom
  const double bs = nhc_half(np->bxi, np->bp, np->bQ, np->bke, np->bdof, Lb, kT, tau_p, dt);
  for (int g = 0; g < np->G; ++g) np->Pb[g] *= bs;
}

// Philox4x32-10 (Salmon et al., SC'11) and Box-Muller normals; stream:
// counter = (q, step, tag, 0) for element block q, key = seed.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ float philox_normal(unsigned long long seed, unsigned step, unsigned tag,
                                               unsigned e) {
  const uint4 x = philox(make_uint4(e >> 2, step, tag, 0u), make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
  const unsigned k = e & 3u;
  const unsigned ua = (k < 2) ? x.x : x.z, ub = (k < 2) ? x.y : x.w;
  const float u1 = (float)ua * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
  const float u2 = (float)ub * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
  const float r = sqrtf(-2.f * logf(u1));
  float sn, cs;
  sincospif(2.f * u2, &sn, &cs);
  return (k & 1u) ? r * sn : r * cs;
}

// BAOAB Langevin up to the force evaluation (routine.py:81-103): B (dt/2
// kick), A (dt/2 drift), O (p = c1 p + c2 sqrt(m) xi, xi zero on fixed atoms,
// the kinetic-energy change added to the thermostat work), A.  Noise: Philox
// stream (seed, step, tag 3), element atom * 3 + component in sorted order.
// shift_im is 1/m with fixed atoms at 0 (the masked shift, md.py:231-234).
__global__ void k_lan_baoa(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                           const float *__restrict__ mass, const float *__restrict__ inv_mass,
                           const float *__restrict__ shift_im, const float *__restrict__ mobile, int N, float dt,
                           float c1, float c2, unsigned long long seed, MdScalars *sc) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double dw = 0.0;
  if (e < N * 3) {
    const int atom = e / 3;
    const float sim = shift_im[atom];
    const float p = mom[e] + 0.5f * dt * force[e];
    float r = pos[e] + 0.5f * dt * p * sim;
    float xi = philox_normal(seed, (unsigned)sc->step, 3u, (unsigned)e);
    if (mobile) xi *= mobile[atom];
    const float pn = c1 * p + c2 * sqrtf(mass[atom]) * xi;
    // kinetic-energy change in FP64, factored to avoid the cancellation of pn^2 - p^2
    dw = 0.5 * ((double)pn - (double)p) * ((double)pn + (double)p) * (double)inv_mass[atom];
    r += 0.5f * dt * pn * sim;
    pos[e] = r;
    mom[e] = pn;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dw += __shfl_xor_sync(0xffffffffu, dw, o);
  if ((threadIdx.x & 31) == 0 && dw != 0.0) atomicAdd(&sc->twork, dw);
}

struct PimdParams {
  int P, N;
  float dt, kT;
  float3 L;
  unsigned long long seed;
  unsigned tag;
};

// B (dt/2 kick), A (dt/2 exact free ring), O (PILE-L), A (dt/2) for one
// (atom, component) column of all beads (deepmd_jax/pimd.py:160-205), then
// the per-bead min_image_unwrap against the previous step (md.py:785).
// C[b][k] (primitive <- normal mode) in shared memory; FP32 columns.
__global__ void k_pimd_baoa(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                            const float *__restrict__ mass, const float *__restrict__ Cg,
                            const float *__restrict__ freqs, const float *__restrict__ gamma, PimdParams pp,
                            MdScalars *sc) {
  __shared__ float C[kMaxBeads * kMaxBeads];
  const int P = pp.P;
  for (int e = threadIdx.x; e < P * P; e += blockDim.x) C[e] = Cg[e];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;  // atom * 3 + comp
  const int N3 = pp.N * 3;
  double dke = 0.0;
  if (col < N3) {
    const int atom = col / 3, comp = col - atom * 3;
    const float Lc = comp == 0 ? pp.L.x : (comp == 1 ? pp.L.y : pp.L.z);
    const float m = mass[atom];
    float R[kMaxBeads], Pm[kMaxBeads], R0[kMaxBeads], Q[kMaxBeads], Pn[kMaxBeads];
    for (int b = 0; b < P; ++b) {
      R0[b] = pos[(size_t)b * N3 + col];
      Pm[b] = mom[(size_t)b * N3 + col] + 0.5f * pp.dt * force[(size_t)b * N3 + col];
    }
    // unwrap across beads onto bead 0's image (pimd.py:210-226)
    for (int b = 0; b < P; ++b) {
      const float d = R0[b] - R0[0];
      R[b] = R0[0] + (d - Lc * rintf(d / Lc));
    }
    const float h = 0.5f * pp.dt;
    for (int pass = 0; pass < 3; ++pass) {
      // to normal modes: Q = C^T R, Pn = C^T P
      for (int k = 0; k < P; ++k) {
        float q = 0.f, pn = 0.f;
        for (int b = 0; b < P; ++b) {
          q = fmaf(C[b * P + k], R[b], q);
          pn = fmaf(C[b * P + k], Pm[b], pn);
        }
        Q[k] = q;
        Pn[k] = pn;
      }
      if (pass == 1) {
        // O: PILE-L in normal modes (pimd.py:92-111)
        for (int k = 0; k < P; ++k) {
          const float c1 = expf(-gamma[k] * pp.dt);
          const float c2 = sqrtf(fmaxf(pp.kT * P * (1.f - c1 * c1), 0.f));
          const unsigned e = (unsigned)(k * N3 + col);
          Pn[k] = c1 * Pn[k] + c2 * sqrtf(m) * philox_normal(pp.seed, (unsigned)sc->step, pp.tag, e);
        }
      } else {
        // A: exact free ring-polymer propagation for h (pimd.py:160-179)
        Q[0] = Q[0] + h * Pn[0] / m;
        for (int k = 1; k < P; ++k) {
          const float w = freqs[k];
          float sn, cs;
          sincosf(w * h, &sn, &cs);
          const float q = Q[k] * cs + Pn[k] * sn / (m * w);
          const float pn = Pn[k] * cs - m * w * Q[k] * sn;
          Q[k] = q;
          Pn[k] = pn;
        }
      }
      // back to primitive coordinates
      for (int b = 0; b < P; ++b) {
        float r = 0.f, pv = 0.f;
        for (int k = 0; k < P; ++k) {
          r = fmaf(C[b * P + k], Q[k], r);
          pv = fmaf(C[b * P + k], Pn[k], pv);
        }
        if (pass == 1) {
          dke += 0.5 * ((double)pv - (double)Pm[b]) * ((double)pv + (double)Pm[b]) / (double)m;
        } else {
          R[b] = r;
        }
        Pm[b] = pv;
      }
    }
    for (int b = 0; b < P; ++b) {
      // min_image_unwrap against the previous step's bead position
      const float d = R[b] - R0[b];
      pos[(size_t)b * N3 + col] = R0[b] + (jmod(d + 0.5f * Lc, Lc) - 0.5f * Lc);
      mom[(size_t)b * N3 + col] = Pm[b];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dke += __shfl_xor_sync(0xffffffffu, dke, o);
  if ((threadIdx.x & 31) == 0 && dke != 0.0) atomicAdd(&sc->twork, dke);
}

// ---------------------------------------------------------------- NPT-PIMD
// deepmd_jax/pimd.py:255-518: Parrinello-Rahman on the centroid mode only,
// internal modes propagated exactly, PILE-L on the beads and a Langevin
// barostat on the box momenta; the barostat is driven by the centroid
// momenta and the centroid-virial dU/d(eps).  Per step: k_nptp_begin (half
// box kick, propagator factors, half box update), k_nptp_a (B, A, O),
// k_nptp_mid (box Langevin, half box update), k_nptp_b (A, unwrap), forces,
// k_nptp_c (internal virial, B, centroid p^2/m), k_nptp_end (dU/d(eps), half
// box kick).  All beads share the box (every row of boxd).

// Box of the current log scales into all P rows of boxd.
__device__ void nptp_set_box(const NptScalars *np, float *boxd, int P) {
  for (int a = 0; a < 3; ++a) {
    const float L = (float)(np->ref[a] * (np->gid[a] >= 0 ? exp(np->Rb[np->gid[a]]) : 1.0));
    for (int b = 0; b < P; ++b) boxd[b * 3 + a] = L;
  }
}

// Factors of the centroid kick exp_iL2_pimd (pimd.py:375-383) and of the
// half-step centroid drift exp_iL1_centroid_pimd (pimd.py:385-398) from the
// current box momenta.
__device__ void nptp_factors(NptScalars *np, double h, double Nf) {
  double Vb[3] = {0.0, 0.0, 0.0}, tr = 0.0;
  for (int g = 0; g < np->G; ++g) {
    Vb[g] = np->Pb[g] / np->Mb[g];
    tr += np->ngrp[g] * Vb[g];
  }
  for (int a = 0; a < 3; ++a) {
    const double va = np->gid[a] >= 0 ? Vb[np->gid[a]] : 0.0;
    const double x = (va + tr / Nf) * h;
    np->a2[a] = exp(-x);
    np->b2[a] = h * sinhx_x(x / 2) * exp(-x / 2);
    const double y = va * h;
    np->e1m1[a] = expm1(y);
    np->b1[a] = h * exp(y / 2) * sinhx_x(y / 2);
  }
}

__global__ void k_nptp_begin(NptScalars *np, float *boxd, int P, double dt, int N) {
  const double h = 0.5 * dt, Nf = 3.0 * N;
  double Ge[3];
  npt_box_force(np, npt_volume(np), Nf, Ge);
  for (int g = 0; g < np->G; ++g) np->Pb[g] += h * Ge[g];
  nptp_factors(np, h, Nf);
  for (int g = 0; g < np->G; ++g) np->Rb[g] += h * np->Pb[g] / np->Mb[g];
  nptp_set_box(np, boxd, P);
}

// Langevin barostat (pimd.py:486-491; normals of tag 2, element g), second
// half box update, factors for the second drift and the last kick.
__global__ void k_nptp_mid(const MdScalars *sc, NptScalars *np, float *boxd, int P, double dt, double kT,
                           double gamma_box, unsigned long long seed, int N) {
  const double h = 0.5 * dt;
  const double c1 = exp(-gamma_box * dt), c2 = sqrt(fmax(kT * (1.0 - c1 * c1), 0.0));
  double dw = 0.0;
  for (int g = 0; g < np->G; ++g) {
    const double old = np->Pb[g];
    np->Pb[g] = c1 * old + c2 * sqrt(np->Mb[g]) * (double)philox_normal(seed, (unsigned)sc->step, 2u, (unsigned)g);
    dw += 0.5 * (np->Pb[g] * np->Pb[g] - old * old) / np->Mb[g];
  }
  np->btwork += dw;
  for (int g = 0; g < np->G; ++g) np->Rb[g] += h * np->Pb[g] / np->Mb[g];
  nptp_set_box(np, boxd, P);
  nptp_factors(np, h, 3.0 * N);
  for (int a = 0; a < 3; ++a) np->ke2[a] = np->intvir[a] = 0.0;
}

// dU/d(eps_g) = (sum_b sum_{a in g} -W_b,aa + sum_{a in g} internal_a) / P
// (pimd.py:332-350), then (kick) the last half box kick.
__global__ void k_nptp_end(NptScalars *np, const double *__restrict__ virial, int P, double dt, int N, int kick) {
  for (int g = 0; g < np->G; ++g) np->dUde[g] = 0.0;
  for (int a = 0; a < 3; ++a) {
    if (np->gid[a] < 0) continue;
    double w = 0.0;
    for (int b = 0; b < P; ++b) w -= virial[b * 9 + a * 3 + a];
    np->dUde[np->gid[a]] += (w + np->intvir[a]) / P;
  }
  if (kick) {
    double Ge[3];
    npt_box_force(np, npt_volume(np), 3.0 * N, Ge);
    for (int g = 0; g < np->G; ++g) np->Pb[g] += 0.5 * dt * Ge[g];
  }
  for (int a = 0; a < 3; ++a) np->intvir[a] = 0.0;
}

// Beads of one column unwrapped onto bead 0's image (pimd.py:210-226).
__device__ __forceinline__ void ring_unwrap(const float *R, float *U, int P, float Lc) {
  for (int b = 0; b < P; ++b) {
    const float d = R[b] - R[0];
    U[b] = R[0] + (d - Lc * rintf(d / Lc));
  }
}

// exp_iL2_pimd of one column: centroid p_c e^-x + h F_c sinh(x/2)/(x/2) e^(-x/2),
// internal modes p - p_c + h (F - F_c).
__device__ __forceinline__ void nptp_kick(float *Pm, const float *F, int P, float a2, float b2, float h) {
  float pc = 0.f, fc = 0.f;
  for (int b = 0; b < P; ++b) {
    pc += Pm[b];
    fc += F[b];
  }
  pc /= (float)P;
  fc /= (float)P;
  const float pcn = pc * a2 + fc * b2;
  for (int b = 0; b < P; ++b) Pm[b] = pcn + (Pm[b] - pc) + h * (F[b] - fc);
}

// Centroid drift: every bead moves by r_c (e^y - 1) + b1 v_c.
__device__ __forceinline__ void nptp_drift(float *R, const float *Pm, float m, int P, float Lc, float e1m1,
                                           float b1) {
  float U[kMaxBeads];
  ring_unwrap(R, U, P, Lc);
  float rc = 0.f, pc = 0.f;
  for (int b = 0; b < P; ++b) {
    rc += U[b];
    pc += Pm[b];
  }
  rc /= (float)P;
  const float d = rc * e1m1 + b1 * (pc / (float)P) / m;
  for (int b = 0; b < P; ++b) R[b] += d;
}

// Exact free propagation of the internal ring-polymer modes for h; the
// centroid normal mode stays (pimd.py:400-415).  C[b][k] in shared memory.
__device__ __forceinline__ void nptp_ring(float *R, float *Pm, float m, int P, float Lc, const float *C,
                                          const float *__restrict__ freqs, float h) {
  float U[kMaxBeads], Q[kMaxBeads], Pn[kMaxBeads];
  ring_unwrap(R, U, P, Lc);
  for (int k = 0; k < P; ++k) {
    float q = 0.f, pn = 0.f;
    for (int b = 0; b < P; ++b) {
      q = fmaf(C[b * P + k], U[b], q);
      pn = fmaf(C[b * P + k], Pm[b], pn);
    }
    Q[k] = q;
    Pn[k] = pn;
  }
  for (int k = 1; k < P; ++k) {
    const float w = freqs[k];
    float sn, cs;
    sincosf(w * h, &sn, &cs);
    const float q = Q[k] * cs + Pn[k] * sn / (m * w);
    const float pn = Pn[k] * cs - m * w * Q[k] * sn;
    Q[k] = q;
    Pn[k] = pn;
  }
  for (int b = 0; b < P; ++b) {
    float r = 0.f, pv = 0.f;
    for (int k = 0; k < P; ++k) {
      r = fmaf(C[b * P + k], Q[k], r);
      pv = fmaf(C[b * P + k], Pn[k], pv);
    }
    R[b] = r;
    Pm[b] = pv;
  }
}

// B (centroid Parrinello-Rahman kick), A (centroid drift + internal ring,
// first box), O (PILE-L, the stream of k_pimd_baoa) of one column.
__global__ void k_nptp_a(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                         float *__restrict__ prev, const float *__restrict__ mass, const float *__restrict__ Cg,
                         const float *__restrict__ freqs, const float *__restrict__ gamma, PimdParams pp,
                         const NptScalars *__restrict__ np, const float *__restrict__ boxd, MdScalars *sc) {
  __shared__ float C[kMaxBeads * kMaxBeads];
  const int P = pp.P;
  for (int e = threadIdx.x; e < P * P; e += blockDim.x) C[e] = Cg[e];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int N3 = pp.N * 3;
  double dke = 0.0;
  if (col < N3) {
    const int atom = col / 3, comp = col - atom * 3;
    const float Lc = boxd[comp], m = mass[atom], h = 0.5f * pp.dt;
    float R[kMaxBeads], Pm[kMaxBeads], F[kMaxBeads], Pn[kMaxBeads];
    for (int b = 0; b < P; ++b) {
      R[b] = pos[(size_t)b * N3 + col];
      prev[(size_t)b * N3 + col] = R[b];
      Pm[b] = mom[(size_t)b * N3 + col];
      F[b] = force[(size_t)b * N3 + col];
    }
    nptp_kick(Pm, F, P, (float)np->a2[comp], (float)np->b2[comp], h);
    nptp_drift(R, Pm, m, P, Lc, (float)np->e1m1[comp], (float)np->b1[comp]);
    nptp_ring(R, Pm, m, P, Lc, C, freqs, h);
    // O: PILE-L in normal modes (pimd.py:471-479)
    for (int k = 0; k < P; ++k) {
      float pn = 0.f;
      for (int b = 0; b < P; ++b) pn = fmaf(C[b * P + k], Pm[b], pn);
      const float c1 = expf(-gamma[k] * pp.dt);
      const float c2 = sqrtf(fmaxf(pp.kT * P * (1.f - c1 * c1), 0.f));
      Pn[k] = c1 * pn + c2 * sqrtf(m) * philox_normal(pp.seed, (unsigned)sc->step, pp.tag, (unsigned)(k * N3 + col));
    }
    for (int b = 0; b < P; ++b) {
      float pv = 0.f;
      for (int k = 0; k < P; ++k) pv = fmaf(C[b * P + k], Pn[k], pv);
      dke += 0.5 * ((double)pv - (double)Pm[b]) * ((double)pv + (double)Pm[b]) / (double)m;
      pos[(size_t)b * N3 + col] = R[b];
      mom[(size_t)b * N3 + col] = pv;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dke += __shfl_xor_sync(0xffffffffu, dke, o);
  if ((threadIdx.x & 31) == 0 && dke != 0.0) atomicAdd(&sc->twork, dke);
}

// A (centroid drift + internal ring, second box), then the per-bead
// min_image_unwrap against the step's initial positions (md.py:785).
__global__ void k_nptp_b(float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ prev,
                         const float *__restrict__ mass, const float *__restrict__ Cg, const float *__restrict__ freqs,
                         PimdParams pp, const NptScalars *__restrict__ np, const float *__restrict__ boxd) {
  __shared__ float C[kMaxBeads * kMaxBeads];
  const int P = pp.P;
  for (int e = threadIdx.x; e < P * P; e += blockDim.x) C[e] = Cg[e];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int N3 = pp.N * 3;
  if (col >= N3) return;
  const int atom = col / 3, comp = col - atom * 3;
  const float Lc = boxd[comp], m = mass[atom], h = 0.5f * pp.dt;
  float R[kMaxBeads], Pm[kMaxBeads];
  for (int b = 0; b < P; ++b) {
    R[b] = pos[(size_t)b * N3 + col];
    Pm[b] = mom[(size_t)b * N3 + col];
  }
  nptp_drift(R, Pm, m, P, Lc, (float)np->e1m1[comp], (float)np->b1[comp]);
  nptp_ring(R, Pm, m, P, Lc, C, freqs, h);
  for (int b = 0; b < P; ++b) {
    const float r0 = prev[(size_t)b * N3 + col];
    pos[(size_t)b * N3 + col] = r0 + (jmod(R[b] - r0 + 0.5f * Lc, Lc) - 0.5f * Lc);
    mom[(size_t)b * N3 + col] = Pm[b];
  }
}

// Internal-mode virial sum_b (r_b - r_c) f_b per axis (pimd.py:344-349),
// then (kick) the last centroid kick, the centroid p_c^2 / m per axis and
// (ke) the kinetic energy of all beads.
__global__ void k_nptp_c(const float *__restrict__ pos, float *__restrict__ mom, const float *__restrict__ force,
                         const float *__restrict__ mass, PimdParams pp, NptScalars *np,
                         const float *__restrict__ boxd, MdScalars *sc, int kick, int ke) {
  const int P = pp.P;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int N3 = pp.N * 3;
  float iv[3] = {0.f, 0.f, 0.f}, k2[3] = {0.f, 0.f, 0.f}, kin = 0.f;
  if (col < N3) {
    const int atom = col / 3, comp = col - atom * 3;
    const float Lc = boxd[comp], m = mass[atom];
    float R[kMaxBeads], U[kMaxBeads], Pm[kMaxBeads], F[kMaxBeads];
    for (int b = 0; b < P; ++b) {
      R[b] = pos[(size_t)b * N3 + col];
      Pm[b] = mom[(size_t)b * N3 + col];
      F[b] = force[(size_t)b * N3 + col];
    }
    ring_unwrap(R, U, P, Lc);
    float rc = 0.f;
    for (int b = 0; b < P; ++b) rc += U[b];
    rc /= (float)P;
    float v = 0.f;
    for (int b = 0; b < P; ++b) v = fmaf(U[b] - rc, F[b], v);
    iv[comp] = v;
    if (kick) {
      nptp_kick(Pm, F, P, (float)np->a2[comp], (float)np->b2[comp], 0.5f * pp.dt);
      for (int b = 0; b < P; ++b) mom[(size_t)b * N3 + col] = Pm[b];
    }
    float pc = 0.f;
    for (int b = 0; b < P; ++b) {
      pc += Pm[b];
      kin += 0.5f * Pm[b] * Pm[b] / m;
    }
    pc /= (float)P;
    k2[comp] = pc * pc / m;
  }
  npt_reduce3(iv[0], iv[1], iv[2], np->intvir, nullptr);
  __syncthreads();
  npt_reduce3(k2[0], k2[1], k2[2], np->ke2, nullptr);
  if (ke) {
    kin = warp_sum(kin);
    if ((threadIdx.x & 31) == 0 && kin != 0.f) atomicAdd(&sc->ke, (double)kin);
  }
}

}  // namespace dpb

using namespace dpb;

struct dpb_md {
  const dpb_model *model;
  dpb_md_desc d;
  int N, P, ntypes, S;
  int type_count[kMaxTypes], sel[kMaxTypes];
  std::vector<int> perm;   // sorted index -> user index
  std::vector<float> mass_sorted;
  float box[3];
  float threshold;
  double kT;
  // device
  float *pos = nullptr, *mom = nullptr, *force = nullptr, *inv_mass = nullptr, *mass = nullptr;
  float *ref_pos = nullptr, *boxd = nullptr;
  int32_t *nbrs = nullptr;
  uint32_t *status = nullptr;
  double *energy = nullptr, *virial = nullptr;
  MdScalars *sc = nullptr;
  NptScalars *np = nullptr, *s_np = nullptr;  // NPT barostat state and its snapshot
  float *s_box = nullptr;
  float *prev = nullptr;  // NPT-PIMD: positions at the start of the step
  int nl_warps = 8;       // centres (warps) per block of the neighbour search (dpb_md_autotune)
  float *box_hist = nullptr;  // NPT: box after each step of the last dpb_md_run (kBoxHist rows)
  float *mobile = nullptr;      // fixed atoms: 1 mobile / 0 fixed per sorted atom (NULL: none fixed)
  float *shift_inv_mass = nullptr;  // fixed atoms: 1/m of mobile atoms, 0 for fixed (the masked shift)
  int n_mobile = 0;
  std::vector<float> mobile_sorted;  // host copy of `mobile`
  float *C = nullptr, *freqs = nullptr, *gamma = nullptr;
  void *nl_ws = nullptr, *ev_ws = nullptr;
  size_t nl_ws_bytes = 0, ev_ws_bytes = 0;
  // snapshot for chunk re-runs
  float *s_pos = nullptr, *s_mom = nullptr, *s_force = nullptr, *s_ref = nullptr;
  MdScalars *s_sc = nullptr;
  // trajectory frames (dpb_md_traj_frames): sorted slot and float64 mass
  // (eV fs^2 / A^2) of each atom in user order
  int32_t *user_slot = nullptr;
  double *user_mass = nullptr;
  std::vector<void *> allocs;
};

static int md_alloc(dpb_md *m, void **p, size_t bytes) {
  if (cudaMalloc(p, bytes < 256 ? 256 : bytes) != cudaSuccess) return DPB_ERR_CUDA;
  m->allocs.push_back(*p);
  return DPB_OK;
}

static int md_alloc_lists(dpb_md *m) {
  size_t NF = (size_t)m->N * m->P;
  if (m->nbrs) {
    cudaFree(m->nbrs);
    m->allocs.erase(std::remove(m->allocs.begin(), m->allocs.end(), (void *)m->nbrs), m->allocs.end());
    m->nbrs = nullptr;
  }
  return md_alloc(m, (void **)&m->nbrs, NF * m->S * sizeof(int32_t));
}

extern "C" int dpb_md_create(const dpb_model *model, const dpb_md_desc *d, dpb_md **out) {
  if (!model || !d || !out || d->natoms <= 0 || d->nbeads <= 0 || !d->type_idx || !d->mass_per_type || !d->sel)
    return DPB_ERR_INVALID_ARG;
  if (d->routine < DPB_MD_NVE || d->routine > DPB_MD_NVT_LANGEVIN) return DPB_ERR_INVALID_ARG;
  if (d->routine == DPB_MD_NVT_LANGEVIN && !(d->tau_t > 0.0)) return DPB_ERR_UNSUPPORTED;
  const bool has_box = d->routine == DPB_MD_NPT_NHC || d->routine == DPB_MD_NPT_PIMD;
  const bool pimd = d->routine == DPB_MD_PIMD_PILE || d->routine == DPB_MD_NPT_PIMD;
  if (d->routine == DPB_MD_NPT_NHC && (d->nbeads != 1 || d->chain_length < 2 || d->chain_length > kMaxChain ||
                                       d->chain_length_p < 2 || d->chain_length_p > kMaxChain))
    return DPB_ERR_UNSUPPORTED;
  if (has_box) {
    if (!(d->tau_p > 0.0)) return DPB_ERR_UNSUPPORTED;
    int G = -1;
    for (int a = 0; a < 3; ++a) {
      if (d->couple_groups[a] < -1 || d->couple_groups[a] > 2) return DPB_ERR_INVALID_ARG;
      G = std::max(G, d->couple_groups[a]);
    }
    if (G < 0) return DPB_ERR_INVALID_ARG;  // no moving axis: use NVT
    for (int g = 0; g <= G; ++g)
      if (d->couple_groups[0] != g && d->couple_groups[1] != g && d->couple_groups[2] != g)
        return DPB_ERR_INVALID_ARG;  // groups must be numbered 0..G-1
  }
  if (pimd && (d->nbeads < 2 || d->nbeads > kMaxBeads || !d->nm_transform || !d->nm_freqs))
    return DPB_ERR_INVALID_ARG;
  if (pimd && d->remove_com_motion) return DPB_ERR_UNSUPPORTED;  // as the reference (md.py:150-151)
  if (!pimd && d->nbeads != 1) return DPB_ERR_INVALID_ARG;
  if (d->routine == DPB_MD_NVT_NHC && (d->chain_length < 2 || d->chain_length > kMaxChain))
    return DPB_ERR_UNSUPPORTED;
  if (d->n_fixed < 0 || (d->n_fixed > 0 && !d->fixed_indices)) return DPB_ERR_INVALID_ARG;
  if (d->n_fixed > 0 && d->routine != DPB_MD_NVE && d->routine != DPB_MD_NVT_NHC &&
      d->routine != DPB_MD_NVT_LANGEVIN)
    return DPB_ERR_UNSUPPORTED;  // fixed atoms: NVE, NVT, NVT Langevin (md.py:146-147,228-229)
  std::vector<char> fixed(d->natoms, 0);
  for (int k = 0; k < d->n_fixed; ++k) {
    const int a = d->fixed_indices[k];
    if (a < 0 || a >= d->natoms) return DPB_ERR_INVALID_ARG;
    fixed[a] = 1;
  }
  int n_mobile = 0;
  for (char c : fixed) n_mobile += c ? 0 : 1;
  if (n_mobile == 0) return DPB_ERR_INVALID_ARG;  // no degree of freedom left
  *out = nullptr;
  dpb_md *m = new dpb_md();
  m->model = model;
  m->d = *d;
  m->N = d->natoms;
  m->P = d->nbeads;
  m->ntypes = model->dm.ntypes;
  std::vector<int> t(d->type_idx, d->type_idx + d->natoms);
  for (int x : t)
    if (x < 0 || x >= m->ntypes) { delete m; return DPB_ERR_INVALID_ARG; }
  m->perm.resize(m->N);
  std::iota(m->perm.begin(), m->perm.end(), 0);
  std::stable_sort(m->perm.begin(), m->perm.end(), [&](int a, int b) { return t[a] < t[b]; });
  for (int k = 0; k < kMaxTypes; ++k) m->type_count[k] = 0;
  for (int x : t) m->type_count[x]++;
  m->S = 0;
  for (int k = 0; k < m->ntypes; ++k) { m->sel[k] = d->sel[k]; m->S += d->sel[k]; }
  for (int k = 0; k < 3; ++k) m->box[k] = (float)d->box[k];
  // soft-update threshold (md.py:733-736), scale_max = 1 at fixed box
  const float rc = model->dm.rcut, skin = (float)d->skin;
  m->threshold = ((rc + skin) - rc) / 2.f - std::min(m->box[0], std::min(m->box[1], m->box[2])) * 1e-6f;
  m->kT = d->temperature * 8.617333e-5;
  const size_t N = m->N, NF = N * m->P;
  int rc_ = DPB_OK;
  rc_ |= md_alloc(m, (void **)&m->pos, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->mom, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->force, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->ref_pos, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->inv_mass, N * 4);
  rc_ |= md_alloc(m, (void **)&m->mass, N * 4);
  rc_ |= md_alloc(m, (void **)&m->boxd, (size_t)m->P * 12);
  rc_ |= md_alloc(m, (void **)&m->status, 4);
  rc_ |= md_alloc(m, (void **)&m->energy, (size_t)m->P * 8);
  rc_ |= md_alloc(m, (void **)&m->virial, (size_t)m->P * 72);
  rc_ |= md_alloc(m, (void **)&m->sc, sizeof(MdScalars));
  rc_ |= md_alloc(m, (void **)&m->s_pos, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->s_mom, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->s_force, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->s_ref, NF * 12);
  rc_ |= md_alloc(m, (void **)&m->s_sc, sizeof(MdScalars));
  rc_ |= md_alloc(m, (void **)&m->user_slot, N * 4);
  rc_ |= md_alloc(m, (void **)&m->user_mass, N * 8);
  if (has_box) {
    rc_ |= md_alloc(m, (void **)&m->np, sizeof(NptScalars));
    rc_ |= md_alloc(m, (void **)&m->s_np, sizeof(NptScalars));
    rc_ |= md_alloc(m, (void **)&m->s_box, (size_t)m->P * 12);
  }
  if (d->routine == DPB_MD_NPT_PIMD) rc_ |= md_alloc(m, (void **)&m->prev, NF * 12);
  if (has_box) rc_ |= md_alloc(m, (void **)&m->box_hist, (size_t)kBoxHist * 12);
  rc_ |= md_alloc_lists(m);
  if (rc_) { dpb_md_destroy(m); return DPB_ERR_CUDA; }
  // masses in eV fs^2 / A^2 (md.py:24), sorted order
  std::vector<float> ms(N), im(N);
  for (size_t k = 0; k < N; ++k) {
    const double mm = d->mass_per_type[t[m->perm[k]]] * 1.036427e2;
    ms[k] = (float)mm;
    im[k] = (float)(1.0 / mm);
  }
  m->mass_sorted = ms;
  cudaMemcpy(m->mass, ms.data(), N * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(m->inv_mass, im.data(), N * 4, cudaMemcpyHostToDevice);
  {  // user order: the sorted slot of each atom and its float64 mass (the host's mass * unit)
    std::vector<int32_t> us(N);
    std::vector<double> um(N);
    for (size_t k = 0; k < N; ++k) {
      const int u = m->perm[k];
      us[u] = (int32_t)k;
      um[u] = d->mass_per_type[t[u]] * 1.036427e2;
    }
    cudaMemcpy(m->user_slot, us.data(), N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(m->user_mass, um.data(), N * 8, cudaMemcpyHostToDevice);
  }
  m->n_mobile = n_mobile;
  if (n_mobile < m->N) {  // fixed atoms: the mask and the masked shift, sorted order
    std::vector<float> mob(N), sim(N);
    for (size_t k = 0; k < N; ++k) {
      mob[k] = fixed[m->perm[k]] ? 0.f : 1.f;
      sim[k] = im[k] * mob[k];
    }
    if (md_alloc(m, (void **)&m->mobile, N * 4) || md_alloc(m, (void **)&m->shift_inv_mass, N * 4)) {
      dpb_md_destroy(m);
      return DPB_ERR_CUDA;
    }
    cudaMemcpy(m->mobile, mob.data(), N * 4, cudaMemcpyHostToDevice);
    m->mobile_sorted = mob;
    cudaMemcpy(m->shift_inv_mass, sim.data(), N * 4, cudaMemcpyHostToDevice);
  }
  std::vector<float> bx(3 * m->P);
  for (int b = 0; b < m->P; ++b)
    for (int k = 0; k < 3; ++k) bx[b * 3 + k] = m->box[k];
  cudaMemcpy(m->boxd, bx.data(), bx.size() * 4, cudaMemcpyHostToDevice);
  MdScalars s0;
  std::memset(&s0, 0, sizeof(s0));
  s0.scale = 1.0;
  s0.dof = 3.0 * (double)n_mobile;
  cudaMemcpy(m->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice);
  cudaMemset(m->status, 0, 4);
  if (pimd) {
    const int P = m->P;
    std::vector<float> C(P * P), fr(P), ga(P);
    for (int i = 0; i < P * P; ++i) C[i] = (float)d->nm_transform[i];
    for (int k = 0; k < P; ++k) {
      fr[k] = (float)d->nm_freqs[k];
      ga[k] = k == 0 ? (float)(1.0 / d->tau_t) : (float)(2.0 * d->pimd_lambda * d->nm_freqs[k]);
    }
    rc_ |= md_alloc(m, (void **)&m->C, C.size() * 4);
    rc_ |= md_alloc(m, (void **)&m->freqs, P * 4);
    rc_ |= md_alloc(m, (void **)&m->gamma, P * 4);
    if (rc_) { dpb_md_destroy(m); return DPB_ERR_CUDA; }
    cudaMemcpy(m->C, C.data(), C.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(m->freqs, fr.data(), P * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(m->gamma, ga.data(), P * 4, cudaMemcpyHostToDevice);
  }
  // workspaces
  if (dpb_nlist_workspace_bytes(m->N, m->P, m->box, (rc + skin) * 0.999f, &m->nl_ws_bytes) ||
      dpb_eval_workspace_bytes(model, m->N, m->P, &m->ev_ws_bytes)) {
    dpb_md_destroy(m);
    return DPB_ERR_INVALID_ARG;
  }
  rc_ |= md_alloc(m, &m->nl_ws, m->nl_ws_bytes);
  rc_ |= md_alloc(m, &m->ev_ws, m->ev_ws_bytes);
  if (rc_) { dpb_md_destroy(m); return DPB_ERR_CUDA; }
  if (cudaDeviceSynchronize() != cudaSuccess) { dpb_md_destroy(m); return DPB_ERR_CUDA; }
  *out = m;
  return DPB_OK;
}

extern "C" int dpb_md_destroy(dpb_md *m) {
  if (!m) return DPB_ERR_INVALID_ARG;
  for (void *p : m->allocs) cudaFree(p);
  delete m;
  return DPB_OK;
}

extern "C" int dpb_md_device_bytes(const dpb_md *m, size_t *bytes) {
  if (!m || !bytes) return DPB_ERR_INVALID_ARG;
  size_t NF = (size_t)m->N * m->P;
  *bytes = NF * (12 * 8 + 4 * m->S) + m->nl_ws_bytes + m->ev_ws_bytes;
  return DPB_OK;
}

// user order (P,N,3) float64 host  <->  sorted device float32
static int md_upload(dpb_md *m, const double *host, float *dev, bool momentum) {
  const int N = m->N, P = m->P;
  std::vector<float> buf((size_t)N * P * 3);
  for (int b = 0; b < P; ++b)
    for (int k = 0; k < N; ++k) {
      const int u = m->perm[k];
      for (int c = 0; c < 3; ++c) {
        double v = host[((size_t)b * N + u) * 3 + c];
        if (momentum) v *= m->mass_sorted[k];
        // setVelocity masks the fixed atoms' momenta (md.py:1029-1030)
        if (momentum && m->mobile && m->mobile_sorted[k] == 0.f) v = 0.0;
        buf[((size_t)b * N + k) * 3 + c] = (float)v;
      }
    }
  // The engine's kernels may run on any stream the caller gives, and a
  // blocking copy from pageable memory orders itself only against the legacy
  // stream (and may return before its DMA lands): wait for the device on both
  // sides.
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  if (cudaMemcpy(dev, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) return DPB_ERR_CUDA;
  return cudaDeviceSynchronize() == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
}

static int md_download(const dpb_md *m, const float *dev, double *host, bool velocity) {
  const int N = m->N, P = m->P;
  std::vector<float> buf((size_t)N * P * 3);
  if (cudaMemcpy(buf.data(), dev, buf.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DPB_ERR_CUDA;
  for (int b = 0; b < P; ++b)
    for (int k = 0; k < N; ++k) {
      const int u = m->perm[k];
      for (int c = 0; c < 3; ++c) {
        double v = buf[((size_t)b * N + k) * 3 + c];
        if (velocity) v /= m->mass_sorted[k];
        host[((size_t)b * N + u) * 3 + c] = v;
      }
    }
  return DPB_OK;
}

extern "C" int dpb_md_set_positions(dpb_md *m, const double *pos) {
  if (!m || !pos) return DPB_ERR_INVALID_ARG;
  return md_upload(m, pos, m->pos, false);
}

extern "C" int dpb_md_set_velocities(dpb_md *m, const double *vel) {
  if (!m || !vel) return DPB_ERR_INVALID_ARG;
  return md_upload(m, vel, m->mom, true);
}

extern "C" int dpb_md_get_state(const dpb_md *m, double *pos, double *vel, double *force) {
  if (!m) return DPB_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  int rc = DPB_OK;
  if (pos) rc |= md_download(m, m->pos, pos, false);
  if (vel) rc |= md_download(m, m->mom, vel, true);
  if (force) rc |= md_download(m, m->force, force, false);
  return rc;
}

// m->box is the neighbour list's reference box; under NPT the current box is
// the device copy m->boxd and the list canonicalises into the reference box.
static int md_build_list(dpb_md *m, const unsigned *gate, cudaStream_t st) {
  const float rc = m->model->dm.rcut + (float)m->d.skin;
  const bool npt = m->np != nullptr;  // the box lives on the device
  return nlist_build_impl(m->pos, nullptr, m->N, m->P, m->ntypes, m->type_count, m->sel, m->box, nullptr, rc,
                          m->nbrs, m->ref_pos, nullptr, m->status, m->nl_ws, m->nl_ws_bytes, gate, st,
                          npt ? m->boxd : nullptr, m->nl_warps);
}

static int md_forces(dpb_md *m, cudaStream_t st) {
  int rc = eval_impl(m->model, m->d.precision, m->pos, nullptr, m->N, m->P, m->type_count, m->boxd, m->nbrs, m->sel,
                     m->energy, nullptr, m->force, m->virial, m->status, m->ev_ws, m->ev_ws_bytes, st);
  if (!rc && m->mobile) {
    k_mask_rows<<<(m->N * 3 + 255) / 256, 256, 0, st>>>(m->force, m->mobile, m->N);
    count_launch();
    DPB_LAUNCH_CHECK();
  }
  return rc;
}

extern "C" int dpb_md_init(dpb_md *m, int reset_thermostat, void *stream) {
  if (!m) return DPB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = md_build_list(m, nullptr, st);
  if (!rc) rc = md_forces(m, st);
  if (rc) return rc;
  // kinetic energy of the initial momenta -> chain state (jax_md nvt init: DOF = 3N)
  MdScalars *sc = m->sc;
  k_md_begin<<<1, 1, 0, st>>>(sc);
  const int NF3 = m->N * m->P * 3;
  std::vector<float> zeros;
  float *tmpF = m->s_force;  // zero "force" to reuse the kick kernel as a pure KE reduction
  DPB_CUDA_TRY(cudaMemsetAsync(tmpF, 0, (size_t)NF3 * 4, st));
  k_vv_kick<<<(NF3 + 255) / 256, 256, 0, st>>>(m->mom, tmpF, m->inv_mass, m->N, m->N * m->P, 0.f, sc);
  count_launch(2);
  DPB_LAUNCH_CHECK();
  if (cudaStreamSynchronize(st) != cudaSuccess) return DPB_ERR_CUDA;
  if (reset_thermostat) {
    MdScalars h;
    cudaMemcpy(&h, sc, sizeof(h), cudaMemcpyDeviceToHost);
    h.chain_ke = h.ke;
    h.dof = 3.0 * (double)m->n_mobile;  // routine.py:119-127: DOF 3 n_mobile, Q0 = kT tau^2 DOF
    for (int k = 0; k < kMaxChain; ++k) {
      h.xi[k] = 0.0;
      h.pxi[k] = 0.0;
      h.Q[k] = k < m->d.chain_length ? m->kT * m->d.tau_t * m->d.tau_t : 0.0;  // chain masses at init
    }
    h.Q[0] *= h.dof;
    h.scale = 1.0;
    h.twork = 0.0;
    // a blocking copy from pageable memory may return before its DMA lands
    // and orders itself only against the legacy stream: wait for it before
    // any step on the caller's stream reads the chain state
    if (cudaMemcpy(sc, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) return DPB_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
    if (m->np) {  // npt init_fn (routine.py:322-350; NPT-PIMD: pimd.py:417-441)
      NptScalars n;
      std::memset(&n, 0, sizeof(n));
      std::vector<double> vir(9);
      cudaMemcpy(vir.data(), m->virial, 72, cudaMemcpyDeviceToHost);
      n.G = 0;
      for (int a = 0; a < 3; ++a) {
        n.gid[a] = m->d.couple_groups[a];
        if (n.gid[a] >= 0) { n.ngrp[n.gid[a]]++; n.G = std::max(n.G, n.gid[a] + 1); }
        n.ref[a] = m->box[a];
      }
      for (int g = 0; g < n.G; ++g) n.Mb[g] = n.ngrp[g] * (m->N + 1.0) * m->kT * m->d.tau_p * m->d.tau_p;
      for (int a = 0; a < 3; ++a)
        if (n.gid[a] >= 0) n.dUde[n.gid[a]] -= vir[a * 3 + a];
      n.pressure = m->d.pressure;
      for (int k = 0; k < m->d.chain_length_p; ++k) n.bQ[k] = m->kT * m->d.tau_p * m->d.tau_p;
      n.bdof = n.G;
      n.bQ[0] *= n.bdof;
      if (cudaMemcpy(m->np, &n, sizeof(n), cudaMemcpyHostToDevice) != cudaSuccess) return DPB_ERR_CUDA;
      if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
      if (m->d.routine == DPB_MD_NPT_PIMD) {
        // centroid-virial dU/d(eps) and centroid p^2/m of the initial state
        PimdParams pp;
        pp.P = m->P; pp.N = m->N; pp.dt = (float)m->d.dt; pp.kT = (float)m->kT;
        pp.L = make_float3(m->box[0], m->box[1], m->box[2]); pp.seed = m->d.seed; pp.tag = 1u;
        k_nptp_c<<<(m->N * 3 + 127) / 128, 128, 0, st>>>(m->pos, m->mom, m->force, m->mass, pp, m->np, m->boxd, sc,
                                                           0, 0);
        k_nptp_end<<<1, 1, 0, st>>>(m->np, m->virial, m->P, m->d.dt, m->N, 0);
        count_launch(2);
        DPB_LAUNCH_CHECK();
        if (cudaStreamSynchronize(st) != cudaSuccess) return DPB_ERR_CUDA;
      }
    }
  }
  return DPB_OK;
}

static int md_step(dpb_md *m, cudaStream_t st, float *traj_pos, float *traj_vel, int k) {
  const int NF = m->N * m->P, NF3 = NF * 3;
  const int nb = (NF + 255) / 256, nb3 = (NF3 + 255) / 256;
  MdScalars *sc = m->sc;
  const float3 L = make_float3(m->box[0], m->box[1], m->box[2]);
  const float dt = (float)m->d.dt;
  prof_begin(PROF_NLIST, st);
  k_md_begin<<<1, 1, 0, st>>>(sc);
  const bool npt = m->np != nullptr;  // the box lives on the device
  k_md_drift<<<nb, 256, 0, st>>>(m->pos, m->mom, m->ref_pos, NF, L, make_float3(1.f, 1.f, 1.f), L, sc, m->status,
                                 npt ? m->boxd : nullptr);
  k_md_decide<<<1, 1, 0, st>>>(sc, m->threshold, npt ? m->boxd : nullptr, L, m->model->dm.rcut, (float)m->d.skin,
                               m->status);
  count_launch(3);
  DPB_LAUNCH_CHECK();
  int rc = md_build_list(m, &sc->rebuild, st);
  if (rc) return rc;
  prof_end(PROF_NLIST, st);
  if (m->d.routine == DPB_MD_NPT_NHC) {  // MTK NPT step (routine.py:403-436)
    const int N = m->N, nbn = (N + 255) / 256;
    const int Lt = m->d.chain_length, Lb = m->d.chain_length_p;
    const double kT = m->kT, tt = m->d.tau_t, tp = m->d.tau_p, dtd = m->d.dt;
    k_npt_begin<<<1, 1, 0, st>>>(sc, m->np, Lt, Lb, kT, tt, tp, dtd, N);
    k_npt_scale_ke2<<<nbn, 256, 0, st>>>(m->mom, m->inv_mass, N, sc, m->np);
    k_npt_box1<<<1, 1, 0, st>>>(m->np, m->boxd, dtd, N);
    k_npt_move<<<nb3, 256, 0, st>>>(m->pos, m->mom, m->force, m->inv_mass, NF3, m->np);
    count_launch(4);
    DPB_LAUNCH_CHECK();
    rc = md_forces(m, st);
    if (rc) return rc;
    k_npt_kick2<<<nbn, 256, 0, st>>>(m->mom, m->force, m->inv_mass, N, sc, m->np);
    k_npt_end<<<1, 1, 0, st>>>(sc, m->np, m->virial, Lt, Lb, kT, tt, tp, dtd, N);
    k_scale_mom<<<nb3, 256, 0, st>>>(m->mom, NF3, sc);
    count_launch(3);
  } else if (m->d.routine == DPB_MD_NPT_PIMD) {  // pimd.py:443-516
    PimdParams pp;
    pp.P = m->P; pp.N = m->N; pp.dt = dt; pp.kT = (float)m->kT; pp.L = L; pp.seed = m->d.seed; pp.tag = 1u;
    const int nc = (m->N * 3 + 127) / 128;
    const double dtd = m->d.dt;
    k_nptp_begin<<<1, 1, 0, st>>>(m->np, m->boxd, m->P, dtd, m->N);
    k_nptp_a<<<nc, 128, 0, st>>>(m->pos, m->mom, m->force, m->prev, m->mass, m->C, m->freqs, m->gamma, pp, m->np,
                                 m->boxd, sc);
    k_nptp_mid<<<1, 1, 0, st>>>(sc, m->np, m->boxd, m->P, dtd, m->kT, 1.0 / m->d.tau_p, m->d.seed, m->N);
    k_nptp_b<<<nc, 128, 0, st>>>(m->pos, m->mom, m->prev, m->mass, m->C, m->freqs, pp, m->np, m->boxd);
    count_launch(4);
    DPB_LAUNCH_CHECK();
    rc = md_forces(m, st);
    if (rc) return rc;
    k_nptp_c<<<nc, 128, 0, st>>>(m->pos, m->mom, m->force, m->mass, pp, m->np, m->boxd, sc, 1, 1);
    k_nptp_end<<<1, 1, 0, st>>>(m->np, m->virial, m->P, dtd, m->N, 1);
    count_launch(2);
  } else if (m->d.routine == DPB_MD_NVT_LANGEVIN) {  // routine.py:81-103
    const double c1 = std::exp(-m->d.dt / m->d.tau_t);
    const double c2 = std::sqrt(std::max(m->kT * (1.0 - c1 * c1), 0.0));
    k_lan_baoa<<<nb3, 256, 0, st>>>(m->pos, m->mom, m->force, m->mass, m->inv_mass,
                                    m->mobile ? m->shift_inv_mass : m->inv_mass, m->mobile, m->N, dt, (float)c1,
                                    (float)c2, m->d.seed, sc);
    count_launch();
    DPB_LAUNCH_CHECK();
    rc = md_forces(m, st);
    if (rc) return rc;
    k_vv_kick<<<nb3, 256, 0, st>>>(m->mom, m->force, m->inv_mass, m->N, NF, dt, sc);
    count_launch();
  } else if (m->d.routine == DPB_MD_PIMD_PILE) {
    PimdParams pp;
    pp.P = m->P; pp.N = m->N; pp.dt = dt; pp.kT = (float)m->kT; pp.L = L; pp.seed = m->d.seed; pp.tag = 1u;
    k_pimd_baoa<<<(m->N * 3 + 127) / 128, 128, 0, st>>>(m->pos, m->mom, m->force, m->mass, m->C, m->freqs,
                                                         m->gamma, pp, sc);
    count_launch();
    DPB_LAUNCH_CHECK();
    rc = md_forces(m, st);
    if (rc) return rc;
    k_vv_kick<<<nb3, 256, 0, st>>>(m->mom, m->force, m->inv_mass, m->N, NF, dt, sc);
    count_launch();
  } else {
    const bool nvt = m->d.routine == DPB_MD_NVT_NHC;
    if (nvt) {
      k_nhc_substep<<<1, 1, 0, st>>>(sc, m->d.chain_length, m->kT, m->d.tau_t, m->d.dt, 1);
      count_launch();
    }
    k_vv_kick_drift<<<nb3, 256, 0, st>>>(m->pos, m->mom, m->force, m->mobile ? m->shift_inv_mass : m->inv_mass,
                                         m->N, NF, dt, sc, nvt ? 1 : 0);
    count_launch();
    DPB_LAUNCH_CHECK();
    rc = md_forces(m, st);
    if (rc) return rc;
    k_vv_kick<<<nb3, 256, 0, st>>>(m->mom, m->force, m->inv_mass, m->N, NF, dt, sc);
    count_launch();
    if (nvt) {
      k_nhc_substep<<<1, 1, 0, st>>>(sc, m->d.chain_length, m->kT, m->d.tau_t, m->d.dt, 2);
      k_scale_mom<<<nb3, 256, 0, st>>>(m->mom, NF3, sc);
      count_launch(2);
    }
  }
  if (m->d.remove_com_motion) {  // after the step, before the frame is emitted (md.py:793-796)
    k_com_sum<<<(m->N + 255) / 256, 256, 0, st>>>(m->mom, m->mass, m->mobile, m->N, sc);
    k_com_sub<<<(m->N + 255) / 256, 256, 0, st>>>(m->mom, m->mass, m->inv_mass, m->mobile,
                                                  m->d.routine != DPB_MD_NVT_LANGEVIN, m->N, sc);
    count_launch(2);
  }
  if (traj_pos) {
    k_copy_frame<<<nb3, 256, 0, st>>>(m->pos, traj_pos, NF3);
    count_launch();
  }
  if (m->box_hist && k < kBoxHist) {  // the box of this step (md.py:784-803 emits it per step)
    k_copy_frame<<<1, 32, 0, st>>>(m->boxd, m->box_hist + (size_t)k * 3, 3);
    count_launch();
  }
  if (traj_vel) {
    k_copy_frame<<<nb3, 256, 0, st>>>(m->mom, traj_vel, NF3);
    count_launch();
  }
  DPB_LAUNCH_CHECK();
  return DPB_OK;
}

extern "C" int dpb_md_run(dpb_md *m, int nsteps, float *traj_pos, float *traj_mom, void *stream) {
  if (!m || nsteps < 0) return DPB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t frame = (size_t)m->N * m->P * 3;
  for (int k = 0; k < nsteps; ++k) {
    int rc = md_step(m, st, traj_pos ? traj_pos + k * frame : nullptr, traj_mom ? traj_mom + k * frame : nullptr, k);
    if (rc) return rc;
  }
  return DPB_OK;
}

extern "C" int dpb_md_report(dpb_md *m, dpb_md_report_t *r) {
  if (!m || !r) return DPB_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  MdScalars h;
  std::vector<double> e(m->P), v(9 * m->P);
  uint32_t st = 0;
  cudaMemcpy(&h, m->sc, sizeof(h), cudaMemcpyDeviceToHost);
  cudaMemcpy(e.data(), m->energy, e.size() * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(v.data(), m->virial, v.size() * 8, cudaMemcpyDeviceToHost);
  if (cudaMemcpy(&st, m->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DPB_ERR_CUDA;
  std::memset(r, 0, sizeof(*r));
  double pe = 0.0;
  for (double x : e) pe += x;
  r->potential_energy = pe;
  for (int k = 0; k < 9; ++k)
    for (int b = 0; b < m->P; ++b) r->virial[k] += v[b * 9 + k];
  r->kinetic_energy = h.ke;
  r->thermostat_work = h.twork;
  r->status = st;
  r->steps = h.step;
  r->rebuilds = h.nrebuild;
  r->rebuild_rate = h.profile;
  r->chain_length = m->d.chain_length;
  r->chain_dof = h.dof;
  for (int k = 0; k < kMaxChain; ++k) { r->chain_xi[k] = h.xi[k]; r->chain_p[k] = h.pxi[k]; r->chain_Q[k] = h.Q[k]; }
  for (int a = 0; a < 3; ++a) r->box[a] = m->box[a];
  if (m->np) {
    NptScalars n;
    cudaMemcpy(&n, m->np, sizeof(n), cudaMemcpyDeviceToHost);
    r->ngroups = n.G;
    for (int a = 0; a < 3; ++a) r->box[a] = n.ref[a] * (n.gid[a] >= 0 ? std::exp(n.Rb[n.gid[a]]) : 1.0);
    for (int g = 0; g < 3; ++g) {
      r->box_position[g] = n.Rb[g];
      r->box_momentum[g] = n.Pb[g];
      r->box_mass[g] = n.Mb[g];
      r->dU_deps[g] = n.dUde[g];
    }
    r->baro_length = m->d.chain_length_p;
    r->box_thermostat_work = n.btwork;
    for (int k = 0; k < kMaxChain; ++k) { r->baro_xi[k] = n.bxi[k]; r->baro_p[k] = n.bp[k]; r->baro_Q[k] = n.bQ[k]; }
  }
  return DPB_OK;
}

extern "C" int dpb_md_clear_status(dpb_md *m, uint32_t keep) {
  if (!m) return DPB_ERR_INVALID_ARG;
  uint32_t st = 0;
  // the word is read after every step in flight on any stream, and the new
  // word has landed before the call returns (see md_upload)
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  if (cudaMemcpy(&st, m->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DPB_ERR_CUDA;
  st &= keep;
  if (cudaMemcpy(m->status, &st, 4, cudaMemcpyHostToDevice) != cudaSuccess) return DPB_ERR_CUDA;
  return cudaDeviceSynchronize() == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
}

extern "C" int dpb_md_snapshot(dpb_md *m, int restore) {
  if (!m) return DPB_ERR_INVALID_ARG;
  const size_t n = (size_t)m->N * m->P * 12;
  cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  // device-to-device cudaMemcpy runs on the legacy stream without host
  // synchronisation, while the steps may run on a non-blocking stream: the
  // state is copied only after every step in flight, and the call returns
  // only when the copies are done
  int bad = cudaDeviceSynchronize() != cudaSuccess;
  if (bad) return DPB_ERR_CUDA;
  if (!restore) {
    bad |= cudaMemcpy(m->s_pos, m->pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_mom, m->mom, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_force, m->force, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_ref, m->ref_pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_sc, m->sc, sizeof(MdScalars), k) != cudaSuccess;
    if (m->np) {
      bad |= cudaMemcpy(m->s_np, m->np, sizeof(NptScalars), k) != cudaSuccess;
      bad |= cudaMemcpy(m->s_box, m->boxd, (size_t)m->P * 12, k) != cudaSuccess;
    }
  } else {
    bad |= cudaMemcpy(m->pos, m->s_pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->mom, m->s_mom, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->force, m->s_force, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->ref_pos, m->s_ref, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->sc, m->s_sc, sizeof(MdScalars), k) != cudaSuccess;
    if (m->np) {
      bad |= cudaMemcpy(m->np, m->s_np, sizeof(NptScalars), k) != cudaSuccess;
      bad |= cudaMemcpy(m->boxd, m->s_box, (size_t)m->P * 12, k) != cudaSuccess;
    }
  }
  bad |= cudaDeviceSynchronize() != cudaSuccess;
  return bad ? DPB_ERR_CUDA : DPB_OK;
}

extern "C" int dpb_md_set_skin(dpb_md *m, double skin, void *stream) {
  if (!m || !(skin > 0.0)) return DPB_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  float cur[3];
  if (cudaMemcpy(cur, m->boxd, 12, cudaMemcpyDeviceToHost) != cudaSuccess) return DPB_ERR_CUDA;
  m->d.skin = skin;
  for (int a = 0; a < 3; ++a) m->box[a] = cur[a];  // the list's new reference box
  const float rc = m->model->dm.rcut, sk = (float)skin;
  m->threshold = ((rc + sk) - rc) / 2.f - std::min(m->box[0], std::min(m->box[1], m->box[2])) * 1e-6f;
  size_t need = 0;
  if (dpb_nlist_workspace_bytes(m->N, m->P, m->box, (rc + sk) * 0.999f, &need)) return DPB_ERR_INVALID_ARG;
  if (need > m->nl_ws_bytes) {
    cudaFree(m->nl_ws);
    m->allocs.erase(std::remove(m->allocs.begin(), m->allocs.end(), m->nl_ws), m->allocs.end());
    m->nl_ws = nullptr;
    m->nl_ws_bytes = need;
    if (md_alloc(m, &m->nl_ws, need)) return DPB_ERR_CUDA;
  }
  return md_build_list(m, nullptr, (cudaStream_t)stream);
}

// Resize the neighbour capacity (overflow resolution, md.py:657-668) and
// rebuild from the current positions.
extern "C" int dpb_md_set_capacity(dpb_md *m, const int *sel, void *stream) {
  if (!m || !sel) return DPB_ERR_INVALID_ARG;
  m->S = 0;
  for (int k = 0; k < m->ntypes; ++k) { m->sel[k] = sel[k]; m->S += sel[k]; }
  int rc = md_alloc_lists(m);
  if (rc) return rc;
  return md_build_list(m, nullptr, (cudaStream_t)stream);
}

extern "C" int dpb_md_box_history(dpb_md *m, int nsteps, double *out) {
  if (!m || !out || nsteps < 0 || nsteps > kBoxHist) return DPB_ERR_INVALID_ARG;
  std::vector<float> h((size_t)nsteps * 3);
  if (m->box_hist) {  // written by the steps on their stream: wait for them
    if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
    if (nsteps && cudaMemcpy(h.data(), m->box_hist, h.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      return DPB_ERR_CUDA;
  } else {
    for (int k = 0; k < nsteps; ++k)
      for (int a = 0; a < 3; ++a) h[(size_t)k * 3 + a] = m->box[a];
  }
  for (size_t e = 0; e < h.size(); ++e) out[e] = h[e];
  return DPB_OK;
}

// Trajectory frames in user atom order as float64, one thread per output
// element (grid-stride): out[f][b][u][c] = frame[f][b][slot[u]][c], the
// momenta divided by the user atom's float64 mass.  Writes are coalesced;
// reads gather 12-byte atom rows.
__global__ void k_traj_frames(const float *__restrict__ tp, const float *__restrict__ tm,
                              const int32_t *__restrict__ slot, const double *__restrict__ mass, int N,
                              size_t total, double *__restrict__ op, double *__restrict__ ov) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
    const size_t row = e / 3;
    const int c = (int)(e - row * 3);
    const size_t fb = row / (size_t)N;
    const int u = (int)(row - fb * (size_t)N);
    const size_t src = (fb * (size_t)N + (size_t)slot[u]) * 3 + c;
    if (op) op[e] = (double)tp[src];
    if (ov) ov[e] = (double)tm[src] / mass[u];
  }
}

extern "C" int dpb_md_traj_frames(dpb_md *m, int nframes, const float *traj_pos, const float *traj_mom,
                                  double *pos_out, double *vel_out, void *stream) {
  if (!m || nframes < 0 || (pos_out && !traj_pos) || (vel_out && !traj_mom)) return DPB_ERR_INVALID_ARG;
  const size_t total = (size_t)nframes * m->P * m->N * 3;
  if (!total || (!pos_out && !vel_out)) return DPB_OK;
  const size_t blocks = std::min<size_t>((total + 255) / 256, (size_t)148 * 16);
  k_traj_frames<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(traj_pos, traj_mom, m->user_slot, m->user_mass,
                                                                    m->N, total, pos_out, vel_out);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
}

extern "C" int dpb_md_eval_model(dpb_md *m, const dpb_model *model, double *energy, double *force) {
  if (!m || !model || !energy || !force) return DPB_ERR_INVALID_ARG;
  if (m->P != 1 || model->dm.ntypes != m->ntypes) return DPB_ERR_UNSUPPORTED;
  size_t wsb = 0;
  int rc = dpb_eval_workspace_bytes(model, m->N, 1, &wsb);
  if (rc) return rc;
  if (cudaDeviceSynchronize() != cudaSuccess) return DPB_ERR_CUDA;
  const size_t N3 = (size_t)m->N * 3;
  char *buf = nullptr;
  const size_t off_f = 0, off_e = (N3 * 4 + 255) & ~(size_t)255, off_v = off_e + 256, off_s = off_v + 256,
               off_w = off_s + 256;
  if (cudaMalloc((void **)&buf, off_w + wsb) != cudaSuccess) return DPB_ERR_CUDA;
  float *F = (float *)(buf + off_f);
  double *E = (double *)(buf + off_e), *W = (double *)(buf + off_v);
  uint32_t *stat = (uint32_t *)(buf + off_s);
  cudaMemset(stat, 0, 4);
  rc = eval_impl(model, m->d.precision, m->pos, nullptr, m->N, 1, m->type_count, m->boxd, m->nbrs, m->sel, E,
                 nullptr, F, W, stat, buf + off_w, wsb, nullptr);
  if (!rc && m->mobile) k_mask_rows<<<(m->N * 3 + 255) / 256, 256>>>(F, m->mobile, m->N);
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = DPB_ERR_CUDA;
  uint32_t hs = 0;
  if (!rc && cudaMemcpy(energy, E, 8, cudaMemcpyDeviceToHost) != cudaSuccess) rc = DPB_ERR_CUDA;
  if (!rc && cudaMemcpy(&hs, stat, 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = DPB_ERR_CUDA;
  if (!rc) rc = md_download(m, F, force, false);
  cudaFree(buf);
  if (!rc && (hs & DPB_ST_NONFINITE)) rc = DPB_ERR_CUDA;
  return rc;
}

// Launch-shape autotuner: each candidate runs on this engine's current state
// (a warm-up, then timed repetitions with CUDA events on the stream) and the
// fastest is kept; shapes never change results.  Ends with the list and
// forces of the current positions, like dpb_md_init.
extern "C" int dpb_md_autotune(dpb_md *m, int *nl_warps, int *dT_warps, int *fit_stages, void *stream) {
  if (!m) return DPB_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t a, b;
  DPB_CUDA_TRY(cudaEventCreate(&a));
  DPB_CUDA_TRY(cudaEventCreate(&b));
  const int cand[3] = {4, 8, 16};
  int best = m->nl_warps, rc = DPB_OK;
  float tbest = 1e30f;
  for (int c = 0; c < 3 && !rc; ++c) {
    m->nl_warps = cand[c];
    int r = md_build_list(m, nullptr, st);
    if (r == DPB_ERR_UNSUPPORTED) continue;  // hit lists of this many warps do not fit in shared memory
    cudaEventRecord(a, st);
    for (int k = 0; k < 3 && !r; ++k) r = md_build_list(m, nullptr, st);
    cudaEventRecord(b, st);
    if (!r && cudaEventSynchronize(b) != cudaSuccess) r = DPB_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (r) rc = r;
    else if (ms < tbest) { tbest = ms; best = cand[c]; }
  }
  m->nl_warps = best;
  int bestT = m->model->dT_warps;
  if (!rc && m->d.precision == DPB_PREC_MIXED) {
    rc = md_forces(m, st);
    if (!rc) {
      const int r = eval_tune_dT(m->model, m->N, m->P, m->ev_ws, st, &bestT);
      if (r && r != DPB_ERR_UNSUPPORTED) rc = r;  // compressed nets have no mixed dE/dT
      if (!r) m->model->dT_warps = bestT;
    }
  }
  // mixed form: the fitting kernel's shallow (2 CTAs per SM) or deep (1 CTA
  // per SM) weight ring, timed over whole evaluations of the current state
  if (!rc && m->d.precision == DPB_PREC_MIXED) {
    int bestd = m->model->fit_deep;
    tbest = 1e30f;
    for (int deep = 0; deep < 2 && !rc; ++deep) {
      m->model->fit_deep = deep;
      int r = md_forces(m, st);  // warm-up
      cudaEventRecord(a, st);
      for (int k = 0; k < 3 && !r; ++k) r = md_forces(m, st);
      cudaEventRecord(b, st);
      if (!r && cudaEventSynchronize(b) != cudaSuccess) r = DPB_ERR_CUDA;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (r) rc = r;
      else if (ms < tbest) { tbest = ms; bestd = deep; }
    }
    m->model->fit_deep = bestd;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!rc) rc = md_build_list(m, nullptr, st);
  if (!rc) rc = md_forces(m, st);
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = DPB_ERR_CUDA;
  if (nl_warps) *nl_warps = m->nl_warps;
  if (dT_warps) *dT_warps = m->model->dT_warps;
  if (fit_stages) *fit_stages = m->d.precision == DPB_PREC_MIXED ? (m->model->fit_deep ? 12 : 4) : 0;
  return rc;
}

extern "C" int dpb_md_device_pointers(dpb_md *m, dpb_md_pointers_t *p) {
  if (!m || !p) return DPB_ERR_INVALID_ARG;
  p->pos = m->pos;
  p->mom = m->mom;
  p->force = m->force;
  p->nbrs = m->nbrs;
  p->energy = m->energy;
  p->virial = m->virial;
  p->status = m->status;
  p->perm_sorted_to_user = nullptr;
  return DPB_OK;
}
