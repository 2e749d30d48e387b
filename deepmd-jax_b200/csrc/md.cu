// Device-resident MD engine: velocity Verlet (NVE), Nose-Hoover chain (NVT)
// and ring-polymer BAOAB with the PILE-L thermostat (PIMD NVT).
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
};

// ---------------------------------------------------------------- kernels
__global__ void k_md_begin(MdScalars *sc) {
  sc->drift_bits = 0u;
  sc->ke = 0.0;
}

// Drift of canonical positions since the last rebuild, reference
// _drift_per_bead: (pos % box) * ref/box against reference_position, minimum
// image in the reference box (utils.py:11-18); also the NaN/Inf check of the
// pre-step state (md.py:638-640).
__global__ void k_md_drift(const float *__restrict__ pos, const float *__restrict__ mom,
                           const float *__restrict__ ref_pos, int NF, float3 L, float3 scale, float3 RB,
                           MdScalars *sc, uint32_t *status) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
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

__global__ void k_md_decide(MdScalars *sc, float threshold) {
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
// nose_hoover_chain, wrapped by deepmd_jax/routine.py:147-158), FP64.
// which == 1: first half step, uses chain_ke; which == 2: second half step,
// chain_ke := KE of the current momenta first.
__global__ void k_nhc_substep(MdScalars *sc, int L, double kT, double tau, double delta, int which) {
  if (which == 2) sc->chain_ke = sc->ke;
  // update_mass (kT fixed): Q = kT tau^2, Q0 *= DOF
  for (int m = 0; m < L; ++m) sc->Q[m] = kT * tau * tau;
  sc->Q[0] *= sc->dof;
  double *p = sc->pxi, *Q = sc->Q;
  const double d2 = delta / 2, d4 = d2 / 2, d8 = d4 / 2;
  const int M = L - 1;
  double G = p[M - 1] * p[M - 1] / Q[M - 1] - kT;
  p[M] += d4 * G;
  for (int m = M - 1; m > 0; --m) {
    G = p[m - 1] * p[m - 1] / Q[m - 1] - kT;
    const double sc_ = exp(-d8 * p[m + 1] / Q[m + 1]);
    p[m] = sc_ * (sc_ * p[m] + d4 * G);
  }
  G = 2.0 * sc->chain_ke - sc->dof * kT;
  double s1 = exp(-d8 * p[1] / Q[1]);
  p[0] = s1 * (s1 * p[0] + d4 * G);
  const double scale = exp(-d2 * p[0] / Q[0]);
  sc->chain_ke *= scale * scale;
  for (int m = 0; m < L; ++m) sc->xi[m] += d2 * p[m] / Q[m];
  G = 2.0 * sc->chain_ke - sc->dof * kT;
  for (int m = 0; m < M; ++m) {
    const double sm = exp(-d8 * p[m + 1] / Q[m + 1]);
    p[m] = sm * (sm * p[m] + d4 * G);
    G = p[m] * p[m] / Q[m] - kT;
  }
  p[M] += d4 * G;
  sc->scale = scale;
}

__global__ void k_scale_mom(float *__restrict__ mom, int n, const MdScalars *__restrict__ sc) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) mom[e] = (float)(mom[e] * sc->scale);
}

__global__ void k_copy_frame(const float *__restrict__ src, float *__restrict__ dst, int n) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dst[e] = src[e];
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
  float dke = 0.f;
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
          dke += 0.5f * (pv * pv - Pm[b] * Pm[b]) / m;
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
  dke = warp_sum(dke);
  if ((threadIdx.x & 31) == 0 && dke != 0.f) atomicAdd(&sc->twork, (double)dke);
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
  float *C = nullptr, *freqs = nullptr, *gamma = nullptr;
  void *nl_ws = nullptr, *ev_ws = nullptr;
  size_t nl_ws_bytes = 0, ev_ws_bytes = 0;
  // snapshot for chunk re-runs
  float *s_pos = nullptr, *s_mom = nullptr, *s_force = nullptr, *s_ref = nullptr;
  MdScalars *s_sc = nullptr;
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
  if (d->routine < DPB_MD_NVE || d->routine > DPB_MD_PIMD_PILE) return DPB_ERR_INVALID_ARG;
  if (d->routine == DPB_MD_PIMD_PILE && (d->nbeads < 2 || d->nbeads > kMaxBeads || !d->nm_transform || !d->nm_freqs))
    return DPB_ERR_INVALID_ARG;
  if (d->routine != DPB_MD_PIMD_PILE && d->nbeads != 1) return DPB_ERR_INVALID_ARG;
  if (d->routine == DPB_MD_NVT_NHC && (d->chain_length < 2 || d->chain_length > kMaxChain))
    return DPB_ERR_UNSUPPORTED;
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
  std::vector<float> bx(3 * m->P);
  for (int b = 0; b < m->P; ++b)
    for (int k = 0; k < 3; ++k) bx[b * 3 + k] = m->box[k];
  cudaMemcpy(m->boxd, bx.data(), bx.size() * 4, cudaMemcpyHostToDevice);
  MdScalars s0;
  std::memset(&s0, 0, sizeof(s0));
  s0.scale = 1.0;
  s0.dof = 3.0 * (double)N;
  cudaMemcpy(m->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice);
  cudaMemset(m->status, 0, 4);
  if (d->routine == DPB_MD_PIMD_PILE) {
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
        buf[((size_t)b * N + k) * 3 + c] = (float)v;
      }
    }
  return cudaMemcpy(dev, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
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

static int md_build_list(dpb_md *m, const unsigned *gate, cudaStream_t st) {
  const float rc = m->model->dm.rcut + (float)m->d.skin;
  return nlist_build_impl(m->pos, nullptr, m->N, m->P, m->ntypes, m->type_count, m->sel, m->box, nullptr, rc,
                          m->nbrs, m->ref_pos, nullptr, m->status, m->nl_ws, m->nl_ws_bytes, gate, st);
}

static int md_forces(dpb_md *m, cudaStream_t st) {
  return eval_impl(m->model, m->d.precision, m->pos, nullptr, m->N, m->P, m->type_count, m->boxd, m->nbrs, m->sel,
                   m->energy, nullptr, m->force, m->virial, m->status, m->ev_ws, m->ev_ws_bytes, st);
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
    h.dof = 3.0 * (double)m->N;
    for (int k = 0; k < kMaxChain; ++k) {
      h.xi[k] = 0.0;
      h.pxi[k] = 0.0;
      h.Q[k] = k < m->d.chain_length ? m->kT * m->d.tau_t * m->d.tau_t : 0.0;  // chain masses at init
    }
    h.Q[0] *= h.dof;
    h.scale = 1.0;
    h.twork = 0.0;
    cudaMemcpy(sc, &h, sizeof(h), cudaMemcpyHostToDevice);
  }
  return DPB_OK;
}

static int md_step(dpb_md *m, cudaStream_t st, float *traj_pos, float *traj_vel) {
  const int NF = m->N * m->P, NF3 = NF * 3;
  const int nb = (NF + 255) / 256, nb3 = (NF3 + 255) / 256;
  MdScalars *sc = m->sc;
  const float3 L = make_float3(m->box[0], m->box[1], m->box[2]);
  const float dt = (float)m->d.dt;
  prof_begin(PROF_NLIST, st);
  k_md_begin<<<1, 1, 0, st>>>(sc);
  k_md_drift<<<nb, 256, 0, st>>>(m->pos, m->mom, m->ref_pos, NF, L, make_float3(1.f, 1.f, 1.f), L, sc, m->status);
  k_md_decide<<<1, 1, 0, st>>>(sc, m->threshold);
  count_launch(3);
  DPB_LAUNCH_CHECK();
  int rc = md_build_list(m, &sc->rebuild, st);
  if (rc) return rc;
  prof_end(PROF_NLIST, st);
  if (m->d.routine == DPB_MD_PIMD_PILE) {
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
    k_vv_kick_drift<<<nb3, 256, 0, st>>>(m->pos, m->mom, m->force, m->inv_mass, m->N, NF, dt, sc, nvt ? 1 : 0);
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
  if (traj_pos) {
    k_copy_frame<<<nb3, 256, 0, st>>>(m->pos, traj_pos, NF3);
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
    int rc = md_step(m, st, traj_pos ? traj_pos + k * frame : nullptr, traj_mom ? traj_mom + k * frame : nullptr);
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
  return DPB_OK;
}

extern "C" int dpb_md_clear_status(dpb_md *m, uint32_t keep) {
  if (!m) return DPB_ERR_INVALID_ARG;
  uint32_t st = 0;
  if (cudaMemcpy(&st, m->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DPB_ERR_CUDA;
  st &= keep;
  return cudaMemcpy(m->status, &st, 4, cudaMemcpyHostToDevice) == cudaSuccess ? DPB_OK : DPB_ERR_CUDA;
}

extern "C" int dpb_md_snapshot(dpb_md *m, int restore) {
  if (!m) return DPB_ERR_INVALID_ARG;
  const size_t n = (size_t)m->N * m->P * 12;
  cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  int bad = 0;
  if (!restore) {
    bad |= cudaMemcpy(m->s_pos, m->pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_mom, m->mom, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_force, m->force, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_ref, m->ref_pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->s_sc, m->sc, sizeof(MdScalars), k) != cudaSuccess;
  } else {
    bad |= cudaMemcpy(m->pos, m->s_pos, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->mom, m->s_mom, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->force, m->s_force, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->ref_pos, m->s_ref, n, k) != cudaSuccess;
    bad |= cudaMemcpy(m->sc, m->s_sc, sizeof(MdScalars), k) != cudaSuccess;
  }
  return bad ? DPB_ERR_CUDA : DPB_OK;
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
