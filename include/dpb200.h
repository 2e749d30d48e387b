/*
 * dpb200.h — C ABI of the B200-native Deep Potential (se_a) evaluation and MD
 * step library (libdpb200.so).
 *
 * Conventions
 *   - Every compute entry point takes caller-owned DEVICE pointers and a
 *     cudaStream_t (passed as void*); nothing is synchronised unless stated.
 *   - Return value: 0 on success, or a DPB_ERR_* code (>= 256) for host-side
 *     failures.  Conditions detected on the device are OR-ed into a caller
 *     owned uint32 status word with the bit meanings of the reference's error
 *     code (deepmd_jax/md.py:618-641): 1 box shrank, 2 neighbour overflow,
 *     4 overflow in a previous chunk, 8 lattice overflow, 16 NaN/Inf.
 *   - Atoms inside a frame are in type-sorted order (stable sort of the user
 *     order, deepmd_jax/utils.py:329-340) unless a permutation is passed.
 *   - Frames: `nframes` frames of `natoms` atoms share type counts; arrays are
 *     frame-major ((F,N,3) positions, (F,N,S) neighbour lists, (F,3) boxes).
 *
 * Reference interfaces each entry point replaces are cited per function.
 */
#ifndef DPB200_H
#define DPB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DPB_API __attribute__((visibility("default")))
#else
#define DPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DPB_OK 0
#define DPB_ST_BOX_SHRUNK 1u
#define DPB_ST_NLIST_OVERFLOW 2u
#define DPB_ST_NLIST_OVERFLOW_PREV 4u
#define DPB_ST_LATTICE_OVERFLOW 8u
#define DPB_ST_NONFINITE 16u

#define DPB_ERR_INVALID_ARG 256
#define DPB_ERR_CUDA 257
#define DPB_ERR_UNSUPPORTED 258
#define DPB_ERR_WORKSPACE 259
#define DPB_ERR_NO_DEVICE 260
#define DPB_ERR_SCRATCH_LIMIT 261

/* Precision of the evaluation.
 * DPB_PREC_FP32:  all arithmetic in FP32 (the reference's float32 with
 *                 jax_default_matmul_precision='float32', deepmd_jax/__init__.py:10).
 * DPB_PREC_MIXED: embedding/fitting contractions in BF16 on the tensor cores
 *                 with FP32 accumulation; s(r), env matrix, first embedding
 *                 layer, per-atom energies and forces in FP32. */
#define DPB_PREC_FP32 0
#define DPB_PREC_MIXED 1

/* Neighbour entries are type-local atom indices (int32, < 2^24); the value
 * natoms marks an empty slot, as in the reference's nbrs_nm padding.
 * Small boxes (some L < 2 * cutoff): an entry means "some periodic image of
 * j lies within the cutoff" and dpb_eval sums every image of j within rcut,
 * the reference's lattice path (deepmd_jax/utils.py:66-78). */
#define DPB_NBR_INDEX_MASK 0x00FFFFFF

typedef struct dpb_model dpb_model;

/* Model description.  Host pointers, float32 arrays in the reference's
 * parameter pytree layout (deepmd_jax/train.py:288-304,
 * deepmd_jax/dpmodel.py:50-81): kernels are (in, out) row-major. */
typedef struct {
  int ntypes;                 /* 1..4 */
  int n_embed;                /* number of embedding layers (3) */
  int embed_widths[4];        /* e.g. 25,50,100 */
  int n_fit;                  /* number of hidden fitting layers (3) */
  int fit_widths[4];          /* e.g. 240,240,240 */
  int axis;                   /* axis_neuron A (16) */
  double rcut;
  double nnbrs;               /* params['Nnbrs'] */
  double out_norm;
  const double *sr_mean;      /* [ntypes] */
  const double *sr_std;       /* [ntypes] */
  const double *ebias;        /* [ntypes] */
  const float *const *embed_kernel; /* [ntypes*ntypes*n_embed], net k = i*ntypes+j */
  const float *const *embed_bias;   /* same */
  const float *tbias;               /* [W] */
  const float *const *fit_kernel;   /* [ntypes*(n_fit+1)] */
  const float *const *fit_bias;     /* same */
  const float *const *fit_dt;       /* [ntypes*n_fit], NULL where the layer has no dt */
  /* Compressed embedding (deepmd_jax/utils.py:126-151, tables made by
   * compress_model, utils.py:250-297).  n_grids > 0 replaces every embedding
   * net k by its piecewise quintic table: cmp_coeff[k] is poly_coeff
   * (n_grids, 6, W) float32 row-major over [cmp_srmin[k], cmp_srmax[k]);
   * embed_kernel / embed_bias may then be NULL.  n_grids = 0: uncompressed. */
  int n_grids;
  const float *const *cmp_coeff;    /* [ntypes*ntypes] or NULL */
  const double *cmp_srmin;          /* [ntypes*ntypes] or NULL */
  const double *cmp_srmax;          /* [ntypes*ntypes] or NULL */
} dpb_model_desc;

/* Upload the weights (FP32 and BF16 copies) to the current device.
 * Replaces: model loading + replication, deepmd_jax/utils.py:230-237. */
DPB_API int dpb_model_create(const dpb_model_desc *desc, dpb_model **out);
DPB_API int dpb_model_destroy(dpb_model *model);

/* ---------------------------------------------------------------- neighbour list */

/* Workspace bytes needed by dpb_nlist_build for one frame layout. */
DPB_API int dpb_nlist_workspace_bytes(int natoms, int nframes, const float box[3],
                              float rcut_plus_skin, size_t *bytes);

/* Typed neighbour list in the reference's nbrs_nm semantics.
 * Replaces: typed_neighbor_list(...).allocate/.update, get_nm
 * (deepmd_jax/md_utils.py:353-461) over jax_md.partition.neighbor_list.
 *   pos        (F,N,3) float32 device; type-sorted order unless perm != NULL
 *   perm       (N) int32 device: sorted index -> user index, or NULL
 *   type_count [ntypes] host; sel [ntypes] host (capacity per neighbour type)
 *   box        [3] host, the current box; ref_box [3] host or NULL (= box)
 *   nbrs       (F,N,sum(sel)) int32 device out: block j holds the type-j
 *              neighbours' type-local indices in ascending order, pad = N
 *   ref_pos    (F,N,3) float32 device out or NULL: canonical coordinates used
 *              for the drift test (reference_position)
 *   counts     (F,N,ntypes) int32 device out or NULL: neighbours per type
 *   status     device word, DPB_ST_NLIST_OVERFLOW is OR-ed in when a count
 *              exceeds sel (the reference's did_buffer_overflow).
 * Boxes with min(L) < 2*rcut_plus_skin list j once if any image of j is
 * within the cutoff (j == i included when a non-zero image is). */
DPB_API int dpb_nlist_build(const float *pos, const int32_t *perm, int natoms, int nframes,
                    int ntypes, const int *type_count, const int *sel,
                    const float box[3], const float *ref_box, float rcut_plus_skin,
                    int32_t *nbrs, float *ref_pos, int32_t *counts, uint32_t *status,
                    void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------- evaluation */

/* Workspace bytes needed by dpb_eval for F frames of N atoms. */
DPB_API int dpb_eval_workspace_bytes(const dpb_model *model, int natoms, int nframes, size_t *bytes);

/* Energy, per-atom energy, forces and virial of F frames.
 * Replaces: DPModel.apply / energy_and_force (deepmd_jax/dpmodel.py:30-108)
 * and the energy_fn / force_fn pair of deepmd_jax/md.py:292,416-444.
 *   pos      (F,N,3) float32 device (type-sorted unless perm != NULL)
 *   perm     (N) int32 device or NULL; outputs are written in the same order
 *            as the positions
 *   box      (F,3) float32 device (orthorhombic box lengths)
 *   nbrs     (F,N,sum(sel)) int32 device, layout of dpb_nlist_build
 *   energy   (F) float64 device out (total energy per frame)
 *   atom_energy (F,N) float32 device out or NULL
 *   force    (F,N,3) float32 device out, -dE/dpos
 *   virial   (F,9) float64 device out or NULL: W_ab = -sum_pairs x_a dE/dx_b
 *            with x = r_j - r_i; trace(W) = -dU/deps of a uniform strain
 *            (deepmd_jax/md_utils.py:139-159)
 *   status   device word (DPB_ST_NONFINITE on NaN/Inf energies). */
DPB_API int dpb_eval(const dpb_model *model, int precision, const float *pos, const int32_t *perm,
             int natoms, int nframes, const int *type_count, const float *box,
             const int32_t *nbrs, const int *sel, double *energy, float *atom_energy,
             float *force, double *virial, uint32_t *status, void *workspace,
             size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------- packed (ragged) batches
 * Many request frames of different atom counts and boxes evaluated by ONE
 * launch sequence (the serving loop's batch).  Replaces: the per-request
 * jit(vmap(energy_and_force)) calls of evaluate()/test()
 * (deepmd_jax/train.py:523-788), which compile and run one shape at a time.
 *
 * Layout ("segments" = request frames, s = 0..nseg-1):
 *   - packed atoms are type-sorted: type block t holds, segment after
 *     segment, each segment's type-t atoms padded with padding atoms to a
 *     multiple of 8 (so every 8-atom block lies in one segment);
 *   - seg[k] (natoms int32) = s for a real atom, -(s+1) for padding;
 *   - perm[k] = slot of packed atom k in pos / force (a bijection on
 *     [0, natoms)); padding atoms get their own slots (any finite position);
 *   - box (nseg, 3) device; energy (nseg) f64; virial (nseg, 9) f64;
 *   - nbrs (natoms, sum(sel)): type-local indices of the packed type blocks,
 *     pad = natoms; padding atoms' rows all pad (dpb_nlist_pack fills it). */
DPB_API int dpb_eval_packed_workspace_bytes(const dpb_model *model, int natoms, int nseg, size_t *bytes);
DPB_API int dpb_eval_packed(const dpb_model *model, int precision, const float *pos, const int32_t *perm,
                            int natoms, const int *type_count, const int32_t *seg, int nseg, const float *box,
                            const int32_t *nbrs, const int *sel, double *energy, float *atom_energy,
                            float *force, double *virial, uint32_t *status, void *workspace, size_t ws_bytes,
                            void *stream);
/* Copy the lists of `nframes` frames of one request (built by
 * dpb_nlist_build: (nframes, natoms, sum(sel)), type-local indices, pad =
 * natoms) into a packed list: frame f's type-t rows go to packed rows
 * row0[t] + f*stride[t] + m and its type-j index v becomes
 * base0[j] + f*stride[j] + v (pad -> packed_natoms).  No reference
 * counterpart (the reference has no packed batches). */
DPB_API int dpb_nlist_pack(const int32_t *src, int natoms, int nframes, int ntypes, const int *type_count,
                           const int *sel, const int *row0, const int *base0, const int *stride,
                           int packed_natoms, int32_t *dst, void *stream);

/* dpb_eval without a caller workspace, for callers that cannot allocate
 * device memory (a host code that keeps the force field inside its own fixed
 * memory pool, a plugin whose process forbids foreign cudaMalloc calls, code
 * that must not allocate between steps).  No counterpart in the reference:
 * its JAX path has no notion of caller-provided scratch.  The scratch is a
 * 64 MiB array inside the library image on each device that loads it; calls
 * whose dpb_eval_workspace_bytes exceed it return DPB_ERR_SCRATCH_LIMIT.
 * The first call on a device resolves the array's address (make it before any
 * stream capture); the address is cached per CUDA context, so after a device
 * reset the next call resolves it again.  Calls share the array: calls that
 * overlap on the GPU race.  Arguments and outputs as dpb_eval.  Allocates
 * nothing. */
DPB_API int dpb_eval_noalloc(const dpb_model *model, int precision, const float *pos, const int32_t *perm,
                             int natoms, int nframes, const int *type_count, const float *box,
                             const int32_t *nbrs, const int *sel, double *energy, float *atom_energy,
                             float *force, double *virial, uint32_t *status, void *stream);

/* ---------------------------------------------------------------- MD engine */

#define DPB_MD_NVE 0
#define DPB_MD_NVT_NHC 1
#define DPB_MD_PIMD_PILE 2
#define DPB_MD_NPT_NHC 3
#define DPB_MD_NPT_PIMD 4  /* NPT path-integral MD: Parrinello-Rahman on the centroid
                              mode, PILE-L, Langevin barostat (deepmd_jax/pimd.py:255-518) */
#define DPB_MD_NVT_LANGEVIN 5  /* BAOAB Langevin, friction 1/tau_t, with the thermostat
                                  work (deepmd_jax/routine.py:46-107, md.py:352-356) */

typedef struct dpb_md dpb_md;

/* Host-side description of an MD run (deepmd_jax/md.py:61-282 constructor
 * arguments).  Units: Angstrom, fs, Dalton, Kelvin. */
typedef struct {
  int routine;                 /* DPB_MD_NVE, DPB_MD_NVT_NHC, DPB_MD_PIMD_PILE, DPB_MD_NPT_NHC,
                                  DPB_MD_NPT_PIMD, DPB_MD_NVT_LANGEVIN */
  int natoms;
  int nbeads;                  /* 1, or P ring-polymer beads for PIMD */
  const int *type_idx;         /* [natoms] user order */
  const double *mass_per_type; /* Dalton */
  const int *sel;              /* neighbour capacity per type */
  double box[3];
  double skin;                 /* neighbour skin (0.3 for NVE/NVT, md.py:203-206) */
  double dt;                   /* fs */
  double temperature;          /* K (NVT / PIMD) */
  int chain_length;            /* Nose-Hoover chain length (3) */
  double tau_t;                /* fs: NHC tau; Langevin and PIMD centroid friction 1/tau_t */
  double pimd_lambda;          /* PILE internal-mode damping scale */
  const double *nm_transform;  /* PIMD: (P,P) C, primitive <- normal mode */
  const double *nm_freqs;      /* PIMD: (P) normal-mode frequencies, 1/fs */
  uint64_t seed;               /* Philox key of the stochastic steps */
  int precision;               /* DPB_PREC_* of the force evaluations */
  /* NPT (DPB_MD_NPT_NHC: MTK barostat + Nose-Hoover chains,
   * deepmd_jax/routine.py:161-456; DPB_MD_NPT_PIMD: Langevin barostat with
   * friction 1/tau_p on the centroid, pimd.py:255-518; orthorhombic, axes in
   * coupled groups) */
  double pressure;             /* target pressure, eV / A^3 */
  double tau_p;                /* barostat time constant, fs */
  int chain_length_p;          /* barostat chain length */
  int couple_groups[3];        /* group of each axis (0..G-1), -1: fixed axis */
  int remove_com_motion;       /* 1: subtract the centre-of-mass velocity after every step
                                  (md.py:793-796; not with PIMD) */
  /* Fixed atoms (md.py:221-236, routine.py:110-136; NVE, NVT and NVT Langevin):
   * user indices of atoms that never move.  Their forces read zero (the
   * stop_gradient of md.py:428-430), their momenta are masked, the chain
   * has 3 (N - n_fixed) degrees of freedom.  NULL / 0: every atom mobile. */
  const int32_t *fixed_indices;
  int n_fixed;
} dpb_md_desc;

typedef struct {
  double potential_energy;     /* sum over beads of the last force evaluation */
  double kinetic_energy;       /* of the current momenta */
  double virial[9];            /* sum over beads */
  double thermostat_work;      /* PILE-L cumulative work */
  uint32_t status;             /* OR of the device status bits */
  uint64_t steps, rebuilds;
  double rebuild_rate;         /* EMA of rebuilds per step (md.py:733) */
  int chain_length;
  double chain_dof;
  double chain_xi[8], chain_p[8], chain_Q[8];
  /* NPT: current box, per-group log box scale / momentum / mass, barostat
   * chain, per-group dU/d(eps) of the last force evaluation */
  double box[3];
  int ngroups;
  double box_position[3], box_momentum[3], box_mass[3];
  int baro_length;
  double baro_xi[8], baro_p[8], baro_Q[8];
  double dU_deps[3];           /* NPT-PIMD: the centroid-virial derivative */
  double box_thermostat_work;  /* NPT-PIMD: Langevin barostat cumulative work */
} dpb_md_report_t;

typedef struct {
  float *pos, *mom, *force;    /* (P,N,3) type-sorted */
  int32_t *nbrs;
  double *energy, *virial;
  uint32_t *status;
  int32_t *perm_sorted_to_user;
} dpb_md_pointers_t;

/* Create an MD context on the current device; allocates the state and the
 * workspaces of the neighbour list and the evaluation.
 * Replaces: Simulation.__init__ state set-up (deepmd_jax/md.py:61-282) and the
 * routine constructors (deepmd_jax/routine.py:139-158, deepmd_jax/pimd.py:114-207). */
DPB_API int dpb_md_create(const dpb_model *model, const dpb_md_desc *desc, dpb_md **out);
DPB_API int dpb_md_destroy(dpb_md *md);
DPB_API int dpb_md_device_bytes(const dpb_md *md, size_t *bytes);
/* State in user atom order, (P,N,3) float64 host arrays; velocities in A/fs.
 * Synchronous (the device is idle before and after each call).
 * Replaces: setPosition / setVelocity / getPosition / getVelocity / getForce
 * (deepmd_jax/md.py:969-1047). */
DPB_API int dpb_md_set_positions(dpb_md *md, const double *pos);
DPB_API int dpb_md_set_velocities(dpb_md *md, const double *vel);
DPB_API int dpb_md_get_state(const dpb_md *md, double *pos, double *vel, double *force);
/* Neighbour list and forces of the current positions; with reset_thermostat
 * the chain / thermostat state restarts from the current kinetic energy (the
 * routine's init_fn).  Synchronous. */
DPB_API int dpb_md_init(dpb_md *md, int reset_thermostat, void *stream);
/* Enqueue nsteps steps (drift test, gated rebuild, status, integrator, force
 * evaluation); no host synchronisation, capturable in a CUDA graph.
 * traj_pos / traj_mom: optional device buffers (nsteps,P,N,3) float32 in
 * type-sorted order.  Replaces: the jitted lax.scan chunk
 * (deepmd_jax/md.py:759-804). */
DPB_API int dpb_md_run(dpb_md *md, int nsteps, float *traj_pos, float *traj_mom, void *stream);
/* Synchronous read of the energies, status word and thermostat state. */
DPB_API int dpb_md_report(dpb_md *md, dpb_md_report_t *report);
DPB_API int dpb_md_clear_status(dpb_md *md, uint32_t keep_bits);
/* restore == 0: save the state (chunk start); 1: restore it (chunk re-run).
 * Synchronous: waits for the device before and after the copies, so the
 * steps may run on any stream. */
DPB_API int dpb_md_snapshot(dpb_md *md, int restore);
/* New neighbour skin and a rebuild whose reference box is the current box
 * (box-shrink resolution, status bit 1; deepmd_jax/md.py:649-654). */
DPB_API int dpb_md_set_skin(dpb_md *md, double skin, void *stream);
/* New neighbour capacity and a rebuild (overflow resolution, md.py:657-668). */
DPB_API int dpb_md_set_capacity(dpb_md *md, const int *sel, void *stream);
DPB_API int dpb_md_device_pointers(dpb_md *md, dpb_md_pointers_t *ptrs);
/* Launch-shape autotuner (no counterpart in the reference, which leaves
 * launch shapes to XLA): times the neighbour search at 4 / 8 / 16 centres
 * per block and, for the mixed form, dE/dT at 2 / 4 / 8 atoms per block and
 * the tensor-core fitting kernel with its shallow weight ring (4 stages, 2
 * CTAs per SM) and its deep one (12 stages, 1 CTA per SM, timed over whole
 * evaluations) on this engine's current state, and keeps the fastest
 * (*nl_warps, *dT_warps and *fit_stages report the choice; *fit_stages is 0
 * for the FP32 form; the dE/dT and ring choices are stored on the model).
 * Results do not depend on the shapes.  Call after dpb_md_init and before
 * capturing dpb_md_run into a graph; ends with the list and forces of the
 * current positions. */
DPB_API int dpb_md_autotune(dpb_md *md, int *nl_warps, int *dT_warps, int *fit_stages, void *stream);
/* Box (3 per step, Angstrom) after each of the first nsteps (<= 1024) steps
 * of the last dpb_md_run call: the per-step box of the reference's scan
 * output (deepmd_jax/md.py:784-803, 938); constant except under NPT. */
DPB_API int dpb_md_box_history(dpb_md *md, int nsteps, double *out);
/* Energy (host, one value) and forces (host, natoms x 3, user order) of
 * another model on the engine's current positions, box and neighbour list,
 * in the engine's precision, fixed atoms' forces zero: one force set of the
 * reference's Model_Devi reporter (deepmd_jax/md.py:299-302,559-567).
 * Synchronous; allocates and frees its scratch; not with beads. */
DPB_API int dpb_md_eval_model(dpb_md *md, const dpb_model *model, double *energy, double *force);
/* Frames written by dpb_md_run (nframes x (P,N,3) float32, type-sorted
 * positions and momenta) as float64 in user atom order: positions, and
 * velocities in A/fs (momenta divided by the float64 mass per atom), in one
 * launch on `stream`; either output may be NULL.  Same values as
 * un-permuting and dividing on the host (float32 -> float64 is exact and the
 * division is correctly rounded).  Replaces: the per-chunk trajectory
 * stacking of the reference's run loop (deepmd_jax/md.py:938-944), whose
 * state is already in user order. */
DPB_API int dpb_md_traj_frames(dpb_md *md, int nframes, const float *traj_pos, const float *traj_mom,
                               double *pos_out, double *vel_out, void *stream);

/* Diagnostics: per-stage CUDA-event timing on the launching stream (off by
 * default; not for use inside graph capture).  Stage ids: 0 neighbour
 * drift/rebuild, 1 embedding forward, 2 fitting chain, 3 embedding adjoint,
 * 4 integrator, 5/6/7 the same three stages of the mixed path, 8 the mixed
 * path's dE/dT kernel. */
DPB_API int dpb_profile_enable(int on);
/* Diagnostics: known-answer test of the tcgen05 tensor-core path, a
 * 128x64x32 BF16 product into TMEM (variant 0: K-major operands, 1: MN-major);
 * out: 128*64 floats (device), err: device int set on a barrier timeout. */
DPB_API int dpb_selftest_tcgen05(int variant, float *out, int *err, void *stream);
DPB_API int dpb_profile_read(int stage, double *ms, uint64_t *count);

/* The descriptor stage alone: T (F,N,10,W) = sum_j R~^T h2 / Nnbrs and
 * G (F,N,A*W) float32, type-sorted atom order (deepmd_jax/dpmodel.py:50-78);
 * err: device int set when a tensor-core wait gave up (mixed path);
 * workspace as for dpb_eval. */
DPB_API int dpb_eval_descriptors(const dpb_model *model, int precision, const float *pos, const int32_t *perm,
                                 int natoms, int nframes, const int *type_count, const float *box,
                                 const int32_t *nbrs, const int *sel, float *T, float *G, int *err,
                                 void *workspace, size_t workspace_bytes, void *stream);

/* Number of kernels the library launched since load (for launch accounting). */
DPB_API uint64_t dpb_kernel_launch_count(void);

/* Library version string. */
DPB_API const char *dpb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DPB200_H */
