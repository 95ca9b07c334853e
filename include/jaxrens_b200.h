/*
 * jaxrens_b200.h -- C-ABI of the B200 nested-sampling walk.
 *
 * Drop-in boundary for jaxrens's jitted NS iteration.  Every buffer is a
 * device pointer owned by the caller (XLA, torch, or plain CUDA); apart from
 * jr_autotune, which clones the state to time launch shapes on, the library
 * allocates nothing on the call path.  All entry points are asynchronous on
 * the given stream and return 0 on success or a negative JR_ERR_* code, with
 * a message available from jr_last_error().
 *
 * Reference interfaces replaced (paths inside the jaxrens source tree):
 *   jr_ns_iterate      <- the jit'd ns_step that _run_loop calls,
 *                         src/jaxrens/sampling/run_loop.py:416-421 and :511-516
 *                         (ns_step, src/jaxrens/sampling/nested_sampling.py:391-686,
 *                         batched by src/jaxrens/sampling/batch_descriptor.py:177-195)
 *   jr_move_trial      <- per_move_fns[k] (src/jaxrens/sampling/mwg.py:152-154),
 *                         used by adjust_step_size
 *                         (src/jaxrens/sampling/adaptation/stepsize_handler.py:246-255)
 *   jr_walk_population <- _one_walk of the burn-in (src/jaxrens/init/burn_in.py:48-127)
 *   jr_energy_forces   <- eval_energy_and_forces on Hamiltonian(LJBackend, EnsembleTerm)
 *                         (src/jaxrens/backends/base.py:74-113,
 *                          src/jaxrens/backends/hamiltonian.py:112-153,
 *                          src/jaxrens/backends/lj.py:125-204,
 *                          src/jaxrens/backends/ensemble.py:34-59)
 *   jr_re_swap         <- replica_exchange_step with EnsembleSwap
 *                         (src/jaxrens/sampling/moves/replica_exchange.py:318-436),
 *                         fired by InterREManager.apply
 *                         (src/jaxrens/sampling/inter_re_manager.py:225-273)
 *
 * Layout (structure-of-arrays, mirroring the MCState leaves of
 * src/jaxrens/state/mc_state.py:70-95 with a leading replica axis P and a
 * padded atom axis Nmax; rows of `cell` are lattice vectors and positions are
 * row vectors, as in src/jaxrens/utils/cell.py):
 *   positions  float [P][K][Nmax][3]     direction float [P][K][Nmax][3]
 *   types      int32 [P][K][Nmax]        cell      float [P][K][3][3]
 *   energy     float [P][K] (float32 view of energy64)
 *   energy64   double[P][K] (full ensemble potential U + P*V - mu*N)
 *   step_sizes float [P][K][M]           n_accepted/n_proposed int32 [P][K][M]
 *   rng_key    uint32[P][2] (jax.random.key_data words)
 *   log_evidence double[P]  iteration int32[P]  emax double[P]
 *   n_atoms int32[P]  pressure float[P]  mu float[P][S] (or NULL)
 */
#ifndef JAXRENS_B200_H
#define JAXRENS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JR_MAX_SPECIES 8
#define JR_MAX_MOVES 8
#define JR_MAX_IMAGES 125
#define JR_MAX_CENTERS 8
#define JR_MAX_ATOMS 256
#define JR_MAX_CULL 32

enum {
  JR_OK = 0,
  JR_ERR_SHAPE = -1,       /* inconsistent or unsupported dimensions */
  JR_ERR_PARAM = -2,       /* invalid parameter value */
  JR_ERR_CUDA = -3,        /* a CUDA runtime call failed */
  JR_ERR_TIMEOUT = -4,     /* a bounded device-side wait gave up */
  JR_ERR_WORKSPACE = -5,   /* workspace missing or too small */
  JR_ERR_UNSUPPORTED = -6  /* a feature the library does not implement */
};

enum { JR_MODEL_LJ = 0, JR_MODEL_GAUSS_MIX = 1, JR_MODEL_SW = 2 };
#define JR_SW_MAX_ATOMS 64
enum { JR_MOVE_GALILEAN = 0, JR_MOVE_VOLUME = 1, JR_MOVE_MORPH = 2,
       JR_MOVE_SWAP = 3, JR_MOVE_SHEAR = 4, JR_MOVE_STRETCH = 5 };

typedef struct JrDims {
  int32_t n_replicas;      /* P */
  int32_t n_walkers;       /* K */
  int32_t n_atoms_max;     /* Nmax (padding stride of the atom axis) */
  int32_t n_moves;         /* M */
  int32_t n_mcmc_steps;    /* T */
  int32_t n_extra;         /* extra walked survivors per iteration */
  int32_t n_cull;          /* culled walkers per iteration, 1..JR_MAX_CULL */
  int32_t shared_move_key; /* 1: move schedule from fold_in(rng_key[0], 1)
                              (VmapRuns); 0: from each run's own key;
                              2: from the caller's key in state.move_key,
                              shared by every run (ns_step's move_key
                              argument; one iteration per call) */
} JrDims;

/* Energy model: LJ with per-species-pair tables (or the Gaussian-mixture
 * validation toy, or Stillinger-Weber).  LJ tables are row-major S x S,
 * already in the float32 form the reference evaluates: eps4 = f32(4*eps_ij),
 * eps24 = f32(24*eps_ij), sig2 = f32(sigma_ij**2).
 * JR_MODEL_SW: Stillinger-Weber (Phys. Rev. B 31, 5262 (1985)) with p = 4,
 * q = 0, one species, n_images = 1, at most JR_SW_MAX_ATOMS atoms; the sw_*
 * fields hold its float32 constants (sigma, a*sigma, gamma*sigma, A*eps, B,
 * lambda*eps) and rc2 = f32(sw_rc**2), has_cutoff = 1.  It has no
 * counterpart in the reference, which plugs potentials in through its
 * EnergyBackend protocol (src/jaxrens/backends/base.py:165-212). */
typedef struct JrModelParams {
  int32_t model;
  int32_t n_species;
  int32_t has_cutoff;
  float rc2;
  float eps4[JR_MAX_SPECIES * JR_MAX_SPECIES];
  float eps24[JR_MAX_SPECIES * JR_MAX_SPECIES];
  float sig2[JR_MAX_SPECIES * JR_MAX_SPECIES];
  int32_t n_images;                  /* supercell image offsets, (0,0,0) included */
  float img_off[JR_MAX_IMAGES * 3];
  int32_t n_centers;
  float centers[JR_MAX_CENTERS * 3];
  float gm_sigma;
  float sw_sigma, sw_rc, sw_gsig, sw_Aeps, sw_B, sw_leps;
} JrModelParams;

typedef struct JrMoveParams {
  int32_t n_moves;
  int32_t type[JR_MAX_MOVES];        /* JR_MOVE_* */
  int32_t n_reflect[JR_MAX_MOVES];   /* galilean */
  float perturb_angle[JR_MAX_MOVES]; /* galilean */
  float cum_probs[JR_MAX_MOVES];     /* float32 cumsum(w / sum(w)) */
  float max_vpa, min_vpa, min_aspect; /* cell-geometry guard */
  int32_t flat_v_prior;
  /* minimum-distance constraint gate (constraints/min_distance.py): applied
   * after move m when gate[m] != 0; dmin is the S x S threshold matrix */
  int32_t gate[JR_MAX_MOVES];
  float dmin[JR_MAX_SPECIES * JR_MAX_SPECIES];
} JrMoveParams;

typedef struct JrParams {
  JrModelParams model;
  JrMoveParams moves;
  double log_alpha;  /* log((K+1-n_cull)/(K+1)) */
  double w_offset[JR_MAX_CULL];  /* log dead-weight offset of cull k of an iteration
                                   (prior_mass.iteration_offsets) */
} JrParams;

typedef struct JrStateBuffers {
  float* positions;
  float* direction;
  int32_t* types;
  float* energy;
  double* energy64;
  float* cell;
  float* step_sizes;
  int32_t* n_accepted;
  int32_t* n_proposed;
  uint32_t* rng_key;
  double* log_evidence;
  int32_t* iteration;
  double* emax;
  const int32_t* n_atoms;
  const float* pressure;
  const float* mu;      /* NULL when the ensemble has no chemical potentials */
  const uint32_t* move_key;  /* [2] explicit move-schedule key words (device), read
                                when dims.shared_move_key == 2, else ignored */
} JrStateBuffers;

/* Per-iteration outputs of jr_ns_iterate, leading axis n_iter then P; the
 * per-cull arrays carry an n_cull axis after P (absent in effect for
 * n_cull = 1), culls in descending energy like the reference's worst_indices.
 * Any pointer may be NULL to skip that output. */
typedef struct JrInfoBuffers {
  int32_t* worst_idx;              /* [n_iter][P][n_cull] */
  int32_t* clone_idx;              /* [n_iter][P][n_cull] */
  double* emax;                    /* [n_iter][P] the new contour (last cull) */
  double* log_evidence;            /* [n_iter][P] after the iteration */
  float* dead_positions;           /* [n_iter][P][n_cull][Nmax][3] */
  int32_t* dead_types;             /* [n_iter][P][n_cull][Nmax] */
  float* dead_cell;                /* [n_iter][P][n_cull][9] */
  int32_t* n_accepted;             /* [n_iter][P][M] */
  int32_t* n_proposed;             /* [n_iter][P][M] */
  int32_t* reject_reason_counts;   /* [n_iter][P][M][4] */
  int32_t* n_evaluations;          /* [n_iter][P][M] */
  int32_t* n_grad_evaluations;     /* [n_iter][P][M] */
  int32_t* rounds;                 /* [P] speculation rounds used (diagnostic) */
  double* dead_energy;             /* [n_iter][P][n_cull] energies of the culled walkers */
  /* [n_iter][P][4] work the iteration's chains evaluated: pairs and
   * triplets of the evaluations with forces, then of the energy-only ones.
   * Pairs are LJ's unique interactions (every image) or Stillinger-Weber's
   * pairs inside the cutoff; triplets are Stillinger-Weber's (zero for LJ).
   * A galilean step evaluates the energy and, only when it reflects off the
   * contour, the forces. */
  int64_t* term_counts;
} JrInfoBuffers;

/* Launch shape of the walk kernels.  threads: CTA size; tpa: threads per
 * atom in the force gather (power of two <= 32); cluster: CTAs per replica
 * (thread-block cluster) serving speculative iterations; warp_walkers: 0 =
 * one walker per CTA, 1 = one walker per warp (threads/32 walkers per CTA).
 * Results do not depend on the launch shape. */
typedef struct JrLaunchConfig {
  int32_t threads;
  int32_t tpa;
  int32_t cluster;
  int32_t warp_walkers;
} JrLaunchConfig;

/* ---- NS iterations (replaces the jit'd ns_step) ---- */
/* Device workspace bytes jr_ns_iterate needs: the snapshot of replica 0's key
 * words (8 bytes) in one 256-byte slot.  The size does not depend on dims in
 * this version; callers ask anyway. */
size_t jr_ns_iterate_workspace_size(const JrDims* dims);

/* Runs n_iter NS iterations on every replica.  `cfg` may be NULL (cached
 * autotune result for these dims, else a heuristic).  `workspace` is device
 * memory of jr_ns_iterate_workspace_size(dims) bytes. */
int jr_ns_iterate(const JrDims* dims, const JrParams* params,
                  const JrStateBuffers* state, const JrInfoBuffers* info,
                  int32_t n_iter, const JrLaunchConfig* cfg, void* workspace,
                  size_t workspace_bytes, void* stream);

/* jr_ns_iterate for callers that cannot allocate device memory (an XLA FFI
 * handler given no scratch operand, a host that forbids allocation after
 * start-up).  It has no counterpart in the reference.  Instead of a caller
 * workspace it uses a 256-byte static __device__ array inside this library;
 * dims whose jr_ns_iterate_workspace_size() exceeds 256 bytes are rejected
 * with JR_ERR_WORKSPACE.  It allocates nothing.  The first call on each
 * device resolves that array's address (cudaGetSymbolAddress, device
 * current) and caches it with the id of the device's CUDA context, so make
 * that first call before any stream capture; after cudaDeviceReset the next
 * call sees a new context and resolves the address again.
 * The scratch is shared by every call on a device: calls that overlap in
 * time (several host threads, or concurrent streams) race on it and must be
 * serialised by the caller. */
int jr_ns_iterate_static(const JrDims* dims, const JrParams* params,
                         const JrStateBuffers* state, const JrInfoBuffers* info,
                         int32_t n_iter, const JrLaunchConfig* cfg, void* stream);

/* ---- burn-in walk of the whole population (replaces _one_walk,
 * src/jaxrens/init/burn_in.py:48-127, called by initial_walk :151-460) ----
 * Every walker k of every run p takes `walklength` MWG steps under the fixed
 * contour emax[p]: chain keys split(split(run_keys[p], K)[k], walklength),
 * move schedule split(move_key, walklength) shared by all walkers and runs.
 * Walkers keep their own step sizes; their acceptance counters advance.
 * run_keys [P][2], move_key [2], emax [P] (device). */
int jr_walk_population(const JrDims* dims, const JrParams* params,
                       const JrStateBuffers* state, int32_t walklength,
                       const uint32_t* run_keys, const uint32_t* move_key,
                       const double* emax, void* stream);

/* ---- one move per (replica, trial) walker (adaptation / burn-in) ---- */
/* walker_idx [P][n_trials], keys [P][n_trials][2], step [P], emax [P];
 * accepted [P][n_trials].  write_back=1 stores the moved walkers in place
 * (burn-in); write_back=0 only reports acceptance (step-size trials).
 * move_idx < 0 draws the move from keys like the MWG step (using
 * move_keys [P][n_trials][2]). */
int jr_move_trial(const JrDims* dims, const JrParams* params,
                  const JrStateBuffers* state, int32_t n_trials,
                  int32_t move_idx, const int32_t* walker_idx,
                  const uint32_t* keys, const uint32_t* move_keys,
                  const float* step, const double* emax, int32_t write_back,
                  int32_t* accepted, int32_t* reject_reason, void* stream);

/* ---- energy + forces of a batch of configurations ---- */
/* positions [B][Nmax][3], types [B][Nmax], cell [B][9], n_atoms [B],
 * pressure [B], mu [B][S] or NULL; energy64 [B] (U + PV - mu N),
 * energy_u [B] (U alone, may be NULL), forces [B][Nmax][3] (may be NULL). */
int jr_energy_forces(const JrParams* params, int32_t n_configs,
                     int32_t n_atoms_max, const float* positions,
                     const int32_t* types, const float* cell,
                     const int32_t* n_atoms, const float* pressure,
                     const float* mu, double* energy64, double* energy_u,
                     float* forces, void* stream);

/* ---- pressure / semi-grand replica exchange pass ---- */
/* key: the swap key words (host values).  acc/att_per_pair [P-1] (may be
 * NULL). Walker-bound fields travel; run-bound fields stay. */
int jr_re_swap(const JrDims* dims, const JrStateBuffers* state,
               uint32_t key0, uint32_t key1, int32_t n_swap_cycles,
               int32_t n_species, int32_t* acc_per_pair,
               int32_t* att_per_pair, void* stream);

/* ---- autotuner: times launch shapes on a scratch copy of `state` ----
 * Every candidate shape walks the same trajectory (restored from a pristine
 * copy before each sample of 4 launches of n_iter_probe iterations), scored
 * by the median of 3 samples; the winner is cached for these dims and used by
 * jr_ns_iterate calls given no launch shape.  The caller's state is not
 * modified.  No counterpart in the reference (the project-written tuner). */
int jr_autotune(const JrDims* dims, const JrParams* params,
                const JrStateBuffers* state, int32_t n_iter_probe,
                JrLaunchConfig* best, void* stream);

/* ---- learned surrogate and the delayed-acceptance walk ----
 * None of these has a counterpart in the reference: the surrogate is a
 * learned energy the walk trains on configurations it evaluated exactly, and
 * uses to screen galilean and volume proposals (two-stage delayed
 * acceptance: the smoothed surrogate constraint first, the exact potential
 * deciding every step).  Descriptors: 16 Gaussian radial functions per atom
 * (centres 1.5..3.8 A, cosine cutoff 3.8 A); network 16-64-64-1 with SiLU,
 * bfloat16 weights and activations in the products, float32 accumulation. */
#define JR_SUR_BASIS 16
#define JR_SUR_HIDDEN 64
/* float32 parameters, flat: W1[16][64] b1[64] W2[64][64] b2[64] w3[64] b3 */
#define JR_SUR_PARAMS 5313

typedef struct JrSurrogate {
  const float* params;       /* device, [JR_SUR_PARAMS] */
  float in_scale[JR_SUR_BASIS], in_shift[JR_SUR_BASIS]; /* x = D in_scale + in_shift */
  float out_scale, out_shift; /* U = sum_i (e_i out_scale + out_shift) */
  float contour_shift;       /* surrogate contour: emax + contour_shift */
  float tau;                 /* width of the smoothed surrogate constraint */
} JrSurrogate;

/* Descriptors D [n_configs][n_atoms][16] (float32) of configurations
 * positions [n_configs][n_atoms][3], cell [n_configs][9] (device),
 * n_atoms <= 128. */
int jr_sur_descriptors(int32_t n_configs, int32_t n_atoms, const float* positions,
                       const float* cell, float* descriptors, void* stream);

/* Device workspace bytes of jr_sur_train_step for a batch of n_batch
 * configurations. */
size_t jr_sur_train_workspace_size(int32_t n_batch, int32_t n_atoms);

/* One Adam step of the surrogate on n_batch configurations: batch_idx
 * [n_batch] picks rows of descriptors [*][n_atoms][16] and targets
 * energy_u [*] (the model energy U).  Loss: mean over the batch of
 * ((sum_i e_i out_scale + n out_shift - U) / n)^2.  params, adam_m, adam_v
 * [JR_SUR_PARAMS] are updated in place (step counts from 1); *loss (device)
 * receives the batch loss before the update.  Forward and backward run on
 * the tensor cores (tcgen05, accumulators in tensor memory).  n_atoms must
 * be 64 (two configurations per 128-row tile).  Workspace layout: an int32
 * error flag (set to 1 if a bounded tensor-core wait gave up; the step's
 * update is then not valid), padded to 256 bytes, then the per-CTA gradient
 * partials. */
int jr_sur_train_step(const JrSurrogate* sur, const float* descriptors, const double* energy_u,
                      const int32_t* batch_idx, int32_t n_batch, int32_t n_atoms,
                      float* params, float* adam_m, float* adam_v, int32_t step, float lr,
                      float* loss, void* workspace, size_t workspace_bytes, void* stream);

/* Surrogate energy (and forces) of a batch of single-species configurations,
 * as the delayed-acceptance walk evaluates it: positions [B][Nmax][3], cell
 * [B][9], n_atoms [B] (<= 64) on the device; energy_u [B] the surrogate U,
 * forces [B][Nmax][3] = -dU/dx (NULL: the energy alone, as the walk's
 * trajectory steps evaluate it).  Radial pairs by the minimum
 * image of the cell (periodic cells need sides > 7.6 A). */
int jr_sur_energy_forces(const JrSurrogate* sur, int32_t n_configs, int32_t n_atoms_max,
                         const float* positions, const float* cell, const int32_t* n_atoms,
                         double* energy_u, float* forces, void* stream);

/* Sample ring of the delayed-acceptance walk: every MWG step of every chain
 * owns one slot, into which a step that evaluated the exact potential stores
 * the evaluated configuration (positions, cell) and its model energy U; a
 * step without an exact evaluation stores energy NaN.  Chain wi (0 = the
 * clone, then the extras) of replica p in the launch's iteration it owns the
 * T slots from base + ((it P + p) W + wi) T, modulo capacity (W = n_cull +
 * n_extra, T = n_mcmc_steps); the caller advances base by n_iter P W T per
 * launch.  Any pointer may be NULL (positions NULL: no recording). */
typedef struct JrSampleRing {
  float* positions;                  /* [capacity][Nmax][3] */
  float* cell;                       /* [capacity][9] */
  double* energy_u;                  /* [capacity] */
  int64_t capacity;
  int64_t base;
  int32_t* n_surrogate_evaluations;  /* [n_iter][P][M] surrogate evaluations */
} JrSampleRing;

/* jr_ns_iterate for the Stillinger-Weber model (params.model.model ==
 * JR_MODEL_SW, one species, walkers of <= 64 atoms, whole-CTA walkers of 512
 * threads) with galilean and volume moves by two-stage delayed acceptance
 * on the surrogate `sur`: stage 1 accepts with the ratio of the smoothed
 * surrogate constraint sigmoid((emax + contour_shift - H_sur) / tau) (galilean
 * trajectories reflect off the surrogate contour at their inner points, never
 * at the final one, so the proposal is symmetric; volume moves take the
 * unclamped prior ratio (V'/V)^N times the surrogate ratio and the cell
 * checks), stage 2 evaluates the exact energy and accepts with
 * 1{E' < emax} min(1, s(x) / s(x')).  Other moves run as in
 * jr_ns_iterate.  info.n_evaluations counts exact evaluations;
 * ring->n_surrogate_evaluations the surrogate's.  `cfg` may be NULL (the
 * heuristic shape). */
int jr_ns_iterate_da(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                     const JrInfoBuffers* info, const JrSurrogate* sur,
                     const JrSampleRing* ring, int32_t n_iter, const JrLaunchConfig* cfg,
                     void* workspace, size_t workspace_bytes, void* stream);

/* ---- measurement utility: FP32 FMA-pipe throughput probe ----
 * Launches n_blocks x 256 threads of independent FMA chains; *flops receives
 * the floating-point operations the launch performs (time it with events).
 * No counterpart in the reference: it supplies the roofline denominator. */
int jr_bench_fma_peak(int n_blocks, int iters, float* scratch, double* flops,
                      void* stream);

const char* jr_last_error(void);
int jr_version(void);

#ifdef __cplusplus
}
#endif
#endif
