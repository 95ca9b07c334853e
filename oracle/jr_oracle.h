/*
 * jr_oracle.h -- CPU oracle for the nested-sampling walk (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it.  It restates, in plain
 * C, the arithmetic of jaxrens's inner nested-sampling walk:
 *
 *   - threefry2x32-20 and the JAX key derivations (split / fold_in /
 *     random_bits / uniform / normal / randint / choice) in the
 *     `jax_threefry_partitionable=True` layout,
 *   - the LJ backend (src/jaxrens/backends/lj.py:125-204) with per-species
 *     tables, triclinic minimum image, supercell images and a hard cutoff,
 *   - the Stillinger-Weber potential (Phys. Rev. B 31, 5262 (1985); no
 *     counterpart in the reference, which plugs such backends in through
 *     src/jaxrens/backends/base.py:165-212) -- parity unpinned against any
 *     external implementation, pinned by its closed forms instead,
 *   - the EnsembleTerm P*V - mu*N (src/jaxrens/backends/ensemble.py:34-59),
 *   - the galilean / volume / alchemical-morph / species-swap moves
 *     (the files under src/jaxrens/sampling/moves/), the MWG step
 *     (src/jaxrens/sampling/mwg.py:227-257), one ns_step iteration
 *     (src/jaxrens/sampling/nested_sampling.py:391-686) and the pressure
 *     replica-exchange pass (src/jaxrens/sampling/moves/replica_exchange.py:318-436).
 *
 * Precision modes:
 *   JRO_DEV   -- the arithmetic contract of the CUDA kernels: FP32 pair terms
 *                with a fixed FMA placement, every reduction accumulated in
 *                FP64 and rounded once.  GPU results must match this mode
 *                bit-for-bit (up to the documented FP64-rounding margin).
 *   JRO_REF32 -- the reference's own FP32 op order (no FMA, FP32 sums in
 *                row-major order), used to state the FP32 error of the
 *                reference against the FP64 oracle and as the CPU baseline.
 *   JRO_F64   -- everything in double (energy/force evaluation only).
 */
#ifndef JR_ORACLE_H
#define JR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { JRO_DEV = 0, JRO_REF32 = 1, JRO_F64 = 2 };
enum { JRO_MOVE_GALILEAN = 0, JRO_MOVE_VOLUME = 1, JRO_MOVE_MORPH = 2,
       JRO_MOVE_SWAP = 3, JRO_MOVE_SHEAR = 4, JRO_MOVE_STRETCH = 5 };
enum { JRO_MODEL_LJ = 0, JRO_MODEL_GAUSS_MIX = 1, JRO_MODEL_SW = 2 };

#define JRO_MAX_SPECIES 8
#define JRO_MAX_MOVES 8
#define JRO_MAX_IMAGES 125
#define JRO_MAX_CENTERS 8

typedef struct JroModel {
  int32_t model;           /* JRO_MODEL_* */
  int32_t n_species;
  int32_t has_cutoff;
  float rc2;               /* float32(cutoff**2) */
  float eps4[JRO_MAX_SPECIES * JRO_MAX_SPECIES];   /* float32(4*eps_ij) */
  float eps24[JRO_MAX_SPECIES * JRO_MAX_SPECIES];  /* float32(24*eps_ij) */
  float sig2[JRO_MAX_SPECIES * JRO_MAX_SPECIES];   /* float32(sigma_ij**2) */
  int32_t n_images;
  float img_off[JRO_MAX_IMAGES * 3];
  /* Gaussian-mixture toy (src/jaxrens/backends/toy.py:163-204) */
  int32_t n_centers;
  float centers[JRO_MAX_CENTERS * 3];
  float gm_sigma;
  /* Stillinger-Weber (p = 4, q = 0, one species): float32 sigma, a*sigma,
   * gamma*sigma, A*eps, B, lambda*eps; rc2 = float32(sw_rc**2) */
  float sw_sigma, sw_rc, sw_gsig, sw_Aeps, sw_B, sw_leps;
} JroModel;

typedef struct JroMoves {
  int32_t n_moves;
  int32_t type[JRO_MAX_MOVES];
  int32_t n_reflect[JRO_MAX_MOVES];
  float perturb_angle[JRO_MAX_MOVES];
  float cum_probs[JRO_MAX_MOVES];  /* float32 cumsum of w / sum(w) */
  /* cell-move guard (src/jaxrens/utils/cell.py:105-125) */
  float max_vpa, min_vpa, min_aspect;
  int32_t flat_v_prior;
  /* minimum-distance gate (constraints/min_distance.py, mwg.py:108-150):
   * applied after move m when gate[m]; dmin is the S x S threshold matrix */
  int32_t gate[JRO_MAX_MOVES];
  float dmin[JRO_MAX_SPECIES * JRO_MAX_SPECIES];
} JroMoves;

/* One replica's population, walker-major, N atoms (no padding). */
typedef struct JroReplica {
  int32_t n_walkers, n_atoms;
  float* positions;   /* [K][N][3] */
  float* direction;   /* [K][N][3] */
  int32_t* types;     /* [K][N] */
  double* energy;     /* [K] full ensemble potential */
  float* cell;        /* [K][9] rows are lattice vectors */
  float* step_sizes;  /* [K][M] */
  int32_t* n_acc;     /* [K][M] */
  int32_t* n_prop;    /* [K][M] */
  uint32_t* rng_key;  /* [2] */
  double* log_evidence;
  int32_t* iteration;
  double* emax;
  float pressure;
  float mu[JRO_MAX_SPECIES];
  int32_t has_mu;
} JroReplica;

typedef struct JroIterInfo {
  int32_t worst_idx, clone_idx;
  double emax;
  double dead_energy;
  int32_t n_acc[JRO_MAX_MOVES], n_prop[JRO_MAX_MOVES];
  int32_t rr[JRO_MAX_MOVES * 4];
  int32_t n_evals[JRO_MAX_MOVES], n_grad[JRO_MAX_MOVES];
  int32_t total_accepted;
} JroIterInfo;

/* ---- RNG ---- */
void jro_threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                      uint32_t out[2]);
void jro_split(const uint32_t key[2], uint32_t index, uint32_t out[2]);
void jro_fold_in(const uint32_t key[2], uint32_t data, uint32_t out[2]);
void jro_split_original(const uint32_t key[2], int32_t n, uint32_t* out);
uint32_t jro_bits32(const uint32_t key[2], uint32_t flat_index);
float jro_uniform(uint32_t bits, float lo, float hi);
float jro_normal(uint32_t bits);
float jro_erfinv(float x);
int32_t jro_randint(const uint32_t key[2], int32_t lo, int32_t hi);
int32_t jro_choice(const uint32_t key[2], const float* cum, int32_t m);
void jro_normal_array(const uint32_t key[2], int32_t n, float* out);
void jro_uniform_array(const uint32_t key[2], int32_t n, float* out);

/* Float32 exp of the Stillinger-Weber kernel contract (Cody-Waite reduction,
 * degree-7 Taylor polynomial), exposed to test its error bound. */
float jro_sw_exp(float x);

/* ---- geometry ---- */
float jro_det3(const float* c);
void jro_inv_cell(const float* c, float* inv);

/* ---- energy ---- */
/* Energy (+ forces when forces != NULL) of one configuration under the
 * model plus the ensemble term.  Returns the full potential (U + PV - mu N);
 * *u_out receives U alone.  forces are -dE/dx, double for every mode. */
double jro_energy(const JroModel* mdl, int32_t mode, int32_t n_atoms,
                  const float* x, const int32_t* types, const float* cell,
                  float pressure, const float* mu, int32_t has_mu,
                  double* forces, double* u_out);

/* ---- moves / NS ---- */
int32_t jro_mwg_step(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                     const uint32_t step_key[2], const uint32_t move_key[2],
                     double emax, int32_t n_atoms, float* x, float* d,
                     int32_t* types, float* cell, double* energy,
                     const float* step_sizes, int32_t* n_acc, int32_t* n_prop,
                     float pressure, const float* mu, int32_t has_mu,
                     int32_t* move_idx_out, int32_t* reason_out,
                     int32_t* n_evals_out, int32_t* n_grad_out);

int32_t jro_move_trial(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                       int32_t move_idx, const uint32_t key[2], float step,
                       double emax, int32_t n_atoms, float* x, float* d,
                       int32_t* types, float* cell, double* energy,
                       float pressure, const float* mu, int32_t has_mu,
                       int32_t* reason_out);

void jro_ns_step(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                 JroReplica* rep, int32_t n_mcmc_steps, int32_t n_extra,
                 const uint32_t* move_key, /* NULL: split from the run key */
                 double log_alpha, double w_offset, JroIterInfo* info,
                 float* dead_positions, int32_t* dead_types, float* dead_cell);

/* ns_step with any n_cull (>= 1): worst/clone [n_cull] indices, dead
 * energies [n_cull], dead walkers [n_cull][...]; w_offsets [n_cull].  Any
 * output may be NULL. */
void jro_ns_step_n(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                   JroReplica* rep, int32_t n_mcmc_steps, int32_t n_cull,
                   int32_t n_extra, const uint32_t* move_key, double log_alpha,
                   const double* w_offsets, JroIterInfo* info, int32_t* worst_out,
                   int32_t* clone_out, double* dead_energy_out, float* dead_positions,
                   int32_t* dead_types, float* dead_cell);

/* Minimum-distance constraint verdict (1 = every pair far enough). */
int32_t jro_min_distance_ok(const JroMoves* mv, int32_t S, int32_t n, const float* x,
                            const int32_t* t, const float* cell, int32_t mode);

/* Burn-in walk of every walker of one run (init/burn_in.py _one_walk). */
void jro_walk_population(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                         JroReplica* rep, int32_t walklength, const uint32_t run_key[2],
                         const uint32_t move_key[2], double emax);

void jro_re_step(JroReplica* reps, int32_t n_reps, const uint32_t key[2],
                 int32_t n_swap_cycles, int32_t mode, int32_t* acc_per_pair,
                 int32_t* att_per_pair);

/* Several replicas, one NS iteration each, threads over replicas. */
void jro_ns_step_batched(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                         JroReplica* reps, int32_t n_reps,
                         int32_t n_mcmc_steps, int32_t n_extra,
                         int32_t shared_move_key, double log_alpha,
                         double w_offset, JroIterInfo* infos, int32_t n_threads);

/* Synthetic uniform-gas walkers (cubic cell, V ~ U(0, v_hi], fractional
 * coordinates U[0,1)^3), walker k drawn from split(key, k). */
void jro_init_walkers(const uint32_t key[2], int32_t n_walkers, int32_t n_atoms,
                      float v_hi, float* positions, float* cell);

#ifdef __cplusplus
}
#endif
#endif
