// jr_host.cuh -- host side shared by the library's translation units:
// argument checks, launch-shape heuristics, shared-memory sizing and the
// launch templates of each model family.  jr_ns.cu defines the shared state
// (error text, attribute cache) and instantiates the pair family; jr_sw.cu
// instantiates the Stillinger-Weber family, jr_swda.cu its delayed-acceptance
// walk.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/jaxrens_b200.h"
#include "jr_kernels.cuh"

namespace jrh {

// Defined in jr_ns.cu.
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
// Raises a kernel's dynamic shared-memory limit (and allows non-portable
// cluster sizes) once per kernel and device context.
cudaError_t ensure_attrs(const void* kern, size_t smem, bool nonportable);

constexpr size_t kMaxDynSmem = 227 * 1024;  // opt-in shared memory per CTA on sm_100

inline int family_of(const JrParams* p) {
  return p->model.model == JR_MODEL_SW ? jr::kFamSW : jr::kFamPair;
}

inline int pow2_floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

inline int warp_tpa(int nmax) {
  int t = pow2_floor(32 / (nmax > 0 ? nmax : 1));
  return t < 1 ? 1 : t;
}

// Small walkers: one warp per walker, four walkers per CTA, one CTA per
// replica; larger walkers (and every Stillinger-Weber walker, whose tables
// fill a CTA's shared memory): one CTA per walker.
inline JrLaunchConfig heuristic_config(const JrDims* d, int fam = jr::kFamPair) {
  JrLaunchConfig c;
  const int nmax = d->n_atoms_max;
  c.cluster = 1;
  if (nmax <= 32 && fam == jr::kFamPair) {
    c.warp_walkers = 1;
    c.threads = 128;
    c.tpa = warp_tpa(nmax);
  } else {
    c.warp_walkers = 0;
    c.threads = 512;
    int tpa = pow2_floor(c.threads / nmax);
    c.tpa = tpa > 16 ? 16 : (tpa < 1 ? 1 : tpa);
  }
  return c;
}

// Speculation depth bound of check_config, without setting the error text.
inline bool spec_fits(const JrLaunchConfig& c, const JrDims* d) {
  if (d->n_cull > 1) return true;  // n_cull > 1 never speculates
  const int W = 1 + d->n_extra;
  const int slots = c.cluster * (c.warp_walkers ? c.threads / 32 : 1);
  if (slots < 2 * W) return true;
  const int D = slots / W < jr::kMaxD ? slots / W : jr::kMaxD;
  return D * d->n_extra <= jr::kMaxWalk && D * W <= jr::kMaxWalk;
}

// Default shape of the NS launch: a CTA per walker chain, 128 threads for
// N <= 16, 256 for N <= 64, 512 above (measured: a 128-thread CTA walks an
// 8-atom chain 8% faster than a warp).  The cluster serves the speculative
// iterations of one run: no more CTAs than one launch's n_iter * (1 + n_extra)
// chains can use, and at most 10 (clusters of 12-16 were measured to share
// SMs between their CTAs, which slows every chain).  A cluster that covers
// the launch's iterations commits them in about one round, which outweighs a
// grid somewhat larger than the SM count (16 runs of 1024 walkers with up to
// 96 atoms: clusters of 10, 160 CTAs, walked 1.4x faster than clusters of 8
// or 9), so the grid is capped at 1.2x the SMs.
inline JrLaunchConfig ns_heuristic_config(const JrDims* d, int n_iter, int fam = jr::kFamPair) {
  JrLaunchConfig c = heuristic_config(d, fam);
  const int nmax = d->n_atoms_max;
  if (nmax <= 64) {
    c.warp_walkers = 0;
    // Stillinger-Weber: 512 threads (the pair scan and the triplet sides
    // spread over twice the lanes; measured 17% faster than 256 on 64 atoms)
    c.threads = jr::sw_family(fam) ? 512 : (nmax <= 16 ? 128 : 256);
    const int tpa = pow2_floor(c.threads / nmax);
    c.tpa = tpa > 16 ? 16 : (tpa < 1 ? 1 : tpa);
  }
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  const int W = d->n_cull + d->n_extra;
  const int cpc = c.warp_walkers ? c.threads / 32 : 1;
  // chains one launch can run at once: n_iter * W speculated (n_cull = 1),
  // otherwise the W chains of one iteration
  const int want = d->n_cull > 1 ? W : (n_iter > 0 ? n_iter : 1) * W;
  int cl = (want + cpc - 1) / cpc;
  const int fit = (sms * 6 / 5) / (d->n_replicas > 0 ? d->n_replicas : 1);
  if (cl > 10) cl = 10;
  if (cl > fit) cl = fit;
  if (cl < 1) cl = 1;
  c.cluster = cl;
  while (c.cluster > 1 && !spec_fits(c, d)) c.cluster -= 1;
  return c;
}

inline int check_params(const JrDims* d, const JrParams* p) {
  if (!d || !p) return fail(JR_ERR_PARAM, "null dims or params");
  if (d->n_replicas < 1 || d->n_walkers < 2 || d->n_atoms_max < 1 ||
      d->n_atoms_max > JR_MAX_ATOMS)
    return fail(JR_ERR_SHAPE, "need n_replicas>=1, n_walkers>=2, 1<=n_atoms_max<=" +
                                  std::to_string(JR_MAX_ATOMS));
  if (d->n_moves < 1 || d->n_moves > JR_MAX_MOVES || d->n_moves != p->moves.n_moves)
    return fail(JR_ERR_SHAPE, "n_moves must be in [1, 8] and match params.moves");
  if (d->n_cull < 1 || d->n_cull > JR_MAX_CULL)
    return fail(JR_ERR_SHAPE, "n_cull must be in [1, " + std::to_string(JR_MAX_CULL) + "]");
  if (d->n_extra < 0 || d->n_extra > d->n_walkers - 2 || d->n_extra + d->n_cull > jr::kMaxWalk)
    return fail(JR_ERR_SHAPE, "n_extra must satisfy 0 <= n_extra <= n_walkers-2 and "
                              "n_cull + n_extra <= 256");
  if (d->n_cull > 1 && 2 * d->n_cull + d->n_extra > d->n_walkers)
    return fail(JR_ERR_SHAPE, "n_cull > 1 needs 2*n_cull + n_extra <= n_walkers "
                              "(nested_sampling.py _select_culls)");
  if (p->model.n_species < 1 || p->model.n_species > JR_MAX_SPECIES)
    return fail(JR_ERR_PARAM, "n_species must be in [1, 8]");
  if (p->model.n_images < 1 || p->model.n_images > JR_MAX_IMAGES)
    return fail(JR_ERR_PARAM, "n_images must be in [1, 125]");
  if (p->model.model < JR_MODEL_LJ || p->model.model > JR_MODEL_SW)
    return fail(JR_ERR_PARAM, "unknown model");
  if (p->model.model == JR_MODEL_SW) {
    if (p->model.n_species != 1 || p->model.n_images != 1)
      return fail(JR_ERR_UNSUPPORTED,
                  "Stillinger-Weber walks take one species and the single minimum image");
    if (d->n_atoms_max > JR_SW_MAX_ATOMS)
      return fail(JR_ERR_SHAPE, "Stillinger-Weber walkers hold at most " +
                                    std::to_string(JR_SW_MAX_ATOMS) + " atoms");
  }
  for (int m = 0; m < d->n_moves; ++m) {
    const int t = p->moves.type[m];
    if (t < 0 || t > JR_MOVE_STRETCH) return fail(JR_ERR_PARAM, "unknown move type");
    if (t == JR_MOVE_GALILEAN && p->moves.n_reflect[m] < 1)
      return fail(JR_ERR_PARAM, "galilean n_reflect must be >= 1");
    if ((t == JR_MOVE_MORPH || t == JR_MOVE_SWAP) && p->model.n_species < 2)
      return fail(JR_ERR_PARAM, "identity moves need n_species >= 2");
  }
  return JR_OK;
}

inline int check_config(const JrLaunchConfig& c, const JrDims* d, int fam = jr::kFamPair) {
  if (c.threads < 32 || c.threads > 512 || (c.threads & 31))
    return fail(JR_ERR_PARAM, "threads must be a multiple of 32 in [32, 512]");
  if (c.tpa < 1 || c.tpa > 32 || (c.tpa & (c.tpa - 1)))
    return fail(JR_ERR_PARAM, "tpa must be a power of two <= 32");
  if (c.cluster < 1 || c.cluster > 16) return fail(JR_ERR_PARAM, "cluster must be in [1, 16]");
  if (c.warp_walkers != 0 && c.warp_walkers != 1)
    return fail(JR_ERR_PARAM, "warp_walkers must be 0 or 1");
  if (c.warp_walkers && jr::sw_family(fam))
    return fail(JR_ERR_PARAM, "Stillinger-Weber walkers are walked by whole CTAs");
  if (!c.warp_walkers && c.tpa > c.threads) return fail(JR_ERR_PARAM, "tpa exceeds the CTA");
  if (c.warp_walkers && c.threads > 128)
    return fail(JR_ERR_PARAM, "warp-walker CTAs hold at most 4 walkers (128 threads)");
  const int W = 1 + d->n_extra;
  const int slots = c.cluster * (c.warp_walkers ? c.threads / 32 : 1);
  if (d->n_cull == 1 && slots >= 2 * W) {
    const int D = slots / W < jr::kMaxD ? slots / W : jr::kMaxD;
    if (D * d->n_extra > jr::kMaxWalk || D * W > jr::kMaxWalk)
      return fail(JR_ERR_PARAM, "speculation depth * n_extra too large");
  }
  return JR_OK;
}

inline size_t ns_dyn_smem(const JrDims* d, const JrParams* p, const JrLaunchConfig& c,
                          int fam = -1) {
  if (fam < 0) fam = family_of(p);
  const int cpc = c.warp_walkers ? c.threads / 32 : 1;
  return jr::dyn_head_bytes(d->n_walkers, d->n_atoms_max, p->model.n_images, d->n_cull, fam) +
         (size_t)cpc * jr::walker_smem_bytes(d->n_atoms_max, p->model.n_images, true, fam);
}

inline size_t group_dyn_smem(int nmax, int nimg, int groups, int fam) {
  return (size_t)groups * (jr::pair_table_bytes(nmax, nimg, fam) +
                           jr::walker_smem_bytes(nmax, nimg, false, fam));
}

inline int check_smem(size_t smem) {
  if (smem > kMaxDynSmem)
    return fail(JR_ERR_SHAPE, "the walkers need " + std::to_string(smem) +
                                  " bytes of shared memory per CTA (at most " +
                                  std::to_string(kMaxDynSmem) + "): fewer walkers per CTA, "
                                  "fewer atoms or fewer live walkers");
  return JR_OK;
}

// Moves outside the lean walk: a constraint gate or a shear/stretch move.
inline bool needs_ext_walk(const JrParams* p) {
  for (int m = 0; m < p->moves.n_moves; ++m)
    if (p->moves.gate[m] || p->moves.type[m] >= JR_MOVE_SHEAR) return true;
  return false;
}

template <class G, int kT, bool kExt>
int launch_ns_as(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                 const JrInfoBuffers& inf, int n_iter, const JrLaunchConfig& c, void* workspace,
                 cudaStream_t s, const jr::DaArgs& da) {
  auto kern = jr::ns_iterate_kernel<G, kT, kExt>;
  const size_t smem = ns_dyn_smem(dims, params, c, G::kFam);
  int rc = check_smem(smem);
  if (rc) return rc;
  cudaError_t e = ensure_attrs(reinterpret_cast<const void*>(kern), smem, c.cluster > 8);
  if (e != cudaSuccess) return cuda_fail(e, "ns_iterate kernel attributes");
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(dims->n_replicas * c.cluster);
  lc.blockDim = dim3(c.threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = c.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  e = cudaLaunchKernelEx(&lc, kern, *dims, *params, *state, inf, n_iter, (int)c.tpa,
                         (int)c.cluster, (const uint32_t*)workspace, da);
  if (e != cudaSuccess) return cuda_fail(e, "ns_iterate launch");
  return JR_OK;
}

// NS launch of model family F, lean (kExt = false) or full walk.  CTA walks of
// at most 256 threads use a kernel bounded at 256 threads: the compiler may
// then keep up to 255 registers per thread (measured: 3% faster chains than
// the 512-bounded kernel at the same 256-thread shape).
template <int F, bool kExt>
int launch_ns_walk(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                   const JrInfoBuffers& inf, int n_iter, const JrLaunchConfig& c, void* workspace,
                   cudaStream_t s, const jr::DaArgs& da) {
  using Cta = jr::CtaG<F>;
  if constexpr (F == jr::kFamPair) {
    if (c.warp_walkers)
      return launch_ns_as<jr::WarpG<F>, 128, kExt>(dims, params, state, inf, n_iter, c,
                                                   workspace, s, da);
  }
  if constexpr (F != jr::kFamSWDA) {
    if (c.threads <= 256)
      return launch_ns_as<Cta, 256, kExt>(dims, params, state, inf, n_iter, c, workspace, s, da);
  }
  return launch_ns_as<Cta, 512, kExt>(dims, params, state, inf, n_iter, c, workspace, s, da);
}

template <int F>
int launch_ns_family(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                     const JrInfoBuffers& inf, int n_iter, const JrLaunchConfig& c,
                     void* workspace, cudaStream_t s, const jr::DaArgs& da) {
  if (needs_ext_walk(params))
    return launch_ns_walk<F, true>(dims, params, state, inf, n_iter, c, workspace, s, da);
  return launch_ns_walk<F, false>(dims, params, state, inf, n_iter, c, workspace, s, da);
}

// One move per (replica, trial) walker, model family F.
template <int F>
int launch_trial_family(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                        int32_t n_trials, int32_t move_idx, const int32_t* walker_idx,
                        const uint32_t* keys, const uint32_t* move_keys, const float* step,
                        const double* emax, int32_t write_back, int32_t* accepted,
                        int32_t* reject_reason, cudaStream_t s) {
  const JrLaunchConfig c = heuristic_config(dims, F);
  const int nimg = params->model.n_images;
  const int total = dims->n_replicas * n_trials;
  cudaError_t e;
  if constexpr (F == jr::kFamPair) {
    if (c.warp_walkers) {
      using G = jr::WarpG<F>;
      const int gpc = c.threads / 32;
      const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, gpc, F);
      int rc = check_smem(smem);
      if (rc) return rc;
      e = ensure_attrs(reinterpret_cast<const void*>(jr::move_trial_kernel<G, 128>), smem, false);
      if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
      jr::move_trial_kernel<G, 128><<<(total + gpc - 1) / gpc, c.threads, smem, s>>>(
          *dims, *params, *state, n_trials, move_idx, walker_idx, keys, move_keys, step, emax,
          write_back, accepted, reject_reason, c.tpa);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "move_trial launch");
      return JR_OK;
    }
  }
  using G = jr::CtaG<F>;
  const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, 1, F);
  int rc = check_smem(smem);
  if (rc) return rc;
  e = ensure_attrs(reinterpret_cast<const void*>(jr::move_trial_kernel<G, 512>), smem, false);
  if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
  jr::move_trial_kernel<G, 512><<<total, c.threads, smem, s>>>(
      *dims, *params, *state, n_trials, move_idx, walker_idx, keys, move_keys, step, emax,
      write_back, accepted, reject_reason, c.tpa);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "move_trial launch");
  return JR_OK;
}

// The burn-in walk of every walker, model family F.
template <int F>
int launch_population_family(const JrDims* dims, const JrParams* params,
                             const JrStateBuffers* state, int32_t walklength,
                             const uint32_t* run_keys, const uint32_t* move_key,
                             const double* emax, cudaStream_t s) {
  const JrLaunchConfig c = heuristic_config(dims, F);
  const int nimg = params->model.n_images;
  const int total = dims->n_replicas * dims->n_walkers;
  cudaError_t e;
  if constexpr (F == jr::kFamPair) {
    if (c.warp_walkers) {
      using G = jr::WarpG<F>;
      const int gpc = c.threads / 32;
      const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, gpc, F);
      int rc = check_smem(smem);
      if (rc) return rc;
      e = ensure_attrs(reinterpret_cast<const void*>(jr::walk_population_kernel<G, 128>), smem,
                       false);
      if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
      jr::walk_population_kernel<G, 128><<<(total + gpc - 1) / gpc, c.threads, smem, s>>>(
          *dims, *params, *state, walklength, run_keys, move_key, emax, c.tpa);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "walk_population launch");
      return JR_OK;
    }
  }
  using G = jr::CtaG<F>;
  const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, 1, F);
  int rc = check_smem(smem);
  if (rc) return rc;
  e = ensure_attrs(reinterpret_cast<const void*>(jr::walk_population_kernel<G, 512>), smem, false);
  if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
  jr::walk_population_kernel<G, 512><<<total, c.threads, smem, s>>>(
      *dims, *params, *state, walklength, run_keys, move_key, emax, c.tpa);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "walk_population launch");
  return JR_OK;
}

// Energy and forces of a batch of configurations, model family F.
template <int F>
int launch_energy_family(const JrParams* params, int32_t n_configs, int32_t n_atoms_max,
                         const float* positions, const int32_t* types, const float* cell,
                         const int32_t* n_atoms, const float* pressure, const float* mu,
                         double* energy64, double* energy_u, float* forces, cudaStream_t s) {
  JrDims d{};
  d.n_atoms_max = n_atoms_max;
  const JrLaunchConfig c = heuristic_config(&d, F);
  const int nimg = params->model.n_images;
  cudaError_t e;
  if constexpr (F == jr::kFamPair) {
    if (c.warp_walkers) {
      using G = jr::WarpG<F>;
      const int gpc = c.threads / 32;
      const size_t smem = group_dyn_smem(n_atoms_max, nimg, gpc, F);
      int rc = check_smem(smem);
      if (rc) return rc;
      e = ensure_attrs(reinterpret_cast<const void*>(jr::energy_kernel<G, 128>), smem, false);
      if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
      jr::energy_kernel<G, 128><<<(n_configs + gpc - 1) / gpc, c.threads, smem, s>>>(
          *params, n_configs, n_atoms_max, positions, types, cell, n_atoms, pressure, mu,
          energy64, energy_u, forces, c.tpa);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "energy launch");
      return JR_OK;
    }
  }
  using G = jr::CtaG<F>;
  const size_t smem = group_dyn_smem(n_atoms_max, nimg, 1, F);
  int rc = check_smem(smem);
  if (rc) return rc;
  e = ensure_attrs(reinterpret_cast<const void*>(jr::energy_kernel<G, 512>), smem, false);
  if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
  jr::energy_kernel<G, 512><<<n_configs, c.threads, smem, s>>>(
      *params, n_configs, n_atoms_max, positions, types, cell, n_atoms, pressure, mu, energy64,
      energy_u, forces, c.tpa);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "energy launch");
  return JR_OK;
}

}  // namespace jrh

// Explicit instantiations, one translation unit each (they compile in
// parallel): jr_ns.cu the pair family's lean NS walk, jr_pair_ext.cu its full
// NS walk, jr_pair_aux.cu its trial, burn-in and energy kernels, jr_sw.cu the
// whole Stillinger-Weber family.
#define JR_NS_WALK_ARGS                                                                      \
  const JrDims*, const JrParams*, const JrStateBuffers*, const JrInfoBuffers&, int,           \
      const JrLaunchConfig&, void*, cudaStream_t, const jr::DaArgs&
#define JR_TRIAL_ARGS                                                                        \
  const JrDims*, const JrParams*, const JrStateBuffers*, int32_t, int32_t, const int32_t*,     \
      const uint32_t*, const uint32_t*, const float*, const double*, int32_t, int32_t*,       \
      int32_t*, cudaStream_t
#define JR_POP_ARGS                                                                          \
  const JrDims*, const JrParams*, const JrStateBuffers*, int32_t, const uint32_t*,            \
      const uint32_t*, const double*, cudaStream_t
#define JR_ENERGY_ARGS                                                                       \
  const JrParams*, int32_t, int32_t, const float*, const int32_t*, const float*,              \
      const int32_t*, const float*, const float*, double*, double*, float*, cudaStream_t

#ifndef JR_INSTANTIATE_PAIR_EXT
extern template int jrh::launch_ns_walk<jr::kFamPair, true>(JR_NS_WALK_ARGS);
#endif
#ifndef JR_INSTANTIATE_PAIR_AUX
extern template int jrh::launch_trial_family<jr::kFamPair>(JR_TRIAL_ARGS);
extern template int jrh::launch_population_family<jr::kFamPair>(JR_POP_ARGS);
extern template int jrh::launch_energy_family<jr::kFamPair>(JR_ENERGY_ARGS);
#endif
#ifndef JR_INSTANTIATE_SW
extern template int jrh::launch_ns_family<jr::kFamSW>(JR_NS_WALK_ARGS);
extern template int jrh::launch_trial_family<jr::kFamSW>(JR_TRIAL_ARGS);
extern template int jrh::launch_population_family<jr::kFamSW>(JR_POP_ARGS);
extern template int jrh::launch_energy_family<jr::kFamSW>(JR_ENERGY_ARGS);
#endif
#ifndef JR_INSTANTIATE_SWDA
extern template int jrh::launch_ns_family<jr::kFamSWDA>(JR_NS_WALK_ARGS);
#endif
