// jr_swda.cu -- the delayed-acceptance walk of the Stillinger-Weber model on
// the learned surrogate (jr_da.cuh): its NS launch (the SW-with-surrogate
// family of the walk kernels, compiled apart from the others), the C-ABI
// entry jr_ns_iterate_da, and jr_sur_energy_forces, the surrogate's energy
// and forces as the walk evaluates them.
#define JR_INSTANTIATE_SWDA
#include "jr_host.cuh"

template int jrh::launch_ns_family<jr::kFamSWDA>(JR_NS_WALK_ARGS);

namespace jr {

// One configuration per 512-thread CTA: the walk's surrogate evaluation on a
// walker loaded from the batch.
__global__ void __launch_bounds__(512, 1)
sur_energy_kernel(const JrModelParams mp, const __grid_constant__ JrSurrogate sur,
                  const int nmax, const float* __restrict__ positions,
                  const float* __restrict__ cell, const int32_t* __restrict__ n_atoms,
                  double* __restrict__ energy_u, float* __restrict__ forces) {
  using G = CtaG<kFamSWDA>;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  const int b = blockIdx.x;
  const size_t ptb = pair_table_bytes(nmax, 1, kFamSWDA);
  char* base = reinterpret_cast<char*>(dyn);
  uint16_t* pij = reinterpret_cast<uint16_t*>(base);
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, nmax, 1, pij, arr, false, kFamSWDA);
  const int n = min(max(n_atoms[b], 2), nmax);
  Walker<G> w{*wsp, arr, tab, n, 1, make_group<G>(red), 0};
  w.sur = &sur;
  sur_load_weights(sur, arr);
  zero_pair_matrix(w.g, arr, nmax);
  build_group_pair_table(w.g, pij, n);
  for (int q = threadIdx.x; q < 3 * n; q += blockDim.x) {
    pos_at(arr.xs, q) = positions[(size_t)b * nmax * 3 + q];
    arr.dir[q] = 0.0f;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) arr.xs[i].w = __int_as_float(0);
  if (threadIdx.x == 0) {
    w.s.cur = 0;
    make_cell_ctx(cell + (size_t)b * 9, w.s.cc[0], arr.T, mp);
  }
  __syncthreads();
  double sff, sfd;
  const double U = forces ? sur_ham<true>(w, 0, 0.0, sff, sfd) : sur_ham<false>(w, 0, 0.0, sff, sfd);
  if (threadIdx.x == 0) energy_u[b] = U;
  if (forces)
    for (int q = threadIdx.x; q < 3 * n; q += blockDim.x)
      forces[(size_t)b * nmax * 3 + q] = arr.F[q];
}

}  // namespace jr

namespace {

int check_surrogate(const JrSurrogate* sur) {
  if (!sur || !sur->params) return jrh::fail(JR_ERR_PARAM, "surrogate or its parameters missing");
  if (!(sur->tau > 0.0f)) return jrh::fail(JR_ERR_PARAM, "surrogate tau must be > 0");
  return JR_OK;
}

size_t sur_smem(int nmax) {
  return jr::pair_table_bytes(nmax, 1, jr::kFamSWDA) +
         jr::walker_smem_bytes(nmax, 1, false, jr::kFamSWDA);
}

}  // namespace

extern "C" {

int jr_sur_energy_forces(const JrSurrogate* sur, int32_t n_configs, int32_t n_atoms_max,
                         const float* positions, const float* cell, const int32_t* n_atoms,
                         double* energy_u, float* forces, void* stream) {
  int rc = check_surrogate(sur);
  if (rc) return rc;
  if (n_configs < 0 || n_atoms_max < 2 || n_atoms_max > JR_SW_MAX_ATOMS)
    return jrh::fail(JR_ERR_SHAPE, "need n_configs >= 0 and 2 <= n_atoms_max <= " +
                                       std::to_string(JR_SW_MAX_ATOMS));
  if (!positions || !cell || !n_atoms || !energy_u)
    return jrh::fail(JR_ERR_PARAM, "null positions, cell, n_atoms or energy_u");
  if (n_configs == 0) return JR_OK;
  JrModelParams mp{};
  mp.model = JR_MODEL_SW;
  mp.n_species = 1;
  mp.n_images = 1;
  const size_t smem = sur_smem(n_atoms_max);
  rc = jrh::check_smem(smem);
  if (rc) return rc;
  cudaError_t e =
      jrh::ensure_attrs(reinterpret_cast<const void*>(jr::sur_energy_kernel), smem, false);
  if (e != cudaSuccess) return jrh::cuda_fail(e, "surrogate energy kernel attributes");
  jr::sur_energy_kernel<<<n_configs, 512, smem, (cudaStream_t)stream>>>(
      mp, *sur, n_atoms_max, positions, cell, n_atoms, energy_u, forces);
  e = cudaGetLastError();
  if (e != cudaSuccess) return jrh::cuda_fail(e, "surrogate energy launch");
  return JR_OK;
}

int jr_ns_iterate_da(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                     const JrInfoBuffers* info, const JrSurrogate* sur,
                     const JrSampleRing* ring, int32_t n_iter, const JrLaunchConfig* cfg,
                     void* workspace, size_t workspace_bytes, void* stream) {
  int rc = jrh::check_params(dims, params);
  if (rc) return rc;
  if (params->model.model != JR_MODEL_SW)
    return jrh::fail(JR_ERR_UNSUPPORTED, "the delayed-acceptance walk runs the "
                                         "Stillinger-Weber model");
  rc = check_surrogate(sur);
  if (rc) return rc;
  if (!state) return jrh::fail(JR_ERR_PARAM, "null state");
  if (n_iter < 1) return jrh::fail(JR_ERR_PARAM, "n_iter must be >= 1");
  if (!workspace || workspace_bytes < jr_ns_iterate_workspace_size(dims))
    return jrh::fail(JR_ERR_WORKSPACE,
                     "workspace missing or smaller than jr_ns_iterate_workspace_size()");
  if (dims->shared_move_key < 0 || dims->shared_move_key > 2)
    return jrh::fail(JR_ERR_PARAM, "shared_move_key must be 0, 1 or 2");
  if (dims->shared_move_key == 2 && (n_iter != 1 || !state->move_key))
    return jrh::fail(JR_ERR_PARAM, "an explicit move key (shared_move_key = 2) needs "
                                   "state.move_key and n_iter = 1");
  jr::DaArgs da{};
  da.sur = *sur;
  if (ring && ring->positions) {
    if (!ring->cell || !ring->energy_u || ring->capacity < 1 || ring->base < 0)
      return jrh::fail(JR_ERR_PARAM, "a recording sample ring needs cell, energy_u, "
                                     "capacity >= 1 and base >= 0");
    da.ring = *ring;
  } else if (ring) {
    da.ring.n_surrogate_evaluations = ring->n_surrogate_evaluations;
  }
  JrLaunchConfig c = cfg ? *cfg : jrh::ns_heuristic_config(dims, n_iter, jr::kFamSWDA);
  rc = jrh::check_config(c, dims, jr::kFamSWDA);
  if (rc) return rc;
  if (c.threads != 512)
    return jrh::fail(JR_ERR_PARAM, "the delayed-acceptance walk needs 512-thread CTAs");
  JrInfoBuffers inf{};
  if (info) inf = *info;
  cudaStream_t s = (cudaStream_t)stream;
  const void* ksrc = dims->shared_move_key == 2 ? (const void*)state->move_key
                                                : (const void*)state->rng_key;
  cudaError_t e = cudaMemcpyAsync(workspace, ksrc, 2 * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return jrh::cuda_fail(e, "key snapshot");
  return jrh::launch_ns_family<jr::kFamSWDA>(dims, params, state, inf, n_iter, c, workspace, s,
                                             da);
}

}  // extern "C"
