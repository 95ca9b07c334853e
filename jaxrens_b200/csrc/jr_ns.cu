// jr_ns.cu -- the C-ABI of the nested-sampling walk and the pair family
// (LJ, the Gaussian-mixture toy) of the walk kernels.
//
// The walk kernels live in jr_kernels.cuh, templated on the walking group,
// which carries the model family; this translation unit instantiates the
// pair family and jr_sw.cu the Stillinger-Weber family.  Kernels defined
// here:
//   re_swap_kernel        pressure / semi-grand replica-exchange pass
//   fma_peak_kernel       FP32 FMA-pipe throughput probe
#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>

#include "../../include/jaxrens_b200.h"
#include "jr_host.cuh"

namespace jr {

// --------------------------------------------------------- RE swaps ----
// Ensemble term of walker (p_conf, slot) under replica p_ens's parameters.
// P*V - mu.N of the walker at (p_conf, slot) under run p_ens's ensemble, one
// warp: lanes count the species, every lane returns the same value.
__device__ double walker_ens(const JrDims& D, const JrStateBuffers& st, int p_conf, int slot,
                             int p_ens, int S, int lane) {
  const int K = D.n_walkers, Nmax = D.n_atoms_max;
  const size_t wb = (size_t)p_conf * K + slot;
  const float vol = fabsf(det3(st.cell + wb * 9));
  double e = (double)st.pressure[p_ens] * (double)vol;
  if (st.mu) {
    const int n = min(max(st.n_atoms[p_conf], 1), Nmax);
    double dot = 0.0;
    for (int q = 0; q < S; ++q) {
      int c = 0;
      for (int i = lane; i < n; i += 32)
        c += min(max(st.types[wb * Nmax + i], 0), S - 1) == q ? 1 : 0;
      c = __reduce_add_sync(0xffffffffu, c);
      dot += (double)st.mu[(size_t)p_ens * S + q] * (double)c;
    }
    e = e - dot;
  }
  return e;
}

template <typename Tp>
__device__ void swap_range(Tp* a, Tp* b, int n, int lane) {
  for (int q = lane; q < n; q += 32) {
    Tp t = a[q];
    a[q] = b[q];
    b[q] = t;
  }
}

// replica_exchange_step with EnsembleSwap (replica_exchange.py:318-436).
// One CTA; within a phase the pairs touch disjoint runs, so warp w serves
// pair slots w, w + nwarps, ...; phases and cycles are separated by a CTA
// barrier because each one sees the swaps of the one before.
__global__ void re_swap_kernel(const JrDims D, const JrStateBuffers st, const Key key,
                               const int n_cycles, const int S, int* acc_pp, int* att_pp) {
  const int R = D.n_replicas, K = D.n_walkers, Nmax = D.n_atoms_max;
  const int n_even = R / 2, n_odd = (R - 1) / 2;
  const int max_pairs = n_even > n_odd ? n_even : n_odd;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int q = threadIdx.x; q < R - 1; q += blockDim.x) {
    if (acc_pp) acc_pp[q] = 0;
    if (att_pp) att_pp[q] = 0;
  }
  __syncthreads();
  for (int cyc = 0; cyc < n_cycles; ++cyc) {
    const Key ck = split(key, (uint32_t)cyc);
    for (int phase = 0; phase < 2; ++phase) {
      const Key pk = split(ck, (uint32_t)phase);
      const int nv = phase == 0 ? n_even : n_odd;
      for (int slot = warp; slot < max_pairs && slot < nv; slot += nwarps) {
        const Key sk = split(pk, (uint32_t)slot);
        const int wi = randint(split(sk, 0u), 0, K);
        const int wj = randint(split(sk, 1u), 0, K);
        const int ri = phase + 2 * slot, rj = ri + 1;
        const size_t bi = (size_t)ri * K + wi, bj = (size_t)rj * K + wj;
        // into_i: walker j re-expressed in run i's ensemble (ensemble.py:62-87)
        const double ej = st.energy64[bj], ei = st.energy64[bi];
        const double into_i = (ej - walker_ens(D, st, rj, wj, rj, S, lane)) +
                              walker_ens(D, st, rj, wj, ri, S, lane);
        const double into_j = (ei - walker_ens(D, st, ri, wi, ri, S, lane)) +
                              walker_ens(D, st, ri, wi, rj, S, lane);
        const bool do_swap = (into_i < st.emax[ri]) && (into_j < st.emax[rj]);
        if (do_swap) {
          swap_range(st.positions + bi * Nmax * 3, st.positions + bj * Nmax * 3, Nmax * 3, lane);
          swap_range(st.direction + bi * Nmax * 3, st.direction + bj * Nmax * 3, Nmax * 3, lane);
          swap_range(st.types + bi * Nmax, st.types + bj * Nmax, Nmax, lane);
          swap_range(st.cell + bi * 9, st.cell + bj * 9, 9, lane);
          if (lane == 0) {
            st.energy64[bi] = into_i;
            st.energy64[bj] = into_j;
            st.energy[bi] = __double2float_rn(into_i);
            st.energy[bj] = __double2float_rn(into_j);
          }
        }
        if (lane == 0) {
          if (acc_pp) acc_pp[ri] += do_swap ? 1 : 0;
          if (att_pp) att_pp[ri] += 1;
        }
      }
      __syncthreads();
    }
  }
}

// Independent FMA chains per thread: the FP32 FMA pipe's attainable rate.
__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float b = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = __fmaf_rn(a0, b, c); a1 = __fmaf_rn(a1, b, c);
      a2 = __fmaf_rn(a2, b, c); a3 = __fmaf_rn(a3, b, c);
      a4 = __fmaf_rn(a4, b, c); a5 = __fmaf_rn(a5, b, c);
      a6 = __fmaf_rn(a6, b, c); a7 = __fmaf_rn(a7, b, c);
    }
  }
  const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace jr

// ================================================================ host ====

namespace jrh {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(JR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Identity of the calling thread's current CUDA context (cuCtxGetId, reached
// through the runtime's driver entry points so the library does not link
// libcuda).  Per-device caches key on it: after cudaDeviceReset the device
// gets a new primary context with a new id, so no cached attribute or symbol
// address outlives the context it was made in.  Returns 0 when the query is
// unavailable (then the caches key on the device ordinal alone).
unsigned long long current_ctx_id() {
  using GetCur = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCur get_cur = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_cur = reinterpret_cast<GetCur>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  });
  if (!get_cur || !get_id) return 0;
  CUcontext ctx = nullptr;
  if (get_cur(&ctx) != CUDA_SUCCESS) return 0;
  if (!ctx) {
    // the runtime makes the primary context current lazily; cudaSetDevice
    // initialises it (CUDA 12) without allocating anything
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess ||
        get_cur(&ctx) != CUDA_SUCCESS || !ctx) {
      cudaGetLastError();
      return 0;
    }
  }
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Kernel attributes already set, per (kernel, device context): the largest
// dynamic shared-memory limit raised so far and whether non-portable cluster
// sizes are allowed.  Setting them once keeps cudaFuncSetAttribute off the
// launch path of every later call.
struct FuncAttrs {
  size_t smem = 0;
  bool nonportable = false;
};
std::mutex g_attr_mu;
std::map<std::tuple<const void*, int, unsigned long long>, FuncAttrs> g_attrs;

cudaError_t ensure_attrs(const void* kern, size_t smem, bool nonportable) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long ctx = current_ctx_id();
  std::lock_guard<std::mutex> lk(g_attr_mu);
  FuncAttrs& a = g_attrs[{kern, dev, ctx}];
  if (smem > a.smem) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    a.smem = smem;
  }
  if (nonportable && !a.nonportable) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    a.nonportable = true;
  }
  return cudaSuccess;
}

}  // namespace jrh

namespace {

using jrh::check_config;
using jrh::check_params;
using jrh::cuda_fail;
using jrh::fail;
using jrh::family_of;

struct TuneKey {
  int P, K, N, M, T, nx, S, nimg, model;
  bool operator<(const TuneKey& o) const {
    return std::tie(P, K, N, M, T, nx, S, nimg, model) <
           std::tie(o.P, o.K, o.N, o.M, o.T, o.nx, o.S, o.nimg, o.model);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, JrLaunchConfig> g_tune_cache;

TuneKey tune_key(const JrDims* d, const JrParams* p) {
  return TuneKey{d->n_replicas, d->n_walkers, d->n_atoms_max, d->n_moves, d->n_mcmc_steps,
                 d->n_extra, p->model.n_species, p->model.n_images, p->model.model};
}

}  // namespace

extern "C" {

const char* jr_last_error(void) { return jrh::g_last_error.c_str(); }

int jr_version(void) { return 3; }

// The workspace holds one thing: the snapshot of replica 0's key words taken
// on the stream before the launch (the shared move schedule of batched runs
// must not see the key the launch itself advances).  8 bytes, kept in one
// 256-byte slot; the size does not depend on the dims.
size_t jr_ns_iterate_workspace_size(const JrDims* dims) {
  (void)dims;
  constexpr size_t kKeySnapshotBytes = 2 * sizeof(uint32_t);
  return (kKeySnapshotBytes + 255) / 256 * 256;
}

int jr_ns_iterate(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                  const JrInfoBuffers* info, int32_t n_iter, const JrLaunchConfig* cfg,
                  void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (!state) return fail(JR_ERR_PARAM, "null state");
  if (n_iter < 1) return fail(JR_ERR_PARAM, "n_iter must be >= 1");
  if (!workspace || workspace_bytes < jr_ns_iterate_workspace_size(dims))
    return fail(JR_ERR_WORKSPACE,
                "workspace missing or smaller than jr_ns_iterate_workspace_size()");
  const int fam = family_of(params);
  JrLaunchConfig c;
  if (cfg) {
    c = *cfg;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(tune_key(dims, params));
    c = it != g_tune_cache.end() ? it->second : jrh::ns_heuristic_config(dims, n_iter, fam);
  }
  rc = check_config(c, dims, fam);
  if (rc) return rc;
  if (dims->shared_move_key < 0 || dims->shared_move_key > 2)
    return fail(JR_ERR_PARAM, "shared_move_key must be 0, 1 or 2");
  if (dims->shared_move_key == 2 && (n_iter != 1 || !state->move_key))
    return fail(JR_ERR_PARAM, "an explicit move key (shared_move_key = 2) needs "
                              "state.move_key and n_iter = 1");
  JrInfoBuffers inf{};
  if (info) inf = *info;
  cudaStream_t s = (cudaStream_t)stream;
  // the move-schedule key: a snapshot of replica 0's key (the shared move
  // schedule of every replica, advanced per iteration in the kernel) or the
  // caller's explicit key
  const void* ksrc = dims->shared_move_key == 2 ? (const void*)state->move_key
                                                : (const void*)state->rng_key;
  cudaError_t e = cudaMemcpyAsync(workspace, ksrc, 2 * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "key snapshot");
  const jr::DaArgs none{};
  if (fam == jr::kFamSW)
    return jrh::launch_ns_family<jr::kFamSW>(dims, params, state, inf, n_iter, c, workspace, s,
                                             none);
  return jrh::launch_ns_family<jr::kFamPair>(dims, params, state, inf, n_iter, c, workspace, s,
                                             none);
}

}  // extern "C"

// Scratch of jr_ns_iterate_static: the same bytes jr_ns_iterate keeps in the
// caller's workspace (the snapshot of replica 0's key, rewritten by every call
// before its launch, so nothing in it has to start at zero).
static constexpr size_t kStaticScratchBytes = 256;
static constexpr int kMaxStaticDevices = 64;
static __device__ __align__(256) unsigned char jr_static_scratch[kStaticScratchBytes];
static std::mutex g_static_mu;
static void* g_static_ptr[kMaxStaticDevices];
static unsigned long long g_static_ctx[kMaxStaticDevices];

extern "C" {

// jr_ns_iterate on the library's own static device scratch instead of a
// caller workspace.  The first call on each device resolves the scratch's
// address with cudaGetSymbolAddress (with that device current) and caches it
// together with the id of the device's context; a call that finds another
// context current (the device was reset) resolves the address again.
int jr_ns_iterate_static(const JrDims* dims, const JrParams* params,
                         const JrStateBuffers* state, const JrInfoBuffers* info, int32_t n_iter,
                         const JrLaunchConfig* cfg, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  // the key snapshot fits today whatever the dims; the check keeps the
  // stated limit enforced should the workspace ever grow
  const size_t need = jr_ns_iterate_workspace_size(dims);
  if (need > kStaticScratchBytes)
    return fail(JR_ERR_WORKSPACE, "jr_ns_iterate_static: these dims need " +
                                      std::to_string(need) + " bytes of scratch; the static "
                                      "scratch holds " + std::to_string(kStaticScratchBytes));
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "jr_ns_iterate_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxStaticDevices)
    return fail(JR_ERR_PARAM, "jr_ns_iterate_static: device ordinal beyond 63");
  const unsigned long long ctx = jrh::current_ctx_id();
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    scratch = g_static_ptr[dev];
    if (!scratch || g_static_ctx[dev] != ctx) {
      e = cudaGetSymbolAddress(&scratch, jr_static_scratch);
      if (e != cudaSuccess)
        return cuda_fail(e, "jr_ns_iterate_static: cudaGetSymbolAddress of the static scratch");
      g_static_ptr[dev] = scratch;
      g_static_ctx[dev] = ctx;
    }
  }
  return jr_ns_iterate(dims, params, state, info, n_iter, cfg, scratch, kStaticScratchBytes,
                       stream);
}

int jr_move_trial(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                  int32_t n_trials, int32_t move_idx, const int32_t* walker_idx,
                  const uint32_t* keys, const uint32_t* move_keys, const float* step,
                  const double* emax, int32_t write_back, int32_t* accepted,
                  int32_t* reject_reason, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (n_trials < 1 || !walker_idx || !keys || !step || !emax || !accepted)
    return fail(JR_ERR_PARAM, "trial buffers missing or n_trials < 1");
  if (move_idx >= dims->n_moves) return fail(JR_ERR_PARAM, "move_idx out of range");
  if (move_idx < 0 && !move_keys) return fail(JR_ERR_PARAM, "move_keys needed when move_idx < 0");
  cudaStream_t s = (cudaStream_t)stream;
  if (family_of(params) == jr::kFamSW)
    return jrh::launch_trial_family<jr::kFamSW>(dims, params, state, n_trials, move_idx,
                                                walker_idx, keys, move_keys, step, emax,
                                                write_back, accepted, reject_reason, s);
  return jrh::launch_trial_family<jr::kFamPair>(dims, params, state, n_trials, move_idx,
                                                walker_idx, keys, move_keys, step, emax,
                                                write_back, accepted, reject_reason, s);
}

int jr_walk_population(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                       int32_t walklength, const uint32_t* run_keys, const uint32_t* move_key,
                       const double* emax, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (!state || !run_keys || !move_key || !emax || walklength < 0)
    return fail(JR_ERR_PARAM, "walk_population: null buffer or walklength < 0");
  if (walklength == 0) return JR_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (family_of(params) == jr::kFamSW)
    return jrh::launch_population_family<jr::kFamSW>(dims, params, state, walklength, run_keys,
                                                     move_key, emax, s);
  return jrh::launch_population_family<jr::kFamPair>(dims, params, state, walklength, run_keys,
                                                     move_key, emax, s);
}

int jr_energy_forces(const JrParams* params, int32_t n_configs, int32_t n_atoms_max,
                     const float* positions, const int32_t* types, const float* cell,
                     const int32_t* n_atoms, const float* pressure, const float* mu,
                     double* energy64, double* energy_u, float* forces, void* stream) {
  if (!params || n_configs < 1 || n_atoms_max < 1 || n_atoms_max > JR_MAX_ATOMS || !positions ||
      !types || !cell || !n_atoms || !pressure || !energy64)
    return fail(JR_ERR_PARAM, "invalid energy_forces arguments");
  if (params->model.n_species < 1 || params->model.n_species > JR_MAX_SPECIES ||
      params->model.n_images < 1 || params->model.n_images > JR_MAX_IMAGES ||
      params->model.model < JR_MODEL_LJ || params->model.model > JR_MODEL_SW)
    return fail(JR_ERR_PARAM, "invalid model parameters");
  cudaStream_t s = (cudaStream_t)stream;
  if (family_of(params) == jr::kFamSW) {
    if (params->model.n_species != 1 || params->model.n_images != 1)
      return fail(JR_ERR_UNSUPPORTED,
                  "Stillinger-Weber takes one species and the single minimum image");
    if (n_atoms_max > JR_SW_MAX_ATOMS)
      return fail(JR_ERR_SHAPE, "Stillinger-Weber configurations hold at most " +
                                    std::to_string(JR_SW_MAX_ATOMS) + " atoms");
    return jrh::launch_energy_family<jr::kFamSW>(params, n_configs, n_atoms_max, positions, types,
                                                 cell, n_atoms, pressure, mu, energy64, energy_u,
                                                 forces, s);
  }
  return jrh::launch_energy_family<jr::kFamPair>(params, n_configs, n_atoms_max, positions,
                                                 types, cell, n_atoms, pressure, mu, energy64,
                                                 energy_u, forces, s);
}

int jr_re_swap(const JrDims* dims, const JrStateBuffers* state, uint32_t key0, uint32_t key1,
               int32_t n_swap_cycles, int32_t n_species, int32_t* acc_per_pair,
               int32_t* att_per_pair, void* stream) {
  if (!dims || !state) return fail(JR_ERR_PARAM, "null dims or state");
  if (n_swap_cycles < 0 || n_species < 1 || n_species > JR_MAX_SPECIES)
    return fail(JR_ERR_PARAM, "invalid swap parameters");
  if (dims->n_replicas < 2) return JR_OK;
  const int max_pairs = dims->n_replicas / 2;  // even-phase pairs, >= the odd ones
  const int warps = max_pairs < 1 ? 1 : (max_pairs > 32 ? 32 : max_pairs);
  jr::re_swap_kernel<<<1, 32 * warps, 0, (cudaStream_t)stream>>>(*dims, *state, jr::Key{key0, key1},
                                                        n_swap_cycles, n_species, acc_per_pair,
                                                        att_per_pair);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "re_swap launch");
  return JR_OK;
}

int jr_bench_fma_peak(int n_blocks, int iters, float* scratch, double* flops, void* stream) {
  if (n_blocks < 1 || iters < 1 || !scratch || !flops)
    return fail(JR_ERR_PARAM, "fma_peak arguments");
  jr::fma_peak_kernel<<<n_blocks, 256, 0, (cudaStream_t)stream>>>(scratch, iters);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fma_peak launch");
  *flops = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * (double)n_blocks;
  return JR_OK;
}

}  // extern "C"

// ============================================================ autotune ====
namespace {

// Device copies of the mutable state made for the autotuner (freed when it
// returns).  `fields` lists, per state field, the copy's pointer and bytes.
struct ScratchState {
  JrStateBuffers b{};
  struct Field {
    void* ptr;
    size_t bytes;
  };
  Field fields[16] = {};
  int nf = 0;
  ~ScratchState() {
    for (int i = 0; i < nf; ++i) cudaFree(fields[i].ptr);
  }
  void* take(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    fields[nf++] = Field{p, bytes};
    return p;
  }
};

// Copy the mutable state fields of `s` into fresh device buffers.
int clone_state(const JrDims* d, const JrStateBuffers* s, ScratchState& out, cudaStream_t st) {
  const size_t PK = (size_t)d->n_replicas * d->n_walkers;
  const size_t N = d->n_atoms_max, M = d->n_moves;
  struct F {
    const void* src;
    size_t bytes;
    void** dst;
  };
  out.b = *s;
  F fields[] = {
      {s->positions, PK * N * 3 * 4, (void**)&out.b.positions},
      {s->direction, PK * N * 3 * 4, (void**)&out.b.direction},
      {s->types, PK * N * 4, (void**)&out.b.types},
      {s->energy, PK * 4, (void**)&out.b.energy},
      {s->energy64, PK * 8, (void**)&out.b.energy64},
      {s->cell, PK * 9 * 4, (void**)&out.b.cell},
      {s->step_sizes, PK * M * 4, (void**)&out.b.step_sizes},
      {s->n_accepted, PK * M * 4, (void**)&out.b.n_accepted},
      {s->n_proposed, PK * M * 4, (void**)&out.b.n_proposed},
      {s->rng_key, (size_t)d->n_replicas * 8, (void**)&out.b.rng_key},
      {s->log_evidence, (size_t)d->n_replicas * 8, (void**)&out.b.log_evidence},
      {s->iteration, (size_t)d->n_replicas * 4, (void**)&out.b.iteration},
      {s->emax, (size_t)d->n_replicas * 8, (void**)&out.b.emax},
  };
  for (auto& f : fields) {
    void* q = out.take(f.bytes);
    if (!q) return fail(JR_ERR_CUDA, "autotune scratch allocation failed");
    cudaError_t e = cudaMemcpyAsync(q, f.src, f.bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "autotune scratch copy");
    *f.dst = q;
  }
  return JR_OK;
}

// dst <- src, field by field (two clones of the same state).
int restore_state(ScratchState& dst, const ScratchState& src, cudaStream_t st) {
  for (int i = 0; i < dst.nf; ++i) {
    cudaError_t e = cudaMemcpyAsync(dst.fields[i].ptr, src.fields[i].ptr, dst.fields[i].bytes,
                                    cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "autotune state restore");
  }
  return JR_OK;
}

}  // namespace

// Times every candidate launch shape on the same trajectory: a pristine copy
// of the caller's state is taken once, and before each timed sample a working
// copy is restored from it, so every candidate walks the same iterations from
// the same walkers (and meets the same speculation outcomes).  A sample is
// kSegs consecutive launches of n_iter_probe iterations -- several segments of
// the trajectory, since one launch's speculation outcome (one or two rounds)
// varies from segment to segment.  Each candidate runs once untimed, then
// kReps samples; its score is their median.  The caller's state is not
// touched.
extern "C" int jr_autotune(const JrDims* dims, const JrParams* params,
                           const JrStateBuffers* state, int32_t n_iter_probe,
                           JrLaunchConfig* best, void* stream) {
  constexpr int kReps = 3;
  constexpr int kSegs = 4;
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (!state || !best || n_iter_probe < 1) return fail(JR_ERR_PARAM, "autotune arguments");
  const int fam = family_of(params);
  cudaStream_t st = (cudaStream_t)stream;
  ScratchState pristine, work;
  rc = clone_state(dims, state, pristine, st);
  if (rc) return rc;
  rc = clone_state(dims, state, work, st);
  if (rc) return rc;
  const size_t wsb = jr_ns_iterate_workspace_size(dims);
  ScratchState ws_owner;
  void* ws = ws_owner.take(wsb);
  if (!ws) return fail(JR_ERR_CUDA, "autotune workspace allocation failed");
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return fail(JR_ERR_CUDA, "autotune events");
  float best_ms = 1e30f;
  JrLaunchConfig bc = jrh::ns_heuristic_config(dims, n_iter_probe, fam);
  const int nmax = dims->n_atoms_max;
  JrLaunchConfig cands[96];
  int nc = 0;
  const int clusters[] = {1, 2, 4, 8, 10, 12, 16};
  if (nmax <= 32 && fam == jr::kFamPair) {  // warp walkers: 1..4 walkers per CTA
    for (int wpc : {1, 2, 4})
      for (int cl : clusters) cands[nc++] = JrLaunchConfig{32 * wpc, jrh::warp_tpa(nmax), cl, 1};
  }
  for (int th : {128, 256, 512})
    for (int cl : clusters) {
      int tpa = jrh::pow2_floor(th / nmax);
      tpa = tpa > 16 ? 16 : (tpa < 1 ? 1 : tpa);
      if (nc < 96) cands[nc++] = JrLaunchConfig{th, tpa, cl, 0};
    }
  for (int i = 0; i < nc; ++i) {
    const JrLaunchConfig c = cands[i];
    if (check_config(c, dims, fam) != JR_OK) continue;
    bool ok = restore_state(work, pristine, st) == JR_OK &&
              jr_ns_iterate(dims, params, &work.b, nullptr, n_iter_probe, &c, ws, wsb, stream) ==
                  JR_OK &&
              cudaStreamSynchronize(st) == cudaSuccess;
    float ms[kReps];
    for (int r = 0; r < kReps && ok; ++r) {
      ok = restore_state(work, pristine, st) == JR_OK && cudaEventRecord(e0, st) == cudaSuccess;
      for (int g = 0; g < kSegs && ok; ++g)
        ok = jr_ns_iterate(dims, params, &work.b, nullptr, n_iter_probe, &c, ws, wsb, stream) ==
             JR_OK;
      ok = ok && cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
           cudaEventElapsedTime(&ms[r], e0, e1) == cudaSuccess;
    }
    if (!ok) {  // shape rejected or failed (e.g. too much shared memory): skip it
      cudaGetLastError();
      cudaStreamSynchronize(st);
      continue;
    }
    // median of kReps
    for (int a = 0; a < kReps; ++a)
      for (int b = a + 1; b < kReps; ++b)
        if (ms[b] < ms[a]) {
          const float t = ms[a];
          ms[a] = ms[b];
          ms[b] = t;
        }
    const float med = ms[kReps / 2];
    if (med < best_ms) {
      best_ms = med;
      bc = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key(dims, params)] = bc;
  }
  *best = bc;
  jrh::g_last_error.clear();
  return JR_OK;
}
