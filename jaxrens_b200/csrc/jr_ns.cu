// jr_ns.cu -- B200 kernels and the C-ABI of the nested-sampling walk.
//
// Kernels
//   ns_iterate_kernel<G>  n_iter NS iterations for every replica in one
//                      launch.  A thread-block cluster of C CTAs serves one
//                      replica; each CTA walks one chain (G = CtaGroup) or one
//                      chain per warp (G = WarpGroup).  Each round predicts
//                      the culls of the next D iterations -- the PRNG stream
//                      is state independent, and the walker culled at
//                      iteration i+d is the (d+1)-th highest energy as long as
//                      the walkers written by iterations < d stay below it --
//                      walks them concurrently, then commits the longest
//                      prefix whose predictions hold.  Committed results are
//                      exactly those of sequential ns_step calls.
//   move_trial_kernel<G>  one move on many walkers (adaptation, burn-in)
//   energy_kernel<G>      energy + forces of a batch of configurations
//   re_swap_kernel        pressure / semi-grand replica-exchange pass
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>

#include "../../include/jaxrens_b200.h"
#include "jr_rng.cuh"
#include "jr_walk.cuh"

namespace cg = cooperative_groups;

namespace jr {

constexpr int kMaxD = 32;     // speculative iterations per round
constexpr int kMaxWalk = 256; // D * (1 + n_extra) bound

struct NsShared {
  int worst[kMaxD];
  int clone[kMaxD];
  double e[kMaxD];
  int spec[kMaxD];
  Key kmcmc[kMaxD];
  Key kmove[kMaxD];
  int extras[kMaxWalk];
  int wset[kMaxWalk];
  int n_wset;
  Key kchain[kMaxD];        // fast predictions: run key of iteration d
  Key k0chain[kMaxD];       // fast predictions: replica-0 key of iteration d
  int cw[JR_MAX_CULL];     // n_cull > 1: culled walkers, descending energy
  int cc[JR_MAX_CULL];     // n_cull > 1: their clone sources
  double ce[JR_MAX_CULL];  // n_cull > 1: culled energies
  double res_E[kMaxWarps];  // final energy of each chain this CTA walked
  unsigned long long u64[2][kMaxWarps];
  int flag[2][kMaxWarps];
};

__device__ __forceinline__ unsigned long long ord_double(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord_double(unsigned long long k) {
  unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)u);
}

// Block max of a u64 and OR of an int flag; uniform result in every thread.
__device__ inline void block_max_u64(NsShared& ns, int& par, unsigned long long& v, int& f) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
    v = o > v ? o : v;
    f |= __shfl_xor_sync(0xffffffffu, f, off);
  }
  if (lane == 0) {
    ns.u64[par][warp] = v;
    ns.flag[par][warp] = f;
  }
  __syncthreads();
  v = 0;
  f = 0;
  for (int q = 0; q < nw; ++q) {
    v = ns.u64[par][q] > v ? ns.u64[par][q] : v;
    f |= ns.flag[par][q];
  }
  par ^= 1;
}

__device__ __forceinline__ bool in_set(const int* set, int n, int k) {
  for (int q = 0; q < n; ++q)
    if (set[q] == k) return true;
  return false;
}

// _find_worst_walker (nested_sampling.py:86-109) over the candidates not in
// `excl`: jnp.max (NaN-propagating), then argmax of uniform noise among the
// exact ties (first index on equal noise).  CTA-wide.
__device__ void cull_select(NsShared& ns, int& par, const double* E, int K, const int* excl,
                            int nexcl, Key kworst, int& worst, double& emax, bool& any_nan) {
  unsigned long long best = 0;
  int nanf = 0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    if (in_set(excl, nexcl, k)) continue;
    const double x = E[k];
    if (isnan(x)) {
      nanf = 1;
    } else {
      const unsigned long long o = ord_double(x);
      best = o > best ? o : best;
    }
  }
  block_max_u64(ns, par, best, nanf);
  any_nan = nanf != 0;
  if (any_nan) {
    emax = __longlong_as_double(0x7ff8000000000000ll);
    worst = 0;
    return;
  }
  emax = unord_double(best);
  unsigned long long tb = 0;
  int dummy = 0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    if (in_set(excl, nexcl, k)) continue;
    if (E[k] == emax) {
      const float nz = uniform01(bits32(kworst, (uint32_t)k));
      const unsigned long long key =
          ((unsigned long long)__float_as_uint(nz) << 32) | (0xFFFFFFFFu - (unsigned)k);
      tb = key > tb ? key : tb;
    }
  }
  block_max_u64(ns, par, tb, dummy);
  worst = (int)(0xFFFFFFFFu - (unsigned)(tb & 0xFFFFFFFFull));
}

// _get_extra_indices (nested_sampling.py:112-133): the n_extra largest uniform
// noises, worst and clone excluded, stable (lower index first on ties).
__device__ void select_extras(NsShared& ns, int& par, float* noise, int K, int worst, int clone,
                              Key kextra, int n_extra, int* out) {
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    noise[k] = (k == worst || k == clone) ? -1.0f : uniform01(bits32(kextra, (uint32_t)k));
  __syncthreads();
  for (int e = 0; e < n_extra; ++e) {
    unsigned long long tb = 0;
    int dummy = 0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      const float nz = noise[k];
      if (nz < 0.0f) continue;
      const unsigned long long key =
          ((unsigned long long)__float_as_uint(nz) << 32) | (0xFFFFFFFFu - (unsigned)k);
      tb = key > tb ? key : tb;
    }
    block_max_u64(ns, par, tb, dummy);
    const int pick = (int)(0xFFFFFFFFu - (unsigned)(tb & 0xFFFFFFFFull));
    if (threadIdx.x == 0) {
      out[e] = pick;
      noise[pick] = -1.0f;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double logaddexp(double a, double b) {
  const double amax = a > b ? a : b;
  const double delta = a - b;
  if (isnan(delta)) return a + b;
  return amax + log1p(exp(-fabs(delta)));
}

// T MWG steps of one chain.  The step keys split(chain_key, t) and the move
// choices (from split(move_key, t)) do not depend on the walk, so each chunk
// of kStepChunk steps draws them up front, one step per thread.
template <bool kExt, class G>
__device__ __forceinline__ void walk_chain(const JrParams& P, Walker<G>& w, int T, Key chain_key,
                                  Key move_key, double emax, float pressure, const float* mu) {
  WalkShared& s = w.s;
  for (int t0 = 0; t0 < T; t0 += kStepChunk) {
    const int nt = T - t0 < kStepChunk ? T - t0 : kStepChunk;
    for (int q = w.g.rank(); q < nt; q += w.g.size()) {
      StepKey sk = make_step_key(split(chain_key, (uint32_t)(t0 + q)));
      const int mi = choice(split(move_key, (uint32_t)(t0 + q)), P.moves.cum_probs,
                            P.moves.n_moves);
      const int ty = P.moves.type[mi];
      if (ty == JR_MOVE_VOLUME) {
        sk.vn = normal(bits32(sk.k0, 0u));
        sk.vu = uniform01(bits32(sk.k1, 0u));
        sk.pre = 1;
      } else if (ty == JR_MOVE_GALILEAN && w.arr.nz) {
        sk.nz = w.arr.nz + (size_t)q * 3 * w.n;
      }
      s.step_key[q] = sk;
      s.step_move[q] = mi;
    }
    w.g.sync();
    // the galilean perturbation normals of the chunk, all threads at once
    if (w.arr.nz) {
      const int n3 = 3 * w.n;
      for (int e = w.g.rank(); e < nt * n3; e += w.g.size()) {
        const int t = e / n3, q = e - t * n3;
        if (s.step_key[t].nz) w.arr.nz[e] = normal(bits32(s.step_key[t].k1, (uint32_t)q));
      }
      w.g.sync();
    }
    for (int t = 0; t < nt; ++t)
      mwg_step<kExt>(P, w, s.step_key[t], s.step_move[t], emax, pressure, mu);
    w.g.sync();
  }
}

// Copy the about-to-be-culled walker of replica p into info row `row`, cull
// `cull` of that iteration.
template <class G>
__device__ inline void write_dead(const G& g, const JrDims& D, const JrStateBuffers& st,
                                  const JrInfoBuffers& info, int row, int p, int slot, int n,
                                  int cull) {
  const int K = D.n_walkers, Nmax = D.n_atoms_max, Pn = D.n_replicas;
  const size_t wb = (size_t)p * K + slot;
  const size_t ib = ((size_t)row * Pn + p) * D.n_cull + cull;
  const int r0 = g.rank(), gs = g.size();
  if (info.dead_positions)
    for (int q = r0; q < 3 * n; q += gs)
      info.dead_positions[ib * Nmax * 3 + q] = st.positions[wb * Nmax * 3 + q];
  if (info.dead_types)
    for (int q = r0; q < n; q += gs) info.dead_types[ib * Nmax + q] = st.types[wb * Nmax + q];
  if (info.dead_cell)
    for (int q = r0; q < 9; q += gs) info.dead_cell[ib * 9 + q] = st.cell[wb * 9 + q];
  g.sync();
}

__device__ inline void copy_params(JrParams& dst, const JrParams& src) {
  const int nw = (int)(sizeof(JrParams) / 4);
  const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int q = threadIdx.x; q < nw; q += blockDim.x) d[q] = s[q];
}

// Dynamic smem of the NS kernel: [K doubles][K floats](n_cull > 1: 3 x
// [K ints])[pair table][walkers].
struct DynLayout {
  double* Epop;
  float* noise;
  int* order;     // n_cull > 1: walkers by descending energy, then survivors
  int* tmp;       // n_cull > 1: shuffle scratch
  uint32_t* u;    // n_cull > 1: shuffle sort keys
  uint16_t* pij;
  char* walkers;
  size_t walker_bytes;
};

__host__ __device__ inline size_t dyn_head_bytes(int K, int nmax, int nimg, int ncull) {
  return align16(8u * (size_t)K) + align16(4u * (size_t)K) +
         (ncull > 1 ? 3u * align16(4u * (size_t)K) : 0u) + pair_table_bytes(nmax, nimg);
}

__device__ inline DynLayout dyn_layout(unsigned char* dyn, int K, int nmax, int nimg, int ncull) {
  DynLayout L;
  char* p = reinterpret_cast<char*>(dyn);
  L.Epop = reinterpret_cast<double*>(p);
  p += align16(8u * (size_t)K);
  L.noise = reinterpret_cast<float*>(p);
  p += align16(4u * (size_t)K);
  L.order = L.tmp = nullptr;
  L.u = nullptr;
  if (ncull > 1) {
    L.order = reinterpret_cast<int*>(p);
    p += align16(4u * (size_t)K);
    L.tmp = reinterpret_cast<int*>(p);
    p += align16(4u * (size_t)K);
    L.u = reinterpret_cast<uint32_t*>(p);
    p += align16(4u * (size_t)K);
  }
  L.pij = use_pair_matrix(nmax, nimg) ? reinterpret_cast<uint16_t*>(p) : nullptr;
  p += pair_table_bytes(nmax, nimg);
  L.walkers = p;
  L.walker_bytes = walker_smem_bytes(nmax, nimg, true);
  return L;
}

// The Dr predictions of a round for n_cull = 1 without extras and K <= 1024,
// identical to Dr sequential cull_select/randint passes but without their
// block barriers: warp 0 walks the run-key chain while warp 1 walks the
// replica-0 key chain, lane d then derives iteration d's keys and raw clone
// draw, and warp 0 selects the Dr culls from registers (walker k in lane
// k % 32, bit k / 32 of a per-lane mask once culled): the maximum energy
// (any NaN poisons it, culling walker 0), exact ties broken by the largest
// uniform noise of that iteration's worst key, then the lowest index.
__device__ void predict_fast(NsShared& ns, const double* E, int K, int Dr, Key key, Key key0,
                             bool shared_mk) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp == 0) {
    Key kd = key;
    for (int d = 0; d < Dr; ++d) {
      if (lane == 0) ns.kchain[d] = kd;
      kd = split(split(kd, 0u), 0u);
    }
  } else if (warp == 1 && shared_mk) {
    Key k0 = key0;
    for (int d = 0; d < Dr; ++d) {
      if (lane == 0) ns.k0chain[d] = k0;
      k0 = advance_iteration(k0);
    }
  }
  __syncthreads();
  if (warp != 0) return;
  // per-iteration keys and raw clone draws, one lane per iteration
  Key my_kw{0u, 0u};
  int my_raw = 0;
  if (lane < Dr) {
    const Key kd = ns.kchain[lane];
    const Key ka = split(kd, 0u);
    my_kw = split(kd, 1u);
    my_raw = randint(split(ka, 1u), 0, K - 1);
    ns.kmcmc[lane] = split(ka, 3u);
    ns.kmove[lane] = shared_mk ? split(ns.k0chain[lane], 1u) : split(ka, 4u);
  }
  const int nslot = (K + 31) >> 5;
  uint32_t taken = 0;
  bool prev_ok = true;
  double prev_e = 0.0;
  // this lane's largest non-culled energy (ordered bits) and NaN flag; only
  // the lane that loses a walker to a cull rescans its entries
  unsigned long long lbest = 0;
  int lnan = 0;
  auto lane_scan = [&]() {
    lbest = 0;
    lnan = 0;
    for (int j = 0; j < nslot; ++j) {
      const int k = lane + 32 * j;
      if (k >= K || ((taken >> j) & 1u)) continue;
      const double x = E[k];
      if (isnan(x)) {
        lnan = 1;
      } else {
        const unsigned long long o = ord_double(x);
        lbest = o > lbest ? o : lbest;
      }
    }
  };
  lane_scan();
  for (int d = 0; d < Dr; ++d) {
    unsigned long long best = lbest;
    int nanf = lnan;
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
      best = o > best ? o : best;
      nanf |= __shfl_xor_sync(0xffffffffu, nanf, off);
    }
    const bool any_nan = nanf != 0;
    int worst = 0;
    double emax = __longlong_as_double(0x7ff8000000000000ll);
    if (!any_nan) {
      emax = unord_double(best);
      // walkers at the maximum: a unique one is the cull whatever the noise;
      // exact ties are broken by the largest noise of this iteration's key
      int nties = 0, idx1 = 0;
      // (== on the values: -0.0 ties with +0.0, as in the reference's E == max)
      if (lbest != 0 && unord_double(lbest) == emax) {
        for (int j = 0; j < nslot; ++j) {
          const int k = lane + 32 * j;
          if (k >= K || ((taken >> j) & 1u) || E[k] != emax) continue;
          ++nties;
          idx1 = k + 1;
        }
      }
      int tot = nties, idx = idx1;
      for (int off = 16; off > 0; off >>= 1) {
        tot += __shfl_xor_sync(0xffffffffu, tot, off);
        const int o = __shfl_xor_sync(0xffffffffu, idx, off);
        idx = o > idx ? o : idx;
      }
      if (tot == 1) {
        worst = idx - 1;
      } else {
        const Key kw{__shfl_sync(0xffffffffu, my_kw.k0, d), __shfl_sync(0xffffffffu, my_kw.k1, d)};
        unsigned long long tb = 0;
        if (nties > 0) {
          for (int j = 0; j < nslot; ++j) {
            const int k = lane + 32 * j;
            if (k >= K || ((taken >> j) & 1u) || E[k] != emax) continue;
            const float nz = uniform01(bits32(kw, (uint32_t)k));
            const unsigned long long t =
                ((unsigned long long)__float_as_uint(nz) << 32) | (0xFFFFFFFFu - (unsigned)k);
            tb = t > tb ? t : tb;
          }
        }
        for (int off = 16; off > 0; off >>= 1) {
          const unsigned long long o = __shfl_xor_sync(0xffffffffu, tb, off);
          tb = o > tb ? o : tb;
        }
        worst = (int)(0xFFFFFFFFu - (unsigned)(tb & 0xFFFFFFFFull));
      }
    }
    int clone = __shfl_sync(0xffffffffu, my_raw, d);
    if (clone >= worst) clone += 1;
    // a clone source culled earlier in the round breaks the prediction chain
    const unsigned cbit = __shfl_sync(0xffffffffu, taken, clone & 31);
    const bool conflict = d > 0 && ((cbit >> (clone >> 5)) & 1u);
    const bool sp = d == 0 || (prev_ok && !any_nan && !isnan(prev_e) && !conflict);
    if (lane == (worst & 31)) {
      taken |= 1u << (worst >> 5);
      if (d + 1 < Dr) lane_scan();
    }
    if (lane == 0) {
      ns.spec[d] = sp ? 1 : 0;
      ns.worst[d] = worst;
      ns.clone[d] = clone;
      ns.e[d] = emax;
      ns.wset[ns.n_wset++] = worst;
    }
    prev_ok = sp;
    prev_e = emax;
  }
}

// _select_culls for n_cull > 1 (nested_sampling.py:195-212).  order = the
// walkers by descending energy (NaN last, as XLA's float sort places it),
// then descending uniform noise, then index (lexsort((-noise, -E)));
// worst = order[:n_cull].  The survivors order[n_cull:] are shuffled like
// jax.random.permutation on an array: ceil(3 ln n / ln(2^32 - 1)) rounds
// (1 for n <= 1625, 2 up to 2642245), each splitting the key and stably
// sorting by 32-bit random bits; clone = survivors[:n_cull], extras =
// survivors[n_cull:n_cull + n_extra].  CTA-wide, ranks by counting.
__device__ void select_culls_multi(NsShared& ns, const DynLayout& L, const double* E, int K,
                                   int ncull, int nx, Key kworst, Key kclone) {
  for (int k = threadIdx.x; k < K; k += blockDim.x) L.noise[k] = uniform01(bits32(kworst, (uint32_t)k));
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const double ek = E[k];
    const bool nk = isnan(ek);
    const float zk = L.noise[k];
    int r = 0;
    for (int j = 0; j < K; ++j) {
      const double ej = E[j];
      const bool nj = isnan(ej);
      bool before;
      if (nj != nk) before = nk;
      else if (!nj && ej != ek) before = ej > ek;
      else if (L.noise[j] != zk) before = L.noise[j] > zk;
      else before = j < k;
      r += before ? 1 : 0;
    }
    L.order[r] = k;
  }
  __syncthreads();
  const int n = K - ncull;
  int* x = L.order + ncull;
  const int rounds = n <= 1 ? 0 : (n <= 1625 ? 1 : 2);
  Key key = kclone;
  for (int rd = 0; rd < rounds; ++rd) {
    const Key sub = split(key, 1u);
    key = split(key, 0u);
    for (int m = threadIdx.x; m < n; m += blockDim.x) L.u[m] = bits32(sub, (uint32_t)m);
    __syncthreads();
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      const uint32_t um = L.u[m];
      int pos = 0;
      for (int q = 0; q < n; ++q) {
        const uint32_t uq = L.u[q];
        pos += (uq < um || (uq == um && q < m)) ? 1 : 0;
      }
      L.tmp[pos] = x[m];
    }
    __syncthreads();
    for (int m = threadIdx.x; m < n; m += blockDim.x) x[m] = L.tmp[m];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int c = 0; c < ncull; ++c) {
      ns.cw[c] = L.order[c];
      ns.cc[c] = x[c];
      ns.ce[c] = E[L.order[c]];
    }
    for (int e = 0; e < nx; ++e) ns.extras[e] = x[ncull + e];
  }
  __syncthreads();
}

template <class G>
__device__ __forceinline__ G make_group(double (*red)[kMaxWarps][3]);
template <>
__device__ __forceinline__ CtaGroup make_group<CtaGroup>(double (*red)[kMaxWarps][3]) {
  return CtaGroup{red};
}
template <>
__device__ __forceinline__ WarpGroup make_group<WarpGroup>(double (*)[kMaxWarps][3]) {
  return WarpGroup{};
}

// Pair decode table of one group's walker (the group's own n).
template <class G>
__device__ inline void build_group_pair_table(const G& g, uint16_t* pij, int n) {
  if (!pij) return;
  const int np = n * (n - 1) / 2;
  for (int q = g.rank(); q < np; q += g.size()) {
    int a = 0;
    while ((a + 1) * (2 * n - a - 2) / 2 <= q) ++a;
    pij[q] = (uint16_t)(a | ((q - a * (2 * n - a - 1) / 2 + a + 1) << 8));
  }
  g.sync();
}

template <class G, int kMaxThreads, bool kExt>
__global__ void __launch_bounds__(kMaxThreads, 1)
ns_iterate_kernel(const JrDims D, const JrParams Pg, const JrStateBuffers st,
                  const JrInfoBuffers info, const int n_iter, const int tpa, const int C,
                  const uint32_t* __restrict__ key0_base) {
  constexpr bool kWarp = std::is_same<G, WarpGroup>::value;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ NsShared ns;
  __shared__ JrParams P;
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  copy_params(P, Pg);
  cg::cluster_group cluster = cg::this_cluster();
  const int p = blockIdx.x / C;
  const int c = blockIdx.x % C;
  const int K = D.n_walkers, M = D.n_moves, T = D.n_mcmc_steps;
  const int nx = D.n_extra, ncull = D.n_cull, W = ncull + nx;
  const int n = min(max(st.n_atoms[p], 1), D.n_atoms_max);
  const int nimg = Pg.model.n_images;
  const int cpc = kWarp ? (int)(blockDim.x >> 5) : 1;  // chains per CTA
  const int my = kWarp ? (int)(threadIdx.x >> 5) : 0;  // this group's chain in the CTA
  const int slots = C * cpc;
  const int s_my = c * cpc + my;
  // speculation needs the n_cull = 1 selection (the top of the order only)
  const int Dmax = (ncull == 1 && slots >= 2 * W) ? (slots / W < kMaxD ? slots / W : kMaxD) : 1;
  DynLayout L = dyn_layout(dyn, K, D.n_atoms_max, nimg, D.n_cull);
  WalkArrays arr;
  WalkShared* wsp = carve_walker(L.walkers + (size_t)my * L.walker_bytes, D.n_atoms_max, nimg,
                                 L.pij, arr, true);
  Walker<G> w{*wsp, arr, tab, n, tpa, make_group<G>(red), 0};
  zero_pair_matrix(w.g, arr, D.n_atoms_max);
  int par = 0;
  __syncthreads();
  load_tables(P, tab);
  build_pair_table(L.pij, n);
  __syncthreads();
  const float pressure = st.pressure[p];
  const float* mu = st.mu ? st.mu + (size_t)p * P.model.n_species : nullptr;
  Key key{st.rng_key[2 * p], st.rng_key[2 * p + 1]};
  Key key0{key0_base[0], key0_base[1]};
  int iter = st.iteration[p];
  double logZ = st.log_evidence[p];
  int committed = 0, rounds = 0;
  while (committed < n_iter) {
    const int Dr = (n_iter - committed) < Dmax ? (n_iter - committed) : Dmax;
    for (int k = threadIdx.x; k < K; k += blockDim.x) L.Epop[k] = st.energy64[(size_t)p * K + k];
    if (threadIdx.x == 0) ns.n_wset = 0;
    __syncthreads();
    // ---- predictions for iterations d < Dr (every CTA, identically) ----
    const bool fast = ncull == 1 && nx == 0 && K <= 1024 && blockDim.x >= 64;
    if (fast) predict_fast(ns, L.Epop, K, Dr, key, key0, D.shared_move_key != 0);
    __syncthreads();
    Key kd = key, k0d = key0;
    for (int d = 0; d < (fast ? 0 : Dr); ++d) {
      const Key ka = split(kd, 0u), kw = split(kd, 1u);
      const Key kclone = split(ka, 1u), kextra = split(ka, 2u);
      const Key kmcmc = split(ka, 3u), kmoves = split(ka, 4u);
      if (ncull > 1) {  // Dr == 1 here
        select_culls_multi(ns, L, L.Epop, K, ncull, nx, kw, kclone);
        if (threadIdx.x == 0) {
          ns.spec[0] = 1;
          ns.worst[0] = ns.cw[0];
          ns.clone[0] = ns.cc[0];
          ns.e[0] = ns.ce[ncull - 1];
          ns.kmcmc[0] = kmcmc;
          ns.kmove[0] = D.shared_move_key ? split(k0d, 1u) : kmoves;
        }
        __syncthreads();
        kd = split(ka, 0u);
        k0d = advance_iteration(k0d);
        continue;
      }
      int worst;
      double emax;
      bool any_nan;
      cull_select(ns, par, L.Epop, K, ns.wset, ns.n_wset, kw, worst, emax, any_nan);
      int clone = randint(kclone, 0, K - 1);
      if (clone >= worst) clone += 1;
      if (nx > 0) select_extras(ns, par, L.noise, K, worst, clone, kextra, nx, ns.extras + d * nx);
      __syncthreads();
      if (threadIdx.x == 0) {
        bool sp = (d == 0);
        if (d > 0) {
          sp = ns.spec[d - 1] && !any_nan && !isnan(ns.e[d - 1]) &&
               !in_set(ns.wset, ns.n_wset, clone);
          for (int e = 0; e < nx && sp; ++e)
            if (in_set(ns.wset, ns.n_wset, ns.extras[d * nx + e])) sp = false;
        }
        ns.spec[d] = sp ? 1 : 0;
        ns.worst[d] = worst;
        ns.clone[d] = clone;
        ns.e[d] = emax;
        ns.kmcmc[d] = kmcmc;
        ns.kmove[d] = D.shared_move_key ? split(k0d, 1u) : kmoves;
        ns.wset[ns.n_wset++] = worst;
        for (int e = 0; e < nx; ++e) ns.wset[ns.n_wset++] = ns.extras[d * nx + e];
      }
      __syncthreads();
      kd = split(ka, 0u);
      k0d = advance_iteration(k0d);
    }
    // ---- walk ----
    if (w.g.leader()) {
      zero_chain_counters(w.s);
      ns.res_E[my] = 0.0;
    }
    __syncthreads();
    if (Dmax == 1) {
      for (int sidx = s_my; sidx < W; sidx += slots) {
        const bool is_clone = sidx < ncull;
        const int src = is_clone ? (ncull > 1 ? ns.cc[sidx] : ns.clone[0]) : ns.extras[sidx - ncull];
        const int dst = is_clone ? (ncull > 1 ? ns.cw[sidx] : ns.worst[0]) : src;
        if (is_clone) write_dead(w.g, D, st, info, committed, p, dst, n, sidx);
        load_walker(P, D, st, w, p, src, is_clone);
        walk_chain<kExt>(P, w, T, split(ns.kmcmc[0], (uint32_t)sidx), ns.kmove[0], ns.e[0],
                         pressure, mu);
        store_walker(D, st, w, p, dst);
      }
    } else {
      const int d = s_my / W, wi = s_my % W;
      if (d < Dr && ns.spec[d]) {
        const int src = wi == 0 ? ns.clone[d] : ns.extras[d * nx + wi - 1];
        load_walker(P, D, st, w, p, src, wi == 0);
        walk_chain<kExt>(P, w, T, split(ns.kmcmc[d], (uint32_t)wi), ns.kmove[d], ns.e[d], pressure,
                         mu);
        if (w.g.leader()) ns.res_E[my] = w.s.E;
      }
    }
    __syncthreads();
    __threadfence();
    cluster.sync();
    // ---- validation: longest prefix whose predicted culls hold ----
    int nval = 1;
    if (Dmax > 1) {
      nval = 0;
      for (int d = 0; d < Dr; ++d) {
        bool ok = ns.spec[d] != 0;
        for (int d2 = 0; d2 < d && ok; ++d2)
          for (int w2 = 0; w2 < W && ok; ++w2) {
            const int sl = d2 * W + w2;
            const double* r = cluster.map_shared_rank(&ns.res_E[sl % cpc], sl / cpc);
            if (!(*r < ns.e[d])) ok = false;
          }
        if (!ok) break;
        ++nval;
      }
      const int d = s_my / W, wi = s_my % W;
      if (d < nval) {
        const int dst = wi == 0 ? ns.worst[d] : ns.extras[d * nx + wi - 1];
        if (wi == 0) write_dead(w.g, D, st, info, committed + d, p, ns.worst[d], n, 0);
        store_walker(D, st, w, p, dst);
      }
    }
    // ---- per-iteration move counters: the group that walked the first slot
    // of a committed iteration sums that iteration's slots and writes them
    // (its own slot from local shared memory), all iterations in parallel ----
    {
      const int d_own = Dmax == 1 ? (s_my == 0 ? 0 : -1)
                                  : ((s_my % W == 0 && s_my / W < nval) ? s_my / W : -1);
      if (d_own >= 0 && w.g.leader()) {
        const size_t ib = (size_t)(committed + d_own) * D.n_replicas + p;
        const int s0 = Dmax == 1 ? 0 : d_own * W;
        const int s1 = Dmax == 1 ? (slots < W ? slots : W) : d_own * W + W;
        for (int m = 0; m < M; ++m) {
          int a = 0, pr = 0, ne = 0, ng = 0, rr[4] = {0, 0, 0, 0};
          for (int sl = s0; sl < s1; ++sl) {
            const WalkShared* local = reinterpret_cast<const WalkShared*>(
                L.walkers + (size_t)(sl % cpc) * L.walker_bytes);
            const WalkShared* rs = sl == s_my ? local : cluster.map_shared_rank(local, sl / cpc);
            a += rs->c_acc[m];
            pr += rs->c_prop[m];
            ne += rs->c_nev[m];
            ng += rs->c_ngr[m];
            for (int q = 0; q < 4; ++q) rr[q] += rs->c_rr[4 * m + q];
          }
          if (info.n_accepted) info.n_accepted[ib * M + m] = a;
          if (info.n_proposed) info.n_proposed[ib * M + m] = pr;
          if (info.n_evaluations) info.n_evaluations[ib * M + m] = ne;
          if (info.n_grad_evaluations) info.n_grad_evaluations[ib * M + m] = ng;
          if (info.reject_reason_counts)
            for (int q = 0; q < 4; ++q) info.reject_reason_counts[(ib * M + m) * 4 + q] = rr[q];
        }
      }
    }
    // ---- per-iteration culls, evidence and replica scalars (CTA 0) ----
    if (c == 0 && threadIdx.x == 0) {
      int it = iter;
      for (int d = 0; d < nval; ++d, ++it) {
        const size_t ib = (size_t)(committed + d) * D.n_replicas + p;
        if (ncull == 1) {
          const double lw = (double)it * P.log_alpha + P.w_offset[0];
          logZ = logaddexp(logZ, lw - ns.e[d]);
          if (info.worst_idx) info.worst_idx[ib] = ns.worst[d];
          if (info.clone_idx) info.clone_idx[ib] = ns.clone[d];
          if (info.dead_energy) info.dead_energy[ib] = ns.e[d];
        } else {
          // logsumexp over the culls (jax.nn.logsumexp with its finite shift)
          double lw[JR_MAX_CULL];
          double amax = -INFINITY;
          for (int q = 0; q < ncull; ++q) {
            lw[q] = (double)it * P.log_alpha + P.w_offset[q] - ns.ce[q];
            if (lw[q] > amax || isnan(lw[q])) amax = lw[q];
          }
          if (!isfinite(amax)) amax = 0.0;
          double sum = 0.0;
          for (int q = 0; q < ncull; ++q) sum += exp(lw[q] - amax);
          logZ = logaddexp(logZ, log(sum) + amax);
          for (int q = 0; q < ncull; ++q) {
            if (info.worst_idx) info.worst_idx[ib * ncull + q] = ns.cw[q];
            if (info.clone_idx) info.clone_idx[ib * ncull + q] = ns.cc[q];
            if (info.dead_energy) info.dead_energy[ib * ncull + q] = ns.ce[q];
          }
        }
        if (info.emax) info.emax[ib] = ns.e[d];
        if (info.log_evidence) info.log_evidence[ib] = logZ;
      }
    }
    if (fast) {
      // the predictions stored the chain: kchain[d] is the key after d
      // iterations, so the committed key is one advance past kchain[nval-1]
      key = advance_iteration(ns.kchain[nval - 1]);
      if (D.shared_move_key) key0 = advance_iteration(ns.k0chain[nval - 1]);
      else
        for (int d = 0; d < nval; ++d) key0 = advance_iteration(key0);
    } else {
      for (int d = 0; d < nval; ++d) {
        key = advance_iteration(key);
        key0 = advance_iteration(key0);
      }
    }
    if (c == 0 && threadIdx.x == 0) {
      st.emax[p] = ns.e[nval - 1];
      st.iteration[p] = iter + nval;
      st.log_evidence[p] = logZ;
      st.rng_key[2 * p] = key.k0;
      st.rng_key[2 * p + 1] = key.k1;
    }
    iter += nval;
    committed += nval;
    ++rounds;
    __syncthreads();
    __threadfence();
    cluster.sync();
  }
  if (c == 0 && threadIdx.x == 0 && info.rounds) info.rounds[p] = rounds;
}

// ------------------------------------------------------------ trials ----
// One walker per group; the grid covers P * n_trials walkers.  Walkers of one
// CTA may belong to different replicas, so every group has its own pair table.
template <class G, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads, 1)
move_trial_kernel(const JrDims D, const JrParams Pg, const JrStateBuffers st, const int n_trials,
                  const int move_idx, const int* walker_idx, const uint32_t* keys,
                  const uint32_t* move_keys, const float* step, const double* emax,
                  const int write_back, int* accepted, int* reject_reason, const int tpa) {
  constexpr bool kWarp = std::is_same<G, WarpGroup>::value;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ JrParams P;
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  copy_params(P, Pg);
  const int gpc = kWarp ? (int)(blockDim.x >> 5) : 1;
  const int my = kWarp ? (int)(threadIdx.x >> 5) : 0;
  const int total = D.n_replicas * n_trials;
  const int t_global = blockIdx.x * gpc + my;
  const int nimg = Pg.model.n_images;
  const size_t ptb = pair_table_bytes(D.n_atoms_max, nimg);
  char* base = reinterpret_cast<char*>(dyn) +
               (size_t)my * (ptb + walker_smem_bytes(D.n_atoms_max, nimg));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, D.n_atoms_max, nimg, pij, arr);
  __syncthreads();
  load_tables(P, tab);
  __syncthreads();
  if (t_global >= total) return;  // whole group leaves together
  const int p = t_global / n_trials;
  const int n = min(max(st.n_atoms[p], 1), D.n_atoms_max);
  Walker<G> w{*wsp, arr, tab, n, tpa, make_group<G>(red), 0};
  zero_pair_matrix(w.g, arr, D.n_atoms_max);
  build_group_pair_table(w.g, pij, n);
  const size_t tb = (size_t)t_global;
  const int slot = walker_idx[tb];
  if (slot < 0 || slot >= D.n_walkers) {  // invalid index: report, touch nothing
    if (w.g.leader()) {
      accepted[tb] = -1;
      if (reject_reason) reject_reason[tb] = -1;
    }
    return;
  }
  load_walker(P, D, st, w, p, slot, false);
  const float* mu = st.mu ? st.mu + (size_t)p * P.model.n_species : nullptr;
  const Key key{keys[2 * tb], keys[2 * tb + 1]};
  int idx = move_idx;
  if (idx < 0) {
    const Key mk{move_keys[2 * tb], move_keys[2 * tb + 1]};
    idx = choice(mk, P.moves.cum_probs, P.moves.n_moves);
  }
  int reason = 0;
  const bool acc = gated_move<true>(P, w, idx, make_step_key(key), step[p], emax[p], st.pressure[p],
                                   mu, reason);
  w.g.sync();
  if (w.g.leader()) {
    accepted[tb] = acc ? 1 : 0;
    if (reject_reason) reject_reason[tb] = acc ? 0 : (reason > 1 ? reason : 1);
    if (write_back) {
      w.s.w_prop[idx] += 1;
      w.s.w_acc[idx] += acc ? 1 : 0;
    }
  }
  if (write_back) store_walker(D, st, w, p, slot);
}

// ------------------------------------------------------- burn-in walk ----
// _one_walk (init/burn_in.py:48-127): every walker k of every run p takes
// `walklength` MWG steps under the fixed contour emax[p], chain keys
// split(split(run_key[p], K)[k], walklength) and the move schedule
// split(move_key, walklength) shared by every walker and run; step sizes
// are the walker's own and its acceptance counters advance.  One group per
// walker, walkers of one CTA may belong to different runs.
template <class G, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads, 1)
walk_population_kernel(const JrDims D, const JrParams Pg, const JrStateBuffers st,
                       const int walklength, const uint32_t* run_keys,
                       const uint32_t* move_key, const double* emax, const int tpa) {
  constexpr bool kWarp = std::is_same<G, WarpGroup>::value;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ JrParams P;
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  copy_params(P, Pg);
  const int gpc = kWarp ? (int)(blockDim.x >> 5) : 1;
  const int my = kWarp ? (int)(threadIdx.x >> 5) : 0;
  const int K = D.n_walkers;
  const int total = D.n_replicas * K;
  const int t_global = blockIdx.x * gpc + my;
  const int nimg = Pg.model.n_images;
  const size_t ptb = pair_table_bytes(D.n_atoms_max, nimg);
  char* base = reinterpret_cast<char*>(dyn) +
               (size_t)my * (ptb + walker_smem_bytes(D.n_atoms_max, nimg));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, D.n_atoms_max, nimg, pij, arr);
  __syncthreads();
  load_tables(P, tab);
  __syncthreads();
  if (t_global >= total) return;  // whole group leaves together
  const int p = t_global / K, slot = t_global % K;
  const int n = min(max(st.n_atoms[p], 1), D.n_atoms_max);
  Walker<G> w{*wsp, arr, tab, n, tpa, make_group<G>(red), 0};
  zero_pair_matrix(w.g, arr, D.n_atoms_max);
  build_group_pair_table(w.g, pij, n);
  load_walker(P, D, st, w, p, slot, false);
  const float* mu = st.mu ? st.mu + (size_t)p * P.model.n_species : nullptr;
  const Key rk{run_keys[2 * p], run_keys[2 * p + 1]};
  const Key mk{move_key[0], move_key[1]};
  walk_chain<true>(P, w, walklength, split(rk, (uint32_t)slot), mk, emax[p], st.pressure[p], mu);
  store_walker(D, st, w, p, slot);
}

// ------------------------------------------------------------ energy ----
template <class G, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads, 1)
energy_kernel(const JrParams Pg, const int n_configs, const int nmax, const float* positions,
              const int32_t* types, const float* cell, const int32_t* n_atoms,
              const float* pressure, const float* mu, double* energy64, double* energy_u,
              float* forces, const int tpa) {
  constexpr bool kWarp = std::is_same<G, WarpGroup>::value;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ JrParams P;
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  copy_params(P, Pg);
  const int gpc = kWarp ? (int)(blockDim.x >> 5) : 1;
  const int my = kWarp ? (int)(threadIdx.x >> 5) : 0;
  const int b = blockIdx.x * gpc + my;
  const int nimg = Pg.model.n_images;
  const size_t ptb = pair_table_bytes(nmax, nimg);
  char* base = reinterpret_cast<char*>(dyn) + (size_t)my * (ptb + walker_smem_bytes(nmax, nimg));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, nmax, nimg, pij, arr);
  __syncthreads();
  load_tables(P, tab);
  __syncthreads();
  if (b >= n_configs) return;
  const int n = min(max(n_atoms[b], 1), nmax);
  const int smax = Pg.model.n_species - 1;
  Walker<G> w{*wsp, arr, tab, n, tpa, make_group<G>(red), 0};
  zero_pair_matrix(w.g, arr, nmax);
  build_group_pair_table(w.g, pij, n);
  const int r0 = w.g.rank(), gs = w.g.size();
  for (int q = r0; q < 3 * n; q += gs) {
    pos_at(arr.xs, q) = positions[(size_t)b * nmax * 3 + q];
    arr.dir[q] = 0.0f;
  }
  for (int i = r0; i < n; i += gs) {
    const int t = types[(size_t)b * nmax + i];
    arr.xs[i].w = __int_as_float(t < 0 ? 0 : (t > smax ? smax : t));
  }
  w.g.sync();
  if (w.g.leader()) {
    for (int q = 0; q < JR_MAX_SPECIES; ++q) w.s.counts[q] = 0;
    for (int i = 0; i < n; ++i) w.s.counts[__float_as_int(arr.xs[i].w)] += 1;
    w.s.cur = 0;
    make_cell_ctx(cell + (size_t)b * 9, w.s.cc[0], arr.T, P.model);
  }
  w.g.sync();
  double U, sff, sfd;
  model_eval<true>(P, w, 0, U, sff, sfd);
  const float* m = mu ? mu + (size_t)b * P.model.n_species : nullptr;
  double E = U;
  if (P.model.model != JR_MODEL_GAUSS_MIX)
    E = U + ensemble_term(w.s, w.s.cc[0].vol, pressure[b], m, P.model.n_species);
  w.g.sync();
  if (w.g.leader()) {
    energy64[b] = E;
    if (energy_u) energy_u[b] = U;
  }
  if (forces)
    for (int q = r0; q < 3 * n; q += gs) forces[(size_t)b * nmax * 3 + q] = arr.F[q];
}

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

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(JR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

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

int pow2_floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

int warp_tpa(int nmax) {
  int t = pow2_floor(32 / (nmax > 0 ? nmax : 1));
  return t < 1 ? 1 : t;
}

// Small walkers: one warp per walker, four walkers per CTA, one CTA per
// replica; larger walkers: one CTA per walker.
JrLaunchConfig heuristic_config(const JrDims* d) {
  JrLaunchConfig c;
  const int nmax = d->n_atoms_max;
  c.cluster = 1;
  if (nmax <= 32) {
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
bool spec_fits(const JrLaunchConfig& c, const JrDims* d) {
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
JrLaunchConfig ns_heuristic_config(const JrDims* d, int n_iter) {
  JrLaunchConfig c = heuristic_config(d);
  const int nmax = d->n_atoms_max;
  if (nmax <= 64) {
    c.warp_walkers = 0;
    c.threads = nmax <= 16 ? 128 : 256;
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

int check_params(const JrDims* d, const JrParams* p) {
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

int check_config(const JrLaunchConfig& c, const JrDims* d) {
  if (c.threads < 32 || c.threads > 512 || (c.threads & 31))
    return fail(JR_ERR_PARAM, "threads must be a multiple of 32 in [32, 512]");
  if (c.tpa < 1 || c.tpa > 32 || (c.tpa & (c.tpa - 1)))
    return fail(JR_ERR_PARAM, "tpa must be a power of two <= 32");
  if (c.cluster < 1 || c.cluster > 16) return fail(JR_ERR_PARAM, "cluster must be in [1, 16]");
  if (c.warp_walkers != 0 && c.warp_walkers != 1)
    return fail(JR_ERR_PARAM, "warp_walkers must be 0 or 1");
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

size_t ns_dyn_smem(const JrDims* d, const JrParams* p, const JrLaunchConfig& c) {
  const int cpc = c.warp_walkers ? c.threads / 32 : 1;
  return jr::dyn_head_bytes(d->n_walkers, d->n_atoms_max, p->model.n_images, d->n_cull) +
         (size_t)cpc * jr::walker_smem_bytes(d->n_atoms_max, p->model.n_images, true);
}

size_t group_dyn_smem(int nmax, int nimg, int groups) {
  return (size_t)groups * (jr::pair_table_bytes(nmax, nimg) + jr::walker_smem_bytes(nmax, nimg));
}

// Moves outside the lean walk: a constraint gate or a shear/stretch move.
bool needs_ext_walk(const JrParams* p) {
  for (int m = 0; m < p->moves.n_moves; ++m)
    if (p->moves.gate[m] || p->moves.type[m] >= JR_MOVE_SHEAR) return true;
  return false;
}

template <class G, int kT, bool kExt>
int launch_ns_as(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                 const JrInfoBuffers& inf, int n_iter, const JrLaunchConfig& c, void* workspace,
                 cudaStream_t s) {
  auto kern = jr::ns_iterate_kernel<G, kT, kExt>;
  const size_t smem = ns_dyn_smem(dims, params, c);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
  if (c.cluster > 8) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return cuda_fail(e, "non-portable cluster attribute");
  }
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
                         (int)c.cluster, (const uint32_t*)workspace);
  if (e != cudaSuccess) return cuda_fail(e, "ns_iterate launch");
  return JR_OK;
}

template <class G>
int launch_ns(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
              const JrInfoBuffers& inf, int n_iter, const JrLaunchConfig& c, void* workspace,
              cudaStream_t s) {
  // CTA walks of at most 256 threads use a kernel bounded at 256 threads: the
  // compiler may then keep up to 255 registers per thread (measured: 3% faster
  // chains than the 512-bounded kernel at the same 256-thread shape)
  const bool ext = needs_ext_walk(params);
  if constexpr (std::is_same<G, jr::WarpGroup>::value) {
    return ext ? launch_ns_as<G, 128, true>(dims, params, state, inf, n_iter, c, workspace, s)
               : launch_ns_as<G, 128, false>(dims, params, state, inf, n_iter, c, workspace, s);
  } else {
    if (c.threads <= 256)
      return ext ? launch_ns_as<G, 256, true>(dims, params, state, inf, n_iter, c, workspace, s)
                 : launch_ns_as<G, 256, false>(dims, params, state, inf, n_iter, c, workspace, s);
    return ext ? launch_ns_as<G, 512, true>(dims, params, state, inf, n_iter, c, workspace, s)
               : launch_ns_as<G, 512, false>(dims, params, state, inf, n_iter, c, workspace, s);
  }
}

}  // namespace

extern "C" {

const char* jr_last_error(void) { return g_last_error.c_str(); }

int jr_version(void) { return 2; }

size_t jr_ns_iterate_workspace_size(const JrDims* dims) {
  (void)dims;
  return 256;
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
  JrLaunchConfig c;
  if (cfg) {
    c = *cfg;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(tune_key(dims, params));
    c = it != g_tune_cache.end() ? it->second : ns_heuristic_config(dims, n_iter);
  }
  rc = check_config(c, dims);
  if (rc) return rc;
  JrInfoBuffers inf{};
  if (info) inf = *info;
  cudaStream_t s = (cudaStream_t)stream;
  // snapshot of replica 0's key: the shared move schedule of every replica
  cudaError_t e = cudaMemcpyAsync(workspace, state->rng_key, 2 * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "key snapshot");
  if (c.warp_walkers)
    return launch_ns<jr::WarpGroup>(dims, params, state, inf, n_iter, c, workspace, s);
  return launch_ns<jr::CtaGroup>(dims, params, state, inf, n_iter, c, workspace, s);
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

extern "C" {

// jr_ns_iterate on the library's own static device scratch instead of a
// caller workspace.  The first call on each device resolves the scratch's
// address with cudaGetSymbolAddress (with that device current) and caches it.
int jr_ns_iterate_static(const JrDims* dims, const JrParams* params,
                         const JrStateBuffers* state, const JrInfoBuffers* info, int32_t n_iter,
                         const JrLaunchConfig* cfg, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
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
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    scratch = g_static_ptr[dev];
    if (!scratch) {
      e = cudaGetSymbolAddress(&scratch, jr_static_scratch);
      if (e != cudaSuccess)
        return cuda_fail(e, "jr_ns_iterate_static: cudaGetSymbolAddress of the static scratch");
      g_static_ptr[dev] = scratch;
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
  const JrLaunchConfig c = heuristic_config(dims);
  const int nimg = params->model.n_images;
  const int total = dims->n_replicas * n_trials;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (c.warp_walkers) {
    const int gpc = c.threads / 32;
    const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, gpc);
    e = cudaFuncSetAttribute(jr::move_trial_kernel<jr::WarpGroup, 128>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::move_trial_kernel<jr::WarpGroup, 128><<<(total + gpc - 1) / gpc, c.threads, smem, s>>>(
        *dims, *params, *state, n_trials, move_idx, walker_idx, keys, move_keys, step, emax,
        write_back, accepted, reject_reason, c.tpa);
  } else {
    const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, 1);
    e = cudaFuncSetAttribute(jr::move_trial_kernel<jr::CtaGroup, 512>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::move_trial_kernel<jr::CtaGroup, 512><<<total, c.threads, smem, s>>>(
        *dims, *params, *state, n_trials, move_idx, walker_idx, keys, move_keys, step, emax,
        write_back, accepted, reject_reason, c.tpa);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "move_trial launch");
  return JR_OK;
}

int jr_walk_population(const JrDims* dims, const JrParams* params, const JrStateBuffers* state,
                       int32_t walklength, const uint32_t* run_keys, const uint32_t* move_key,
                       const double* emax, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (!state || !run_keys || !move_key || !emax || walklength < 0)
    return fail(JR_ERR_PARAM, "walk_population: null buffer or walklength < 0");
  if (walklength == 0) return JR_OK;
  const JrLaunchConfig c = heuristic_config(dims);
  const int nimg = params->model.n_images;
  const int total = dims->n_replicas * dims->n_walkers;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (c.warp_walkers) {
    const int gpc = c.threads / 32;
    const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, gpc);
    e = cudaFuncSetAttribute(jr::walk_population_kernel<jr::WarpGroup, 128>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::walk_population_kernel<jr::WarpGroup, 128><<<(total + gpc - 1) / gpc, c.threads, smem, s>>>(
        *dims, *params, *state, walklength, run_keys, move_key, emax, c.tpa);
  } else {
    const size_t smem = group_dyn_smem(dims->n_atoms_max, nimg, 1);
    e = cudaFuncSetAttribute(jr::walk_population_kernel<jr::CtaGroup, 512>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::walk_population_kernel<jr::CtaGroup, 512><<<total, c.threads, smem, s>>>(
        *dims, *params, *state, walklength, run_keys, move_key, emax, c.tpa);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "walk_population launch");
  return JR_OK;
}

int jr_energy_forces(const JrParams* params, int32_t n_configs, int32_t n_atoms_max,
                     const float* positions, const int32_t* types, const float* cell,
                     const int32_t* n_atoms, const float* pressure, const float* mu,
                     double* energy64, double* energy_u, float* forces, void* stream) {
  if (!params || n_configs < 1 || n_atoms_max < 1 || n_atoms_max > JR_MAX_ATOMS || !positions ||
      !types || !cell || !n_atoms || !pressure || !energy64)
    return fail(JR_ERR_PARAM, "invalid energy_forces arguments");
  if (params->model.n_species < 1 || params->model.n_species > JR_MAX_SPECIES ||
      params->model.n_images < 1 || params->model.n_images > JR_MAX_IMAGES)
    return fail(JR_ERR_PARAM, "invalid model parameters");
  JrDims d{};
  d.n_atoms_max = n_atoms_max;
  const JrLaunchConfig c = heuristic_config(&d);
  const int nimg = params->model.n_images;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (c.warp_walkers) {
    const int gpc = c.threads / 32;
    const size_t smem = group_dyn_smem(n_atoms_max, nimg, gpc);
    e = cudaFuncSetAttribute(jr::energy_kernel<jr::WarpGroup, 128>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::energy_kernel<jr::WarpGroup, 128><<<(n_configs + gpc - 1) / gpc, c.threads, smem, s>>>(
        *params, n_configs, n_atoms_max, positions, types, cell, n_atoms, pressure, mu, energy64,
        energy_u, forces, c.tpa);
  } else {
    const size_t smem = group_dyn_smem(n_atoms_max, nimg, 1);
    e = cudaFuncSetAttribute(jr::energy_kernel<jr::CtaGroup, 512>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
    jr::energy_kernel<jr::CtaGroup, 512><<<n_configs, c.threads, smem, s>>>(
        *params, n_configs, n_atoms_max, positions, types, cell, n_atoms, pressure, mu, energy64,
        energy_u, forces, c.tpa);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "energy launch");
  return JR_OK;
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

struct ScratchState {
  JrStateBuffers b{};
  void* blocks[16] = {};
  int nblk = 0;
  ~ScratchState() {
    for (int i = 0; i < nblk; ++i) cudaFree(blocks[i]);
  }
  void* take(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    blocks[nblk++] = p;
    return p;
  }
};

// Scratch copy of the mutable state so candidate launch shapes can be timed
// without touching the caller's walkers.  Freed before jr_autotune returns.
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

}  // namespace

extern "C" int jr_autotune(const JrDims* dims, const JrParams* params,
                           const JrStateBuffers* state, int32_t n_iter_probe,
                           JrLaunchConfig* best, void* stream) {
  int rc = check_params(dims, params);
  if (rc) return rc;
  if (!state || !best || n_iter_probe < 1) return fail(JR_ERR_PARAM, "autotune arguments");
  cudaStream_t st = (cudaStream_t)stream;
  ScratchState scratch;
  rc = clone_state(dims, state, scratch, st);
  if (rc) return rc;
  const size_t wsb = jr_ns_iterate_workspace_size(dims);
  void* ws = scratch.take(wsb);
  if (!ws) return fail(JR_ERR_CUDA, "autotune workspace allocation failed");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  JrLaunchConfig bc = ns_heuristic_config(dims, n_iter_probe);
  const int nmax = dims->n_atoms_max;
  JrLaunchConfig cands[96];
  int nc = 0;
  const int clusters[] = {1, 2, 4, 8, 10, 12, 16};
  if (nmax <= 32) {  // warp walkers: 1..8 walkers per CTA
    for (int wpc : {1, 2, 4})
      for (int cl : clusters) cands[nc++] = JrLaunchConfig{32 * wpc, warp_tpa(nmax), cl, 1};
  }
  for (int th : {128, 256, 512})
    for (int cl : clusters) {
      int tpa = pow2_floor(th / nmax);
      tpa = tpa > 16 ? 16 : (tpa < 1 ? 1 : tpa);
      if (nc < 96) cands[nc++] = JrLaunchConfig{th, tpa, cl, 0};
    }
  for (int i = 0; i < nc; ++i) {
    const JrLaunchConfig c = cands[i];
    if (check_config(c, dims) != JR_OK) continue;
    rc = jr_ns_iterate(dims, params, &scratch.b, nullptr, 1, &c, ws, wsb, stream);
    if (rc != JR_OK || cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaEventRecord(e0, st);
    rc = jr_ns_iterate(dims, params, &scratch.b, nullptr, n_iter_probe, &c, ws, wsb, stream);
    cudaEventRecord(e1, st);
    if (rc != JR_OK || cudaEventSynchronize(e1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
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
  g_last_error.clear();
  return JR_OK;
}
