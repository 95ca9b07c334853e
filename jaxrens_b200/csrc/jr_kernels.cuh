// jr_kernels.cuh -- the walk kernels, templated on the walking group (which
// carries the model family), shared by the translation units of the library.
//
// Kernels
//   ns_iterate_kernel<G>  n_iter NS iterations for every replica in one
//                      launch.  A thread-block cluster of C CTAs serves one
//                      replica; each CTA walks one chain (G = CtaG) or one
//                      chain per warp (G = WarpG).  Each round predicts
//                      the culls of the next D iterations -- the PRNG stream
//                      is state independent, and the walker culled at
//                      iteration i+d is the (d+1)-th highest energy as long as
//                      the walkers written by iterations < d stay below it --
//                      walks them concurrently, then commits the longest
//                      prefix whose predictions hold.  Committed results are
//                      exactly those of sequential ns_step calls.
//   move_trial_kernel<G>  one move on many walkers (adaptation, burn-in)
//   walk_population_kernel<G>  the burn-in walk of every walker
//   energy_kernel<G>      energy + forces of a batch of configurations
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

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
  double vE[kMaxWalk];      // validation: every slot's final energy, gathered once
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
__device__ inline void cull_select(NsShared& ns, int& par, const double* E, int K, const int* excl,
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
__device__ inline void select_extras(NsShared& ns, int& par, float* noise, int K, int worst, int clone,
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
  if constexpr (G::kFam == kFamSWDA) {
    // the surrogate energy of the loaded walker
    double d0, d1;
    const double ens = ensemble_term(s, s.cc[s.cur].vol, pressure, mu, P.model.n_species);
    const double Hs = sur_ham<false>(w, s.cur, ens, d0, d1);
    if (w.g.leader()) s.Esur = Hs;
    w.g.sync();
  }
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
    for (int t = 0; t < nt; ++t) {
      w.ring_step = t0 + t;
      mwg_step<kExt>(P, w, s.step_key[t], s.step_move[t], emax, pressure, mu);
    }
    w.g.sync();
  }
  {
    // the chain's evaluated pairs and triplets, summed over threads
    double a = w.tc[0], b = w.tc[1], c = w.tc[2], d = w.tc[3], z0 = 0.0, z1 = 0.0;
    w.g.sum3(a, b, c, 1, w.par);
    w.g.sum3(d, z0, z1, 1, w.par);
    if (w.g.leader()) {
      s.c_terms[0] += (long long)a;
      s.c_terms[1] += (long long)b;
      s.c_terms[2] += (long long)c;
      s.c_terms[3] += (long long)d;
    }
    for (int q = 0; q < 4; ++q) w.tc[q] = 0;
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

__host__ __device__ inline size_t dyn_head_bytes(int K, int nmax, int nimg, int ncull, int fam) {
  return align16(8u * (size_t)K) + align16(4u * (size_t)K) +
         (ncull > 1 ? 3u * align16(4u * (size_t)K) : 0u) + pair_table_bytes(nmax, nimg, fam);
}

__device__ inline DynLayout dyn_layout(unsigned char* dyn, int K, int nmax, int nimg, int ncull,
                                       int fam) {
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
  L.pij = pair_table_bytes(nmax, nimg, fam) ? reinterpret_cast<uint16_t*>(p) : nullptr;
  p += pair_table_bytes(nmax, nimg, fam);
  L.walkers = p;
  L.walker_bytes = walker_smem_bytes(nmax, nimg, true, fam);
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
__device__ inline void predict_fast(NsShared& ns, const double* E, int K, int Dr, Key key, Key key0,
                                    int mk_mode) {
  const bool shared_mk = mk_mode != 0;
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
    ns.kmove[lane] = mk_mode == 2 ? ns.k0chain[lane]
                                  : (shared_mk ? split(ns.k0chain[lane], 1u) : split(ka, 4u));
  }
  const int nslot = (K + 31) >> 5;
  uint32_t taken = 0;
  bool prev_ok = true;
  double prev_e = 0.0;
  // this lane's largest non-culled energy (ordered bits) and NaN flag; only
  // the lane that loses a walker to a cull rescans its entries
  unsigned long long lbest = 0;
  int lnan = 0;
  // and how many of the lane's entries equal its largest value (== on the
  // values: -0.0 ties with +0.0), with 1 + the largest such index
  int lties = 0, lidx = 0;
  auto lane_scan = [&]() {
    lbest = 0;
    lnan = 0;
    lties = 0;
    lidx = 0;
    for (int j = 0; j < nslot; ++j) {
      const int k = lane + 32 * j;
      if (k >= K || ((taken >> j) & 1u)) continue;
      const double x = E[k];
      if (isnan(x)) {
        lnan = 1;
      } else {
        const unsigned long long o = ord_double(x);
        if (o > lbest) {
          const bool eq = lbest != 0 && x == unord_double(lbest);
          lbest = o;
          lties = eq ? lties + 1 : 1;
          lidx = k + 1;
        } else if (x == unord_double(lbest)) {
          ++lties;
          lidx = k + 1;
        }
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
        nties = lties;
        idx1 = lidx;
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
__device__ inline void select_culls_multi(NsShared& ns, const DynLayout& L, const double* E, int K,
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

// The key of iteration d's move schedule: the run's own split(ka, 4)
// (mode 0), fold_in(replica 0's key, 1) (mode 1, batched runs; k0d is replica
// 0's key at iteration d), or the caller's explicit key (mode 2, k0d holds it).
__device__ __forceinline__ Key move_schedule_key(int mode, Key k0d, Key kmoves) {
  return mode == 2 ? k0d : (mode == 1 ? split(k0d, 1u) : kmoves);
}

template <class G>
__device__ __forceinline__ G make_group(double (*red)[kMaxWarps][3]) {
  if constexpr (G::kIsWarp) {
    (void)red;
    return G{};
  } else {
    return G{red};
  }
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

// The surrogate and the sample ring of the delayed-acceptance walk (unused
// by the other families).
struct DaArgs {
  JrSurrogate sur;
  JrSampleRing ring;
};

template <class G, int kMaxThreads, bool kExt>
__global__ void __launch_bounds__(kMaxThreads, 1)
ns_iterate_kernel(const JrDims D, const JrParams Pg, const JrStateBuffers st,
                  const JrInfoBuffers info, const int n_iter, const int tpa, const int C,
                  const uint32_t* __restrict__ key0_base, const __grid_constant__ DaArgs da) {
  constexpr bool kWarp = G::kIsWarp;
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
  DynLayout L = dyn_layout(dyn, K, D.n_atoms_max, nimg, D.n_cull, G::kFam);
  WalkArrays arr;
  WalkShared* wsp = carve_walker(L.walkers + (size_t)my * L.walker_bytes, D.n_atoms_max, nimg,
                                 L.pij, arr, true, G::kFam);
  Walker<G> w{*wsp, arr, tab, n, tpa, make_group<G>(red), 0};
  if constexpr (G::kFam == kFamSWDA) {
    w.sur = &da.sur;
    if (da.ring.positions) {
      w.ring_pos = da.ring.positions;
      w.ring_cell = da.ring.cell;
      w.ring_u = da.ring.energy_u;
      w.ring_nmax = D.n_atoms_max;
      w.ring_cap = da.ring.capacity;
    }
    sur_load_weights(da.sur, arr);
  }
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
    if (fast) predict_fast(ns, L.Epop, K, Dr, key, key0, D.shared_move_key);
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
          ns.kmove[0] = move_schedule_key(D.shared_move_key, k0d, kmoves);
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
        ns.kmove[d] = move_schedule_key(D.shared_move_key, k0d, kmoves);
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
        w.ring_chain = da.ring.base + ((long long)committed * D.n_replicas + p) * W * T +
                       (long long)sidx * T;
        walk_chain<kExt>(P, w, T, split(ns.kmcmc[0], (uint32_t)sidx), ns.kmove[0], ns.e[0],
                         pressure, mu);
        store_walker(D, st, w, p, dst);
      }
    } else {
      const int d = s_my / W, wi = s_my % W;
      if (d < Dr && ns.spec[d]) {
        const int src = wi == 0 ? ns.clone[d] : ns.extras[d * nx + wi - 1];
        load_walker(P, D, st, w, p, src, wi == 0);
        w.ring_chain = da.ring.base + ((long long)(committed + d) * D.n_replicas + p) * W * T +
                       (long long)wi * T;
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
      // every slot's final energy, one remote load per thread, then the
      // prefix test on the local copy
      for (int sl = threadIdx.x; sl < Dr * W; sl += blockDim.x)
        ns.vE[sl] = *cluster.map_shared_rank(&ns.res_E[sl % cpc], sl / cpc);
      __syncthreads();
      nval = 0;
      for (int d = 0; d < Dr; ++d) {
        bool ok = ns.spec[d] != 0;
        for (int sl = 0; sl < d * W && ok; ++sl)
          if (!(ns.vE[sl] < ns.e[d])) ok = false;
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
          int a = 0, pr = 0, ne = 0, ng = 0, nsur = 0, rr[4] = {0, 0, 0, 0};
          for (int sl = s0; sl < s1; ++sl) {
            const WalkShared* local = reinterpret_cast<const WalkShared*>(
                L.walkers + (size_t)(sl % cpc) * L.walker_bytes);
            const WalkShared* rs = sl == s_my ? local : cluster.map_shared_rank(local, sl / cpc);
            a += rs->c_acc[m];
            pr += rs->c_prop[m];
            ne += rs->c_nev[m];
            ng += rs->c_ngr[m];
            nsur += rs->c_nsur[m];
            for (int q = 0; q < 4; ++q) rr[q] += rs->c_rr[4 * m + q];
          }
          if (da.ring.n_surrogate_evaluations) da.ring.n_surrogate_evaluations[ib * M + m] = nsur;
          if (info.n_accepted) info.n_accepted[ib * M + m] = a;
          if (info.n_proposed) info.n_proposed[ib * M + m] = pr;
          if (info.n_evaluations) info.n_evaluations[ib * M + m] = ne;
          if (info.n_grad_evaluations) info.n_grad_evaluations[ib * M + m] = ng;
          if (info.reject_reason_counts)
            for (int q = 0; q < 4; ++q) info.reject_reason_counts[(ib * M + m) * 4 + q] = rr[q];
        }
        if (info.term_counts) {
          long long tc[4] = {0, 0, 0, 0};
          for (int sl = s0; sl < s1; ++sl) {
            const WalkShared* local = reinterpret_cast<const WalkShared*>(
                L.walkers + (size_t)(sl % cpc) * L.walker_bytes);
            const WalkShared* rs = sl == s_my ? local : cluster.map_shared_rank(local, sl / cpc);
            for (int q = 0; q < 4; ++q) tc[q] += rs->c_terms[q];
          }
          for (int q = 0; q < 4; ++q) info.term_counts[ib * 4 + q] = tc[q];
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
  constexpr bool kWarp = G::kIsWarp;
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
  const size_t ptb = pair_table_bytes(D.n_atoms_max, nimg, G::kFam);
  char* base = reinterpret_cast<char*>(dyn) +
               (size_t)my * (ptb + walker_smem_bytes(D.n_atoms_max, nimg, false, G::kFam));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, D.n_atoms_max, nimg, pij, arr, false, G::kFam);
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
  constexpr bool kWarp = G::kIsWarp;
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
  const size_t ptb = pair_table_bytes(D.n_atoms_max, nimg, G::kFam);
  char* base = reinterpret_cast<char*>(dyn) +
               (size_t)my * (ptb + walker_smem_bytes(D.n_atoms_max, nimg, false, G::kFam));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, D.n_atoms_max, nimg, pij, arr, false, G::kFam);
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
  constexpr bool kWarp = G::kIsWarp;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ JrParams P;
  __shared__ PairTables tab;
  __shared__ double red[2][kMaxWarps][3];
  copy_params(P, Pg);
  const int gpc = kWarp ? (int)(blockDim.x >> 5) : 1;
  const int my = kWarp ? (int)(threadIdx.x >> 5) : 0;
  const int b = blockIdx.x * gpc + my;
  const int nimg = Pg.model.n_images;
  const size_t ptb = pair_table_bytes(nmax, nimg, G::kFam);
  char* base = reinterpret_cast<char*>(dyn) +
               (size_t)my * (ptb + walker_smem_bytes(nmax, nimg, false, G::kFam));
  uint16_t* pij = ptb ? reinterpret_cast<uint16_t*>(base) : nullptr;
  WalkArrays arr;
  WalkShared* wsp = carve_walker(base + ptb, nmax, nimg, pij, arr, false, G::kFam);
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


}  // namespace jr
