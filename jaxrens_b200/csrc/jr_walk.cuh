// jr_walk.cuh -- one walker resident in shared memory, walked by a thread
// group: a whole CTA (large walkers) or a single warp (small walkers, several
// walkers per CTA).
//
// Arithmetic contract (shared with the CPU oracle's DEV mode):
//   * pair terms in float32 with a fixed FMA placement (explicit intrinsics,
//     the translation unit is compiled with -fmad=false),
//   * every sum (energy, forces, norms, dot products) accumulated in float64
//     and rounded to float32 once where a float32 value is needed.
// The float64 sums of float32 terms are exact whenever a configuration's pair
// terms span < 2^29 in magnitude, so results do not depend on the thread
// mapping (launch shape) and match the oracle bit-for-bit; beyond that range
// (overlapping atoms) float64 energies can differ in their last bit.
#pragma once
#include <cstdint>

#include "../../include/jaxrens_b200.h"
#include "jr_rng.cuh"

namespace jr {

constexpr int kMaxWarps = 32;
constexpr int kStepChunk = 64;  // steps whose keys and moves are drawn at once

// Model families, fixed at compile time per kernel instantiation (carried by
// the group type): the pair family (LJ and the Gaussian-mixture toy) and the
// Stillinger-Weber family.  A kernel of one family compiles no code of the
// other, so each family's walk keeps its own registers and instruction
// stream.
constexpr int kFamPair = 0;
constexpr int kFamSW = 1;
// Stillinger-Weber with the learned surrogate: galilean and volume moves by
// two-stage delayed acceptance, the exact SW energy deciding every step
constexpr int kFamSWDA = 2;

__host__ __device__ constexpr bool sw_family(int fam) { return fam == kFamSW || fam == kFamSWDA; }

// The key of one MWG step with its two first-level subkeys, split(k, 0) and
// split(k, 1), which every move draws from (galilean: initial direction and
// perturbation; volume and cell moves: proposal and prior; identity moves:
// atom and species).
struct StepKey {
  Key k, k0, k1;
  // draws of the step made ahead of the walk (they depend on the keys only):
  // nz, when set, holds the galilean perturbation normals normal(bits(k1, q));
  // with pre set, vn = normal(bits(k0, 0)) and vu = uniform(bits(k1, 0)) of a
  // volume step
  const float* nz;
  float vn, vu;
  int pre;
};

__device__ __forceinline__ StepKey make_step_key(Key k) {
  return StepKey{k, split(k, 0u), split(k, 1u), nullptr, 0.0f, 0.0f, 0};
}

// The largest walker (atoms) whose NS chains get a buffer for the galilean
// normals of a chunk of steps (kStepChunk x 3 n floats).
constexpr int kNormalAtomsMax = 32;
constexpr int kSWMaxAtoms = 64;  // Stillinger-Weber walkers: one 64-bit neighbour mask per atom
constexpr int kSWCandSlack = 16 * 32;  // per-warp segment rounding of the SW candidate list
// offset of the dense candidate list after the per-warp segments
constexpr int kSWCandDense = kSWMaxAtoms * (kSWMaxAtoms - 1) / 2 + kSWCandSlack;
constexpr int kPairMatMax = 96;  // walkers up to this size use the pair matrix
                                 // (12 n pm_stride(n) bytes: 112 KB at 96; measured faster than
                                 // the ordered pairs from 32 to 96 atoms)

// ------------------------------------------------------------- groups ----

// A whole CTA walking one walker.  sum3 reduces three doubles across the
// block through two alternating shared buffers (one barrier per reduction).
template <int kFamily>
struct CtaG {
  static constexpr int kFam = kFamily;
  static constexpr bool kIsWarp = false;
  double (*red)[kMaxWarps][3];  // smem [2][kMaxWarps][3]
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
  // lanes hold partials only at multiples of `stride` (a power of two)
  __device__ __forceinline__ void sum3(double& a, double& b, double& c, int stride,
                                       int& par) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    for (int off = 16; off >= stride; off >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, off);
      b += __shfl_xor_sync(0xffffffffu, b, off);
      c += __shfl_xor_sync(0xffffffffu, c, off);
    }
    double (*buf)[3] = red[par];
    if (lane == 0) {
      buf[warp][0] = a;
      buf[warp][1] = b;
      buf[warp][2] = c;
    }
    __syncthreads();
    // every thread sums the warp partials itself: the pairwise tree over the
    // lowest next_pow2(nw) warps (zeros above), no shuffle chain after the
    // barrier
    if (nw <= 8) {
      a = tree_sum<8>(buf, nw, 0);
      b = tree_sum<8>(buf, nw, 1);
      c = tree_sum<8>(buf, nw, 2);
    } else {
      a = tree_sum<16>(buf, nw, 0);
      b = tree_sum<16>(buf, nw, 1);
      c = tree_sum<16>(buf, nw, 2);
    }
    par ^= 1;
  }
  // sum3 of one value: the same tree for `a`, a third of the shuffles
  __device__ __forceinline__ void sum1(double& a, int stride, int& par) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    for (int off = 16; off >= stride; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    double (*buf)[3] = red[par];
    if (lane == 0) buf[warp][0] = a;
    __syncthreads();
    // every thread sums the warp partials itself, in the pairwise order of
    // sum3's butterfly (zeros past nw; x + 0 leaves x unchanged): no shuffle
    // chain and no broadcast after the barrier
    a = nw <= 8 ? tree_sum<8>(buf, nw, 0) : tree_sum<16>(buf, nw, 0);
    par ^= 1;
  }
  // the pairwise sum of buf[0..nw)[k] padded with zeros to W entries (the
  // launch bound of 512 threads keeps nw <= 16); the order of the butterfly
  // over next_pow2(nw) lanes, since x + 0 leaves x unchanged
  template <int W>
  __device__ __forceinline__ static double tree_sum(const double (*buf)[3], int nw, int k) {
    double v[W];
#pragma unroll
    for (int q = 0; q < W; ++q) v[q] = q < nw ? buf[q][k] : 0.0;
#pragma unroll
    for (int st = 1; st < W; st <<= 1)
#pragma unroll
      for (int q = 0; q + st < W; q += 2 * st) v[q] += v[q + st];
    return v[0];
  }
};

// One warp walking one walker: register shuffles only, no block barriers.
template <int kFamily>
struct WarpG {
  static constexpr int kFam = kFamily;
  static constexpr bool kIsWarp = true;
  __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  __device__ __forceinline__ bool leader() const { return (threadIdx.x & 31) == 0; }
  __device__ __forceinline__ void sum3(double& a, double& b, double& c, int stride,
                                       int& par) const {
    for (int off = 16; off >= stride; off >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, off);
      b += __shfl_xor_sync(0xffffffffu, b, off);
      c += __shfl_xor_sync(0xffffffffu, c, off);
    }
    if (stride > 1) {
      a = __shfl_sync(0xffffffffu, a, 0);
      b = __shfl_sync(0xffffffffu, b, 0);
      c = __shfl_sync(0xffffffffu, c, 0);
    }
    (void)par;
  }
  __device__ __forceinline__ void sum1(double& a, int stride, int& par) const {
    for (int off = 16; off >= stride; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    if (stride > 1) a = __shfl_sync(0xffffffffu, a, 0);
    (void)par;
  }
};

using CtaGroup = CtaG<kFamPair>;
using WarpGroup = WarpG<kFamPair>;

// ----------------------------------------------------------- walker ----

// Geometry of one cell: the matrix, its inverse and the image translations.
struct CellCtx {
  float raw[9];  // the cell as stored (rows are lattice vectors)
  float h[9];    // the cell used for geometry (1e10*I when det == 0)
  float inv[9];
  int diag;
  float vol;  // |det| of the stored cell (ensemble term)
};

// Per-walker scalar state (one per walking group).
struct WalkShared {
  CellCtx cc[2];  // [cur], [trial]
  int cur;        // index of the current cell context
  double E;       // current full potential of the walker
  float step_sizes[JR_MAX_MOVES];
  int counts[JR_MAX_SPECIES];
  // per-walker MWG counters (MCState.n_accepted / n_proposed)
  int w_acc[JR_MAX_MOVES];
  int w_prop[JR_MAX_MOVES];
  // per-chain info counters (ns_step info dict), summed over steps
  int c_acc[JR_MAX_MOVES];
  int c_prop[JR_MAX_MOVES];
  int c_rr[JR_MAX_MOVES * 4];
  int c_nev[JR_MAX_MOVES];
  int c_ngr[JR_MAX_MOVES];
  // step keys and move choices of the next steps of a chain
  StepKey step_key[kStepChunk];
  int step_move[kStepChunk];
  int cell_ok;  // cell-geometry verdict of the pending cell move
  int sw_cand[kMaxWarps];  // Stillinger-Weber: pairs inside the cutoff found by each warp
  // work of the chain's evaluations: [pairs with forces, triplets with
  // forces, energy-only pairs, energy-only triplets]; pairs are LJ's unique
  // interactions or Stillinger-Weber's pairs inside the cutoff
  long long c_terms[4];
  // pre-move copy for the constraint gate
  double E_save;
  int cur_save;
  int counts_save[JR_MAX_SPECIES];
  // surrogate walk: the surrogate potential (with the ensemble term) of the
  // current walker, and the exact / surrogate evaluations of the last move
  double Esur;
  int step_nev, step_nsur;
  int c_nsur[JR_MAX_MOVES];  // per-chain surrogate evaluations per move
};

// Pair tables of the model, shared by every walker of a CTA.
struct PairTables {
  float sig2[JR_MAX_SPECIES * JR_MAX_SPECIES];
  float eps4[JR_MAX_SPECIES * JR_MAX_SPECIES];
  float eps24[JR_MAX_SPECIES * JR_MAX_SPECIES];
};

// Per-walker arrays in dynamic shared memory.  Walkers with one image and at
// most kPairMatMax atoms also get the antisymmetric pair-force matrix, three
// float planes [n][n|1] (the odd row stride keeps the row gather free of bank
// conflicts); the pair decode table is shared by all walkers of a CTA (same
// atom count).
struct WalkArrays {
  float4* xs;           // [Nmax] position + type bits (current / trial positions)
  float4* xsave;        // [Nmax] pre-move copy of xs for the constraint gate
  float* x0;            // [3 Nmax] saved positions
  float* dir;           // [3 Nmax] direction
  float* dp;            // [3 Nmax] perturbed direction (flip target on reject)
  float* F;             // [3 Nmax] forces
  float* T;             // [2][3 n_img] image translations for cc[0], cc[1]
  float* pm;            // [3][n][pm_stride(n)] pair force terms g*dr_ij, or nullptr
  const uint16_t* pij;  // [Nmax(Nmax-1)/2] pair decode a | b << 8, or nullptr
  float* nz;            // [kStepChunk][3 n] galilean normals drawn ahead, or nullptr
  // Stillinger-Weber tables (the SW family only), one record per unordered
  // pair of the row-major upper triangle:
  float4* swr0;         // [n(n-1)/2] (dr, 1/r) of pairs inside the cutoff
  float4* swr1;         // [n(n-1)/2] (g, g'/(g r), phi2'/r, phi2)
  float4* swq;          // [n(n-1)/2] pair force share Q_ab
  uint64_t* nbm;        // [2][kSWMaxAtoms] neighbour masks (alternating evaluations)
  uint16_t* cand;       // [kSWCandDense + n(n-1)/2] pairs inside the cutoff: per-warp
                        // segments, then (from kSWCandDense) the dense list
  // surrogate network (the SW-with-surrogate family only): bfloat16 operand
  // tiles of the warp-level products, row-major with padded rows
  uint16_t* sw1t;       // [64][kSurLdX]   W1^T (n = hidden, k = input)
  uint16_t* sw2t;       // [64][kSurLdH]   W2^T (n = out, k = in)
  uint16_t* sw2k;       // [64][kSurLdH]   W2   (n = in, k = out)
  uint16_t* sw1k;       // [16][kSurLdH]   W1   (n = input, k = hidden)
  uint16_t* sx;         // [64][kSurLdX]   network input rows
  uint16_t* sh1;        // [64][kSurLdH]   first hidden layer
  uint16_t* sg2;        // [64][kSurLdH]   gradient at the second layer
  uint16_t* sg1;        // [64][kSurLdH]   gradient at the first layer
  float* sbias;         // [3][64] b1, b2, w3
  float* sdx;           // [64][kSurLdG] gradient of the energy at the descriptors
};

// Padded row strides (bfloat16 elements) of the surrogate's operand tiles:
// the warp-level fragment loads of 8 rows x 4 columns fall on distinct banks;
// kSurLdG (floats) spreads the dU/dD rows of neighbouring atoms over banks.
constexpr int kSurLdX = 24, kSurLdH = 72, kSurLdG = 17;

__host__ __device__ inline size_t sur_table_bytes() {
  return 2u * (64u * kSurLdX * 2u + 64u * kSurLdH * 5u + 16u * kSurLdH) + 4u * (3u * 64u) +
         4u * (64u * kSurLdG);
}

__host__ __device__ inline bool use_pair_matrix(int nmax, int nimg, int fam = kFamPair) {
  return fam == kFamPair && nimg == 1 && nmax <= kPairMatMax;
}

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Row stride of the pair-force matrix: n rounded up to the 8-partner gather
// blocks, made odd (an odd stride keeps the warp's row reads and the pair
// stores on distinct banks).  Columns n.. and the diagonal are never written
// by the pair loop and stay +0.0 from zero_pair_matrix, so the gather reads
// whole blocks unconditionally: an absent partner contributes +0.0, as the
// canonical order prescribes.
__host__ __device__ inline int pm_stride(int n) { return ((n + 7) & ~7) | 1; }

__host__ __device__ inline size_t pair_count(int nmax) {
  return (size_t)nmax * (size_t)(nmax - 1) / 2;
}

// Bytes of one walker: WalkShared + arrays (+ pair buffer) (+ the buffer of
// normals drawn ahead, for the NS chains of small walkers).
__host__ __device__ inline bool use_normal_buffer(int nmax, bool normals) {
  return normals && nmax <= kNormalAtomsMax;
}

// Bytes of the Stillinger-Weber tables of one walker.
__host__ __device__ inline size_t sw_table_bytes(int nmax) {
  const size_t np = pair_count(nmax);
  return 3u * 16u * np + 2u * 8u * (size_t)kSWMaxAtoms +
         align16(2u * ((size_t)kSWCandDense + np));
}

__host__ __device__ inline size_t walker_smem_bytes(int nmax, int nimg, bool normals = false,
                                                    int fam = kFamPair) {
  size_t b = align16(sizeof(WalkShared));
  b += 2u * 16u * (size_t)nmax + 4u * 12u * (size_t)nmax;
  b += align16(2u * 3u * 4u * (size_t)nimg);
  if (use_pair_matrix(nmax, nimg, fam)) b += align16(12u * (size_t)nmax * (size_t)pm_stride(nmax));
  if (sw_family(fam)) b += sw_table_bytes(nmax);
  if (fam == kFamSWDA) b += align16(sur_table_bytes());
  if (use_normal_buffer(nmax, normals)) b += align16(12u * (size_t)kStepChunk * (size_t)nmax);
  return align16(b);
}

// Bytes of the CTA-shared pair decode table (the pair-matrix path and every
// Stillinger-Weber walk).
__host__ __device__ inline size_t pair_table_bytes(int nmax, int nimg, int fam = kFamPair) {
  return (use_pair_matrix(nmax, nimg, fam) || sw_family(fam)) ? align16(2u * pair_count(nmax)) : 0;
}

__device__ inline WalkShared* carve_walker(char* p, int nmax, int nimg, const uint16_t* pij,
                                           WalkArrays& a, bool normals = false,
                                           int fam = kFamPair) {
  WalkShared* s = reinterpret_cast<WalkShared*>(p);
  p += align16(sizeof(WalkShared));
  a.xs = (float4*)p; p += 16 * nmax;
  a.xsave = (float4*)p; p += 16 * nmax;
  a.x0 = (float*)p; p += 12 * nmax;
  a.dir = (float*)p; p += 12 * nmax;
  a.dp = (float*)p; p += 12 * nmax;
  a.F = (float*)p; p += 12 * nmax;
  a.T = (float*)p; p += align16(2 * 3 * 4 * nimg);
  a.pm = nullptr;
  a.pij = nullptr;
  a.swr0 = a.swr1 = a.swq = nullptr;
  a.nbm = nullptr;
  a.cand = nullptr;
  a.sw1t = a.sw2t = a.sw2k = a.sw1k = a.sx = a.sh1 = a.sg2 = a.sg1 = nullptr;
  a.sbias = a.sdx = nullptr;
  if (use_pair_matrix(nmax, nimg, fam)) {
    a.pm = (float*)p;
    a.pij = pij;
    p += align16(12u * (size_t)nmax * (size_t)pm_stride(nmax));
  }
  if (sw_family(fam)) {
    const size_t np = pair_count(nmax);
    a.pij = pij;
    a.swr0 = (float4*)p; p += 16u * np;
    a.swr1 = (float4*)p; p += 16u * np;
    a.swq = (float4*)p; p += 16u * np;
    a.nbm = (uint64_t*)p; p += 2u * 8u * kSWMaxAtoms;
    a.cand = (uint16_t*)p; p += align16(2u * ((size_t)kSWCandDense + np));
  }
  if (fam == kFamSWDA) {
    char* q = p;
    a.sw1t = (uint16_t*)q; q += 2 * 64 * kSurLdX;
    a.sx = (uint16_t*)q; q += 2 * 64 * kSurLdX;
    a.sw2t = (uint16_t*)q; q += 2 * 64 * kSurLdH;
    a.sw2k = (uint16_t*)q; q += 2 * 64 * kSurLdH;
    a.sh1 = (uint16_t*)q; q += 2 * 64 * kSurLdH;
    a.sg2 = (uint16_t*)q; q += 2 * 64 * kSurLdH;
    a.sg1 = (uint16_t*)q; q += 2 * 64 * kSurLdH;
    a.sw1k = (uint16_t*)q; q += 2 * 16 * kSurLdH;
    a.sbias = (float*)q; q += 4 * 3 * 64;
    a.sdx = (float*)q; q += 4 * 64 * kSurLdG;
    p += align16(sur_table_bytes());
  }
  a.nz = use_normal_buffer(nmax, normals) ? (float*)p : nullptr;
  return s;
}

// Zero a walker's whole pair-force matrix (sized for nmax), group-wide; the
// group synchronises before the first evaluation.
template <class G>
__device__ inline void zero_pair_matrix(const G& g, const WalkArrays& a, int nmax) {
  if (a.nbm != nullptr)
    for (int q = g.rank(); q < 2 * kSWMaxAtoms; q += g.size()) a.nbm[q] = 0ull;
  if (a.pm == nullptr) return;
  const int words = 3 * nmax * pm_stride(nmax);
  for (int q = g.rank(); q < words; q += g.size()) a.pm[q] = 0.0f;
}

// Fill the pair decode table for n atoms (pairs a < b, row-major), CTA-wide.
__device__ inline void build_pair_table(uint16_t* pij, int n) {
  if (!pij) return;
  const int np = n * (n - 1) / 2;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    int a = (int)((2.0f * n - 1.0f - sqrtf((2.0f * n - 1.0f) * (2.0f * n - 1.0f) - 8.0f * p)) * 0.5f);
    if (a < 0) a = 0;
    if (a > n - 2) a = n - 2;
    while (a > 0 && a * (2 * n - a - 1) / 2 > p) --a;
    while (a < n - 2 && (a + 1) * (2 * n - a - 2) / 2 <= p) ++a;
    const int b = p - a * (2 * n - a - 1) / 2 + a + 1;
    pij[p] = (uint16_t)(a | (b << 8));
  }
}

// Per-thread view of one walker and the group that walks it.  `par` is this
// thread's copy of the block-reduction buffer parity (group-uniform).
template <class G>
struct Walker {
  WalkShared& s;
  WalkArrays arr;
  const PairTables& tab;
  int n;
  int tpa;
  G g;
  int par;
  int swpar = 0;  // Stillinger-Weber: which neighbour-mask buffer the next evaluation uses
  // this thread's share of the chain's evaluated work since the chain began:
  // pairs (LJ: unique interactions; Stillinger-Weber: pairs inside the
  // cutoff) and triplets, with forces, then energy-only
  int tc[4] = {0, 0, 0, 0};
  // sample ring of exactly evaluated configurations (recording when
  // ring_pos is set): step t of the chain owns slot (ring_chain + t) mod
  // ring_cap; ring_step is the current step (every thread's copy)
  float* ring_pos = nullptr;   // [cap][Nmax][3]
  float* ring_cell = nullptr;  // [cap][9]
  double* ring_u = nullptr;    // [cap] model energy U, NaN: slot holds no evaluation
  int ring_nmax = 0;
  long long ring_cap = 0;
  long long ring_chain = 0;
  int ring_step = 0;
  // surrogate walk: the CTA's copy of the surrogate's scalars
  const JrSurrogate* sur = nullptr;
};

__device__ __forceinline__ float& pos_at(float4* xs, int idx) {
  return reinterpret_cast<float*>(xs)[4 * (idx / 3) + (idx % 3)];
}

// jnp.linalg.det of a 3x3 (jax _det_3x3), float32, left to right.
__device__ __forceinline__ float det3(const float* a) {
  float t1 = __fmul_rn(__fmul_rn(a[0], a[4]), a[8]);
  float t2 = __fmul_rn(__fmul_rn(a[1], a[5]), a[6]);
  float t3 = __fmul_rn(__fmul_rn(a[2], a[3]), a[7]);
  float t4 = __fmul_rn(__fmul_rn(a[2], a[4]), a[6]);
  float t5 = __fmul_rn(__fmul_rn(a[0], a[5]), a[7]);
  float t6 = __fmul_rn(__fmul_rn(a[1], a[3]), a[8]);
  float s = __fadd_rn(t1, t2);
  s = __fadd_rn(s, t3);
  s = __fsub_rn(s, t4);
  s = __fsub_rn(s, t5);
  s = __fsub_rn(s, t6);
  return s;
}

// Fill a cell context: det==0 substitutes 1e10*I (lj.py:136-137); a diagonal
// cell inverts with float32 division, any other through the double adjugate.
__device__ inline void make_cell_ctx(const float* h_in, CellCtx& cc, float* T,
                                     const JrModelParams& mp) {
  cc.vol = fabsf(det3(h_in));
  for (int q = 0; q < 9; ++q) cc.raw[q] = h_in[q];
  float h[9];
  if (det3(h_in) == 0.0f) {
    for (int q = 0; q < 9; ++q) h[q] = 0.0f;
    h[0] = h[4] = h[8] = 1.0e10f;
  } else {
    for (int q = 0; q < 9; ++q) h[q] = h_in[q];
  }
  for (int q = 0; q < 9; ++q) cc.h[q] = h[q];
  const bool diag = h[1] == 0.0f && h[2] == 0.0f && h[3] == 0.0f &&
                    h[5] == 0.0f && h[6] == 0.0f && h[7] == 0.0f;
  cc.diag = diag;
  if (diag) {
    for (int q = 0; q < 9; ++q) cc.inv[q] = 0.0f;
    cc.inv[0] = __fdiv_rn(1.0f, h[0]);
    cc.inv[4] = __fdiv_rn(1.0f, h[4]);
    cc.inv[8] = __fdiv_rn(1.0f, h[8]);
  } else {
    double a[9], cof[9];
    for (int q = 0; q < 9; ++q) a[q] = (double)h[q];
    cof[0] = __dsub_rn(__dmul_rn(a[4], a[8]), __dmul_rn(a[5], a[7]));
    cof[1] = __dsub_rn(__dmul_rn(a[5], a[6]), __dmul_rn(a[3], a[8]));
    cof[2] = __dsub_rn(__dmul_rn(a[3], a[7]), __dmul_rn(a[4], a[6]));
    cof[3] = __dsub_rn(__dmul_rn(a[2], a[7]), __dmul_rn(a[1], a[8]));
    cof[4] = __dsub_rn(__dmul_rn(a[0], a[8]), __dmul_rn(a[2], a[6]));
    cof[5] = __dsub_rn(__dmul_rn(a[1], a[6]), __dmul_rn(a[0], a[7]));
    cof[6] = __dsub_rn(__dmul_rn(a[1], a[5]), __dmul_rn(a[2], a[4]));
    cof[7] = __dsub_rn(__dmul_rn(a[2], a[3]), __dmul_rn(a[0], a[5]));
    cof[8] = __dsub_rn(__dmul_rn(a[0], a[4]), __dmul_rn(a[1], a[3]));
    double det = __dadd_rn(__dadd_rn(__dmul_rn(a[0], cof[0]), __dmul_rn(a[1], cof[1])),
                           __dmul_rn(a[2], cof[2]));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        cc.inv[i * 3 + j] = __double2float_rn(__ddiv_rn(cof[j * 3 + i], det));
  }
  for (int k = 0; k < mp.n_images; ++k) {
    const float* o = mp.img_off + 3 * k;
    for (int q = 0; q < 3; ++q) {
      float v = __fmul_rn(o[0], h[q]);
      v = __fmaf_rn(o[1], h[3 + q], v);
      v = __fmaf_rn(o[2], h[6 + q], v);
      T[3 * k + q] = v;
    }
  }
}

// Triclinic minimum image: dr - round(dr @ inv) @ h (lj.py:147-154).  The
// diagonal branch is the general formula with the zero terms dropped, which
// leaves every result bit unchanged.
__device__ __forceinline__ void mic(const CellCtx& cc, float& dx, float& dy, float& dz) {
  if (cc.diag) {
    float n0 = rintf(__fmul_rn(dx, cc.inv[0]));
    float n1 = rintf(__fmul_rn(dy, cc.inv[4]));
    float n2 = rintf(__fmul_rn(dz, cc.inv[8]));
    dx = __fsub_rn(dx, __fmul_rn(n0, cc.h[0]));
    dy = __fsub_rn(dy, __fmul_rn(n1, cc.h[4]));
    dz = __fsub_rn(dz, __fmul_rn(n2, cc.h[8]));
  } else {
    float n[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float f = __fmul_rn(dx, cc.inv[q]);
      f = __fmaf_rn(dy, cc.inv[3 + q], f);
      f = __fmaf_rn(dz, cc.inv[6 + q], f);
      n[q] = rintf(f);
    }
    float s[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float v = __fmul_rn(n[0], cc.h[q]);
      v = __fmaf_rn(n[1], cc.h[3 + q], v);
      v = __fmaf_rn(n[2], cc.h[6 + q], v);
      s[q] = v;
    }
    dx = __fsub_rn(dx, s[0]);
    dy = __fsub_rn(dy, s[1]);
    dz = __fsub_rn(dz, s[2]);
  }
}

// Register copy of the geometry the minimum image needs; for a diagonal cell
// only the six diagonal entries are read (the rest are never loaded).
struct MicRegs {
  float inv[9];
  float h[9];
};

template <bool kDiag>
__device__ __forceinline__ MicRegs load_mic(const CellCtx& cc) {
  MicRegs m;
  if (kDiag) {
    m.inv[0] = cc.inv[0]; m.inv[4] = cc.inv[4]; m.inv[8] = cc.inv[8];
    m.h[0] = cc.h[0]; m.h[4] = cc.h[4]; m.h[8] = cc.h[8];
  } else {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      m.inv[q] = cc.inv[q];
      m.h[q] = cc.h[q];
    }
  }
  return m;
}

// mic() with the cell in registers; bit-identical to mic() for either branch.
template <bool kDiag>
__device__ __forceinline__ void mic_r(const MicRegs& m, float& dx, float& dy, float& dz) {
  if (kDiag) {
    const float n0 = rintf(__fmul_rn(dx, m.inv[0]));
    const float n1 = rintf(__fmul_rn(dy, m.inv[4]));
    const float n2 = rintf(__fmul_rn(dz, m.inv[8]));
    dx = __fsub_rn(dx, __fmul_rn(n0, m.h[0]));
    dy = __fsub_rn(dy, __fmul_rn(n1, m.h[4]));
    dz = __fsub_rn(dz, __fmul_rn(n2, m.h[8]));
  } else {
    float n[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float f = __fmul_rn(dx, m.inv[q]);
      f = __fmaf_rn(dy, m.inv[3 + q], f);
      f = __fmaf_rn(dz, m.inv[6 + q], f);
      n[q] = rintf(f);
    }
    float sh[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float v = __fmul_rn(n[0], m.h[q]);
      v = __fmaf_rn(n[1], m.h[3 + q], v);
      v = __fmaf_rn(n[2], m.h[6 + q], v);
      sh[q] = v;
    }
    dx = __fsub_rn(dx, sh[0]);
    dy = __fsub_rn(dy, sh[1]);
    dz = __fsub_rn(dz, sh[2]);
  }
}

// 1/x for the pair loop: a bit-pattern seed refined by three Newton-Raphson
// steps y <- y + y*(1 - x*y), all in fused multiply-adds, so the result is the
// same on any IEEE machine with an FMA (the CPU check reproduces it bit for
// bit).  The seed y0 = as_float(C - as_int(x)) is the piecewise-linear
// reciprocal of the float bit pattern (the exponent negated, the mantissa
// reflected); C sets its offset.  Scanning every C over the mantissas of one
// binade, the largest relative error max|x*y0 - 1| is smallest at C =
// 0x7EF311C2 (5.0510%), and C = 0x7EF311C3, used here, is within 2e-8 of it.
// Each Newton step squares the relative error: 5.05% -> 2.6e-3 -> 6.5e-6 ->
// 4e-11, below half an ulp before the last rounding.  Max error 0.501 ulp
// over normal inputs; inputs outside [2^-120, 2^120] (zero, denormals, inf,
// NaN) take the correctly rounded reciprocal.
__device__ __noinline__ inline float rcp_rare(float x) { return __frcp_rn(x); }

__device__ __forceinline__ float rcp_nr(float x) {
  float y = __int_as_float(0x7EF311C3 - __float_as_int(x));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float e = __fmaf_rn(-x, y, 1.0f);
    y = __fmaf_rn(y, e, y);
  }
  // rare: a branch to an out-of-line call keeps the correctly rounded
  // reciprocal's instructions off the common path
  if (__builtin_expect(!(x >= 0x1p-120f && x <= 0x1p120f), 0)) y = rcp_rare(x);
  return y;
}

// One LJ pair term (lj.py:191-203), float32: energy e and the force
// coefficient g with F_i += g * dr_ij; e = g = 0 beyond the cutoff.  Written
// branch-free (compute, then select) so a warp never splits on the cutoff.
__device__ __forceinline__ void lj_pair(float dx, float dy, float dz, float sig2, float eps4,
                                        float eps24, bool has_cut, float rc2, float& e,
                                        float& g) {
  float r2 = __fmul_rn(dx, dx);
  r2 = __fmaf_rn(dy, dy, r2);
  r2 = __fmaf_rn(dz, dz, r2);
  const bool inside = !has_cut || (r2 < rc2);
  const float ri = rcp_nr(r2);
  const float s2 = __fmul_rn(sig2, ri);
  const float s4 = __fmul_rn(s2, s2);
  const float s6 = __fmul_rn(s4, s2);
  const float s12 = __fmul_rn(s6, s6);
  const float ev = __fmul_rn(eps4, __fsub_rn(s12, s6));
  const float t = __fmaf_rn(2.0f, s12, -s6);
  const float a = __fmul_rn(eps24, ri);
  const float gv = -__fmul_rn(a, t);
  e = inside ? ev : 0.0f;
  g = inside ? gv : 0.0f;
}

// Ensemble term P*V - mu*N (ensemble.py:34-59) in float64.
__device__ __forceinline__ double ensemble_term(const WalkShared& s, float vol, float pressure,
                                                const float* mu, int nsp) {
  double e = (double)pressure * (double)vol;
  if (mu) {
    double dot = 0.0;
    for (int q = 0; q < nsp; ++q) dot += (double)mu[q] * (double)s.counts[q];
    e = e - dot;
  }
  return e;
}

// Gaussian-mixture toy (toy.py:163-204), float64, forces rounded to float32.
__device__ inline double gauss_mix_energy(const JrModelParams& mp, const float4* xs, int n,
                                          float* F, bool forces) {
  double com[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    com[0] += (double)xs[i].x;
    com[1] += (double)xs[i].y;
    com[2] += (double)xs[i].z;
  }
  for (int q = 0; q < 3; ++q) com[q] /= (double)n;
  const double s2 = (double)mp.gm_sigma * (double)mp.gm_sigma;
  const double lnorm = 1.5 * log(2.0 * 3.141592653589793 * s2);
  double l[JR_MAX_CENTERS], lmax = -INFINITY;
  for (int k = 0; k < mp.n_centers; ++k) {
    double ds = 0.0;
    for (int q = 0; q < 3; ++q) {
      double df = com[q] - (double)mp.centers[3 * k + q];
      ds += df * df;
    }
    l[k] = -0.5 * ds / s2 - lnorm;
    if (l[k] > lmax) lmax = l[k];
  }
  double z = 0.0;
  for (int k = 0; k < mp.n_centers; ++k) z += exp(l[k] - lmax);
  const double E = -(lmax + log(z));
  if (forces) {
    double g[3] = {0, 0, 0};
    for (int k = 0; k < mp.n_centers; ++k) {
      double p = exp(l[k] - lmax) / z;
      for (int q = 0; q < 3; ++q) g[q] += p * (com[q] - (double)mp.centers[3 * k + q]) / s2;
    }
    for (int i = 0; i < n; ++i)
      for (int q = 0; q < 3; ++q) F[3 * i + q] = (float)(-g[q] / (double)n);
  }
  return E;
}

__device__ __forceinline__ int center_image(const JrModelParams& mp) {
  for (int k = 0; k < mp.n_images; ++k)
    if (mp.img_off[3 * k] == 0.0f && mp.img_off[3 * k + 1] == 0.0f &&
        mp.img_off[3 * k + 2] == 0.0f)
      return k;
  return -1;
}

// Force gather contract: F_i is accumulated in float32 in a canonical order
// that depends only on n -- partners j in blocks of 8 (sequential, ascending
// j, then ascending image), then the block partials combined pairwise
// ((P0+P1)+(P2+P3))+... over L = next_pow2(ceil(n/8)) lanes.  The lanes of
// one atom are adjacent in a warp; the pairwise tree is the xor butterfly.
__device__ __forceinline__ int gather_lanes(int n) {
  const int nb = (n + 7) >> 3;
  int L = 1;
  while (L < nb) L <<= 1;
  return L;
}

__device__ __forceinline__ void gather_tree(float& fx, float& fy, float& fz, int L) {
  for (int off = 1; off < L; off <<= 1) {
    fx = __fadd_rn(fx, __shfl_xor_sync(0xffffffffu, fx, off));
    fy = __fadd_rn(fy, __shfl_xor_sync(0xffffffffu, fy, off));
    fz = __fadd_rn(fz, __shfl_xor_sync(0xffffffffu, fz, off));
  }
}

// Unordered pairs a < b once each (pair matrix path): the force term g*dr of
// pair (a,b) goes to M[a][b] and its negation to M[b][a] (the float32 term of
// the mirrored ordered pair is exactly the negation); atom i then gathers its
// row in the canonical order.  U is the float64 sum over pairs.
template <bool kForces, bool kS1, bool kDiag, class G>
__device__ __forceinline__ void pairs_matrix(const JrParams& P, Walker<G>& w, const MicRegs& cc,
                                             double& U, double& sff, double& sfd) {
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int nsp = P.model.n_species;
  const bool has_cut = P.model.has_cutoff != 0;
  const float rc2 = P.model.rc2;
  const float sig2_1 = w.tab.sig2[0], eps4_1 = w.tab.eps4[0], eps24_1 = w.tab.eps24[0];
  const int np = n * (n - 1) / 2;
  const int tid = w.g.rank(), gs = w.g.size();
  const int S = pm_stride(n), plane = n * S;
  double ep = 0.0;
  // Two pairs per trip with every shared-memory load issued before any store,
  // so the pairs overlap (the compiler cannot move loads above the stores).
  auto term = [&](const float4 xa, const float4 xb, float& e, float& vx, float& vy, float& vz) {
    float dx = __fsub_rn(xb.x, xa.x);
    float dy = __fsub_rn(xb.y, xa.y);
    float dz = __fsub_rn(xb.z, xa.z);
    mic_r<kDiag>(cc, dx, dy, dz);
    float sig2 = sig2_1, eps4 = eps4_1, eps24 = eps24_1;
    if (!kS1) {
      const int pt = __float_as_int(xa.w) * nsp + __float_as_int(xb.w);
      sig2 = w.tab.sig2[pt];
      eps4 = w.tab.eps4[pt];
      eps24 = w.tab.eps24[pt];
    }
    float g;
    lj_pair(dx, dy, dz, sig2, eps4, eps24, has_cut, rc2, e, g);
    vx = __fmul_rn(g, dx);
    vy = __fmul_rn(g, dy);
    vz = __fmul_rn(g, dz);
  };
  auto put = [&](int a, int b, float vx, float vy, float vz) {
    const int ab = a * S + b, ba = b * S + a;
    arr.pm[ab] = vx;
    arr.pm[ba] = -vx;
    arr.pm[plane + ab] = vy;
    arr.pm[plane + ba] = -vy;
    arr.pm[2 * plane + ab] = vz;
    arr.pm[2 * plane + ba] = -vz;
  };
  for (int p0 = tid; p0 < np; p0 += 2 * gs) {
    const int p1 = p0 + gs;
    const bool two = p1 < np;
    const uint32_t ab0 = arr.pij[p0];
    const uint32_t ab1 = two ? arr.pij[p1] : ab0;
    const int a0 = ab0 & 255, b0 = ab0 >> 8, a1 = ab1 & 255, b1 = ab1 >> 8;
    const float4 xa0 = arr.xs[a0], xb0 = arr.xs[b0], xa1 = arr.xs[a1], xb1 = arr.xs[b1];
    float e0, vx0, vy0, vz0, e1, vx1, vy1, vz1;
    term(xa0, xb0, e0, vx0, vy0, vz0);
    term(xa1, xb1, e1, vx1, vy1, vz1);
    ep += (double)e0;
    if (two) ep += (double)e1;
    if (kForces) {
      put(a0, b0, vx0, vy0, vz0);
      if (two) put(a1, b1, vx1, vy1, vz1);
    }
  }
  if (tid == 0) w.tc[kForces ? 0 : 2] += np;
  if (!kForces) {
    w.g.sum1(ep, 1, w.par);
    U = ep;
    sff = 0.0;
    sfd = 0.0;
    return;
  }
  w.g.sync();
  const int L = gather_lanes(n);
  const int apb = gs / L;
  const int blk = tid & (L - 1);
  double ff_part = 0.0, fd_part = 0.0;
  // The energy partials are first summed over the L lanes of an atom group
  // (every lane of the group ends with the group sum), so the group
  // reduction below starts at stride L, where ff and fd live.  Warps that
  // gather do it while their row loads are in flight.
  bool ep_folded = false;
  auto fold_ep = [&]() {
    for (int off = 1; off < L; off <<= 1) ep += __shfl_xor_sync(0xffffffffu, ep, off);
    ep_folded = true;
  };
  for (int base = 0; base < n; base += apb) {
    const int i = base + tid / L;
    // warps whose atoms all lie beyond n leave the issue slots to the others
    if (!__any_sync(0xffffffffu, i < n)) continue;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    // partners j0..j0+7 in ascending order; an absent partner (the atom
    // itself, or a column past n) adds +0, which leaves the running sum
    // unchanged (it is never -0); all 24 loads issue before the adds.
    const int j0 = blk * 8;
    const int ic = i < n ? i : 0;
    const float d0 = arr.dir[3 * ic], d1 = arr.dir[3 * ic + 1], d2 = arr.dir[3 * ic + 2];
    float vx[8], vy[8], vz[8];
    if (j0 < n) {
      // partners j0..j0+7 of row i: the diagonal and the columns past n hold
      // +0.0 (lanes of atoms past n read row 0; their sums are discarded)
      const float* row = arr.pm + ic * S + j0;
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        vx[jj] = row[jj];
        vy[jj] = row[plane + jj];
        vz[jj] = row[2 * plane + jj];
      }
    } else {
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) vx[jj] = vy[jj] = vz[jj] = 0.0f;
    }
    if (!ep_folded) fold_ep();
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      fx = __fadd_rn(fx, vx[jj]);
      fy = __fadd_rn(fy, vy[jj]);
      fz = __fadd_rn(fz, vz[jj]);
    }
    gather_tree(fx, fy, fz, L);
    if (blk == 0 && i < n) {
      arr.F[3 * i] = fx;
      arr.F[3 * i + 1] = fy;
      arr.F[3 * i + 2] = fz;
      const double dx = fx, dy = fy, dz = fz;
      ff_part = __fma_rn(dx, dx, __fma_rn(dy, dy, __fma_rn(dz, dz, ff_part)));
      fd_part = __fma_rn(dx, (double)d0, __fma_rn(dy, (double)d1, __fma_rn(dz, (double)d2, fd_part)));
    }
  }
  if (!ep_folded) fold_ep();
  double e_part = ep;
  w.g.sum3(e_part, ff_part, fd_part, L, w.par);
  U = e_part;
  sff = ff_part;
  sfd = fd_part;
}

// Ordered pairs (i, j), every image; gather_lanes(n) lanes per atom i, each
// lane one block of 8 partners (the canonical gather order above).
template <bool kForces, bool kS1, bool kDiag, class G>
__device__ __forceinline__ void pairs_ordered(const JrParams& P, Walker<G>& w, const MicRegs& cc,
                                              const float* T, double& U, double& sff,
                                              double& sfd) {
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const JrModelParams& mp = P.model;
  const int nimg = mp.n_images;
  const bool has_cut = mp.has_cutoff != 0;
  const float rc2 = mp.rc2;
  const int nsp = mp.n_species;
  const float sig2_1 = w.tab.sig2[0], eps4_1 = w.tab.eps4[0], eps24_1 = w.tab.eps24[0];
  const int tid = w.g.rank();
  const int L = gather_lanes(n);
  const int apb = w.g.size() / L;
  const int blk = tid & (L - 1);
  const int center = center_image(mp);
  // unique interactions: every image of every pair once, no self term in
  // the centre image
  if (tid == 0) w.tc[kForces ? 0 : 2] += (nimg * n * n - n) / 2;
  double e_part = 0.0, ff_part = 0.0, fd_part = 0.0;
  for (int base = 0; base < n; base += apb) {
    const int i = base + tid / L;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (i < n) {
      const float4 xi = arr.xs[i];
      const int ti = __float_as_int(xi.w);
      const int j0 = blk * 8;
      const int j1 = j0 + 8 < n ? j0 + 8 : n;
      for (int j = j0; j < j1; ++j) {
        const float4 xj = arr.xs[j];
        float dx = __fsub_rn(xj.x, xi.x);
        float dy = __fsub_rn(xj.y, xi.y);
        float dz = __fsub_rn(xj.z, xi.z);
        mic_r<kDiag>(cc, dx, dy, dz);
        float sig2 = sig2_1, eps4 = eps4_1, eps24 = eps24_1;
        if (!kS1) {
          const int pt = ti * nsp + __float_as_int(xj.w);
          sig2 = w.tab.sig2[pt];
          eps4 = w.tab.eps4[pt];
          eps24 = w.tab.eps24[pt];
        }
        if (nimg == 1) {
          if (j != i) {
            float e, g;
            lj_pair(dx, dy, dz, sig2, eps4, eps24, has_cut, rc2, e, g);
            e_part += (double)e;
            if (kForces) {
              fx = __fadd_rn(fx, __fmul_rn(g, dx));
              fy = __fadd_rn(fy, __fmul_rn(g, dy));
              fz = __fadd_rn(fz, __fmul_rn(g, dz));
            }
          }
        } else {
          for (int k = 0; k < nimg; ++k) {
            if (k == center && i == j) continue;
            const float ex = __fadd_rn(dx, T[3 * k]);
            const float ey = __fadd_rn(dy, T[3 * k + 1]);
            const float ez = __fadd_rn(dz, T[3 * k + 2]);
            float e, g;
            lj_pair(ex, ey, ez, sig2, eps4, eps24, has_cut, rc2, e, g);
            e_part += (double)e;
            if (kForces && i != j) {
              fx = __fadd_rn(fx, __fmul_rn(g, ex));
              fy = __fadd_rn(fy, __fmul_rn(g, ey));
              fz = __fadd_rn(fz, __fmul_rn(g, ez));
            }
          }
        }
      }
    }
    if (kForces) {
      gather_tree(fx, fy, fz, L);
      if (blk == 0 && i < n) {
        arr.F[3 * i] = fx;
        arr.F[3 * i + 1] = fy;
        arr.F[3 * i + 2] = fz;
        ff_part += (double)fx * (double)fx + (double)fy * (double)fy + (double)fz * (double)fz;
        fd_part += (double)fx * (double)arr.dir[3 * i] + (double)fy * (double)arr.dir[3 * i + 1] +
                   (double)fz * (double)arr.dir[3 * i + 2];
      }
    }
  }
  if (kForces) w.g.sum3(e_part, ff_part, fd_part, 1, w.par);
  else w.g.sum1(e_part, 1, w.par);
  U = 0.5 * e_part;
  sff = ff_part;
  sfd = fd_part;
}

}  // namespace jr

#include "jr_sw.cuh"

namespace jr {

// The pair family's models: the Gaussian-mixture toy and LJ.
template <bool kForces, class G>
__device__ __forceinline__ void model_eval_pair(const JrParams& P, Walker<G>& w, int cidx,
                                                double& U, double& sff, double& sfd) {
  const WalkArrays& arr = w.arr;
  const JrModelParams& mp = P.model;
  if (mp.model == JR_MODEL_GAUSS_MIX) {
    double e = 0.0, a = 0.0, b = 0.0;
    if (w.g.leader()) {
      e = gauss_mix_energy(mp, arr.xs, w.n, arr.F, kForces);
      if (kForces) {
        for (int q = 0; q < 3 * w.n; ++q) {
          a += (double)arr.F[q] * (double)arr.F[q];
          b += (double)arr.F[q] * (double)arr.dir[q];
        }
      }
    }
    w.g.sum3(e, a, b, 1, w.par);
    U = e;
    sff = a;
    sfd = b;
    w.g.sync();
    return;
  }
  const CellCtx& ccs = w.s.cc[cidx];
  const bool s1 = mp.n_species == 1;
  const bool diag = ccs.diag != 0;
  if (arr.pm != nullptr && mp.n_images == 1 && w.n <= kPairMatMax) {
    if (diag) {
      const MicRegs cc = load_mic<true>(ccs);
      if (s1) pairs_matrix<kForces, true, true>(P, w, cc, U, sff, sfd);
      else pairs_matrix<kForces, false, true>(P, w, cc, U, sff, sfd);
    } else {
      const MicRegs cc = load_mic<false>(ccs);
      if (s1) pairs_matrix<kForces, true, false>(P, w, cc, U, sff, sfd);
      else pairs_matrix<kForces, false, false>(P, w, cc, U, sff, sfd);
    }
  } else {
    const float* T = arr.T + cidx * 3 * mp.n_images;
    if (diag) {
      const MicRegs cc = load_mic<true>(ccs);
      if (s1) pairs_ordered<kForces, true, true>(P, w, cc, T, U, sff, sfd);
      else pairs_ordered<kForces, false, true>(P, w, cc, T, U, sff, sfd);
    } else {
      const MicRegs cc = load_mic<false>(ccs);
      if (s1) pairs_ordered<kForces, true, false>(P, w, cc, T, U, sff, sfd);
      else pairs_ordered<kForces, false, false>(P, w, cc, T, U, sff, sfd);
    }
  }
}

// Model energy U (forces into arr.F when kForces) of the walker; also sum(F^2)
// and sum(F . dir) for the galilean reflection.  Results are group-uniform.
template <bool kForces, class G>
__device__ __forceinline__ void model_eval(const JrParams& P, Walker<G>& w, int cidx, double& U, double& sff,
                           double& sfd) {
  if constexpr (sw_family(G::kFam)) {
    const CellCtx& ccs = w.s.cc[cidx];
    if (ccs.diag) sw_eval<kForces, true>(P, w, load_mic<true>(ccs), U, sff, sfd);
    else sw_eval<kForces, false>(P, w, load_mic<false>(ccs), U, sff, sfd);
  } else {
    model_eval_pair<kForces>(P, w, cidx, U, sff, sfd);
  }
}

// Full potential of the walker for cell context cidx: U + (P*V - mu*N).
template <bool kForces, class G>
__device__ __forceinline__ double ham_eval(const JrParams& P, Walker<G>& w, int cidx,
                                           float pressure, const float* mu, double& sff,
                                           double& sfd) {
  double U;
  model_eval<kForces>(P, w, cidx, U, sff, sfd);
  if (P.model.model == JR_MODEL_GAUSS_MIX) return U;
  return U + ensemble_term(w.s, w.s.cc[cidx].vol, pressure, mu, P.model.n_species);
}

template <class G>
__device__ __forceinline__ double group_sum1(Walker<G>& w, double v) {
  w.g.sum1(v, 1, w.par);
  return v;
}

// ---------------------------------------------------------------- moves --

// The R position updates and evaluations of one galilean trajectory.  The
// pair path, the species branch and the cell geometry are chosen once for
// the trajectory (the cell is fixed during the move), so each evaluation
// starts directly on the pair loop; ens is the fixed P V - mu N share.
// Returns the final potential (NaN read as +inf); the direction is reflected
// off the contour in place.
constexpr int kTrajModel = 0, kTrajMatrix = 1, kTrajOrdered = 2, kTrajSW = 3;

template <int kPath, bool kS1, bool kDiag, class G>
__device__ __forceinline__ double galilean_trajectory(const JrParams& P, Walker<G>& w, float step,
                                                      int R, double emax, double ens) {
  const WalkArrays& arr = w.arr;
  const int n3 = 3 * w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const int cidx = w.s.cur;
  MicRegs cc;
  if (kPath != kTrajModel) cc = load_mic<kDiag>(w.s.cc[cidx]);
  const float* T = arr.T + cidx * 3 * P.model.n_images;
  double E = w.s.E;
  // a reflection off the contour is applied by the coordinate's owner thread
  // together with the next position update (d is reused from the register)
  bool refl = false;
  float coef = 0.0f;
  for (int r = 0; r < R; ++r) {
    for (int q = r0; q < n3; q += gs) {
      float d = arr.dir[q];
      if (refl) {
        d = __fmaf_rn(-coef, arr.F[q], d);
        arr.dir[q] = d;
      }
      float& x = pos_at(arr.xs, q);
      x = __fmaf_rn(step, d, x);
    }
    w.g.sync();
    // Forces only steer a reflection, so each step first evaluates the
    // energy alone and evaluates the forces (at the same positions) only when
    // the step lands on or above the contour -- a few percent of the steps
    // on the benchmark workloads.  The walk is the same as evaluating both
    // every step: the decision reads the energy, the reflection the forces.
    double U, sff = 0.0, sfd = 0.0;
    if constexpr (kPath == kTrajSW) {
      sw_eval<false, kDiag>(P, w, cc, U, sff, sfd);
      E = U + ens;
    } else if (kPath == kTrajMatrix) {
      pairs_matrix<false, kS1, kDiag>(P, w, cc, U, sff, sfd);
      E = U + ens;
    } else if (kPath == kTrajOrdered) {
      pairs_ordered<false, kS1, kDiag>(P, w, cc, T, U, sff, sfd);
      E = U + ens;
    } else {
      model_eval<true>(P, w, cidx, U, sff, sfd);
      E = U;
    }
    if (isnan(E)) E = INFINITY;
    refl = E >= emax;
    if (refl) {
      if constexpr (kPath == kTrajSW) sw_eval<true, kDiag>(P, w, cc, U, sff, sfd);
      else if constexpr (kPath == kTrajMatrix) pairs_matrix<true, kS1, kDiag>(P, w, cc, U, sff, sfd);
      else if constexpr (kPath == kTrajOrdered)
        pairs_ordered<true, kS1, kDiag>(P, w, cc, T, U, sff, sfd);
      // d <- d - [2 (F.d) / max(|F|^2, 1e-20)] F, the scalar in float32
      const float ffs = __double2float_rn(sff);
      coef = __fmul_rn(2.0f * __double2float_rn(sfd), rcp_nr(ffs > 1e-20f ? ffs : 1e-20f));
    }
  }
  if (refl)
    for (int q = r0; q < n3; q += gs) arr.dir[q] = __fmaf_rn(-coef, arr.F[q], arr.dir[q]);
  return E;
}

// Galilean move (galilean.py:142-300) with forces-based reflection.  The
// reflection d - 2 (f.d) f with f = F/|F| is evaluated as
// d - [2 (F.d) / max(|F|,1e-10)^2] F from two float64 sums.
template <class G>
__device__ __forceinline__ bool move_galilean(const JrParams& P, Walker<G>& w, const StepKey& key, float step, int R,
                              float pa, double emax, float pressure, const float* mu) {
  const WalkArrays& arr = w.arr;
  const int n3 = 3 * w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const Key ki = key.k0, kp = key.k1;
  // |d|^2 and |d + pa * normal|^2 in one group reduction; a direction of
  // norm < 1e-8 (a walker's first galilean move) then redraws a fresh normal
  // direction and reduces its norm separately.  The sums are the ones of
  // the two-pass form (same partials, same tree).
  double sq = 0.0, sv = 0.0, zero = 0.0;
  for (int q = r0; q < n3; q += gs) {
    const float d = arr.dir[q];
    const float g = key.nz ? key.nz[q] : normal(bits32(kp, (uint32_t)q));
    const float v = __fmaf_rn(pa, g, d);
    sq += (double)d * (double)d;
    sv += (double)v * (double)v;
    arr.dir[q] = v;
  }
  w.g.sum3(sq, sv, zero, 1, w.par);
  if (__double2float_rn(sqrt(sq)) < 1e-8f) {
    sv = 0.0;
    for (int q = r0; q < n3; q += gs) {
      const float v = normal(bits32(ki, (uint32_t)q));
      arr.dir[q] = v;
      sv += (double)v * (double)v;
    }
    sv = group_sum1(w, sv);
  }
  const float nv = __double2float_rn(sqrt(sv));
  const float den = nv > 1e-10f ? nv : 1e-10f;
  for (int q = r0; q < n3; q += gs) {
    const float v = __fdiv_rn(arr.dir[q], den);
    arr.dir[q] = v;
    arr.dp[q] = v;
    arr.x0[q] = pos_at(arr.xs, q);
  }
  const double E0 = w.s.E;
  double E;
  const JrModelParams& mp = P.model;
  if constexpr (sw_family(G::kFam)) {
    const double ens = ensemble_term(w.s, w.s.cc[w.s.cur].vol, pressure, mu, mp.n_species);
    if (w.s.cc[w.s.cur].diag) E = galilean_trajectory<kTrajSW, true, true>(P, w, step, R, emax, ens);
    else E = galilean_trajectory<kTrajSW, true, false>(P, w, step, R, emax, ens);
  } else if (mp.model == JR_MODEL_GAUSS_MIX) {
    E = galilean_trajectory<kTrajModel, true, true>(P, w, step, R, emax, 0.0);
  } else {
    // the cell, the species counts and so P V - mu N are fixed for the move
    const double ens = ensemble_term(w.s, w.s.cc[w.s.cur].vol, pressure, mu, mp.n_species);
    const bool s1 = mp.n_species == 1;
    const bool diag = w.s.cc[w.s.cur].diag != 0;
    if (arr.pm != nullptr && mp.n_images == 1 && w.n <= kPairMatMax) {
      if (diag) E = s1 ? galilean_trajectory<kTrajMatrix, true, true>(P, w, step, R, emax, ens)
                       : galilean_trajectory<kTrajMatrix, false, true>(P, w, step, R, emax, ens);
      else E = s1 ? galilean_trajectory<kTrajMatrix, true, false>(P, w, step, R, emax, ens)
                  : galilean_trajectory<kTrajMatrix, false, false>(P, w, step, R, emax, ens);
    } else {
      if (diag) E = s1 ? galilean_trajectory<kTrajOrdered, true, true>(P, w, step, R, emax, ens)
                       : galilean_trajectory<kTrajOrdered, false, true>(P, w, step, R, emax, ens);
      else E = s1 ? galilean_trajectory<kTrajOrdered, true, false>(P, w, step, R, emax, ens)
                  : galilean_trajectory<kTrajOrdered, false, false>(P, w, step, R, emax, ens);
    }
  }
  const bool acc = E < emax;
  if (!acc) {
    for (int q = r0; q < n3; q += gs) {
      pos_at(arr.xs, q) = arr.x0[q];
      arr.dir[q] = -arr.dp[q];
    }
  }
  // every thread read s.E before the trajectory's barriers
  if (w.g.leader()) w.s.E = acc ? E : E0;
  w.g.sync();
  return acc;
}

// check_cell_shape (utils/cell.py:80-125), float32 with float64 sums.
__device__ inline bool cell_valid(const float* c, int n, const JrMoveParams& mv) {
  const float vol = fabsf(det3(c));
  const float vpa = __fdiv_rn(vol, (float)n);
  const float vc = __double2float_rn(pow((double)vol, (double)(1.0f / 3.0f)));
  const int pr[3][3] = {{0, 1, 2}, {1, 2, 0}, {0, 2, 1}};
  float amin = INFINITY;
  for (int p = 0; p < 3; ++p) {
    const float* a = c + 3 * pr[p][0];
    const float* b = c + 3 * pr[p][1];
    const float* e = c + 3 * pr[p][2];
    float cr[3];
    cr[0] = __fsub_rn(__fmul_rn(a[1], b[2]), __fmul_rn(a[2], b[1]));
    cr[1] = __fsub_rn(__fmul_rn(a[2], b[0]), __fmul_rn(a[0], b[2]));
    cr[2] = __fsub_rn(__fmul_rn(a[0], b[1]), __fmul_rn(a[1], b[0]));
    double sq = 0.0;
    for (int q = 0; q < 3; ++q) sq += (double)cr[q] * (double)cr[q];
    const float nrm = __double2float_rn(sqrt(sq));
    float cn[3];
    for (int q = 0; q < 3; ++q) cn[q] = __fdiv_rn(cr[q], nrm);
    double hd = (double)cn[0] * (double)e[0];
    hd = hd + (double)cn[1] * (double)e[1];
    hd = hd + (double)cn[2] * (double)e[2];
    const float h = fabsf(__double2float_rn(hd));
    const float ratio = __fdiv_rn(h, vc);
    if (ratio < amin || isnan(ratio)) amin = ratio;
  }
  return (vpa <= mv.max_vpa) && (vpa >= mv.min_vpa) && (amin >= mv.min_aspect);
}

// The volume prior's ratio: 1 for a flat prior, else ratio**N by
// lax.integer_pow's binary exponentiation, in float64.
__device__ __forceinline__ double volume_jacobian(float ratio, int n, bool flat) {
  if (flat) return 1.0;
  double acc = 1.0, b = (double)ratio;
  bool first = true;
  int y = n;
  while (y > 0) {
    if (y & 1) {
      acc = first ? b : acc * b;
      first = false;
    }
    y >>= 1;
    if (y > 0) b = b * b;
  }
  return acc;
}

// Acceptance probability of the volume prior: min(1, volume_jacobian).
__device__ __forceinline__ double volume_prior(float ratio, int n, bool flat) {
  const double j = volume_jacobian(ratio, n, flat);
  return j < 1.0 ? j : 1.0;
}

// Volume move (volume.py:49-109 + _common.py:16-93).  Returns acceptance and
// the reject reason (priority energy > cell > prior).
template <class G>
__device__ __forceinline__ bool move_volume(const JrParams& P, Walker<G>& w, const StepKey& key, float step, double emax,
                            float pressure, const float* mu, int& reason) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const JrMoveParams& mv = P.moves;
  const Key k1 = key.k0, k2 = key.k1;
  const int cur = s.cur, tr = cur ^ 1;
  const float* h = s.cc[cur].raw;
  const float oldV = s.cc[cur].vol;
  const float sn = __fmul_rn(step, (float)n);
  const float dV = __fmul_rn(sn, key.pre ? key.vn : normal(bits32(k1, 0u)));
  const float newV = fabsf(__fadd_rn(oldV, dV));
  const float ratio = __fdiv_rn(newV, oldV);
  const float scale = __double2float_rn(pow((double)ratio, (double)(1.0f / 3.0f)));
  float nc[9];
  for (int q = 0; q < 9; ++q) nc[q] = __fmul_rn(h[q], scale);
  const int n3 = 3 * n;
  for (int q = r0; q < n3; q += gs) {
    float& x = pos_at(arr.xs, q);
    arr.x0[q] = x;
    x = __fmul_rn(x, scale);
  }
  // the trial cell context and the cell-geometry check, side by side on two
  // threads (of different warps when the group has them)
  const int helper = gs > 32 ? 32 : 1;
  if (w.g.leader()) make_cell_ctx(nc, s.cc[tr], arr.T + tr * 3 * P.model.n_images, P.model);
  else if (r0 == helper % gs) s.cell_ok = cell_valid(nc, n, mv) ? 1 : 0;
  w.g.sync();
  double d0, d1;
  const double En = ham_eval<false>(P, w, tr, pressure, mu, d0, d1);
  const bool valid = s.cell_ok != 0;
  const float u = key.pre ? key.vu : uniform01(bits32(k2, 0u));
  const bool prior_ok = (double)u < volume_prior(ratio, n, mv.flat_v_prior != 0);
  const bool energy_ok = En < emax;
  const bool acc = energy_ok && valid && prior_ok;
  reason = acc ? 0 : (!energy_ok ? 1 : (!valid ? 2 : 3));
  if (!acc) {
    for (int q = r0; q < n3; q += gs) pos_at(arr.xs, q) = arr.x0[q];
  }
  // cur and tr are held in registers; nothing reads s.cur or s.E before this
  // barrier
  if (w.g.leader() && acc) {
    s.cur = tr;
    s.E = En;
  }
  w.g.sync();
  return acc;
}

// Cell-move tail shared by shear and stretch (moves/_common.py:16-93 without
// a prior): positions x' = x . T (float32, the FMA order of the oracle), one
// energy-only evaluation with the new cell, the cell-geometry guard; accept
// iff the energy is under the contour and the cell is valid (energy > cell).
template <class G>
__device__ __forceinline__ bool move_cell(const JrParams& P, Walker<G>& w, const float* nc,
                                          const float* T, double emax, float pressure,
                                          const float* mu, int& reason) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const int cur = s.cur, tr = cur ^ 1;
  for (int i = r0; i < n; i += gs) {
    const float4 x = arr.xs[i];
    arr.x0[3 * i] = x.x;
    arr.x0[3 * i + 1] = x.y;
    arr.x0[3 * i + 2] = x.z;
    float y[3];
    for (int q = 0; q < 3; ++q)
      y[q] = __fmaf_rn(x.z, T[6 + q], __fmaf_rn(x.y, T[3 + q], __fmul_rn(x.x, T[q])));
    arr.xs[i] = make_float4(y[0], y[1], y[2], x.w);
  }
  w.g.sync();
  if (w.g.leader()) make_cell_ctx(nc, s.cc[tr], arr.T + tr * 3 * P.model.n_images, P.model);
  w.g.sync();
  double d0, d1;
  const double En = ham_eval<false>(P, w, tr, pressure, mu, d0, d1);
  const bool valid = cell_valid(nc, n, P.moves);
  const bool energy_ok = En < emax;
  const bool acc = energy_ok && valid;
  reason = acc ? 0 : (!energy_ok ? 1 : 2);
  if (!acc) {
    for (int q = r0; q < 3 * n; q += gs) pos_at(arr.xs, q) = arr.x0[q];
  }
  w.g.sync();
  if (w.g.leader() && acc) {
    s.cur = tr;
    s.E = En;
  }
  w.g.sync();
  return acc;
}

// float32 norm of a 3-vector from a float64 sum of squares.
__device__ __forceinline__ float norm3_f(const float* v) {
  double q = __dadd_rn(0.0, __dmul_rn((double)v[0], (double)v[0]));
  q = __dadd_rn(q, __dmul_rn((double)v[1], (double)v[1]));
  q = __dadd_rn(q, __dmul_rn((double)v[2], (double)v[2]));
  return __double2float_rn(__dsqrt_rn(q));
}

// shear (moves/shear.py:18-127): row a = randint(k1, 0, 3) moves by
// rv1 v1n + rv2 v2n within the plane of the other two rows, (rv1, rv2) =
// step * normal(k2, (2,)); T = solve(old, new) in float64.
template <class G>
__device__ __forceinline__ bool move_shear(const JrParams& P, Walker<G>& w, const StepKey& key, float step,
                                           double emax, float pressure, const float* mu,
                                           int& reason) {
  const Key k1 = key.k0, k2 = key.k1;
  const int a = randint(k1, 0, 3);
  const float rv1 = __fmul_rn(step, normal(bits32(k2, 0u)));
  const float rv2 = __fmul_rn(step, normal(bits32(k2, 1u)));
  const float* h = w.s.cc[w.s.cur].raw;
  const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
  const float* v1 = h + 3 * b;
  const float* v2 = h + 3 * c;
  float v1n[3], v2p[3], v2n[3];
  const float n1 = norm3_f(v1);
  for (int k = 0; k < 3; ++k) v1n[k] = __fdiv_rn(v1[k], n1);
  double dd = __dadd_rn(0.0, __dmul_rn((double)v2[0], (double)v1n[0]));
  dd = __dadd_rn(dd, __dmul_rn((double)v2[1], (double)v1n[1]));
  dd = __dadd_rn(dd, __dmul_rn((double)v2[2], (double)v1n[2]));
  const float dot = __double2float_rn(dd);
  for (int k = 0; k < 3; ++k) v2p[k] = __fmaf_rn(-dot, v1n[k], v2[k]);
  const float n2 = norm3_f(v2p);
  for (int k = 0; k < 3; ++k) v2n[k] = __fdiv_rn(v2p[k], n2);
  float nc[9];
  for (int q = 0; q < 9; ++q) nc[q] = h[q];
  for (int k = 0; k < 3; ++k)
    nc[3 * a + k] = __fmaf_rn(rv2, v2n[k], __fmaf_rn(rv1, v1n[k], h[3 * a + k]));
  double o[9], cof[9];
  for (int q = 0; q < 9; ++q) o[q] = (double)h[q];
  cof[0] = __dsub_rn(__dmul_rn(o[4], o[8]), __dmul_rn(o[5], o[7]));
  cof[1] = __dsub_rn(__dmul_rn(o[5], o[6]), __dmul_rn(o[3], o[8]));
  cof[2] = __dsub_rn(__dmul_rn(o[3], o[7]), __dmul_rn(o[4], o[6]));
  cof[3] = __dsub_rn(__dmul_rn(o[2], o[7]), __dmul_rn(o[1], o[8]));
  cof[4] = __dsub_rn(__dmul_rn(o[0], o[8]), __dmul_rn(o[2], o[6]));
  cof[5] = __dsub_rn(__dmul_rn(o[1], o[6]), __dmul_rn(o[0], o[7]));
  cof[6] = __dsub_rn(__dmul_rn(o[1], o[5]), __dmul_rn(o[2], o[4]));
  cof[7] = __dsub_rn(__dmul_rn(o[2], o[3]), __dmul_rn(o[0], o[5]));
  cof[8] = __dsub_rn(__dmul_rn(o[0], o[4]), __dmul_rn(o[1], o[3]));
  const double det = __dadd_rn(__dadd_rn(__dmul_rn(o[0], cof[0]), __dmul_rn(o[1], cof[1])),
                               __dmul_rn(o[2], cof[2]));
  float T[9];
  for (int k = 0; k < 3; ++k)
    for (int q = 0; q < 3; ++q) {
      double v = 0.0;
      for (int m = 0; m < 3; ++m)
        v = __dadd_rn(v, __dmul_rn(__ddiv_rn(cof[3 * m + k], det), (double)nc[3 * m + q]));
      T[3 * k + q] = __double2float_rn(v);
    }
  return move_cell(P, w, nc, T, emax, pressure, mu, reason);
}

// stretch (moves/stretch.py:18-104): axes (i, j) = [(0,1), (0,2), (1,2)]
// [randint(k1, 0, 3)], rv = step * normal(k2); T = diag with exp(rv) at i
// and exp(-rv) at j (float64 exp rounded to float32); cell . T, x . T.
template <class G>
__device__ __forceinline__ bool move_stretch(const JrParams& P, Walker<G>& w, const StepKey& key,
                                             float step, double emax, float pressure,
                                             const float* mu, int& reason) {
  const Key k1 = key.k0, k2 = key.k1;
  const int pr = randint(k1, 0, 3);
  const int ai = pr == 2 ? 1 : 0, aj = pr == 0 ? 1 : 2;
  const float rv = __fmul_rn(step, normal(bits32(k2, 0u)));
  float dg[3] = {1.0f, 1.0f, 1.0f};
  dg[ai] = __double2float_rn(exp((double)rv));
  dg[aj] = __double2float_rn(exp(-(double)rv));
  const float* h = w.s.cc[w.s.cur].raw;
  float T[9], nc[9];
  for (int q = 0; q < 9; ++q) T[q] = 0.0f;
  for (int k = 0; k < 3; ++k) T[4 * k] = dg[k];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) nc[3 * r + q] = __fmul_rn(h[3 * r + q], dg[q]);
  return move_cell(P, w, nc, T, emax, pressure, mu, reason);
}

// alchemical_morph (alchemical.py:40-79).
template <class G>
__device__ __forceinline__ bool move_morph(const JrParams& P, Walker<G>& w, const StepKey& key, double emax,
                           float pressure, const float* mu) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int atom = randint(key.k0, 0, w.n);
  const int curt = __float_as_int(arr.xs[atom].w);
  const int cand = randint(key.k1, 0, P.model.n_species - 1);
  const int nt = cand + (cand >= curt ? 1 : 0);
  w.g.sync();
  if (w.g.leader()) {
    arr.xs[atom].w = __int_as_float(nt);
    s.counts[curt] -= 1;
    s.counts[nt] += 1;
  }
  w.g.sync();
  double d0, d1;
  const double En = ham_eval<false>(P, w, s.cur, pressure, mu, d0, d1);
  const bool acc = En < emax;
  w.g.sync();
  if (w.g.leader()) {
    if (acc) {
      s.E = En;
    } else {
      arr.xs[atom].w = __int_as_float(curt);
      s.counts[curt] += 1;
      s.counts[nt] -= 1;
    }
  }
  w.g.sync();
  return acc;
}

// species_swap over all species (swap.py:177-260).
template <class G>
__device__ __forceinline__ bool move_swap(const JrParams& P, Walker<G>& w, const StepKey& key, double emax, float pressure,
                          const float* mu) {
  constexpr int kMaxPairs = JR_MAX_SPECIES * (JR_MAX_SPECIES - 1) / 2;
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int S = P.model.n_species;
  const Key kp = key.k0, klo = key.k1, khi = split(key.k, 2u);
  int counts[JR_MAX_SPECIES];
  for (int q = 0; q < S; ++q) counts[q] = s.counts[q];
  uint8_t plo[kMaxPairs], phi[kMaxPairs];
  float cum[kMaxPairs];
  int np = 0;
  float total = 0.0f;
  for (int a = 0; a < S; ++a)
    for (int b = a + 1; b < S; ++b) {
      plo[np] = (uint8_t)a;
      phi[np] = (uint8_t)b;
      total = __fadd_rn(total, (float)(counts[a] * counts[b]));
      cum[np] = total;
      ++np;
    }
  const bool has_pair = total > 0.0f;
  const float u = __fmul_rn(uniform01(bits32(kp, 0u)), has_pair ? total : 1.0f);
  int pidx = 0;
  while (pidx < np && cum[pidx] <= u) ++pidx;
  if (pidx > np - 1) pidx = np - 1;
  const int clo = plo[pidx], chi = phi[pidx];
  const int klo_i = randint(klo, 0, counts[clo] > 1 ? counts[clo] : 1);
  const int khi_i = randint(khi, 0, counts[chi] > 1 ? counts[chi] : 1);
  int ilo = n - 1, ihi = n - 1;
  {
    int run = 0;
    for (int i = 0; i < n; ++i) {
      run += (__float_as_int(arr.xs[i].w) == clo);
      if (run >= klo_i + 1) { ilo = i; break; }
    }
    run = 0;
    for (int i = 0; i < n; ++i) {
      run += (__float_as_int(arr.xs[i].w) == chi);
      if (run >= khi_i + 1) { ihi = i; break; }
    }
  }
  const int tlo = __float_as_int(arr.xs[ilo].w), thi = __float_as_int(arr.xs[ihi].w);
  w.g.sync();
  if (w.g.leader()) {
    arr.xs[ilo].w = __int_as_float(chi);
    arr.xs[ihi].w = __int_as_float(clo);
  }
  w.g.sync();
  double d0, d1;
  const double En = ham_eval<false>(P, w, s.cur, pressure, mu, d0, d1);
  const bool acc = (En < emax) && has_pair;
  w.g.sync();
  if (w.g.leader()) {
    if (acc) {
      s.E = En;
    } else {
      arr.xs[ilo].w = __int_as_float(tlo);
      arr.xs[ihi].w = __int_as_float(thi);
    }
  }
  w.g.sync();
  return acc;
}

}  // namespace jr

#include "jr_da.cuh"

namespace jr {

// One move of type P.moves.type[idx]; returns acceptance and reject reason.
// The surrogate family walks its galilean and volume moves by delayed
// acceptance.
template <class G>
__device__ __forceinline__ bool run_move(const JrParams& P, Walker<G>& w, int idx, const StepKey& key,
                                         float step, double emax, float pressure,
                                         const float* mu, int& reason) {
  reason = 0;
  if constexpr (G::kFam == kFamSWDA) {
    if (P.moves.type[idx] == JR_MOVE_GALILEAN)
      return da_galilean(P, w, key, step, P.moves.n_reflect[idx], P.moves.perturb_angle[idx],
                         emax, pressure, mu, reason);
    if (P.moves.type[idx] == JR_MOVE_VOLUME)
      return da_volume(P, w, key, step, emax, pressure, mu, reason);
  }
  switch (P.moves.type[idx]) {
    case JR_MOVE_GALILEAN:
      return move_galilean(P, w, key, step, P.moves.n_reflect[idx], P.moves.perturb_angle[idx],
                           emax, pressure, mu);
    case JR_MOVE_VOLUME:
      return move_volume(P, w, key, step, emax, pressure, mu, reason);
    case JR_MOVE_MORPH:
      return move_morph(P, w, key, emax, pressure, mu);
    case JR_MOVE_SWAP: {
      const bool a = move_swap(P, w, key, emax, pressure, mu);
      reason = a ? 0 : 1;
      return a;
    }
  }
  return false;
}

// Minimum-distance constraint (constraints/min_distance.py:25-47 with the
// MIC of backends/geometry.py:18-69): every pair i != j must be at least
// dmin[t_i][t_j] apart.  Periodic iff |det(cell)| > 1e-10: fractional
// coordinates f = x . inv(cell) (float32, FMA order of the pair MIC),
// df = f_i - f_j - rint(f_i - f_j), delta = df . cell; otherwise the raw
// difference; the distance is the correctly rounded sqrt of |delta|^2.
// Group-uniform result.
template <class G>
__device__ inline bool min_distance_ok(const JrParams& P, Walker<G>& w) {
  const CellCtx& cc = w.s.cc[w.s.cur];
  const bool periodic = cc.vol > 1e-10f;
  const float4* xs = w.arr.xs;
  const int n = w.n, S = P.model.n_species;
  double bad = 0.0;
  for (int q = w.g.rank(); q < n * n; q += w.g.size()) {
    const int i = q / n, j = q - i * n;
    if (j <= i) continue;
    const float4 a = xs[i], b = xs[j];
    const float thr = P.moves.dmin[__float_as_int(a.w) * S + __float_as_int(b.w)];
    float d[3];
    if (periodic) {
      float fa[3], fb[3];
      for (int k = 0; k < 3; ++k) {
        fa[k] = __fmaf_rn(a.z, cc.inv[6 + k], __fmaf_rn(a.y, cc.inv[3 + k], __fmul_rn(a.x, cc.inv[k])));
        fb[k] = __fmaf_rn(b.z, cc.inv[6 + k], __fmaf_rn(b.y, cc.inv[3 + k], __fmul_rn(b.x, cc.inv[k])));
      }
      float df[3];
      for (int k = 0; k < 3; ++k) {
        df[k] = __fsub_rn(fa[k], fb[k]);
        df[k] = __fsub_rn(df[k], rintf(df[k]));
      }
      for (int k = 0; k < 3; ++k)
        d[k] = __fmaf_rn(df[2], cc.raw[6 + k], __fmaf_rn(df[1], cc.raw[3 + k], __fmul_rn(df[0], cc.raw[k])));
    } else {
      d[0] = __fsub_rn(a.x, b.x);
      d[1] = __fsub_rn(a.y, b.y);
      d[2] = __fsub_rn(a.z, b.z);
    }
    const float r2 = __fmaf_rn(d[2], d[2], __fmaf_rn(d[1], d[1], __fmul_rn(d[0], d[0])));
    if (__fsqrt_rn(r2) < thr) bad = 1.0;
  }
  return group_sum1(w, bad) == 0.0;
}

// One move through the _wrap gate (mwg.py:108-150): a move that the
// minimum-distance constraint applies to (gate[idx], set by the host from the
// move's `mutates` and the constraint's `depends_on`) and that was accepted
// into a violating configuration is undone -- positions, cell, types and
// energy back to the pre-move state, the direction kept -- and reports
// reject reason 4.  kExt = false compiles the lean walk (galilean, volume,
// identity moves, no gate), which the host launches whenever no move is
// gated and no shear/stretch move is present: the extra code, inlined into
// the walk loop, was measured to slow every chain by about 9%.
template <bool kExt, class G>
__device__ __forceinline__ bool gated_move(const JrParams& P, Walker<G>& w, int idx, const StepKey& key,
                                           float step, double emax, float pressure,
                                           const float* mu, int& reason) {
  if constexpr (!kExt) {
    return run_move(P, w, idx, key, step, emax, pressure, mu, reason);
  } else {
    const int t = P.moves.type[idx];
    auto body = [&]() -> bool {
      reason = 0;
      if (t == JR_MOVE_SHEAR) return move_shear(P, w, key, step, emax, pressure, mu, reason);
      if (t == JR_MOVE_STRETCH) return move_stretch(P, w, key, step, emax, pressure, mu, reason);
      return run_move(P, w, idx, key, step, emax, pressure, mu, reason);
    };
    if (!P.moves.gate[idx]) return body();
    WalkShared& s = w.s;
    const int n = w.n;
    w.g.sync();
    for (int i = w.g.rank(); i < n; i += w.g.size()) w.arr.xsave[i] = w.arr.xs[i];
    if (w.g.leader()) {
      s.E_save = s.E;
      s.cur_save = s.cur;
      for (int q = 0; q < JR_MAX_SPECIES; ++q) s.counts_save[q] = s.counts[q];
    }
    w.g.sync();
    bool acc = body();
    w.g.sync();
    if (acc && !min_distance_ok(P, w)) {
      for (int i = w.g.rank(); i < n; i += w.g.size()) w.arr.xs[i] = w.arr.xsave[i];
      w.g.sync();
      if (w.g.leader()) {
        s.E = s.E_save;
        s.cur = s.cur_save;
        for (int q = 0; q < JR_MAX_SPECIES; ++q) s.counts[q] = s.counts_save[q];
      }
      w.g.sync();
      acc = false;
      reason = 4;
    }
    return acc;
  }
}

// MWG step (mwg.py:227-257 with the _wrap counters of mwg.py:108-150) plus
// the ns_step scan-body counters (nested_sampling.py:541-609).
template <bool kExt, class G>
__device__ __forceinline__ void mwg_step(const JrParams& P, Walker<G>& w, const StepKey& step_key, int idx,
                                         double emax, float pressure, const float* mu) {
  WalkShared& s = w.s;
  int reason = 0;
  if (G::kFam == kFamSWDA && w.g.leader()) {
    s.step_nev = 1;
    s.step_nsur = 0;
  }
  const bool acc = gated_move<kExt>(P, w, idx, step_key, s.step_sizes[idx], emax, pressure, mu,
                                   reason);
  if constexpr (G::kFam == kFamSWDA) {
    const int ty = P.moves.type[idx];
    if ((ty != JR_MOVE_GALILEAN && ty != JR_MOVE_VOLUME) || reason == 4) {
      // another move (or the constraint gate's undo) changed the walker: its
      // surrogate energy anew
      double d0, d1;
      const double ens = ensemble_term(s, s.cc[s.cur].vol, pressure, mu, P.model.n_species);
      const double Hs = sur_ham<false>(w, s.cur, ens, d0, d1);
      if (w.g.leader()) s.Esur = Hs;
    }
    if (w.g.leader()) {
      // the step's ring slot holds no exact evaluation
      if (w.ring_pos && ((ty != JR_MOVE_GALILEAN && ty != JR_MOVE_VOLUME) || s.step_nev == 0))
        w.ring_u[(w.ring_chain + w.ring_step) % w.ring_cap] = __longlong_as_double(
            0x7ff8000000000000ll);
      s.c_prop[idx] += 1;
      s.c_nsur[idx] += s.step_nsur;
      s.c_nev[idx] += s.step_nev;
      s.w_prop[idx] += 1;
      s.w_acc[idx] += acc ? 1 : 0;
      s.c_acc[idx] += acc ? 1 : 0;
      const int col = acc ? 0 : (reason > 1 ? reason : 1);
      if (col < 4) s.c_rr[idx * 4 + col] += 1;
    }
    return;
  }
  if (w.g.leader()) {
    s.w_prop[idx] += 1;
    s.w_acc[idx] += acc ? 1 : 0;
    s.c_prop[idx] += 1;
    s.c_acc[idx] += acc ? 1 : 0;
    // reason 4 (a constraint) lies outside the 4 buckets: the reference's
    // scatter drops it (nested_sampling.py:562-570)
    const int col = acc ? 0 : (reason > 1 ? reason : 1);
    if (col < 4) s.c_rr[idx * 4 + col] += 1;
    const bool gal = P.moves.type[idx] == JR_MOVE_GALILEAN;
    const int ne = gal ? P.moves.n_reflect[idx] : 1;
    s.c_nev[idx] += ne;
    s.c_ngr[idx] += gal ? ne : 0;
  }
}

// ------------------------------------------------------ load / store ----

__device__ inline void load_tables(const JrParams& P, PairTables& t) {
  const int SS = P.model.n_species * P.model.n_species;
  for (int q = threadIdx.x; q < SS; q += blockDim.x) {
    t.sig2[q] = P.model.sig2[q];
    t.eps4[q] = P.model.eps4[q];
    t.eps24[q] = P.model.eps24[q];
  }
}

// Load walker `slot` of replica p.  zero_counters: a fresh clone
// (nested_sampling.py:507-512).
template <class G>
__device__ __forceinline__ void load_walker(const JrParams& P, const JrDims& D, const JrStateBuffers& st,
                                   Walker<G>& w, int p, int slot, bool zero_counters) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const int K = D.n_walkers, Nmax = D.n_atoms_max, M = D.n_moves;
  const size_t wb = (size_t)p * K + slot;
  const float* gx = st.positions + wb * Nmax * 3;
  const float* gd = st.direction + wb * Nmax * 3;
  const int32_t* gt = st.types + wb * Nmax;
  w.g.sync();
  for (int q = r0; q < 3 * n; q += gs) {
    pos_at(arr.xs, q) = gx[q];
    arr.dir[q] = gd[q];
  }
  const int smax = P.model.n_species - 1;
  for (int i = r0; i < n; i += gs) {
    // out-of-range species clamp like a JAX gather index
    const int t = gt[i];
    arr.xs[i].w = __int_as_float(t < 0 ? 0 : (t > smax ? smax : t));
  }
  if (w.g.leader()) {
    for (int q = 0; q < JR_MAX_SPECIES; ++q) s.counts[q] = 0;
    s.E = st.energy64[wb];
    for (int m = 0; m < M; ++m) {
      s.step_sizes[m] = st.step_sizes[wb * M + m];
      s.w_acc[m] = zero_counters ? 0 : st.n_accepted[wb * M + m];
      s.w_prop[m] = zero_counters ? 0 : st.n_proposed[wb * M + m];
    }
    s.cur = 0;
    make_cell_ctx(st.cell + wb * 9, s.cc[0], arr.T, P.model);
  }
  w.g.sync();
  if (w.g.leader())
    for (int i = 0; i < n; ++i) s.counts[__float_as_int(arr.xs[i].w)] += 1;
  w.g.sync();
}

// Store the walker into `slot` of replica p.
template <class G>
__device__ __forceinline__ void store_walker(const JrDims& D, const JrStateBuffers& st, Walker<G>& w,
                                    int p, int slot) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const int n = w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const int K = D.n_walkers, Nmax = D.n_atoms_max, M = D.n_moves;
  const size_t wb = (size_t)p * K + slot;
  float* gx = st.positions + wb * Nmax * 3;
  float* gd = st.direction + wb * Nmax * 3;
  int32_t* gt = st.types + wb * Nmax;
  w.g.sync();
  for (int q = r0; q < 3 * n; q += gs) {
    gx[q] = pos_at(arr.xs, q);
    gd[q] = arr.dir[q];
  }
  for (int i = r0; i < n; i += gs) gt[i] = __float_as_int(arr.xs[i].w);
  if (w.g.leader()) {
    st.energy64[wb] = s.E;
    st.energy[wb] = __double2float_rn(s.E);
    for (int q = 0; q < 9; ++q) st.cell[wb * 9 + q] = s.cc[s.cur].raw[q];
    for (int m = 0; m < M; ++m) {
      st.step_sizes[wb * M + m] = s.step_sizes[m];
      st.n_accepted[wb * M + m] = s.w_acc[m];
      st.n_proposed[wb * M + m] = s.w_prop[m];
    }
  }
}

__device__ inline void zero_chain_counters(WalkShared& s) {
  for (int q = 0; q < 4; ++q) s.c_terms[q] = 0;
  for (int m = 0; m < JR_MAX_MOVES; ++m) {
    s.c_acc[m] = s.c_prop[m] = s.c_nev[m] = s.c_ngr[m] = s.c_nsur[m] = 0;
    s.c_rr[4 * m] = s.c_rr[4 * m + 1] = s.c_rr[4 * m + 2] = s.c_rr[4 * m + 3] = 0;
  }
}

}  // namespace jr
