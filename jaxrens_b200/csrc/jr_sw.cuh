// jr_sw.cuh -- Stillinger-Weber energy and forces of one walker resident in
// shared memory (included by jr_walk.cuh).
//
// Model (F. H. Stillinger and T. A. Weber, Phys. Rev. B 31, 5262 (1985)),
// one species, exponents p = 4 and q = 0:
//   E = sum_{i<j} phi2(r_ij) + sum_i sum_{j<k in nb(i)} h(i; j, k)
//   phi2(r)   = A eps (B (sigma/r)^4 - 1) exp(sigma / (r - a sigma))
//   h(i;j,k)  = lambda eps (cos theta_jik + 1/3)^2 g(r_ij) g(r_ik),
//   g(r)      = exp(gamma sigma / (r - a sigma)),
// every term zero beyond r_c = a sigma.  Periodic cells use the single
// minimum image of the LJ path (dr - rint(dr . inv) . h).
//
// Evaluation, one walker, one thread group:
//   1. pair pass over the n(n-1)/2 unordered pairs: a cheap scan (minimum
//      image, r^2 < rc2) sets the neighbour bits of both atoms and compacts
//      the pairs inside the cutoff into per-warp segments, then every thread
//      takes a share of those for the per-pair record (dr, 1/r, g,
//      u = g'/(g r), the two-body force coefficient c2 = phi2'/r); two-body
//      energies summed;
//   2. triplet pass, the two centre sides of each neighbour pair {a, b} on
//      two adjacent lanes: V_ab = force on b from the triplets centred on a
//      (other leg k ascending) on one lane, V_ba likewise on the other, and
//      the triplet energies whose smaller leg is the pair's other atom (each
//      triplet once); Q_ab = c2 dr_ab + V_ba - V_ab is the whole
//      antisymmetric pair share of the force, F_i = sum_j Q_ij;
//   3. gather, one lane per atom: F_i = sum of +-Q_ij over the neighbours j
//      of i in ascending order, sequentially in float32.
// Every float32 operation is an explicit IEEE intrinsic; the CPU oracle's
// DEV mode restates the same sequence, so forces match it bit for bit.  The
// float64 energy sum of float32 terms is order-dependent here (terms near
// the cutoff are tiny), so energies match the oracle to rounding of the sum.
#pragma once

namespace jr {

// exp(x) in float32, written for this project (used for the SW radial
// factors, x <= 0): Cody-Waite argument reduction x = k ln2 + r with k =
// rint(x log2(e)) and ln2 split into LN2_HI (float32 ln2 with its 12 low
// mantissa bits cleared, so k * LN2_HI is exact for |k| < 2^12) plus LN2_LO =
// float32(ln2 - LN2_HI); then the degree-7 Taylor polynomial of e^r (the
// coefficients are 1/n! rounded to float32) in Horner form with fused
// multiply-adds, |r| <= ln2/2 where the truncation error is 5e-9 relative;
// scaled by 2^k through the exponent bits, in two steps below the normal
// range.  Each step is one IEEE operation, so the result is the same on any
// machine with an FMA.  Tested against double-precision exp (<= 2 ulp).
__device__ __forceinline__ float sw_exp(float x) {
  if (!(x > -104.0f)) return 0.0f;          // below the smallest denormal (and NaN)
  if (x > 88.5f) return __int_as_float(0x7f800000);
  const float k = rintf(__fmul_rn(x, 0x1.715476p+0f));
  float r = __fmaf_rn(-k, 0x1.62ep-1f, x);
  r = __fmaf_rn(-k, 0x1.0bfbe8p-15f, r);
  float p = 0x1.a01a02p-13f;                // 1/7!
  p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);     // 1/6!
  p = __fmaf_rn(p, r, 0x1.111112p-7f);      // 1/5!
  p = __fmaf_rn(p, r, 0x1.555556p-5f);      // 1/4!
  p = __fmaf_rn(p, r, 0x1.555556p-3f);      // 1/3!
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  const int ki = (int)k;
  if (ki >= -126) return __fmul_rn(p, __int_as_float((ki + 127) << 23));
  // 2^k = 2^(k + 64) * 2^-64 for the denormal results
  return __fmul_rn(__fmul_rn(p, __int_as_float((ki + 64 + 127) << 23)), 0x1p-64f);
}

// Float32 constants of the model, in registers.
struct SwConsts {
  float rc, rc2, sig, gsig, Aeps, B, leps;
};

__device__ __forceinline__ SwConsts sw_consts(const JrModelParams& mp) {
  return SwConsts{mp.sw_rc, mp.rc2, mp.sw_sigma, mp.sw_gsig, mp.sw_Aeps, mp.sw_B, mp.sw_leps};
}

// Index of the unordered pair (lo, hi), lo < hi, in the row-major upper
// triangle of n atoms.
__device__ __forceinline__ int sw_pidx(int lo, int hi, int n) {
  return lo * (2 * n - lo - 1) / 2 + (hi - lo - 1);
}

// Pair record of one pair inside the cutoff, r2 < rc2 (float32, fixed op
// order): r = sqrt(r2), 1/r, 1/(rc - r), the two exponentials, phi2, c2 =
// phi2'/r and u = g'/(g r).  The host sets rc2 to the largest float32 whose
// correctly rounded square root lies below rc, so r < rc holds here.
__device__ __forceinline__ void sw_pair_terms(const SwConsts& c, float r2, float& inv_r, float& g,
                                              float& u, float& c2, float& e2) {
  // r2 < rc2, and rc2 is chosen by the host so that then r < rc
  const float r = __fsqrt_rn(r2);
  inv_r = rcp_nr(r);
  const float md = __fsub_rn(c.rc, r);          // rc - r > 0
  const float inv_md = rcp_nr(md);
  const float ex = sw_exp(-__fmul_rn(c.sig, inv_md));
  g = sw_exp(-__fmul_rn(c.gsig, inv_md));
  const float s = __fmul_rn(c.sig, inv_r);
  const float s2 = __fmul_rn(s, s);
  const float s4 = __fmul_rn(s2, s2);
  const float bq = __fmaf_rn(c.B, s4, -1.0f);   // B s^4 - 1
  const float aex = __fmul_rn(c.Aeps, ex);
  e2 = __fmul_rn(aex, bq);
  // phi2'(r) = A eps ex [-4 B s^4 / r - (B s^4 - 1) sigma / (r - rc)^2]
  const float w = __fmul_rn(__fmul_rn(c.sig, inv_md), inv_md);
  const float t1 = __fmul_rn(__fmul_rn(-4.0f, __fmul_rn(c.B, s4)), inv_r);
  const float dphi = __fmul_rn(aex, __fmaf_rn(-bq, w, t1));
  c2 = __fmul_rn(dphi, inv_r);
  // g'/g = -gamma sigma / (r - rc)^2
  u = __fmul_rn(-__fmul_rn(__fmul_rn(c.gsig, inv_md), inv_md), inv_r);
}

// One triplet seen from leg j of centre c (other leg k): the force on j
// subtracted from (vx, vy, vz); the triplet energy h returned.
//   cos = (dr_cj . dr_ck) / (r_j r_k), t = cos + 1/3, G = lambda eps g_j g_k,
//   F_j = -[tG (t u_j - 2 cos / r_j^2)] dr_cj - [2 tG / (r_j r_k)] dr_ck.
template <bool kForces>
__device__ __forceinline__ float sw_triplet(float leps, float jx, float jy, float jz, float ij,
                                            float gj, float uj, float kx, float ky, float kz,
                                            float ik, float gk, float& vx, float& vy, float& vz) {
  const float dot = __fmaf_rn(jz, kz, __fmaf_rn(jy, ky, __fmul_rn(jx, kx)));
  const float cs = __fmul_rn(__fmul_rn(dot, ij), ik);
  const float t = __fadd_rn(cs, 0x1.555556p-2f);
  const float G = __fmul_rn(__fmul_rn(leps, gj), gk);
  const float tG = __fmul_rn(t, G);
  if (kForces) {
    const float ij2 = __fmul_rn(ij, ij);
    const float p2 = __fmul_rn(__fmul_rn(2.0f, cs), ij2);
    const float A = __fmul_rn(tG, __fmaf_rn(t, uj, -p2));
    const float Bc = __fmul_rn(__fmul_rn(2.0f, tG), __fmul_rn(ij, ik));
    vx = __fsub_rn(vx, __fmaf_rn(A, jx, __fmul_rn(Bc, kx)));
    vy = __fsub_rn(vy, __fmaf_rn(A, jy, __fmul_rn(Bc, ky)));
    vz = __fsub_rn(vz, __fmaf_rn(A, jz, __fmul_rn(Bc, kz)));
  }
  return __fmul_rn(tG, t);
}

// The centre-c side of neighbour pair (c, j): V = force on j from every
// triplet (c; j, k), k over nb(c) \ {j} ascending; adds to e3 the energies
// of the triplets with k > j.  (jx, jy, jz) = dr_cj.
template <bool kForces>
__device__ __forceinline__ void sw_side(const SwConsts& sc, const float4* r0, const float4* r1,
                                        uint64_t mask, int c, int j, int n, float jx, float jy,
                                        float jz, float ij, float gj, float uj, float& vx,
                                        float& vy, float& vz, double& e3, int& ntrip) {
  mask &= ~(1ull << j);
  while (mask) {
    const int k = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    const bool fwd = c < k;
    const int pk = fwd ? sw_pidx(c, k, n) : sw_pidx(k, c, n);
    const float4 a = r0[pk];
    const float4 b = r1[pk];
    const float kx = fwd ? a.x : -a.x, ky = fwd ? a.y : -a.y, kz = fwd ? a.z : -a.z;
    if (kForces || k > j) {
      const float h = sw_triplet<kForces>(sc.leps, jx, jy, jz, ij, gj, uj, kx, ky, kz, a.w, b.x,
                                          vx, vy, vz);
      if (k > j) {
        e3 += (double)h;
        ++ntrip;
      }
    }
  }
}

// Neighbour bits of the pair (a, b) this lane scanned, if inside the cutoff
// (native 32-bit shared atomics on the two halves of each 64-bit mask).
__device__ __forceinline__ void sw_mask_bits(uint64_t* nbm, bool in, int a, int b) {
  if (!in) return;
  unsigned* m32 = reinterpret_cast<unsigned*>(nbm);
  atomicOr(m32 + 2 * a + (b >> 5), 1u << (b & 31));
  atomicOr(m32 + 2 * b + (a >> 5), 1u << (a & 31));
}

// Candidate q of the per-warp segments: `incl` is this lane's inclusive
// prefix of the segment counts (lane l < nwarps holds warps 0..l), so the
// segment of q is the number of lanes whose prefix is <= q.
__device__ __forceinline__ int sw_cand_pair(const uint16_t* cand, int per_warp, int incl,
                                            int nwarps, int q) {
  // the first warp whose inclusive count exceeds q (counts ascend; the last
  // is M > q), by a binary search of fixed depth so every lane takes part in
  // every shuffle
  int lo = 0, hi = nwarps - 1;
#pragma unroll
  for (int it = 0; it < 5; ++it) {
    const int mid = (lo + hi) >> 1;
    const int v = __shfl_sync(0xffffffffu, incl, mid);
    if (lo < hi) {
      if (v > q) hi = mid;
      else lo = mid + 1;
    }
  }
  const int below = __shfl_sync(0xffffffffu, incl, lo > 0 ? lo - 1 : 0);
  const int base = lo > 0 ? below : 0;
  return cand[lo * per_warp + (q - base)];
}

// Energy (U) of the walker, forces into arr.F when kForces, and the sums
// F.F and F.dir.  Group-uniform results.
template <bool kForces, bool kDiag, class G>
__device__ __forceinline__ void sw_eval(const JrParams& P, Walker<G>& w, const MicRegs& cc,
                                        double& U, double& sff, double& sfd) {
  const WalkArrays& arr = w.arr;
  WalkShared& s = w.s;
  const int n = w.n;
  const int np = n * (n - 1) / 2;
  const int tid = w.g.rank(), gs = w.g.size();
  const SwConsts sc = sw_consts(P.model);
  uint64_t* nbm = arr.nbm + (w.swpar & 1) * kSWMaxAtoms;
  uint64_t* nbm_next = arr.nbm + ((w.swpar + 1) & 1) * kSWMaxAtoms;
  w.swpar ^= 1;
  double ep = 0.0;
  const int lane = tid & 31, warp = tid >> 5, nwarps = gs >> 5;
  const int per_warp = ((np + gs - 1) / gs) * 32;  // pairs one warp scans, at most
  // ---- 1a. scan of every pair, two per trip with the loads of both issued
  // first: minimum image and r^2.  The pairs inside the cutoff are appended
  // to their warp's segment of the candidate list in scan order (so the list
  // does not depend on timing), with (dr, r^2) in their record.
  {
    uint16_t* seg = arr.cand + warp * per_warp;
    int cw = 0;
    for (int p0 = warp * 32; p0 < np; p0 += 2 * gs) {
      const int pa = p0 + lane, pb = p0 + gs + lane;
      const bool va = pa < np, vb = pb < np;
      const uint32_t aba = va ? arr.pij[pa] : 0u;
      const uint32_t abb = vb ? arr.pij[pb] : 0u;
      const float4 x0 = arr.xs[aba & 255], x1 = arr.xs[aba >> 8];
      const float4 y0 = arr.xs[abb & 255], y1 = arr.xs[abb >> 8];
      float ax = __fsub_rn(x1.x, x0.x), ay = __fsub_rn(x1.y, x0.y), az = __fsub_rn(x1.z, x0.z);
      float bx = __fsub_rn(y1.x, y0.x), by = __fsub_rn(y1.y, y0.y), bz = __fsub_rn(y1.z, y0.z);
      mic_r<kDiag>(cc, ax, ay, az);
      mic_r<kDiag>(cc, bx, by, bz);
      float ra2 = __fmul_rn(ax, ax);
      ra2 = __fmaf_rn(ay, ay, ra2);
      ra2 = __fmaf_rn(az, az, ra2);
      float rb2 = __fmul_rn(bx, bx);
      rb2 = __fmaf_rn(by, by, rb2);
      rb2 = __fmaf_rn(bz, bz, rb2);
      const bool ina = va && ra2 < sc.rc2, inb = vb && rb2 < sc.rc2;
      const unsigned bala = __ballot_sync(0xffffffffu, ina);
      const unsigned balb = __ballot_sync(0xffffffffu, inb);
      const unsigned lt = (1u << lane) - 1u;
      if (ina) {
        seg[cw + __popc(bala & lt)] = (uint16_t)pa;
        arr.swr0[pa] = make_float4(ax, ay, az, ra2);
      }
      cw += __popc(bala);
      if (inb) {
        seg[cw + __popc(balb & lt)] = (uint16_t)pb;
        arr.swr0[pb] = make_float4(bx, by, bz, rb2);
      }
      cw += __popc(balb);
      sw_mask_bits(nbm, ina, aba & 255, aba >> 8);
      sw_mask_bits(nbm, inb, abb & 255, abb >> 8);
    }
    if (lane == 0) s.sw_cand[warp] = cw;
  }
  w.g.sync();
  // prefix of the segment counts, in every warp (lane l: warps 0..l)
  int incl = lane < nwarps ? s.sw_cand[lane] : 0;
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  const int M = __shfl_sync(0xffffffffu, incl, nwarps - 1);
  // ---- 1b. pair records of the candidates, spread over every thread: r,
  // 1/r, the exponentials, phi2, the force coefficients; neighbour bits.
  uint16_t* dense = arr.cand + kSWCandDense;
  for (int base = tid - lane; base < M; base += gs) {
    const int q = base + lane;
    const int p = sw_cand_pair(arr.cand, per_warp, incl, nwarps, q < M ? q : M - 1);
    if (q < M) {
      dense[q] = (uint16_t)p;
      const float4 d = arr.swr0[p];
      float inv_r, g, u, c2, e2;
      sw_pair_terms(sc, d.w, inv_r, g, u, c2, e2);
      arr.swr0[p] = make_float4(d.x, d.y, d.z, inv_r);
      arr.swr1[p] = make_float4(g, u, c2, e2);
      ep += (double)e2;
      w.tc[kForces ? 0 : 2] += 1;
    }
  }
  w.g.sync();
  // ---- 2. triplet pass: the two centre sides of neighbour pair q on
  // adjacent lanes (2q: centre a, 2q + 1: centre b), joined by one shuffle ----
  for (int q = tid; q < n; q += gs) nbm_next[q] = 0ull;  // the next evaluation's masks
  double e3 = 0.0;
  int ntrip = 0;
  for (int base = tid - lane; base < 2 * M; base += gs) {
    const int u = base + lane;
    const bool act = u < 2 * M;
    const int side = u & 1;
    const int p = act ? dense[u >> 1] : 0;
    const uint32_t ab = arr.pij[p];
    const int a = ab & 255, b = ab >> 8;
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    float4 ra = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float c2 = 0.0f;
    if (act) {
      ra = arr.swr0[p];
      const float4 rb = arr.swr1[p];
      c2 = rb.z;
      // side 0: V_ab, force on b from the triplets centred on a; side 1:
      // V_ba, force on a from those centred on b (dr_ba = -dr_ab)
      const float sg = side ? -1.0f : 1.0f;
      sw_side<kForces>(sc, arr.swr0, arr.swr1, nbm[side ? b : a], side ? b : a, side ? a : b, n,
                       sg * ra.x, sg * ra.y, sg * ra.z, ra.w, rb.x, rb.y, vx, vy, vz, e3, ntrip);
    }
    if (kForces) {
      const float ox = __shfl_xor_sync(0xffffffffu, vx, 1);
      const float oy = __shfl_xor_sync(0xffffffffu, vy, 1);
      const float oz = __shfl_xor_sync(0xffffffffu, vz, 1);
      if (act && side == 0) {
        // Q_ab = c2 dr_ab + V_ba - V_ab
        const float qx = __fsub_rn(__fmaf_rn(c2, ra.x, ox), vx);
        const float qy = __fsub_rn(__fmaf_rn(c2, ra.y, oy), vy);
        const float qz = __fsub_rn(__fmaf_rn(c2, ra.z, oz), vz);
        arr.swq[p] = make_float4(qx, qy, qz, 0.0f);
      }
    }
  }
  w.tc[kForces ? 1 : 3] += ntrip;
  ep += e3;
  if (!kForces) {
    w.g.sum1(ep, 1, w.par);
    U = ep;
    sff = 0.0;
    sfd = 0.0;
    return;
  }
  w.g.sync();
  // ---- 3. gather, one lane per atom: F_i = sum over the neighbours j of i
  // in ascending order of +-Q, a sequential float32 sum from +0 ----
  double ff_part = 0.0, fd_part = 0.0;
  for (int i = tid; i < n; i += gs) {
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (uint64_t m = nbm[i]; m; m &= m - 1) {
      const int j = __ffsll((long long)m) - 1;
      const bool fwd = i < j;
      const float4 q = arr.swq[fwd ? sw_pidx(i, j, n) : sw_pidx(j, i, n)];
      fx = __fadd_rn(fx, fwd ? q.x : -q.x);
      fy = __fadd_rn(fy, fwd ? q.y : -q.y);
      fz = __fadd_rn(fz, fwd ? q.z : -q.z);
    }
    arr.F[3 * i] = fx;
    arr.F[3 * i + 1] = fy;
    arr.F[3 * i + 2] = fz;
    const double dx = fx, dy = fy, dz = fz;
    ff_part = __fma_rn(dx, dx, __fma_rn(dy, dy, __fma_rn(dz, dz, ff_part)));
    fd_part = __fma_rn(dx, (double)arr.dir[3 * i],
                       __fma_rn(dy, (double)arr.dir[3 * i + 1],
                                __fma_rn(dz, (double)arr.dir[3 * i + 2], fd_part)));
  }
  w.g.sum3(ep, ff_part, fd_part, 1, w.par);
  U = ep;
  sff = ff_part;
  sfd = fd_part;
}

}  // namespace jr
