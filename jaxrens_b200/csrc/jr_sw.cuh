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
//   1. pair pass over the n(n-1)/2 unordered pairs: minimum image, and for
//      pairs inside r_c the per-pair record (dr, 1/r, g, u = g'/(g r), the
//      two-body force coefficient c2 = phi2'/r) and the neighbour bits of
//      both atoms; two-body energies summed;
//   2. list pass (one warp): the neighbour pairs a < b in ascending (a, b)
//      order, and the pair and triplet counts of the evaluation;
//   3. triplet pass, one neighbour pair {a, b} per thread: V_ab = force on b
//      from the triplets centred on a (other leg k ascending), V_ba likewise,
//      and the triplet energies whose smaller leg is the pair's other atom
//      (each triplet once); Q_ab = c2 dr_ab + V_ba - V_ab is the whole
//      antisymmetric pair share of the force, F_i = sum_j Q_ij;
//   4. gather: F_i in the canonical order of the pair-matrix path (partners
//      in blocks of 8, ascending, then the xor tree over the blocks).
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

// Pair record of one pair inside the cutoff (float32, fixed op order):
// r = sqrt(r2), 1/r, 1/(rc - r), the two exponentials, phi2, c2 = phi2'/r
// and u = g'/(g r).  Returns false (nothing written) outside the cutoff.
__device__ __forceinline__ bool sw_pair_terms(const SwConsts& c, float r2, float& inv_r, float& g,
                                              float& u, float& c2, float& e2) {
  if (!(r2 < c.rc2)) return false;
  const float r = __fsqrt_rn(r2);
  if (!(r < c.rc)) return false;
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
  return true;
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
                                        float& vy, float& vz, double& e3) {
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
      if (k > j) e3 += (double)h;
    }
  }
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
  // ---- 1. pair pass ----
  for (int p = tid; p < np; p += gs) {
    const uint32_t ab = arr.pij[p];
    const int a = ab & 255, b = ab >> 8;
    const float4 xa = arr.xs[a], xb = arr.xs[b];
    float dx = __fsub_rn(xb.x, xa.x);
    float dy = __fsub_rn(xb.y, xa.y);
    float dz = __fsub_rn(xb.z, xa.z);
    mic_r<kDiag>(cc, dx, dy, dz);
    float r2 = __fmul_rn(dx, dx);
    r2 = __fmaf_rn(dy, dy, r2);
    r2 = __fmaf_rn(dz, dz, r2);
    float inv_r, g, u, c2, e2;
    if (sw_pair_terms(sc, r2, inv_r, g, u, c2, e2)) {
      arr.swr0[p] = make_float4(dx, dy, dz, inv_r);
      arr.swr1[p] = make_float4(g, u, c2, e2);
      atomicOr(reinterpret_cast<unsigned long long*>(nbm + a), 1ull << b);
      atomicOr(reinterpret_cast<unsigned long long*>(nbm + b), 1ull << a);
      ep += (double)e2;
    }
  }
  w.g.sync();
  // ---- 2. list pass: neighbour pairs in ascending (a, b) order (warp 0) ----
  if (tid < 32) {
    const int lane = tid;
    const int a0 = lane, a1 = lane + 32;
    const uint64_t m0 = a0 < n ? nbm[a0] : 0ull, m1 = a1 < n ? nbm[a1] : 0ull;
    // partners above each atom
    const uint64_t up0 = a0 >= 63 ? 0ull : (m0 >> (a0 + 1)) << (a0 + 1);
    const uint64_t up1 = a1 >= 63 ? 0ull : (m1 >> (a1 + 1)) << (a1 + 1);
    const int c0 = __popcll(up0), c1 = __popcll(up1);
    // exclusive scan of c0 over lanes, then of c1 after all c0
    int x0 = c0;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x0, off);
      if (lane >= off) x0 += y;
    }
    const int tot0 = __shfl_sync(0xffffffffu, x0, 31);
    int x1 = c1;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x1, off);
      if (lane >= off) x1 += y;
    }
    const int tot1 = __shfl_sync(0xffffffffu, x1, 31);
    int o0 = x0 - c0, o1 = tot0 + x1 - c1;
    for (uint64_t m = up0; m; m &= m - 1)
      arr.items[o0++] = (uint16_t)(a0 | ((__ffsll((long long)m) - 1) << 8));
    for (uint64_t m = up1; m; m &= m - 1)
      arr.items[o1++] = (uint16_t)(a1 | ((__ffsll((long long)m) - 1) << 8));
    // pair and triplet counts of this evaluation
    const int d0 = __popcll(m0), d1 = __popcll(m1);
    int pairs = d0 + d1;
    int trip = d0 * (d0 - 1) / 2 + d1 * (d1 - 1) / 2;
    for (int off = 16; off > 0; off >>= 1) {
      pairs += __shfl_xor_sync(0xffffffffu, pairs, off);
      trip += __shfl_xor_sync(0xffffffffu, trip, off);
    }
    if (lane == 0) {
      s.sw_nitems = tot0 + tot1;
      s.c_terms[kForces ? 0 : 2] += pairs / 2;
      s.c_terms[kForces ? 1 : 3] += trip;
    }
  }
  w.g.sync();
  // ---- 3. triplet pass ----
  const int nitems = s.sw_nitems;
  double e3 = 0.0;
  for (int q = tid; q < n; q += gs) nbm_next[q] = 0ull;  // the next evaluation's masks
  for (int q = tid; q < nitems; q += gs) {
    const uint32_t it = arr.items[q];
    const int a = it & 255, b = it >> 8;
    const int p = sw_pidx(a, b, n);
    const float4 ra = arr.swr0[p];
    const float4 rb = arr.swr1[p];
    float vabx = 0.0f, vaby = 0.0f, vabz = 0.0f;  // force on b, centre a
    float vbax = 0.0f, vbay = 0.0f, vbaz = 0.0f;  // force on a, centre b
    sw_side<kForces>(sc, arr.swr0, arr.swr1, nbm[a], a, b, n, ra.x, ra.y, ra.z, ra.w, rb.x, rb.y,
                     vabx, vaby, vabz, e3);
    sw_side<kForces>(sc, arr.swr0, arr.swr1, nbm[b], b, a, n, -ra.x, -ra.y, -ra.z, ra.w, rb.x,
                     rb.y, vbax, vbay, vbaz, e3);
    if (kForces) {
      // Q_ab = c2 dr_ab + V_ba - V_ab
      const float qx = __fsub_rn(__fmaf_rn(rb.z, ra.x, vbax), vabx);
      const float qy = __fsub_rn(__fmaf_rn(rb.z, ra.y, vbay), vaby);
      const float qz = __fsub_rn(__fmaf_rn(rb.z, ra.z, vbaz), vabz);
      arr.swq[p] = make_float4(qx, qy, qz, 0.0f);
    }
  }
  ep += e3;
  if (!kForces) {
    double z0 = 0.0, z1 = 0.0;
    w.g.sum3(ep, z0, z1, 1, w.par);
    U = ep;
    sff = 0.0;
    sfd = 0.0;
    return;
  }
  w.g.sync();
  // ---- 4. gather: F_i = sum_j Q_ij, partners in blocks of 8 ascending ----
  const int L = gather_lanes(n);
  const int apb = gs / L;
  const int blk = tid & (L - 1);
  for (int off = 1; off < L; off <<= 1) ep += __shfl_xor_sync(0xffffffffu, ep, off);
  double ff_part = 0.0, fd_part = 0.0;
  for (int base = 0; base < n; base += apb) {
    const int i = base + tid / L;
    if (!__any_sync(0xffffffffu, i < n)) continue;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    const int j0 = blk * 8;
    if (i < n && j0 < n) {
      uint64_t m = (nbm[i] >> j0) & 0xffull;
      while (m) {
        const int j = j0 + __ffsll((long long)m) - 1;
        m &= m - 1;
        const bool fwd = i < j;
        const float4 q = arr.swq[fwd ? sw_pidx(i, j, n) : sw_pidx(j, i, n)];
        fx = __fadd_rn(fx, fwd ? q.x : -q.x);
        fy = __fadd_rn(fy, fwd ? q.y : -q.y);
        fz = __fadd_rn(fz, fwd ? q.z : -q.z);
      }
    }
    gather_tree(fx, fy, fz, L);
    if (blk == 0 && i < n) {
      arr.F[3 * i] = fx;
      arr.F[3 * i + 1] = fy;
      arr.F[3 * i + 2] = fz;
      const double dx = fx, dy = fy, dz = fz;
      ff_part = __fma_rn(dx, dx, __fma_rn(dy, dy, __fma_rn(dz, dz, ff_part)));
      fd_part = __fma_rn(dx, (double)arr.dir[3 * i],
                         __fma_rn(dy, (double)arr.dir[3 * i + 1],
                                  __fma_rn(dz, (double)arr.dir[3 * i + 2], fd_part)));
    }
  }
  w.g.sum3(ep, ff_part, fd_part, L, w.par);
  U = ep;
  sff = ff_part;
  sfd = fd_part;
}

}  // namespace jr
