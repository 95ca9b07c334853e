// jr_da.cuh -- the delayed-acceptance walk of the Stillinger-Weber-with-
// surrogate family (included by jr_walk.cuh): the learned surrogate
// (jr_sur.cuh) evaluated inside the walk on the walker resident in shared
// memory, and the galilean and volume moves in two stages.
//
// Surrogate evaluation, one walker (n <= 64 atoms) on a 512-thread CTA:
//   1. pair scan within the descriptor cutoff (minimum image, r^2), compacted
//      in per-warp segments, with the neighbour masks; 2. per pair r and the
//      cosine cutoff; 3. descriptors, thread (atom i, basis pair k) summing
//      its neighbours in ascending order, standardised and rounded to
//      bfloat16; 4. the two hidden layers as warp-level tensor-core products
//      (mma.sync m16n8k16, bfloat16 operands, float32 accumulation; warp w
//      owns rows 16 (w / 4).. and columns 16 (w % 4)..), SiLU, per-row
//      energies; 5. with forces only: the backward products, dU/dD, the pair
//      force coefficients sum_k (dU/dD_ik + dU/dD_jk) dphi_k(r) / r and the
//      per-atom gather of the Stillinger-Weber path.
//
// Delayed acceptance (J. A. Christen and C. Fox, J. Comput. Graph. Stat. 14,
// 795 (2005)) with the smoothed surrogate constraint
//   s(x) = sigmoid((emax + contour_shift - H_sur(x)) / tau),
// H_sur = surrogate U + the exact ensemble term.  Galilean: the trajectory is
// walked on the surrogate (reflections off its contour, forces only on
// reflecting steps); stage 1 accepts with min(1, s(x') / s(x)), stage 2
// evaluates the exact energy and accepts with 1{E(x') < emax} min(1, s(x) /
// s(x')).  Volume: stage 1 with min(1, prior ratio s(x') / s(x)) and the exact
// cell checks, stage 2 as above.  The exact energy decides every step; the
// stored energy of every walker is exact.
#pragma once

#include "jr_sur.cuh"

namespace jr {

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment (16 x 16, row-major rows row0.., columns k0..) of a bfloat16
// tile with row stride ld; B fragment (16 x 8) of an n-major tile (rows are
// the n index, k contiguous) at n0, k0.
__device__ __forceinline__ void frag_a(const uint16_t* t, int ld, int row0, int k0, int lane,
                                       uint32_t* a) {
  const int g = lane >> 2, c = 2 * (lane & 3);
  a[0] = *reinterpret_cast<const uint32_t*>(t + (row0 + g) * ld + k0 + c);
  a[1] = *reinterpret_cast<const uint32_t*>(t + (row0 + g + 8) * ld + k0 + c);
  a[2] = *reinterpret_cast<const uint32_t*>(t + (row0 + g) * ld + k0 + c + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(t + (row0 + g + 8) * ld + k0 + c + 8);
}

__device__ __forceinline__ void frag_b(const uint16_t* t, int ld, int n0, int k0, int lane,
                                       uint32_t* b) {
  const int g = lane >> 2, c = 2 * (lane & 3);
  b[0] = *reinterpret_cast<const uint32_t*>(t + (n0 + g) * ld + k0 + c);
  b[1] = *reinterpret_cast<const uint32_t*>(t + (n0 + g) * ld + k0 + c + 8);
}

// Load the surrogate (bfloat16 operand tiles, float32 biases) into the
// walker's shared memory, CTA-wide.
__device__ inline void sur_load_weights(const JrSurrogate& S, const WalkArrays& a) {
  const float* P = S.params;
  for (int q = threadIdx.x; q < kSurBasis * kSurHidden; q += blockDim.x) {
    const int d = q / kSurHidden, h = q % kSurHidden;
    const uint16_t v = sur_bf16(P[kSurOffW1 + q]);
    a.sw1t[h * kSurLdX + d] = v;
    a.sw1k[d * kSurLdH + h] = v;
  }
  for (int q = threadIdx.x; q < kSurHidden * kSurHidden; q += blockDim.x) {
    const int i = q / kSurHidden, o = q % kSurHidden;
    const uint16_t v = sur_bf16(P[kSurOffW2 + q]);
    a.sw2t[o * kSurLdH + i] = v;
    a.sw2k[i * kSurLdH + o] = v;
  }
  for (int q = threadIdx.x; q < kSurHidden; q += blockDim.x) {
    a.sbias[q] = P[kSurOffB1 + q];
    a.sbias[64 + q] = P[kSurOffB2 + q];
    a.sbias[128 + q] = P[kSurOffW3 + q];
  }
}

// Surrogate potential U_sur of the walker (cell context from cc), and with
// kForces its forces into arr.F and the sums F.F, F.dir.  Group-uniform.
// Requires a 512-thread CTA group.
template <bool kForces, bool kDiag, class G>
__device__ __forceinline__ void sur_eval(Walker<G>& w, const MicRegs& cc, double& U, double& sff,
                                         double& sfd) {
  const WalkArrays& arr = w.arr;
  WalkShared& s = w.s;
  const JrSurrogate& S = *w.sur;
  const int n = w.n;
  const int np = n * (n - 1) / 2;
  const int tid = w.g.rank(), gs = w.g.size();
  const int lane = tid & 31, warp = tid >> 5, nwarps = gs >> 5;
  uint64_t* nbm = arr.nbm + (w.swpar & 1) * kSWMaxAtoms;
  uint64_t* nbm_next = arr.nbm + ((w.swpar + 1) & 1) * kSWMaxAtoms;
  w.swpar ^= 1;
  const float rc2 = kSurRc * kSurRc;
  const int per_warp = ((np + gs - 1) / gs) * 32;
  // ---- 1. scan: candidates within the cutoff, their (dr, r^2), masks ----
  {
    uint16_t* seg = arr.cand + warp * per_warp;
    int cw = 0;
    for (int p0 = warp * 32; p0 < np; p0 += gs) {
      const int p = p0 + lane;
      bool in = false;
      float dx = 0.0f, dy = 0.0f, dz = 0.0f, r2 = 0.0f;
      uint32_t ab = 0;
      if (p < np) {
        ab = arr.pij[p];
        const float4 xa = arr.xs[ab & 255], xb = arr.xs[ab >> 8];
        dx = __fsub_rn(xb.x, xa.x);
        dy = __fsub_rn(xb.y, xa.y);
        dz = __fsub_rn(xb.z, xa.z);
        mic_r<kDiag>(cc, dx, dy, dz);
        r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        in = r2 < rc2 && r2 > 0.0f;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, in);
      if (in) {
        seg[cw + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)p;
        arr.swr0[p] = make_float4(dx, dy, dz, r2);
        unsigned* m32 = reinterpret_cast<unsigned*>(nbm);
        const int a = ab & 255, b = ab >> 8;
        atomicOr(m32 + 2 * a + (b >> 5), 1u << (b & 31));
        atomicOr(m32 + 2 * b + (a >> 5), 1u << (a & 31));
      }
      cw += __popc(bal);
    }
    if (lane == 0) s.sw_cand[warp] = cw;
  }
  w.g.sync();
  int incl = lane < nwarps ? s.sw_cand[lane] : 0;
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  const int M = __shfl_sync(0xffffffffu, incl, nwarps - 1);
  // ---- 2. per pair: r, the cutoff and its derivative; the dense list ----
  uint16_t* dense = arr.cand + kSWCandDense;
  for (int base = tid - lane; base < M; base += gs) {
    const int q = base + lane;
    const int p = sw_cand_pair(arr.cand, per_warp, incl, nwarps, q < M ? q : M - 1);
    if (q < M) {
      dense[q] = (uint16_t)p;
      const float4 d = arr.swr0[p];
      const float r = sqrtf(d.w);
      float fc, dfc;
      sur_cutoff(r, fc, dfc);
      arr.swr0[p] = make_float4(d.x, d.y, d.z, r);
      arr.swr1[p] = make_float4(fc, dfc, 0.0f, 0.0f);
    }
  }
  w.g.sync();
  for (int q = tid; q < n; q += gs) nbm_next[q] = 0ull;  // the next evaluation's masks
  // ---- 3. descriptors: thread (atom i, basis pair kk), neighbours ascending ----
  for (int t = tid; t < 64 * 8; t += gs) {
    const int i = t >> 3, k0 = 2 * (t & 7);
    float d0 = 0.0f, d1 = 0.0f;
    if (i < n) {
      for (uint64_t m = nbm[i]; m; m &= m - 1) {
        const int j = __ffsll((long long)m) - 1;
        const int p = i < j ? sw_pidx(i, j, n) : sw_pidx(j, i, n);
        const float r = arr.swr0[p].w;
        const float4 c = arr.swr1[p];
        float phi, dphi;
        sur_basis(r, c.x, c.y, k0, phi, dphi);
        d0 += phi;
        sur_basis(r, c.x, c.y, k0 + 1, phi, dphi);
        d1 += phi;
      }
      d0 = d0 * S.in_scale[k0] + S.in_shift[k0];
      d1 = d1 * S.in_scale[k0 + 1] + S.in_shift[k0 + 1];
    }
    *reinterpret_cast<uint32_t*>(arr.sx + i * kSurLdX + k0) =
        i < n ? sur_pack_bf16(d0, d1) : 0u;
  }
  w.g.sync();
  // ---- 4. hidden layers: warp w owns row tile mt = w / 4 and the column
  // tiles nt0 = 2 (w % 4), nt0 + 1 ----
  const int mt = warp >> 2, nt0 = 2 * (warp & 3);
  const int g = lane >> 2, cq = 2 * (lane & 3);
  const int row_a = 16 * mt + g, row_b = row_a + 8;
  float ds1[8], g2[8];
  {
    uint32_t af[4], bf[2];
    frag_a(arr.sx, kSurLdX, 16 * mt, 0, lane, af);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      frag_b(arr.sw1t, kSurLdX, 8 * (nt0 + u), 0, lane, bf);
      mma_bf16(c, af, bf);
      const int col = 8 * (nt0 + u) + cq;
      const float z00 = c[0] + arr.sbias[col], z01 = c[1] + arr.sbias[col + 1];
      const float z10 = c[2] + arr.sbias[col], z11 = c[3] + arr.sbias[col + 1];
      ds1[4 * u] = sur_dsilu(z00);
      ds1[4 * u + 1] = sur_dsilu(z01);
      ds1[4 * u + 2] = sur_dsilu(z10);
      ds1[4 * u + 3] = sur_dsilu(z11);
      *reinterpret_cast<uint32_t*>(arr.sh1 + row_a * kSurLdH + col) =
          sur_pack_bf16(sur_silu(z00), sur_silu(z01));
      *reinterpret_cast<uint32_t*>(arr.sh1 + row_b * kSurLdH + col) =
          sur_pack_bf16(sur_silu(z10), sur_silu(z11));
    }
  }
  w.g.sync();
  {
    float c[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t af[4], bf[2];
      frag_a(arr.sh1, kSurLdH, 16 * mt, 16 * ks, lane, af);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        frag_b(arr.sw2t, kSurLdH, 8 * (nt0 + u), 16 * ks, lane, bf);
        mma_bf16(c[u], af, bf);
      }
    }
    float ea = 0.0f, eb = 0.0f;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int col = 8 * (nt0 + u) + cq;
      const float b0 = arr.sbias[64 + col], b1 = arr.sbias[64 + col + 1];
      const float w0 = arr.sbias[128 + col], w1 = arr.sbias[128 + col + 1];
      const float z00 = c[u][0] + b0, z01 = c[u][1] + b1, z10 = c[u][2] + b0, z11 = c[u][3] + b1;
      ea += sur_silu(z00) * w0 + sur_silu(z01) * w1;
      eb += sur_silu(z10) * w0 + sur_silu(z11) * w1;
      g2[4 * u] = S.out_scale * w0 * sur_dsilu(z00);
      g2[4 * u + 1] = S.out_scale * w1 * sur_dsilu(z01);
      g2[4 * u + 2] = S.out_scale * w0 * sur_dsilu(z10);
      g2[4 * u + 3] = S.out_scale * w1 * sur_dsilu(z11);
    }
    // the four lanes of a row hold its 16 columns of this warp
    ea += __shfl_xor_sync(0xffffffffu, ea, 1);
    ea += __shfl_xor_sync(0xffffffffu, ea, 2);
    eb += __shfl_xor_sync(0xffffffffu, eb, 1);
    eb += __shfl_xor_sync(0xffffffffu, eb, 2);
    if ((lane & 3) == 0) {
      arr.separt[(warp & 3) * 64 + row_a] = ea;
      arr.separt[(warp & 3) * 64 + row_b] = eb;
    }
  }
  w.g.sync();
  // ---- 5. energy: U = sum_i (e_i out_scale + out_shift), rows i < n ----
  double e_part = 0.0;
  if (tid < n) {
    const float e = ((arr.separt[tid] + arr.separt[64 + tid]) +
                     (arr.separt[128 + tid] + arr.separt[192 + tid])) +
                    S.params[kSurOffB3];
    e_part = (double)e * (double)S.out_scale + (double)S.out_shift;
  }
  if constexpr (!kForces) {
    double z0 = 0.0, z1 = 0.0;
    w.g.sum3(e_part, z0, z1, 1, w.par);
    U = e_part;
    sff = 0.0;
    sfd = 0.0;
  } else {
    // ---- 6. backward: G2 -> G1 = (G2 W2^T) silu'(z1) -> dU/dx = G1 W1^T ----
  #pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int col = 8 * (nt0 + u) + cq;
      *reinterpret_cast<uint32_t*>(arr.sg2 + row_a * kSurLdH + col) =
          sur_pack_bf16(g2[4 * u], g2[4 * u + 1]);
      *reinterpret_cast<uint32_t*>(arr.sg2 + row_b * kSurLdH + col) =
          sur_pack_bf16(g2[4 * u + 2], g2[4 * u + 3]);
    }
    w.g.sync();
    {
      float c[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
  #pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        uint32_t af[4], bf[2];
        frag_a(arr.sg2, kSurLdH, 16 * mt, 16 * ks, lane, af);
  #pragma unroll
        for (int u = 0; u < 2; ++u) {
          frag_b(arr.sw2k, kSurLdH, 8 * (nt0 + u), 16 * ks, lane, bf);
          mma_bf16(c[u], af, bf);
        }
      }
  #pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int col = 8 * (nt0 + u) + cq;
        *reinterpret_cast<uint32_t*>(arr.sg1 + row_a * kSurLdH + col) =
            sur_pack_bf16(c[u][0] * ds1[4 * u], c[u][1] * ds1[4 * u + 1]);
        *reinterpret_cast<uint32_t*>(arr.sg1 + row_b * kSurLdH + col) =
            sur_pack_bf16(c[u][2] * ds1[4 * u + 2], c[u][3] * ds1[4 * u + 3]);
      }
    }
    w.g.sync();
    if (warp < 8) {  // dU/dx [64][16]: row tile warp / 2, column tile warp % 2
      const int m2 = warp >> 1, n2 = warp & 1;
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  #pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        uint32_t af[4], bf[2];
        frag_a(arr.sg1, kSurLdH, 16 * m2, 16 * ks, lane, af);
        frag_b(arr.sw1k, kSurLdH, 8 * n2, 16 * ks, lane, bf);
        mma_bf16(c, af, bf);
      }
      const int col = 8 * n2 + cq, ra = 16 * m2 + g;
      arr.sdx[ra * 16 + col] = c[0] * S.in_scale[col];          // dU/dD
      arr.sdx[ra * 16 + col + 1] = c[1] * S.in_scale[col + 1];
      arr.sdx[(ra + 8) * 16 + col] = c[2] * S.in_scale[col];
      arr.sdx[(ra + 8) * 16 + col + 1] = c[3] * S.in_scale[col + 1];
    }
    w.g.sync();
    // ---- 7. pair forces: Q_ab = [sum_k (gD_ak + gD_bk) dphi_k(r) / r] dr_ab ----
    for (int q = tid; q < M; q += gs) {
      const int p = dense[q];
      const uint32_t ab = arr.pij[p];
      const int a = ab & 255, b = ab >> 8;
      const float4 d = arr.swr0[p];
      const float4 cf = arr.swr1[p];
      float sk = 0.0f;
  #pragma unroll
      for (int k = 0; k < kSurBasis; ++k) {
        float phi, dphi;
        sur_basis(d.w, cf.x, cf.y, k, phi, dphi);
        sk += (arr.sdx[a * 16 + k] + arr.sdx[b * 16 + k]) * dphi;
      }
      const float coef = sk / d.w;
      arr.swq[p] = make_float4(coef * d.x, coef * d.y, coef * d.z, 0.0f);
    }
    w.g.sync();
    // ---- 8. gather, one lane per atom, neighbours ascending ----
    double ff_part = 0.0, fd_part = 0.0;
    for (int i = tid; i < n; i += gs) {
      float fx = 0.0f, fy = 0.0f, fz = 0.0f;
      for (uint64_t m = nbm[i]; m; m &= m - 1) {
        const int j = __ffsll((long long)m) - 1;
        const bool fwd = i < j;
        const float4 q = arr.swq[fwd ? sw_pidx(i, j, n) : sw_pidx(j, i, n)];
        fx += fwd ? q.x : -q.x;
        fy += fwd ? q.y : -q.y;
        fz += fwd ? q.z : -q.z;
      }
      arr.F[3 * i] = fx;
      arr.F[3 * i + 1] = fy;
      arr.F[3 * i + 2] = fz;
      const double dx = fx, dy = fy, dz = fz;
      ff_part += dx * dx + dy * dy + dz * dz;
      fd_part += dx * arr.dir[3 * i] + dy * arr.dir[3 * i + 1] + dz * arr.dir[3 * i + 2];
    }
    w.g.sum3(e_part, ff_part, fd_part, 1, w.par);
    U = e_part;
    sff = ff_part;
    sfd = fd_part;
  }
}

// Surrogate potential (with the ensemble term) of the walker for cell
// context cidx.
template <bool kForces, class G>
__device__ __forceinline__ double sur_ham(Walker<G>& w, int cidx, double ens, double& sff,
                                          double& sfd) {
  const CellCtx& ccs = w.s.cc[cidx];
  double U;
  if (ccs.diag) sur_eval<kForces, true>(w, load_mic<true>(ccs), U, sff, sfd);
  else sur_eval<kForces, false>(w, load_mic<false>(ccs), U, sff, sfd);
  return U + ens;
}

// log s(H) = -softplus((H - contour) / tau)
__device__ __forceinline__ float sur_log_s(double H, double contour, float tau) {
  const float z = (float)((H - contour) / (double)tau);
  if (isnan(z)) return -INFINITY;
  return -(fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z))));
}

// Store the walker's positions, the cell of context cidx and the model
// energy U in the sample ring slot of this step (group-wide; no-op when the
// walk is not recording).
template <class G>
__device__ __forceinline__ void ring_put(Walker<G>& w, int cidx, double U) {
  if (w.ring_pos == nullptr) return;
  const long long slot = (w.ring_chain + w.ring_step) % w.ring_cap;
  float* dst = w.ring_pos + slot * (long long)w.ring_nmax * 3;
  for (int q = w.g.rank(); q < 3 * w.n; q += w.g.size()) dst[q] = pos_at(w.arr.xs, q);
  if (w.g.leader()) {
    for (int q = 0; q < 9; ++q) w.ring_cell[slot * 9 + q] = w.s.cc[cidx].raw[q];
    w.ring_u[slot] = U;
  }
}

// Galilean move by delayed acceptance: the direction as in move_galilean,
// the trajectory on the surrogate, stage 1 on the smoothed surrogate
// constraint, stage 2 on the exact energy.
template <class G>
__device__ __forceinline__ bool da_galilean(const JrParams& P, Walker<G>& w, const StepKey& key,
                                            float step, int R, float pa, double emax,
                                            float pressure, const float* mu, int& reason) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const JrSurrogate& S = *w.sur;
  const int n3 = 3 * w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const Key ki = key.k0, kp = key.k1;
  double sq = 0.0, sv = 0.0, zero = 0.0;
  for (int q = r0; q < n3; q += gs) {
    const float d = arr.dir[q];
    const float gz = key.nz ? key.nz[q] : normal(bits32(kp, (uint32_t)q));
    const float v = __fmaf_rn(pa, gz, d);
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
  const int cidx = s.cur;
  const double ens = ensemble_term(s, s.cc[cidx].vol, pressure, mu, P.model.n_species);
  const double contour = emax + (double)S.contour_shift;
  const double Hs0 = s.Esur;
  double Hs = Hs0;
  bool refl = false;
  float coef = 0.0f;
  int nsur = 0;
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
    double sff = 0.0, sfd = 0.0;
    Hs = sur_ham<false>(w, cidx, ens, sff, sfd);
    ++nsur;
    if (isnan(Hs)) Hs = INFINITY;
    refl = Hs >= contour;
    if (refl) {
      sur_ham<true>(w, cidx, ens, sff, sfd);
      ++nsur;
      const float ffs = __double2float_rn(sff);
      coef = __fmul_rn(2.0f * __double2float_rn(sfd), rcp_nr(ffs > 1e-20f ? ffs : 1e-20f));
    }
  }
  if (refl)
    for (int q = r0; q < n3; q += gs) arr.dir[q] = __fmaf_rn(-coef, arr.F[q], arr.dir[q]);
  const float ls1 = sur_log_s(Hs, contour, S.tau), ls0 = sur_log_s(Hs0, contour, S.tau);
  const float u1 = uniform01(bits32(split(key.k, 3u), 0u));
  const bool stage1 = logf(u1) < fminf(0.0f, ls1 - ls0);
  bool acc = false;
  double E = s.E;
  int nev = 0;
  reason = 3;
  if (stage1) {
    double d0, d1;
    E = ham_eval<false>(P, w, cidx, pressure, mu, d0, d1);
    nev = 1;
    ring_put(w, cidx, E - ens);
    const float u2 = uniform01(bits32(split(key.k, 4u), 0u));
    const bool energy_ok = E < emax;
    acc = energy_ok && logf(u2) < fminf(0.0f, ls0 - ls1);
    reason = acc ? 0 : (energy_ok ? 3 : 1);
  }
  if (!acc) {
    for (int q = r0; q < n3; q += gs) {
      pos_at(arr.xs, q) = arr.x0[q];
      arr.dir[q] = -arr.dp[q];
    }
  }
  if (w.g.leader()) {
    if (acc) {
      s.E = E;
      s.Esur = Hs;
    }
    s.step_nev = nev;
    s.step_nsur = nsur;
  }
  w.g.sync();
  return acc;
}

// Volume move by delayed acceptance: the proposal and the cell checks of
// move_volume; stage 1 with min(1, prior ratio s(x') / s(x)) on the
// surrogate, stage 2 on the exact energy.
template <class G>
__device__ __forceinline__ bool da_volume(const JrParams& P, Walker<G>& w, const StepKey& key,
                                          float step, double emax, float pressure,
                                          const float* mu, int& reason) {
  WalkShared& s = w.s;
  const WalkArrays& arr = w.arr;
  const JrSurrogate& S = *w.sur;
  const int n = w.n;
  const int r0 = w.g.rank(), gs = w.g.size();
  const JrMoveParams& mv = P.moves;
  const int cur = s.cur, tr = cur ^ 1;
  const float* h = s.cc[cur].raw;
  const float oldV = s.cc[cur].vol;
  const float sn = __fmul_rn(step, (float)n);
  const float dV = __fmul_rn(sn, key.pre ? key.vn : normal(bits32(key.k0, 0u)));
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
  const int helper = gs > 32 ? 32 : 1;
  if (w.g.leader()) make_cell_ctx(nc, s.cc[tr], arr.T + tr * 3 * P.model.n_images, P.model);
  else if (r0 == helper % gs) s.cell_ok = cell_valid(nc, n, mv) ? 1 : 0;
  w.g.sync();
  const double ens1 = ensemble_term(s, s.cc[tr].vol, pressure, mu, P.model.n_species);
  const double contour = emax + (double)S.contour_shift;
  double d0, d1;
  const double Hs1 = sur_ham<false>(w, tr, ens1, d0, d1);
  const double Hs0 = s.Esur;
  const float ls1 = sur_log_s(Hs1, contour, S.tau), ls0 = sur_log_s(Hs0, contour, S.tau);
  // log of min(1, ratio^N) (flat prior: 0)
  const double pa = volume_prior(ratio, n, mv.flat_v_prior != 0);
  const bool valid = s.cell_ok != 0;
  const float u1 = key.pre ? key.vu : uniform01(bits32(key.k1, 0u));
  // u1 < min(1, pa s(x') / s(x)); a flat surrogate constraint leaves the
  // prior test of the exact move
  const double r1 = pa * exp((double)ls1 - (double)ls0);
  const bool stage1 = valid && (double)u1 < (r1 < 1.0 ? r1 : 1.0);
  bool acc = false;
  double En = s.E;
  int nev = 0;
  reason = valid ? 3 : 2;
  if (stage1) {
    En = ham_eval<false>(P, w, tr, pressure, mu, d0, d1);
    nev = 1;
    ring_put(w, tr, En - ens1);
    const float u2 = uniform01(bits32(split(key.k, 4u), 0u));
    const bool energy_ok = En < emax;
    acc = energy_ok && logf(u2) < fminf(0.0f, ls0 - ls1);
    reason = acc ? 0 : (energy_ok ? 3 : 1);
  }
  if (!acc)
    for (int q = r0; q < n3; q += gs) pos_at(arr.xs, q) = arr.x0[q];
  if (w.g.leader()) {
    if (acc) {
      s.cur = tr;
      s.E = En;
      s.Esur = Hs1;
    }
    s.step_nev = nev;
    s.step_nsur = 1;
  }
  w.g.sync();
  return acc;
}

}  // namespace jr
