// jr_da.cuh -- the delayed-acceptance walk of the Stillinger-Weber-with-
// surrogate family (included by jr_walk.cuh): the learned surrogate
// (jr_sur.cuh) evaluated inside the walk on the walker resident in shared
// memory, and the galilean and volume moves in two stages.
//
// Surrogate evaluation, one walker (n <= 64 atoms) on a 512-thread CTA, no
// pair list: 1. descriptors, eight threads per atom, each over every eighth
// other atom (minimum image, r^2 test, the 16 basis values by a two-exponential
// product recurrence), summed over the eight threads, standardised and
// rounded to bfloat16; 2.-3. the two hidden layers as warp-level tensor-core
// products (mma.sync m16n8k16, bfloat16 operands, float32 accumulation; warp
// w owns rows 16 (w / 4).. and columns 16 (w % 4)..; the four warps of a row
// tile meet at a named barrier), SiLU, the energy; 4. with forces only: the
// backward products down to dU/dD; 5. each atom's force from its neighbours
// (both sides of every pair evaluated, so no scatter), summed over its eight
// threads.

// Delayed acceptance (J. A. Christen and C. Fox, J. Comput. Graph. Stat. 14,
// 795 (2005)) with the smoothed surrogate constraint
//   s(x) = sigmoid((emax + contour_shift - H_sur(x)) / tau),
// H_sur = surrogate U + the exact ensemble term.  Galilean: the trajectory is
// walked on the surrogate (reflections off its contour at the inner points,
// forces only on reflecting steps; the final point does not reflect, which
// makes the trajectory its own reverse and the proposal symmetric); stage 1
// accepts with min(1, s(x') / s(x)), stage 2
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

// Barrier of the 4 warps (128 threads) that own row tile `grp` of the
// surrogate's products (named barriers 1..4; barrier 0 is the CTA's).
__device__ __forceinline__ void rows_sync(int grp) {
  asm volatile("bar.sync %0, 128;" ::"r"(grp + 1) : "memory");
}

// The 16 radial basis values g_k = exp(-(t - k)^2 / 2), t = (r - mu_0) / dmu,
// scaled by e^60, by a product recurrence from k = 0 (two exponentials per
// distance): g'_0 = exp(60 - t^2 / 2), g'_{k+1} = g'_k R_k with R_0 =
// exp(t - 1/2) and R_{k+1} = R_k / e.  The scale keeps every value a normal
// float for the distances inside the cutoff (t in [-9.8, 15]: g'_k between
// about e^-53 and e^60); callers fold e^-60 into the cutoff factor.
constexpr float kSurGScale = 8.75651076269652e-27f;  // e^-60

__device__ __forceinline__ void sur_gauss16(float t, float* g) {
  constexpr float kInvE = 0.36787944117144233f;
  float h = __expf(60.0f - 0.5f * t * t);
  float R = __expf(t - 0.5f);
  g[0] = h;
#pragma unroll
  for (int k = 1; k < 16; ++k) {
    h *= R;
    R *= kInvE;
    g[k] = h;
  }
}

// Sum v[0..15] over the 8 lanes sub = lane & 7 of an aligned group
// (reduce-scatter: 14 shuffles); lane sub ends with the totals of entries
// 2 sub and 2 sub + 1 in v[0], v[1].
__device__ __forceinline__ void sum16_over8(float* v, int sub) {
  const bool h4 = (sub & 4) != 0, h2 = (sub & 2) != 0, h1 = (sub & 1) != 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const float send = h4 ? v[q] : v[q + 8];
    const float keep = h4 ? v[q + 8] : v[q];
    v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float send = h2 ? v[q] : v[q + 4];
    const float keep = h2 ? v[q + 4] : v[q];
    v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float send = h1 ? v[q] : v[q + 2];
    const float keep = h1 ? v[q + 2] : v[q];
    v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
  }
}

// Surrogate potential U_sur of the walker (cell context from cc), and with
// kForces its forces into arr.F and the sums F.F, F.dir.  Group-uniform.
// Requires a 512-thread CTA: thread t serves atom t / 8 with the neighbours
// j = t mod 8, t mod 8 + 8, ..., and warp w the row tile w / 4 of the
// products; the four warps of a row tile meet at their own named barrier.
// Every sum runs in a fixed order (deterministic results).
template <bool kForces, bool kDiag, class G>
__device__ __forceinline__ void sur_eval(Walker<G>& w, const MicRegs& cc, double& U, double& sff,
                                         double& sfd) {
  const WalkArrays& arr = w.arr;
  const JrSurrogate& S = *w.sur;
  const int n = w.n;
  const int tid = w.g.rank();
  const int lane = tid & 31, warp = tid >> 5;
  const int grp = warp >> 2;
  const int ai = tid >> 3, sub = tid & 7;
  constexpr float kRc2 = kSurRc * kSurRc;
  constexpr float kInvDmu = 1.0f / kSurDmu;
  const float4 xi = arr.xs[ai < n ? ai : 0];
  // ---- 1. descriptors of atom ai over its neighbour share, then the sum
  // over the atom's 8 threads ----
  {
    float ds[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) ds[k] = 0.0f;
    if (ai < n) {
      for (int j = sub; j < n; j += 8) {
        const float4 xj = arr.xs[j];
        float dx = __fsub_rn(xj.x, xi.x), dy = __fsub_rn(xj.y, xi.y), dz = __fsub_rn(xj.z, xi.z);
        mic_r<kDiag>(cc, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (j != ai && r2 < kRc2 && r2 > 0.0f) {
          const float r = sqrtf(r2);
          float fc, dfc, g[16];
          sur_cutoff(r, fc, dfc);
          sur_gauss16((r - kSurMu0) * kInvDmu, g);
          fc *= kSurGScale;
#pragma unroll
          for (int k = 0; k < 16; ++k) ds[k] = fmaf(g[k], fc, ds[k]);
        }
      }
    }
    sum16_over8(ds, sub);
    const int k0 = 2 * sub;
    const float x0 = ai < n ? fmaf(ds[0], S.in_scale[k0], S.in_shift[k0]) : 0.0f;
    const float x1 = ai < n ? fmaf(ds[1], S.in_scale[k0 + 1], S.in_shift[k0 + 1]) : 0.0f;
    *reinterpret_cast<uint32_t*>(arr.sx + ai * kSurLdX + k0) = sur_pack_bf16(x0, x1);
  }
  rows_sync(grp);
  // ---- 2. first layer: warp w owns row tile grp, column tiles nt0, nt0+1 ----
  const int nt0 = 2 * (warp & 3);
  const int g8 = lane >> 2, cq = 2 * (lane & 3);
  const int row_a = 16 * grp + g8, row_b = row_a + 8;
  float ds1[8], g2[8];
  {
    uint32_t af[4], bf[2];
    frag_a(arr.sx, kSurLdX, 16 * grp, 0, lane, af);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      frag_b(arr.sw1t, kSurLdX, 8 * (nt0 + u), 0, lane, bf);
      mma_bf16(c, af, bf);
      const int col = 8 * (nt0 + u) + cq;
      const float z00 = c[0] + arr.sbias[col], z01 = c[1] + arr.sbias[col + 1];
      const float z10 = c[2] + arr.sbias[col], z11 = c[3] + arr.sbias[col + 1];
      if (kForces) {
        ds1[4 * u] = sur_dsilu(z00);
        ds1[4 * u + 1] = sur_dsilu(z01);
        ds1[4 * u + 2] = sur_dsilu(z10);
        ds1[4 * u + 3] = sur_dsilu(z11);
      }
      *reinterpret_cast<uint32_t*>(arr.sh1 + row_a * kSurLdH + col) =
          sur_pack_bf16(sur_silu(z00), sur_silu(z01));
      *reinterpret_cast<uint32_t*>(arr.sh1 + row_b * kSurLdH + col) =
          sur_pack_bf16(sur_silu(z10), sur_silu(z11));
    }
  }
  rows_sync(grp);
  // ---- 3. second layer and the per-row energies of this warp's columns ----
  double e_part = 0.0;
  {
    float c[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t af[4], bf[2];
      frag_a(arr.sh1, kSurLdH, 16 * grp, 16 * ks, lane, af);
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
      if (kForces) {
        g2[4 * u] = S.out_scale * w0 * sur_dsilu(z00);
        g2[4 * u + 1] = S.out_scale * w1 * sur_dsilu(z01);
        g2[4 * u + 2] = S.out_scale * w0 * sur_dsilu(z10);
        g2[4 * u + 3] = S.out_scale * w1 * sur_dsilu(z11);
      }
    }
    ea += __shfl_xor_sync(0xffffffffu, ea, 1);
    ea += __shfl_xor_sync(0xffffffffu, ea, 2);
    eb += __shfl_xor_sync(0xffffffffu, eb, 1);
    eb += __shfl_xor_sync(0xffffffffu, eb, 2);
    // U = out_scale sum_{rows < n} (h2 . w3) + n (b3 out_scale + out_shift)
    if ((lane & 3) == 0) e_part = (double)(row_a < n ? ea : 0.0f) + (double)(row_b < n ? eb : 0.0f);
    e_part *= (double)S.out_scale;
    if (tid == 0)
      e_part += (double)n * ((double)S.params[kSurOffB3] * (double)S.out_scale +
                             (double)S.out_shift);
  }
  if constexpr (!kForces) {
    w.g.sum1(e_part, 1, w.par);
    U = e_part;
    sff = 0.0;
    sfd = 0.0;
  } else {
    // ---- 4. backward: G2 -> G1 = (G2 W2^T) silu'(z1) -> dU/dx = G1 W1^T ----
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int col = 8 * (nt0 + u) + cq;
      *reinterpret_cast<uint32_t*>(arr.sg2 + row_a * kSurLdH + col) =
          sur_pack_bf16(g2[4 * u], g2[4 * u + 1]);
      *reinterpret_cast<uint32_t*>(arr.sg2 + row_b * kSurLdH + col) =
          sur_pack_bf16(g2[4 * u + 2], g2[4 * u + 3]);
    }
    rows_sync(grp);
    {
      float c[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        uint32_t af[4], bf[2];
        frag_a(arr.sg2, kSurLdH, 16 * grp, 16 * ks, lane, af);
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
    rows_sync(grp);
    if ((warp & 3) < 2) {  // dU/dD of the row tile: column tile warp & 1
      const int n2 = warp & 1;
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        uint32_t af[4], bf[2];
        frag_a(arr.sg1, kSurLdH, 16 * grp, 16 * ks, lane, af);
        frag_b(arr.sw1k, kSurLdH, 8 * n2, 16 * ks, lane, bf);
        mma_bf16(c, af, bf);
      }
      const int col = 8 * n2 + cq;
      arr.sdx[row_a * kSurLdG + col] = c[0] * S.in_scale[col];
      arr.sdx[row_a * kSurLdG + col + 1] = c[1] * S.in_scale[col + 1];
      arr.sdx[row_b * kSurLdG + col] = c[2] * S.in_scale[col];
      arr.sdx[row_b * kSurLdG + col + 1] = c[3] * S.in_scale[col + 1];
    }
    w.g.sync();
    // ---- 5. forces: F_i = sum_j c_ij (x_j - x_i), c_ij = sum_k (dU/dD_ik +
    // dU/dD_jk) dphi_k(r_ij) / r_ij, atom ai over its neighbour share, then
    // the sum over its 8 threads ----
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (ai < n) {
      float gi[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) gi[k] = arr.sdx[ai * kSurLdG + k];
      for (int j = sub; j < n; j += 8) {
        const float4 xj = arr.xs[j];
        float dx = __fsub_rn(xj.x, xi.x), dy = __fsub_rn(xj.y, xi.y), dz = __fsub_rn(xj.z, xi.z);
        mic_r<kDiag>(cc, dx, dy, dz);
        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (j != ai && r2 < kRc2 && r2 > 0.0f) {
          const float r = sqrtf(r2);
          const float t = (r - kSurMu0) * kInvDmu;
          float fc, dfc, g[16];
          sur_cutoff(r, fc, dfc);
          sur_gauss16(t, g);
          fc *= kSurGScale;
          dfc *= kSurGScale;
          float sk = 0.0f;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const float dphi = g[k] * fmaf(-fc * kInvDmu, t - (float)k, dfc);
            sk = fmaf(gi[k] + arr.sdx[j * kSurLdG + k], dphi, sk);
          }
          const float coef = sk / r;
          fx = fmaf(coef, dx, fx);
          fy = fmaf(coef, dy, fy);
          fz = fmaf(coef, dz, fz);
        }
      }
    }
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, off);
      fy += __shfl_xor_sync(0xffffffffu, fy, off);
      fz += __shfl_xor_sync(0xffffffffu, fz, off);
    }
    double ff_part = 0.0, fd_part = 0.0;
    if (sub == 0 && ai < n) {
      arr.F[3 * ai] = fx;
      arr.F[3 * ai + 1] = fy;
      arr.F[3 * ai + 2] = fz;
      const double dfx = fx, dfy = fy, dfz = fz;
      ff_part = dfx * dfx + dfy * dfy + dfz * dfz;
      fd_part = dfx * arr.dir[3 * ai] + dfy * arr.dir[3 * ai + 1] + dfz * arr.dir[3 * ai + 2];
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
    // reflections at the inner points only: the final point never reflects,
    // so the trajectory retraces itself from (x', -d') back to (x, -d) (the
    // proposal is symmetric, as delayed acceptance needs); the exact walk
    // gets this from its acceptance test, which the surrogate trajectory
    // does not make
    refl = r + 1 < R && Hs >= contour;
    if (refl) {
      sur_ham<true>(w, cidx, ens, sff, sfd);
      ++nsur;
      const float ffs = __double2float_rn(sff);
      coef = __fmul_rn(2.0f * __double2float_rn(sfd), rcp_nr(ffs > 1e-20f ? ffs : 1e-20f));
    }
  }
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
  const double jac = volume_jacobian(ratio, n, mv.flat_v_prior != 0);
  const bool valid = s.cell_ok != 0;
  const float u1 = key.pre ? key.vu : uniform01(bits32(key.k1, 0u));
  // u1 < min(1, J s(x') / s(x)) with J = ratio**N the prior ratio (the
  // first-stage acceptance of delayed acceptance, which the second stage's
  // min(1, s(x) / s(x')) assumes); a flat surrogate constraint leaves the
  // prior test of the exact move, u1 < min(1, J)
  const double r1 = jac * exp((double)ls1 - (double)ls0);
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
