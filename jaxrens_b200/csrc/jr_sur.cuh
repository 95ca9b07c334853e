// jr_sur.cuh -- the learned surrogate energy: radial descriptors and the
// 16-64-64-1 SiLU network, shared by the training kernels (jr_sur.cu) and the
// delayed-acceptance walk.
//
// Descriptor of atom i (one species, single minimum image):
//   D[i][k] = sum_{j != i, r_ij < rc} exp(-eta (r_ij - mu_k)^2) fc(r_ij),
//   fc(r) = (cos(pi r / rc) + 1) / 2, mu_k = 1.5 + k (3.8 - 1.5) / 15 A
//   (k = 0..15), eta = 1 / (2 dmu^2), rc = 3.8 A.
// Network: x = D in_scale + in_shift, h1 = silu(x W1 + b1),
//   h2 = silu(h1 W2 + b2), e = h2 . w3 + b3, U = sum_i (e_i out_scale +
//   out_shift); the matrix products in bfloat16 with float32 accumulation.
// No counterpart in the reference: a learned part the walk adds to screen
// proposals, the exact potential deciding every step.
#pragma once
#include <cstdint>

#include "../../include/jaxrens_b200.h"

namespace jr {

constexpr int kSurBasis = 16;
constexpr int kSurHidden = 64;
constexpr float kSurRc = 3.8f;
constexpr float kSurMu0 = 1.5f;
constexpr float kSurDmu = (3.8f - 1.5f) / 15.0f;
constexpr float kSurEta = 1.0f / (2.0f * kSurDmu * kSurDmu);
constexpr float kSurPi = 3.14159265358979f;

// Offsets of the float32 parameters in the flat layout [W1 16x64][b1 64]
// [W2 64x64][b2 64][w3 64][b3 1] (gradients and Adam moments use it too).
constexpr int kSurOffW1 = 0;
constexpr int kSurOffB1 = kSurOffW1 + kSurBasis * kSurHidden;
constexpr int kSurOffW2 = kSurOffB1 + kSurHidden;
constexpr int kSurOffB2 = kSurOffW2 + kSurHidden * kSurHidden;
constexpr int kSurOffW3 = kSurOffB2 + kSurHidden;
constexpr int kSurOffB3 = kSurOffW3 + kSurHidden;
constexpr int kSurParams = kSurOffB3 + 1;
static_assert(kSurParams == JR_SUR_PARAMS, "flat parameter layout");

// SiLU and its derivative with the approximate exponential and division
// (a few ulp; the network's products round to bfloat16 anyway).
__device__ __forceinline__ float sur_silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

__device__ __forceinline__ float sur_dsilu(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Cosine cutoff and its derivative, r < rc.
__device__ __forceinline__ void sur_cutoff(float r, float& fc, float& dfc) {
  float sn, cs;
  __sincosf(kSurPi * r / kSurRc, &sn, &cs);
  fc = 0.5f * (cs + 1.0f);
  dfc = -0.5f * (kSurPi / kSurRc) * sn;
}

// Basis k at distance r (times the cutoff) and its r-derivative.
__device__ __forceinline__ void sur_basis(float r, float fc, float dfc, int k, float& phi,
                                          float& dphi) {
  const float d = r - (kSurMu0 + (float)k * kSurDmu);
  const float g = __expf(-kSurEta * d * d);
  phi = g * fc;
  dphi = g * (dfc - 2.0f * kSurEta * d * fc);
}

// bfloat16 bits of x, round to nearest even (NaN kept quiet).
__device__ __forceinline__ uint16_t sur_bf16(float x) {
  const uint32_t u = __float_as_uint(x);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
  return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

__device__ __forceinline__ uint32_t sur_pack_bf16(float lo, float hi) {
  return (uint32_t)sur_bf16(lo) | ((uint32_t)sur_bf16(hi) << 16);
}

}  // namespace jr
