// jr_rng.cuh -- JAX threefry2x32 streams on the device.
//
// Restates the PRNG the reference draws from (jax.random with
// jax_threefry_partitionable=True, the default of the pinned jax>=0.9):
// threefry2x32-20 (Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC'11), split/fold_in as hash(key, (0, i)), 32-bit random_bits
// as y0 ^ y1, and the float transforms of jax.random.uniform / normal /
// randint / choice.  Every float operation uses an explicit round-to-nearest
// intrinsic so that the stream is independent of FMA contraction.
#pragma once
#include <cstdint>

namespace jr {

struct Key {
  uint32_t k0, k1;
};

__host__ __device__ __forceinline__ uint32_t rotl(uint32_t x, int r) {
#ifdef __CUDA_ARCH__
  return __funnelshift_l(x, x, r);
#else
  return (x << r) | (x >> (32 - r));
#endif
}

// threefry2x32 with 20 rounds; rotation constants and key-injection schedule
// of the Random123 specification.
__host__ __device__ __forceinline__ void threefry(Key k, uint32_t c0, uint32_t c1,
                                                  uint32_t& o0, uint32_t& o1) {
  const uint32_t ks2 = 0x1BD11BDAu ^ k.k0 ^ k.k1;
  uint32_t x0 = c0 + k.k0;
  uint32_t x1 = c1 + k.k1;
#define JR_TF_ROUND(r) \
  x0 += x1;            \
  x1 = rotl(x1, r);    \
  x1 ^= x0;
  JR_TF_ROUND(13) JR_TF_ROUND(15) JR_TF_ROUND(26) JR_TF_ROUND(6)
  x0 += k.k1; x1 += ks2 + 1u;
  JR_TF_ROUND(17) JR_TF_ROUND(29) JR_TF_ROUND(16) JR_TF_ROUND(24)
  x0 += ks2; x1 += k.k0 + 2u;
  JR_TF_ROUND(13) JR_TF_ROUND(15) JR_TF_ROUND(26) JR_TF_ROUND(6)
  x0 += k.k0; x1 += k.k1 + 3u;
  JR_TF_ROUND(17) JR_TF_ROUND(29) JR_TF_ROUND(16) JR_TF_ROUND(24)
  x0 += k.k1; x1 += ks2 + 4u;
  JR_TF_ROUND(13) JR_TF_ROUND(15) JR_TF_ROUND(26) JR_TF_ROUND(6)
  x0 += ks2; x1 += k.k0 + 5u;
#undef JR_TF_ROUND
  o0 = x0;
  o1 = x1;
}

// jax.random.split(key, n)[i]  ==  jax.random.fold_in(key, i)
__host__ __device__ __forceinline__ Key split(Key k, uint32_t i) {
  Key o;
  threefry(k, 0u, i, o.k0, o.k1);
  return o;
}

// random_bits(key, 32, shape) at row-major flat index i (shapes < 2^32).
__host__ __device__ __forceinline__ uint32_t bits32(Key k, uint32_t i) {
  uint32_t a, b;
  threefry(k, 0u, i, a, b);
  return a ^ b;
}

// One NS-iteration key advance of ns_step (nested_sampling.py:465-466):
// key, _ = split(key); key, ... = split(key, 5)  ->  new key.
__host__ __device__ __forceinline__ Key advance_iteration(Key k) {
  return split(split(k, 0u), 0u);
}

#ifdef __CUDACC__
__device__ __forceinline__ float unit_from_bits(uint32_t bits) {
  return __fsub_rn(__uint_as_float((bits >> 9) | 0x3F800000u), 1.0f);
}

// jax.random.uniform(key, minval=lo, maxval=hi) element from its 32 bits.
__device__ __forceinline__ float uniform(uint32_t bits, float lo, float hi) {
  float f = unit_from_bits(bits);
  float r = __fadd_rn(__fmul_rn(f, __fsub_rn(hi, lo)), lo);
  return r > lo ? r : lo;
}

__device__ __forceinline__ float uniform01(uint32_t bits) {
  return uniform(bits, 0.0f, 1.0f);
}

// Single-precision inverse error function of M. Giles, "Approximating the
// erfinv function" (GPU Computing Gems Jade, 2011) -- the approximation
// XLA lowers jax.lax.erf_inv to for float32 -- with the log1p term taken in
// double and rounded once.
__device__ __forceinline__ float erfinv_giles(float x) {
  float xx = __fmul_rn(x, x);
  float w = -__double2float_rn(log1p((double)(-xx)));
  float p;
  if (w < 5.0f) {
    w = __fsub_rn(w, 2.5f);
    p = 2.81022636e-08f;
    p = __fadd_rn(3.43273939e-07f, __fmul_rn(p, w));
    p = __fadd_rn(-3.5233877e-06f, __fmul_rn(p, w));
    p = __fadd_rn(-4.39150654e-06f, __fmul_rn(p, w));
    p = __fadd_rn(0.00021858087f, __fmul_rn(p, w));
    p = __fadd_rn(-0.00125372503f, __fmul_rn(p, w));
    p = __fadd_rn(-0.00417768164f, __fmul_rn(p, w));
    p = __fadd_rn(0.246640727f, __fmul_rn(p, w));
    p = __fadd_rn(1.50140941f, __fmul_rn(p, w));
  } else {
    w = __fsub_rn(__fsqrt_rn(w), 3.0f);
    p = -0.000200214257f;
    p = __fadd_rn(0.000100950558f, __fmul_rn(p, w));
    p = __fadd_rn(0.00134934322f, __fmul_rn(p, w));
    p = __fadd_rn(-0.00367342844f, __fmul_rn(p, w));
    p = __fadd_rn(0.00573950773f, __fmul_rn(p, w));
    p = __fadd_rn(-0.0076224613f, __fmul_rn(p, w));
    p = __fadd_rn(0.00943887047f, __fmul_rn(p, w));
    p = __fadd_rn(1.00167406f, __fmul_rn(p, w));
    p = __fadd_rn(2.83297682f, __fmul_rn(p, w));
  }
  if (fabsf(x) == 1.0f) return __fmul_rn(x, 3.40282347e38f);
  return __fmul_rn(p, x);
}

// jax.random.normal element: sqrt(2) * erf_inv(uniform(lo=nextafter(-1,0), 1)).
__device__ __forceinline__ float normal(uint32_t bits) {
  const float lo = -0.99999994f;  // nextafter(-1, 0) in float32
  float u = uniform(bits, lo, 1.0f);
  return __fmul_rn(1.41421354f, erfinv_giles(u));
}

// jax.random.randint(key, (), lo, hi) for int32.
__device__ __forceinline__ int32_t randint(Key k, int32_t lo, int32_t hi) {
  uint32_t higher = bits32(split(k, 0u), 0u);
  uint32_t lower = bits32(split(k, 1u), 0u);
  uint32_t span = hi > lo ? (uint32_t)(hi - lo) : 1u;
  uint32_t mult = 65536u % span;
  mult = (mult * mult) % span;
  uint32_t off = (higher % span) * mult + (lower % span);
  off = off % span;
  return lo + (int32_t)off;
}

// jax.random.choice(key, m, p) with replacement: searchsorted(cum, cum[-1]*(1-u)).
__device__ __forceinline__ int choice(Key k, const float* cum, int m) {
  float u = unit_from_bits(bits32(k, 0u));
  float r = __fmul_rn(cum[m - 1], __fsub_rn(1.0f, u));
  int idx = 0;
  while (idx < m && cum[idx] < r) ++idx;
  return idx;
}
#endif

}  // namespace jr
