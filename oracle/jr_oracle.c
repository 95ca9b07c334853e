/*
 * jr_oracle.c -- CPU oracle for jaxrens's nested-sampling walk.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, the smoke check and bench.py's CPU
 * baseline leg are the only callers; the product library never links it.
 * See jr_oracle.h for the precision modes.  Every function cites the
 * reference file:line it restates (paths relative to the jaxrens tree).
 *
 * Build with -ffp-contract=off: the FP32 arithmetic here must be exactly
 * the sequence of IEEE operations written, with fmaf() only where an FMA is
 * part of the kernel contract.
 */
#include "jr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ------------------------------------------------------------------ */
/* threefry2x32-20 (Salmon et al., SC'11; Random123 threefry.h).       */
/* JAX: jax._src.prng.threefry2x32 (dependency jax>=0.9, not vendored). */
/* ------------------------------------------------------------------ */
static inline uint32_t rotl32(uint32_t x, int r) {
  return (x << r) | (x >> (32 - r));
}

void jro_threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                      uint32_t out[2]) {
  static const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
  const uint32_t ks[3] = {k0, k1, 0x1BD11BDAu ^ k0 ^ k1};
  uint32_t x0 = c0 + ks[0];
  uint32_t x1 = c1 + ks[1];
  for (int r = 0; r < 20; ++r) {
    x0 += x1;
    x1 = rotl32(x1, rot[r & 7]);
    x1 ^= x0;
    if ((r & 3) == 3) {
      const uint32_t s = (uint32_t)((r >> 2) + 1);
      x0 += ks[s % 3];
      x1 += ks[(s + 1) % 3] + s;
    }
  }
  out[0] = x0;
  out[1] = x1;
}

/* split(key, n)[index] with jax_threefry_partitionable=True: the counter of
 * element i of shape (n,) is the 64-bit iota value i split as (hi, lo). */
void jro_split(const uint32_t key[2], uint32_t index, uint32_t out[2]) {
  jro_threefry2x32(key[0], key[1], 0u, index, out);
}

/* fold_in(key, d) = threefry_2x32(key, threefry_seed(d)) = hash(key,(0,d)). */
void jro_fold_in(const uint32_t key[2], uint32_t data, uint32_t out[2]) {
  jro_threefry2x32(key[0], key[1], 0u, data, out);
}

/* The pre-0.5 (non-partitionable) split: counts = iota(2n) hashed as the
 * pairs (i, n+i); output words laid out [y0..., y1...] then reshaped (n,2).
 * Kept only to pin the cipher against JAX's documented split(key(0)). */
void jro_split_original(const uint32_t key[2], int32_t n, uint32_t* out) {
  uint32_t* flat = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)n);
  for (int32_t i = 0; i < n; ++i) {
    uint32_t y[2];
    jro_threefry2x32(key[0], key[1], (uint32_t)i, (uint32_t)(n + i), y);
    flat[i] = y[0];
    flat[n + i] = y[1];
  }
  memcpy(out, flat, sizeof(uint32_t) * 2 * (size_t)n);
  free(flat);
}

/* random_bits(key, 32, shape)[flat] (partitionable): bits1 ^ bits2. */
uint32_t jro_bits32(const uint32_t key[2], uint32_t flat_index) {
  uint32_t y[2];
  jro_threefry2x32(key[0], key[1], 0u, flat_index, y);
  return y[0] ^ y[1];
}

static inline float bits_to_unit(uint32_t bits) {
  uint32_t b = (bits >> 9) | 0x3F800000u;
  float f;
  memcpy(&f, &b, 4);
  return f - 1.0f;
}

/* jax.random.uniform (jax._src.random._uniform): mantissa fill, then
 * floats * (maxval - minval) + minval, then max(minval, .). */
float jro_uniform(uint32_t bits, float lo, float hi) {
  float f = bits_to_unit(bits);
  float span = hi - lo;
  float r = f * span;
  r = r + lo;
  return r > lo ? r : lo;
}

/* XLA's float32 ErfInv: M. Giles, "Approximating the erfinv function",
 * GPU Computing Gems Jade Edition (2011), single-precision branch with the
 * polynomial evaluated as p = c_i + p*w (separate multiply and add).
 * log1p is evaluated in double and rounded once, the same contract the
 * kernels use, so CPU and GPU agree except at float rounding ties. */
float jro_erfinv(float x) {
  static const float lt5[9] = {2.81022636e-08f,  3.43273939e-07f,
                               -3.5233877e-06f,  -4.39150654e-06f,
                               0.00021858087f,   -0.00125372503f,
                               -0.00417768164f,  0.246640727f,
                               1.50140941f};
  static const float ge5[9] = {-0.000200214257f, 0.000100950558f,
                               0.00134934322f,   -0.00367342844f,
                               0.00573950773f,   -0.0076224613f,
                               0.00943887047f,   1.00167406f,
                               2.83297682f};
  float xx = x * x;
  float w = -(float)log1p((double)(-xx));
  float p;
  if (w < 5.0f) {
    w = w - 2.5f;
    p = lt5[0];
    for (int i = 1; i < 9; ++i) {
      float pw = p * w;
      p = lt5[i] + pw;
    }
  } else {
    w = sqrtf(w) - 3.0f;
    p = ge5[0];
    for (int i = 1; i < 9; ++i) {
      float pw = p * w;
      p = ge5[i] + pw;
    }
  }
  if (fabsf(x) == 1.0f) return x * FLT_MAX;
  return p * x;
}

/* jax.random.normal (jax._src.random._normal_real):
 * sqrt(2) * erf_inv(uniform(key, lo=nextafter(-1, 0), hi=1)). */
float jro_normal(uint32_t bits) {
  const float lo = nextafterf(-1.0f, 0.0f);
  float u = jro_uniform(bits, lo, 1.0f);
  return 1.41421354f * jro_erfinv(u);
}

/* jax.random.randint, int32, scalar shape (jax._src.random._randint). */
int32_t jro_randint(const uint32_t key[2], int32_t lo, int32_t hi) {
  uint32_t k1[2], k2[2];
  jro_split(key, 0, k1);
  jro_split(key, 1, k2);
  uint32_t higher = jro_bits32(k1, 0);
  uint32_t lower = jro_bits32(k2, 0);
  uint32_t span = (uint32_t)(hi - lo);
  if (hi <= lo) span = 1u;
  uint32_t mult = 65536u % span;
  mult = (uint32_t)(mult * mult) % span;
  uint32_t off = (uint32_t)((higher % span) * mult + (lower % span));
  off = off % span;
  return lo + (int32_t)off;
}

/* jax.random.choice(key, m, p=p) with replace=True:
 * r = cum[-1] * (1 - uniform(key)); index = searchsorted(cum, r, 'left'). */
int32_t jro_choice(const uint32_t key[2], const float* cum, int32_t m) {
  float u = bits_to_unit(jro_bits32(key, 0));
  float one_minus = 1.0f - u;
  float r = cum[m - 1] * one_minus;
  int32_t idx = 0;
  while (idx < m && cum[idx] < r) ++idx;
  return idx;
}

void jro_normal_array(const uint32_t key[2], int32_t n, float* out) {
  for (int32_t i = 0; i < n; ++i) out[i] = jro_normal(jro_bits32(key, (uint32_t)i));
}

void jro_uniform_array(const uint32_t key[2], int32_t n, float* out) {
  for (int32_t i = 0; i < n; ++i)
    out[i] = jro_uniform(jro_bits32(key, (uint32_t)i), 0.0f, 1.0f);
}

/* ------------------------------------------------------------------ */
/* Geometry                                                            */
/* ------------------------------------------------------------------ */

/* jnp.linalg.det for 3x3 (jax._src.numpy.linalg._det_3x3), float32,
 * evaluated left to right as written there. */
float jro_det3(const float* a) {
  float t1 = (a[0] * a[4]) * a[8];
  float t2 = (a[1] * a[5]) * a[6];
  float t3 = (a[2] * a[3]) * a[7];
  float t4 = (a[2] * a[4]) * a[6];
  float t5 = (a[0] * a[5]) * a[7];
  float t6 = (a[1] * a[3]) * a[8];
  float s = t1 + t2;
  s = s + t3;
  s = s - t4;
  s = s - t5;
  s = s - t6;
  return s;
}

static int is_diag(const float* c) {
  return c[1] == 0.0f && c[2] == 0.0f && c[3] == 0.0f && c[5] == 0.0f &&
         c[6] == 0.0f && c[7] == 0.0f;
}

/* Kernel contract for inv(cell): a diagonal cell inverts element-wise with
 * float32 division (what LU-solve produces for a diagonal matrix); any other
 * cell uses the double adjugate divided by the double determinant, rounded
 * once to float32.  The reference (lj.py:156) uses jnp.linalg.inv. */
void jro_inv_cell(const float* c, float* inv) {
  if (is_diag(c)) {
    memset(inv, 0, 9 * sizeof(float));
    inv[0] = 1.0f / c[0];
    inv[4] = 1.0f / c[4];
    inv[8] = 1.0f / c[8];
    return;
  }
  double a[9];
  for (int i = 0; i < 9; ++i) a[i] = (double)c[i];
  double cof[9];
  cof[0] = a[4] * a[8] - a[5] * a[7];
  cof[1] = a[5] * a[6] - a[3] * a[8];
  cof[2] = a[3] * a[7] - a[4] * a[6];
  cof[3] = a[2] * a[7] - a[1] * a[8];
  cof[4] = a[0] * a[8] - a[2] * a[6];
  cof[5] = a[1] * a[6] - a[0] * a[7];
  cof[6] = a[1] * a[5] - a[2] * a[4];
  cof[7] = a[2] * a[3] - a[0] * a[5];
  cof[8] = a[0] * a[4] - a[1] * a[3];
  double det = a[0] * cof[0] + a[1] * cof[1] + a[2] * cof[2];
  /* inv[i][j] = cof[j][i] / det */
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) inv[i * 3 + j] = (float)(cof[j * 3 + i] / det);
}

static void inv_cell_f64(const double* a, double* inv) {
  double cof[9];
  cof[0] = a[4] * a[8] - a[5] * a[7];
  cof[1] = a[5] * a[6] - a[3] * a[8];
  cof[2] = a[3] * a[7] - a[4] * a[6];
  cof[3] = a[2] * a[7] - a[1] * a[8];
  cof[4] = a[0] * a[8] - a[2] * a[6];
  cof[5] = a[1] * a[6] - a[0] * a[7];
  cof[6] = a[1] * a[5] - a[2] * a[4];
  cof[7] = a[2] * a[3] - a[0] * a[5];
  cof[8] = a[0] * a[4] - a[1] * a[3];
  double det = a[0] * cof[0] + a[1] * cof[1] + a[2] * cof[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) inv[i * 3 + j] = cof[j * 3 + i] / det;
}

/* ------------------------------------------------------------------ */
/* Lennard-Jones (backends/lj.py:125-204)                              */
/* ------------------------------------------------------------------ */

static int center_image(const JroModel* m) {
  for (int k = 0; k < m->n_images; ++k)
    if (m->img_off[3 * k] == 0.0f && m->img_off[3 * k + 1] == 0.0f &&
        m->img_off[3 * k + 2] == 0.0f)
      return k;
  return -1;
}

/* Kernel reciprocal: bit-pattern seed + three FMA Newton-Raphson steps
 * (max 0.501 ulp); outside [2^-120, 2^120] the correctly rounded 1/x.  The
 * seed as_float(C - as_int(x)) is the piecewise-linear reciprocal of the bit
 * pattern; C = 0x7EF311C3 is within 2e-8 of the offset that minimises its
 * largest relative error over a binade (5.05%, found by scanning C), and each
 * Newton step squares that error. */
static inline float rcp_nr(float x) {
  if (!(x >= 0x1p-120f && x <= 0x1p120f)) return 1.0f / x;
  uint32_t u;
  memcpy(&u, &x, 4);
  u = 0x7EF311C3u - u;
  float y;
  memcpy(&y, &u, 4);
  for (int k = 0; k < 3; ++k) {
    float e = fmaf(-x, y, 1.0f);
    y = fmaf(y, e, y);
  }
  return y;
}

/* DEV contract, one ordered pair: r2 by FMA chain, reciprocal, LJ powers. */
static inline void dev_pair(const JroModel* m, int ti, int tj, float dx,
                            float dy, float dz, float* e, float* g) {
  float r2 = dx * dx;
  r2 = fmaf(dy, dy, r2);
  r2 = fmaf(dz, dz, r2);
  if (m->has_cutoff && !(r2 < m->rc2)) {
    *e = 0.0f;
    *g = 0.0f;
    return;
  }
  const int S = m->n_species;
  float sig2 = m->sig2[ti * S + tj];
  float eps4 = m->eps4[ti * S + tj];
  float eps24 = m->eps24[ti * S + tj];
  float ri = rcp_nr(r2);
  float s2 = sig2 * ri;
  float s4 = s2 * s2;
  float s6 = s4 * s2;
  float s12 = s6 * s6;
  float diff = s12 - s6;
  *e = eps4 * diff;
  float t = fmaf(2.0f, s12, -s6);
  float a = eps24 * ri;
  *g = -(a * t);
}

static double lj_dev(const JroModel* m, int n, const float* x,
                     const int32_t* t, const float* cell_in, double* F) {
  float safe[9];
  const float* c = cell_in;
  if (jro_det3(cell_in) == 0.0f) {
    memset(safe, 0, sizeof(safe));
    safe[0] = safe[4] = safe[8] = 1.0e10f;
    c = safe;
  }
  float inv[9];
  jro_inv_cell(c, inv);
  const int nimg = m->n_images;
  const int ctr = center_image(m);
  float T[JRO_MAX_IMAGES * 3];
  for (int k = 0; k < nimg; ++k) {
    const float* o = m->img_off + 3 * k;
    for (int q = 0; q < 3; ++q) {
      float v = o[0] * c[q];
      v = fmaf(o[1], c[3 + q], v);
      v = fmaf(o[2], c[6 + q], v);
      T[3 * k + q] = v;
    }
  }
  /* Energy: float64 sum of the float32 pair terms.  Forces: float32 in the
   * canonical order -- partners in blocks of 8 (ascending j, then image),
   * block partials combined pairwise over L = next_pow2(ceil(n/8)) slots. */
  int nb = (n + 7) / 8, L = 1;
  while (L < nb) L <<= 1;
  double E = 0.0;
  for (int i = 0; i < n; ++i) {
    float Pb[32][3];
    memset(Pb, 0, sizeof(Pb));
    for (int b = 0; b < L; ++b) {
      const int j0 = 8 * b, j1 = j0 + 8 < n ? j0 + 8 : n;
      for (int j = j0; j < j1; ++j) {
        float dr[3], d[3];
        for (int q = 0; q < 3; ++q) dr[q] = x[3 * j + q] - x[3 * i + q];
        float nn[3];
        for (int q = 0; q < 3; ++q) {
          float f = dr[0] * inv[q];
          f = fmaf(dr[1], inv[3 + q], f);
          f = fmaf(dr[2], inv[6 + q], f);
          nn[q] = rintf(f);
        }
        for (int q = 0; q < 3; ++q) {
          float s = nn[0] * c[q];
          s = fmaf(nn[1], c[3 + q], s);
          s = fmaf(nn[2], c[6 + q], s);
          d[q] = dr[q] - s;
        }
        for (int k = 0; k < nimg; ++k) {
          if (k == ctr && i == j) continue;
          float dd[3];
          if (nimg > 1) {
            for (int q = 0; q < 3; ++q) dd[q] = d[q] + T[3 * k + q];
          } else {
            dd[0] = d[0]; dd[1] = d[1]; dd[2] = d[2];
          }
          float e, g;
          dev_pair(m, t[i], t[j], dd[0], dd[1], dd[2], &e, &g);
          E += (double)e;
          if (F && i != j)
            for (int q = 0; q < 3; ++q) {
              float term = g * dd[q];
              Pb[b][q] = Pb[b][q] + term;
            }
        }
      }
    }
    if (F) {
      for (int s = 1; s < L; s <<= 1) {
        float Q[32][3];
        for (int b = 0; b < L; ++b)
          for (int q = 0; q < 3; ++q) Q[b][q] = Pb[b][q] + Pb[b ^ s][q];
        memcpy(Pb, Q, sizeof(float) * 3 * L);
      }
      for (int q = 0; q < 3; ++q) F[3 * i + q] = (double)Pb[0][q];
    }
  }
  return 0.5 * E;
}

/* REF32: the reference's float32 op order (no FMA, f32 row-major sums). */
static double lj_ref32(const JroModel* m, int n, const float* x,
                       const int32_t* t, const float* cell_in, double* F) {
  float safe[9];
  const float* c = cell_in;
  if (jro_det3(cell_in) == 0.0f) {
    memset(safe, 0, sizeof(safe));
    safe[0] = safe[4] = safe[8] = 1.0e10f;
    c = safe;
  }
  float inv[9];
  jro_inv_cell(c, inv);
  const int nimg = m->n_images;
  const int ctr = center_image(m);
  const int S = m->n_species;
  float T[JRO_MAX_IMAGES * 3];
  for (int k = 0; k < nimg; ++k) {
    const float* o = m->img_off + 3 * k;
    for (int q = 0; q < 3; ++q) {
      float v = o[0] * c[q] + o[1] * c[3 + q];
      v = v + o[2] * c[6 + q];
      T[3 * k + q] = v;
    }
  }
  float Esum = 0.0f;
  float* Fs = NULL;
  if (F) Fs = (float*)calloc((size_t)3 * n, sizeof(float));
  for (int k = 0; k < nimg; ++k) {
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) {
        float dr[3], d[3], nn[3];
        for (int q = 0; q < 3; ++q) dr[q] = x[3 * j + q] - x[3 * i + q];
        for (int q = 0; q < 3; ++q) {
          float f = dr[0] * inv[q] + dr[1] * inv[3 + q];
          f = f + dr[2] * inv[6 + q];
          nn[q] = rintf(f);
        }
        for (int q = 0; q < 3; ++q) {
          float s = nn[0] * c[q] + nn[1] * c[3 + q];
          s = s + nn[2] * c[6 + q];
          d[q] = dr[q] - s;
        }
        if (k == ctr && i == j) continue;
        float dd[3];
        for (int q = 0; q < 3; ++q) dd[q] = d[q] + T[3 * k + q];
        float r2 = dd[0] * dd[0] + dd[1] * dd[1];
        r2 = r2 + dd[2] * dd[2];
        if (m->has_cutoff && !(r2 < m->rc2)) continue;
        float sig2 = m->sig2[t[i] * S + t[j]];
        float s2 = sig2 / r2;
        float s6 = s2 * (s2 * s2);
        float s12 = s6 * s6;
        float e = m->eps4[t[i] * S + t[j]] * (s12 - s6);
        Esum = Esum + e;
        if (Fs && i != j) {
          float coef = (m->eps24[t[i] * S + t[j]] / r2) * (2.0f * s12 - s6);
          for (int q = 0; q < 3; ++q) Fs[3 * i + q] = Fs[3 * i + q] - coef * dd[q];
        }
      }
    }
  }
  if (F) {
    for (int i = 0; i < 3 * n; ++i) F[i] = (double)Fs[i];
    free(Fs);
  }
  return (double)(0.5f * Esum);
}

/* Everything in double: the error yardstick for the FP32 paths. */
static double lj_f64(const JroModel* m, int n, const float* x,
                     const int32_t* t, const float* cell_in, double* F) {
  double c[9], inv[9];
  for (int i = 0; i < 9; ++i) c[i] = (double)cell_in[i];
  if (jro_det3(cell_in) == 0.0f) {
    memset(c, 0, sizeof(c));
    c[0] = c[4] = c[8] = 1.0e10;
  }
  inv_cell_f64(c, inv);
  const int nimg = m->n_images;
  const int ctr = center_image(m);
  const int S = m->n_species;
  double T[JRO_MAX_IMAGES * 3];
  for (int k = 0; k < nimg; ++k) {
    const float* o = m->img_off + 3 * k;
    for (int q = 0; q < 3; ++q)
      T[3 * k + q] = o[0] * c[q] + o[1] * c[3 + q] + o[2] * c[6 + q];
  }
  double E = 0.0;
  if (F) memset(F, 0, sizeof(double) * 3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      double dr[3], d[3], nn[3];
      for (int q = 0; q < 3; ++q) dr[q] = (double)x[3 * j + q] - (double)x[3 * i + q];
      for (int q = 0; q < 3; ++q)
        nn[q] = nearbyint(dr[0] * inv[q] + dr[1] * inv[3 + q] + dr[2] * inv[6 + q]);
      for (int q = 0; q < 3; ++q)
        d[q] = dr[q] - (nn[0] * c[q] + nn[1] * c[3 + q] + nn[2] * c[6 + q]);
      for (int k = 0; k < nimg; ++k) {
        if (k == ctr && i == j) continue;
        double dd[3];
        for (int q = 0; q < 3; ++q) dd[q] = d[q] + T[3 * k + q];
        double r2 = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
        if (m->has_cutoff && !(r2 < (double)m->rc2)) continue;
        double sig2 = (double)m->sig2[t[i] * S + t[j]];
        double eps4 = (double)m->eps4[t[i] * S + t[j]];
        double s2 = sig2 / r2, s6 = s2 * s2 * s2, s12 = s6 * s6;
        E += eps4 * (s12 - s6);
        if (F && i != j) {
          double coef = (6.0 * eps4 / r2) * (2.0 * s12 - s6);
          for (int q = 0; q < 3; ++q) F[3 * i + q] -= coef * dd[q];
        }
      }
    }
  }
  return 0.5 * E;
}

/* ------------------------------------------------------------------ */
/* Stillinger-Weber (Phys. Rev. B 31, 5262 (1985)), p = 4, q = 0        */
/* ------------------------------------------------------------------ */

/* exp(x) of the kernel contract: Cody-Waite reduction x = k ln2 + r with
 * k = rint(x log2 e), ln2 = LN2_HI + LN2_LO (LN2_HI: float32 ln2 with its 12
 * low mantissa bits cleared), the degree-7 Taylor polynomial of e^r (1/n! in
 * float32) in FMA Horner form, scaled by 2^k (two steps below the normal
 * range). */
float jro_sw_exp(float x) {
  if (!(x > -104.0f)) return 0.0f;
  if (x > 88.5f) return INFINITY;
  const float k = rintf(x * 0x1.715476p+0f);
  float r = fmaf(-k, 0x1.62ep-1f, x);
  r = fmaf(-k, 0x1.0bfbe8p-15f, r);
  float p = 0x1.a01a02p-13f;
  p = fmaf(p, r, 0x1.6c16c2p-10f);
  p = fmaf(p, r, 0x1.111112p-7f);
  p = fmaf(p, r, 0x1.555556p-5f);
  p = fmaf(p, r, 0x1.555556p-3f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  const int ki = (int)k;
  uint32_t b;
  float sc;
  if (ki >= -126) {
    b = (uint32_t)(ki + 127) << 23;
    memcpy(&sc, &b, 4);
    return p * sc;
  }
  b = (uint32_t)(ki + 64 + 127) << 23;
  memcpy(&sc, &b, 4);
  return (p * sc) * 0x1p-64f;
}

typedef struct SwPair {
  float dx, dy, dz, inv_r, g, u, c2, e2;
} SwPair;

static inline int sw_pidx(int lo, int hi, int n) { return lo * (2 * n - lo - 1) / 2 + (hi - lo - 1); }

/* The kernel's pair record (float32, the kernel's op order). */
static int sw_pair_dev(const JroModel* m, float r2, SwPair* q) {
  /* rc2 is the smallest float32 whose square root reaches rc, so r2 < rc2
   * is exactly sqrt(r2) < rc */
  if (!(r2 < m->rc2)) return 0;
  const float r = sqrtf(r2);
  q->inv_r = rcp_nr(r);
  const float md = m->sw_rc - r;
  const float inv_md = rcp_nr(md);
  const float ex = jro_sw_exp(-(m->sw_sigma * inv_md));
  q->g = jro_sw_exp(-(m->sw_gsig * inv_md));
  const float sg = m->sw_sigma * q->inv_r;
  const float s2 = sg * sg;
  const float s4 = s2 * s2;
  const float bq = fmaf(m->sw_B, s4, -1.0f);
  const float aex = m->sw_Aeps * ex;
  q->e2 = aex * bq;
  const float w = (m->sw_sigma * inv_md) * inv_md;
  const float t1 = (-4.0f * (m->sw_B * s4)) * q->inv_r;
  const float dphi = aex * fmaf(-bq, w, t1);
  q->c2 = dphi * q->inv_r;
  q->u = (-((m->sw_gsig * inv_md) * inv_md)) * q->inv_r;
  return 1;
}

/* One triplet seen from leg j (other leg k): force on j subtracted from v,
 * energy returned (the kernel's sw_triplet). */
static float sw_triplet_dev(float leps, const float* jv, float ij, float gj, float uj,
                            const float* kv, float ik, float gk, float* v, int forces) {
  const float dot = fmaf(jv[2], kv[2], fmaf(jv[1], kv[1], jv[0] * kv[0]));
  const float cs = (dot * ij) * ik;
  const float t = cs + 0x1.555556p-2f;
  const float G = (leps * gj) * gk;
  const float tG = t * G;
  if (forces) {
    const float ij2 = ij * ij;
    const float p2 = (2.0f * cs) * ij2;
    const float A = tG * fmaf(t, uj, -p2);
    const float Bc = (2.0f * tG) * (ij * ik);
    for (int q = 0; q < 3; ++q) v[q] = v[q] - fmaf(A, jv[q], Bc * kv[q]);
  }
  return tG * t;
}

/* The kernel contract (DEV): pair records, per neighbour pair {a<b} the two
 * centre sides with the other leg ascending, Q_ab = c2 dr_ab + V_ba - V_ab,
 * F_i the sequential float32 sum of +-Q_ij over the neighbours j ascending.  Also
 * used for REF32: the reference has no Stillinger-Weber to take an op order
 * from.  *n_pairs / *n_trip receive the evaluation's counts (may be NULL). */
static double sw_dev(const JroModel* m, int n, const float* x, const float* cell_in, double* F,
                     int64_t* n_pairs, int64_t* n_trip) {
  float safe[9];
  const float* c = cell_in;
  if (jro_det3(cell_in) == 0.0f) {
    memset(safe, 0, sizeof(safe));
    safe[0] = safe[4] = safe[8] = 1.0e10f;
    c = safe;
  }
  float inv[9];
  jro_inv_cell(c, inv);
  const int np = n * (n - 1) / 2;
  SwPair* pr = (SwPair*)calloc((size_t)(np > 0 ? np : 1), sizeof(SwPair));
  float* Q = (float*)calloc((size_t)(np > 0 ? np : 1) * 3, sizeof(float));
  uint64_t nbm[64];
  memset(nbm, 0, sizeof(nbm));
  double E = 0.0;
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      float dr[3], d[3], nn[3];
      for (int q = 0; q < 3; ++q) dr[q] = x[3 * b + q] - x[3 * a + q];
      for (int q = 0; q < 3; ++q) {
        float f = dr[0] * inv[q];
        f = fmaf(dr[1], inv[3 + q], f);
        f = fmaf(dr[2], inv[6 + q], f);
        nn[q] = rintf(f);
      }
      for (int q = 0; q < 3; ++q) {
        float sv = nn[0] * c[q];
        sv = fmaf(nn[1], c[3 + q], sv);
        sv = fmaf(nn[2], c[6 + q], sv);
        d[q] = dr[q] - sv;
      }
      float r2 = d[0] * d[0];
      r2 = fmaf(d[1], d[1], r2);
      r2 = fmaf(d[2], d[2], r2);
      SwPair* q = pr + sw_pidx(a, b, n);
      if (sw_pair_dev(m, r2, q)) {
        q->dx = d[0];
        q->dy = d[1];
        q->dz = d[2];
        nbm[a] |= 1ull << b;
        nbm[b] |= 1ull << a;
        E += (double)q->e2;
      }
    }
  int64_t pairs = 0, trip = 0;
  for (int i = 0; i < n; ++i) {
    const int dg = __builtin_popcountll(nbm[i]);
    pairs += dg;
    trip += dg * (dg - 1) / 2;
  }
  if (n_pairs) *n_pairs = pairs / 2;
  if (n_trip) *n_trip = trip;
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      if (!((nbm[a] >> b) & 1ull)) continue;
      const int p = sw_pidx(a, b, n);
      const SwPair* ab = pr + p;
      float vab[3] = {0.0f, 0.0f, 0.0f}, vba[3] = {0.0f, 0.0f, 0.0f};
      for (int side = 0; side < 2; ++side) {
        const int ctr = side == 0 ? a : b, leg = side == 0 ? b : a;
        const float sg = side == 0 ? 1.0f : -1.0f;
        const float jv[3] = {sg * ab->dx, sg * ab->dy, sg * ab->dz};
        float* v = side == 0 ? vab : vba;
        for (int k = 0; k < n; ++k) {
          if (k == leg || !((nbm[ctr] >> k) & 1ull)) continue;
          const int fwd = ctr < k;
          const SwPair* ck = pr + (fwd ? sw_pidx(ctr, k, n) : sw_pidx(k, ctr, n));
          const float kv[3] = {fwd ? ck->dx : -ck->dx, fwd ? ck->dy : -ck->dy,
                               fwd ? ck->dz : -ck->dz};
          if (F || k > leg) {
            const float h = sw_triplet_dev(m->sw_leps, jv, ab->inv_r, ab->g, ab->u, kv,
                                           ck->inv_r, ck->g, v, F != NULL);
            if (k > leg) E += (double)h;
          }
        }
      }
      if (F) {
        const float dv[3] = {ab->dx, ab->dy, ab->dz};
        for (int q = 0; q < 3; ++q) Q[3 * p + q] = fmaf(ab->c2, dv[q], vba[q]) - vab[q];
      }
    }
  if (F) {
    for (int i = 0; i < n; ++i) {
      float f[3] = {0.0f, 0.0f, 0.0f};
      for (int j = 0; j < n; ++j) {
        if (!((nbm[i] >> j) & 1ull)) continue;
        const int fwd = i < j;
        const float* qv = Q + 3 * (fwd ? sw_pidx(i, j, n) : sw_pidx(j, i, n));
        for (int q = 0; q < 3; ++q) f[q] = f[q] + (fwd ? qv[q] : -qv[q]);
      }
      for (int q = 0; q < 3; ++q) F[3 * i + q] = (double)f[q];
    }
  }
  free(pr);
  free(Q);
  return E;
}

/* Everything in double, written independently of the kernel's organisation:
 * pair sum over i < j, triplet sum over centres i and leg pairs j < k, forces
 * from the analytic gradient of each term added to the three atoms. */
static double sw_f64(const JroModel* m, int n, const float* x, const float* cell_in, double* F) {
  double c[9], inv[9];
  for (int i = 0; i < 9; ++i) c[i] = (double)cell_in[i];
  if (jro_det3(cell_in) == 0.0f) {
    memset(c, 0, sizeof(c));
    c[0] = c[4] = c[8] = 1.0e10;
  }
  inv_cell_f64(c, inv);
  const double sig = m->sw_sigma, rc = m->sw_rc, gsig = m->sw_gsig, Ae = m->sw_Aeps,
               B = m->sw_B, le = m->sw_leps;
  double* D = (double*)calloc((size_t)n * n * 3, sizeof(double));  /* MIC dr_ij = x_j - x_i */
  double* R = (double*)calloc((size_t)n * n, sizeof(double));
  if (F) memset(F, 0, sizeof(double) * 3 * (size_t)n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      double dr[3], nn[3];
      for (int q = 0; q < 3; ++q) dr[q] = (double)x[3 * j + q] - (double)x[3 * i + q];
      for (int q = 0; q < 3; ++q)
        nn[q] = nearbyint(dr[0] * inv[q] + dr[1] * inv[3 + q] + dr[2] * inv[6 + q]);
      for (int q = 0; q < 3; ++q)
        D[3 * (i * n + j) + q] = dr[q] - (nn[0] * c[q] + nn[1] * c[3 + q] + nn[2] * c[6 + q]);
      const double* d = D + 3 * (i * n + j);
      R[i * n + j] = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
  double E = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double r = R[i * n + j];
      if (!(r < rc)) continue;
      const double s4 = pow(sig / r, 4.0);
      const double ex = exp(sig / (r - rc));
      E += Ae * (B * s4 - 1.0) * ex;
      if (F) {
        const double dphi = Ae * ex * (-4.0 * B * s4 / r - (B * s4 - 1.0) * sig / ((r - rc) * (r - rc)));
        const double* d = D + 3 * (i * n + j);
        for (int q = 0; q < 3; ++q) {
          F[3 * i + q] += dphi * d[q] / r;
          F[3 * j + q] -= dphi * d[q] / r;
        }
      }
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      if (j == i || !(R[i * n + j] < rc)) continue;
      for (int k = j + 1; k < n; ++k) {
        if (k == i || !(R[i * n + k] < rc)) continue;
        const double* dj = D + 3 * (i * n + j);
        const double* dk = D + 3 * (i * n + k);
        const double rj = R[i * n + j], rk = R[i * n + k];
        const double cs = (dj[0] * dk[0] + dj[1] * dk[1] + dj[2] * dk[2]) / (rj * rk);
        const double gj = exp(gsig / (rj - rc)), gk = exp(gsig / (rk - rc));
        const double t = cs + 1.0 / 3.0;
        E += le * t * t * gj * gk;
        if (F) {
          /* dh/dx_j = le gj gk [t^2 g'j/gj drj/rj + 2t dcos/dx_j] */
          const double lj = -gsig / ((rj - rc) * (rj - rc)), lk = -gsig / ((rk - rc) * (rk - rc));
          const double G = le * gj * gk;
          double hj[3], hk[3];
          for (int q = 0; q < 3; ++q) {
            const double dcj = dk[q] / (rj * rk) - cs * dj[q] / (rj * rj);
            const double dck = dj[q] / (rj * rk) - cs * dk[q] / (rk * rk);
            hj[q] = G * (t * t * lj * dj[q] / rj + 2.0 * t * dcj);
            hk[q] = G * (t * t * lk * dk[q] / rk + 2.0 * t * dck);
          }
          for (int q = 0; q < 3; ++q) {
            F[3 * j + q] -= hj[q];
            F[3 * k + q] -= hk[q];
            F[3 * i + q] += hj[q] + hk[q];
          }
        }
      }
    }
  free(D);
  free(R);
  return E;
}

/* Gaussian-mixture toy (backends/toy.py:163-204), evaluated in double. */
static double gauss_mix(const JroModel* m, int n, const float* x, double* F) {
  double com[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < 3; ++q) com[q] += (double)x[3 * i + q];
  for (int q = 0; q < 3; ++q) com[q] /= (double)n;
  const double s2 = (double)m->gm_sigma * (double)m->gm_sigma;
  const double lnorm = 1.5 * log(2.0 * M_PI * s2);
  double l[JRO_MAX_CENTERS], lmax = -INFINITY;
  for (int k = 0; k < m->n_centers; ++k) {
    double ds = 0.0;
    for (int q = 0; q < 3; ++q) {
      double df = com[q] - (double)m->centers[3 * k + q];
      ds += df * df;
    }
    l[k] = -0.5 * ds / s2 - lnorm;
    if (l[k] > lmax) lmax = l[k];
  }
  double z = 0.0;
  for (int k = 0; k < m->n_centers; ++k) z += exp(l[k] - lmax);
  double E = -(lmax + log(z));
  if (F) {
    double gcom[3] = {0, 0, 0};
    for (int k = 0; k < m->n_centers; ++k) {
      double p = exp(l[k] - lmax) / z;
      for (int q = 0; q < 3; ++q)
        gcom[q] += p * (com[q] - (double)m->centers[3 * k + q]) / s2;
    }
    for (int i = 0; i < n; ++i)
      for (int q = 0; q < 3; ++q) F[3 * i + q] = (double)(float)(-gcom[q] / (double)n);
  }
  return E;
}

/* EnsembleTerm (backends/ensemble.py:34-59) + Hamiltonian sum
 * (backends/hamiltonian.py:112-153). */
double jro_energy(const JroModel* mdl, int32_t mode, int32_t n, const float* x,
                  const int32_t* types, const float* cell, float pressure,
                  const float* mu, int32_t has_mu, double* forces,
                  double* u_out) {
  double U;
  if (mdl->model == JRO_MODEL_GAUSS_MIX) {
    U = gauss_mix(mdl, n, x, forces);
  } else if (mdl->model == JRO_MODEL_SW) {
    U = mode == JRO_F64 ? sw_f64(mdl, n, x, cell, forces)
                        : sw_dev(mdl, n, x, cell, forces, NULL, NULL);
  } else if (mode == JRO_DEV) {
    U = lj_dev(mdl, n, x, types, cell, forces);
  } else if (mode == JRO_REF32) {
    U = lj_ref32(mdl, n, x, types, cell, forces);
  } else {
    U = lj_f64(mdl, n, x, types, cell, forces);
  }
  if (u_out) *u_out = U;
  if (mdl->model == JRO_MODEL_GAUSS_MIX) return U;
  int32_t counts[JRO_MAX_SPECIES] = {0};
  for (int i = 0; i < n; ++i) counts[types[i]]++;
  float V = fabsf(jro_det3(cell));
  if (mode == JRO_REF32) {
    float ens = pressure * V;
    if (has_mu) {
      float dot = 0.0f;
      for (int s = 0; s < mdl->n_species; ++s) dot = dot + mu[s] * (float)counts[s];
      ens = ens - dot;
    }
    return (double)((float)U + ens);
  }
  double ens = (double)pressure * (double)V;
  if (has_mu) {
    double dot = 0.0;
    for (int s = 0; s < mdl->n_species; ++s) dot += (double)mu[s] * (double)counts[s];
    ens = ens - dot;
  }
  return U + ens;
}

/* ------------------------------------------------------------------ */
/* Move helpers                                                        */
/* ------------------------------------------------------------------ */

static float vnorm(const float* v, int n, int mode) {
  if (mode == JRO_REF32) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s = s + v[i] * v[i];
    return sqrtf(s);
  }
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += (double)v[i] * (double)v[i];
  return (float)sqrt(s);
}

static void vnormalize(float* v, int n, int mode) {
  float nv = vnorm(v, n, mode);
  float den = nv > 1e-10f ? nv : 1e-10f;
  for (int i = 0; i < n; ++i) v[i] = v[i] / den;
}

static double eval_energy(const JroModel* mdl, int mode, int n, const float* x,
                          const int32_t* t, const float* cell, float P,
                          const float* mu, int has_mu, double* F) {
  return jro_energy(mdl, mode, n, x, t, cell, P, mu, has_mu, F, NULL);
}

/* Galilean move (sampling/moves/galilean.py:142-300). */
static int move_galilean(const JroModel* mdl, int mode, const uint32_t key[2],
                         float step, int R, float pa, double emax, int n,
                         float* x, float* d, int32_t* t, float* cell,
                         double* energy, float P, const float* mu, int has_mu) {
  const int n3 = 3 * n;
  uint32_t k_init[2], k_pert[2];
  jro_split(key, 0, k_init);
  jro_split(key, 1, k_pert);
  float* v = (float*)calloc((size_t)(n3 > 0 ? n3 : 1), sizeof(float));
  float* x0 = (float*)malloc(sizeof(float) * n3);
  float* dp = (float*)malloc(sizeof(float) * n3);
  double* F = (double*)malloc(sizeof(double) * n3);
  float* Ff = (float*)malloc(sizeof(float) * n3);
  float dn = vnorm(d, n3, mode);
  if (dn < 1e-8f) {
    for (int i = 0; i < n3; ++i) v[i] = jro_normal(jro_bits32(k_init, (uint32_t)i));
  } else {
    for (int i = 0; i < n3; ++i) {
      float z = jro_normal(jro_bits32(k_pert, (uint32_t)i));
      if (mode == JRO_REF32) {
        float noise = pa * z;
        v[i] = d[i] + noise;
      } else {
        v[i] = fmaf(pa, z, d[i]);
      }
    }
  }
  vnormalize(v, n3, mode);
  memcpy(x0, x, sizeof(float) * n3);
  memcpy(dp, v, sizeof(float) * n3);
  double E0 = *energy;
  double E = E0;
  for (int r = 0; r < R; ++r) {
    for (int i = 0; i < n3; ++i) {
      if (mode == JRO_REF32) {
        float sv = step * v[i];
        x[i] = x[i] + sv;
      } else {
        x[i] = fmaf(step, v[i], x[i]);
      }
    }
    E = eval_energy(mdl, mode, n, x, t, cell, P, mu, has_mu, F);
    if (isnan(E)) E = INFINITY;
    if (E >= emax) {
      for (int i = 0; i < n3; ++i) Ff[i] = (float)F[i];
      if (mode == JRO_REF32) {
        float fn = vnorm(Ff, n3, mode);
        float den = fn > 1e-10f ? fn : 1e-10f;
        float dot = 0.0f;
        for (int i = 0; i < n3; ++i) Ff[i] = Ff[i] / den;
        for (int i = 0; i < n3; ++i) dot = dot + Ff[i] * v[i];
        float two = 2.0f * dot;
        for (int i = 0; i < n3; ++i) v[i] = v[i] - two * Ff[i];
      } else {
        double sff = 0.0, sfd = 0.0;
        for (int i = 0; i < n3; ++i) {
          sff += (double)Ff[i] * (double)Ff[i];
          sfd += (double)Ff[i] * (double)v[i];
        }
        /* coefficient 2 (F.d) / max(|F|^2, 1e-20) with the scalar in float32 */
        float ffs = (float)sff;
        float coef = (2.0f * (float)sfd) * rcp_nr(ffs > 1e-20f ? ffs : 1e-20f);
        for (int i = 0; i < n3; ++i) v[i] = fmaf(-coef, Ff[i], v[i]);
      }
    }
  }
  int acc = E < emax;
  if (acc) {
    *energy = E;
    memcpy(d, v, sizeof(float) * n3);
  } else {
    memcpy(x, x0, sizeof(float) * n3);
    *energy = E0;
    for (int i = 0; i < n3; ++i) d[i] = -dp[i];
  }
  free(v); free(x0); free(dp); free(F); free(Ff);
  return acc;
}

/* utils/cell.py:80-125 check_cell_shape (float32; reductions per contract) */
static int cell_valid(const float* c, int n, float max_vpa, float min_vpa,
                      float min_aspect, int mode) {
  float vol = fabsf(jro_det3(c));
  float vpa = vol / (float)n;
  float vc = (float)pow((double)vol, (double)(1.0f / 3.0f));
  static const int pr[3][3] = {{0, 1, 2}, {1, 2, 0}, {0, 2, 1}};
  float amin = INFINITY;
  for (int p = 0; p < 3; ++p) {
    const float* a = c + 3 * pr[p][0];
    const float* b = c + 3 * pr[p][1];
    const float* e = c + 3 * pr[p][2];
    float cr[3];
    cr[0] = a[1] * b[2] - a[2] * b[1];
    cr[1] = a[2] * b[0] - a[0] * b[2];
    cr[2] = a[0] * b[1] - a[1] * b[0];
    float nrm = vnorm(cr, 3, mode);
    float cn[3] = {cr[0] / nrm, cr[1] / nrm, cr[2] / nrm};
    float h;
    if (mode == JRO_REF32) {
      h = cn[0] * e[0] + cn[1] * e[1];
      h = h + cn[2] * e[2];
    } else {
      h = (float)((double)cn[0] * e[0] + (double)cn[1] * e[1] + (double)cn[2] * e[2]);
    }
    h = fabsf(h);
    float ratio = h / vc;
    if (ratio < amin || isnan(ratio)) amin = ratio;
  }
  return (vpa <= max_vpa) && (vpa >= min_vpa) && (amin >= min_aspect);
}

/* Volume move (sampling/moves/volume.py:49-109, moves/_common.py:16-93). */
static int move_volume(const JroModel* mdl, const JroMoves* mv, int mode,
                       const uint32_t key[2], float step, double emax, int n,
                       float* x, int32_t* t, float* cell, double* energy,
                       float P, const float* mu, int has_mu, int* reason) {
  uint32_t k1[2], k2[2];
  jro_split(key, 0, k1);
  jro_split(key, 1, k2);
  float oldV = fabsf(jro_det3(cell));
  float sn = step * (float)n;
  float dV = sn * jro_normal(jro_bits32(k1, 0));
  float newV = fabsf(oldV + dV);
  float ratio = newV / oldV;
  float scale = (float)pow((double)ratio, (double)(1.0f / 3.0f));
  float nc[9];
  for (int i = 0; i < 9; ++i) nc[i] = cell[i] * scale;
  float* nx = (float*)malloc(sizeof(float) * 3 * n);
  for (int i = 0; i < 3 * n; ++i) nx[i] = x[i] * scale;
  double En = eval_energy(mdl, mode, n, nx, t, nc, P, mu, has_mu, NULL);
  int valid = cell_valid(nc, n, mv->max_vpa, mv->min_vpa, mv->min_aspect, mode);
  int prior_ok;
  float u = jro_uniform(jro_bits32(k2, 0), 0.0f, 1.0f);
  if (mv->flat_v_prior) {
    prior_ok = u < 1.0f;
  } else if (mode == JRO_REF32) {
    /* lax.integer_pow by binary exponentiation, float32 */
    float acc = 1.0f, b = ratio;
    int first = 1, y = n;
    while (y > 0) {
      if (y & 1) { acc = first ? b : acc * b; first = 0; }
      y >>= 1;
      if (y > 0) b = b * b;
    }
    float pa = acc < 1.0f ? acc : 1.0f;
    prior_ok = u < pa;
  } else {
    double acc = 1.0, b = (double)ratio;
    int first = 1, y = n;
    while (y > 0) {
      if (y & 1) { acc = first ? b : acc * b; first = 0; }
      y >>= 1;
      if (y > 0) b = b * b;
    }
    double pa = acc < 1.0 ? acc : 1.0;
    prior_ok = (double)u < pa;
  }
  int energy_ok = En < emax;
  int acc = energy_ok && valid && prior_ok;
  *reason = acc ? 0 : (!energy_ok ? 1 : (!valid ? 2 : 3));
  if (acc) {
    memcpy(cell, nc, sizeof(nc));
    memcpy(x, nx, sizeof(float) * 3 * n);
    *energy = En;
  }
  free(nx);
  return acc;
}

/* Cell move common tail (sampling/moves/_common.py:16-93 without a prior):
 * positions x' = x . T, one energy, the cell-geometry guard, accept iff the
 * energy is under the contour and the cell is valid (reason energy > cell). */
static int cell_move_finish(const JroModel* mdl, const JroMoves* mv, int mode, double emax,
                            int n, float* x, int32_t* t, float* cell, double* energy,
                            float P, const float* mu, int has_mu, const float* nc,
                            const float* T, int* reason) {
  float* nx = (float*)malloc(sizeof(float) * 3 * n);
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < 3; ++q) {
      const float* xi = x + 3 * i;
      nx[3 * i + q] = mode == JRO_REF32
                          ? xi[0] * T[q] + xi[1] * T[3 + q] + xi[2] * T[6 + q]
                          : fmaf(xi[2], T[6 + q], fmaf(xi[1], T[3 + q], xi[0] * T[q]));
    }
  double En = eval_energy(mdl, mode, n, nx, t, nc, P, mu, has_mu, NULL);
  int valid = cell_valid(nc, n, mv->max_vpa, mv->min_vpa, mv->min_aspect, mode);
  int energy_ok = En < emax;
  int acc = energy_ok && valid;
  *reason = acc ? 0 : (!energy_ok ? 1 : 2);
  if (acc) {
    memcpy(cell, nc, sizeof(float) * 9);
    memcpy(x, nx, sizeof(float) * 3 * n);
    *energy = En;
  }
  free(nx);
  return acc;
}

/* shear (sampling/moves/shear.py:18-127): row a = randint(k1, 0, 3) moves by
 * rv1 v1n + rv2 v2n in the plane of the other two rows (v1n the first of them
 * normalised, v2n the second orthogonalised against it and normalised),
 * (rv1, rv2) = step * normal(k2, (2,)); T = solve(old, new) in float64. */
static int move_shear(const JroModel* mdl, const JroMoves* mv, int mode, const uint32_t key[2],
                      float step, double emax, int n, float* x, int32_t* t, float* cell,
                      double* energy, float P, const float* mu, int has_mu, int* reason) {
  uint32_t k1[2], k2[2];
  jro_split(key, 0, k1);
  jro_split(key, 1, k2);
  const int a = jro_randint(k1, 0, 3);
  const float rv1 = step * jro_normal(jro_bits32(k2, 0));
  const float rv2 = step * jro_normal(jro_bits32(k2, 1));
  const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
  const float* v1 = cell + 3 * b;
  const float* v2 = cell + 3 * c;
  float v1n[3], v2p[3], v2n[3];
  const float n1 = vnorm(v1, 3, mode);
  for (int k = 0; k < 3; ++k) v1n[k] = v1[k] / n1;
  float dot;
  if (mode == JRO_REF32) {
    dot = v2[0] * v1n[0] + v2[1] * v1n[1] + v2[2] * v1n[2];
  } else {
    double d = 0.0;
    for (int k = 0; k < 3; ++k) d += (double)v2[k] * (double)v1n[k];
    dot = (float)d;
  }
  for (int k = 0; k < 3; ++k)
    v2p[k] = mode == JRO_REF32 ? v2[k] - dot * v1n[k] : fmaf(-dot, v1n[k], v2[k]);
  const float n2 = vnorm(v2p, 3, mode);
  for (int k = 0; k < 3; ++k) v2n[k] = v2p[k] / n2;
  float nc[9];
  memcpy(nc, cell, sizeof(nc));
  for (int k = 0; k < 3; ++k)
    nc[3 * a + k] = mode == JRO_REF32 ? cell[3 * a + k] + rv1 * v1n[k] + rv2 * v2n[k]
                                      : fmaf(rv2, v2n[k], fmaf(rv1, v1n[k], cell[3 * a + k]));
  double o[9], inv[9];
  for (int q = 0; q < 9; ++q) o[q] = (double)cell[q];
  inv_cell_f64(o, inv);
  float T[9];
  for (int k = 0; k < 3; ++k)
    for (int q = 0; q < 3; ++q) {
      double v = 0.0;
      for (int m = 0; m < 3; ++m) v += inv[3 * k + m] * (double)nc[3 * m + q];
      T[3 * k + q] = (float)v;
    }
  return cell_move_finish(mdl, mv, mode, emax, n, x, t, cell, energy, P, mu, has_mu, nc, T,
                          reason);
}

/* stretch (sampling/moves/stretch.py:18-104): axes (i, j) = [(0,1), (0,2),
 * (1,2)][randint(k1, 0, 3)], rv = step * normal(k2); T = diag with
 * exp(rv) at i and exp(-rv) at j (float64 exp rounded to float32);
 * new cell = cell . T, positions x . T. */
static int move_stretch(const JroModel* mdl, const JroMoves* mv, int mode, const uint32_t key[2],
                        float step, double emax, int n, float* x, int32_t* t, float* cell,
                        double* energy, float P, const float* mu, int has_mu, int* reason) {
  uint32_t k1[2], k2[2];
  jro_split(key, 0, k1);
  jro_split(key, 1, k2);
  const int pr = jro_randint(k1, 0, 3);
  const int ai = pr == 2 ? 1 : 0, aj = pr == 0 ? 1 : 2;
  const float rv = step * jro_normal(jro_bits32(k2, 0));
  float dg[3] = {1.0f, 1.0f, 1.0f};
  dg[ai] = (float)exp((double)rv);
  dg[aj] = (float)exp(-(double)rv);
  float T[9] = {0}, nc[9];
  for (int k = 0; k < 3; ++k) T[4 * k] = dg[k];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) nc[3 * r + q] = cell[3 * r + q] * dg[q];
  return cell_move_finish(mdl, mv, mode, emax, n, x, t, cell, energy, P, mu, has_mu, nc, T,
                          reason);
}

/* alchemical_morph (sampling/moves/alchemical.py:40-79). */
static int move_morph(const JroModel* mdl, int mode, const uint32_t key[2],
                      double emax, int n, float* x, int32_t* t, float* cell,
                      double* energy, float P, const float* mu, int has_mu) {
  uint32_t ka[2], ks[2];
  jro_split(key, 0, ka);
  jro_split(key, 1, ks);
  int atom = jro_randint(ka, 0, n);
  int cur = t[atom];
  int cand = jro_randint(ks, 0, mdl->n_species - 1);
  int nt = cand + (cand >= cur ? 1 : 0);
  int32_t* tt = (int32_t*)malloc(sizeof(int32_t) * n);
  memcpy(tt, t, sizeof(int32_t) * n);
  tt[atom] = nt;
  double En = eval_energy(mdl, mode, n, x, tt, cell, P, mu, has_mu, NULL);
  int acc = En < emax;
  if (acc) {
    memcpy(t, tt, sizeof(int32_t) * n);
    *energy = En;
  }
  free(tt);
  return acc;
}

/* species_swap over every species (sampling/moves/swap.py:177-260). */
static int move_swap(const JroModel* mdl, int mode, const uint32_t key[2],
                     double emax, int n, float* x, int32_t* t, float* cell,
                     double* energy, float P, const float* mu, int has_mu) {
  const int S = mdl->n_species;
  uint32_t kp[2], klo[2], khi[2];
  jro_split(key, 0, kp);
  jro_split(key, 1, klo);
  jro_split(key, 2, khi);
  int counts[JRO_MAX_SPECIES] = {0};
  for (int i = 0; i < n; ++i) counts[t[i]]++;
  int plo[JRO_MAX_SPECIES * JRO_MAX_SPECIES], phi[JRO_MAX_SPECIES * JRO_MAX_SPECIES];
  int np = 0;
  for (int a = 0; a < S; ++a)
    for (int b = 0; b < S; ++b)
      if (a < b) { plo[np] = a; phi[np] = b; ++np; }
  float cum[JRO_MAX_SPECIES * JRO_MAX_SPECIES];
  float total = 0.0f;
  for (int p = 0; p < np; ++p) {
    float w = (float)(counts[plo[p]] * counts[phi[p]]);
    total = total + w;
    cum[p] = total;
  }
  int has_pair = total > 0.0f;
  float u = jro_uniform(jro_bits32(kp, 0), 0.0f, 1.0f) * (has_pair ? total : 1.0f);
  int pidx = 0;
  while (pidx < np && cum[pidx] <= u) ++pidx; /* searchsorted side='right' */
  if (pidx > np - 1) pidx = np - 1;
  int clo = plo[pidx], chi = phi[pidx];
  int klo_i = jro_randint(klo, 0, counts[clo] > 1 ? counts[clo] : 1);
  int khi_i = jro_randint(khi, 0, counts[chi] > 1 ? counts[chi] : 1);
  int ilo = n - 1, ihi = n - 1, run = 0;
  for (int i = 0; i < n; ++i) {
    run += (t[i] == clo);
    if (run >= klo_i + 1) { ilo = i; break; }
  }
  run = 0;
  for (int i = 0; i < n; ++i) {
    run += (t[i] == chi);
    if (run >= khi_i + 1) { ihi = i; break; }
  }
  int32_t* tt = (int32_t*)malloc(sizeof(int32_t) * n);
  memcpy(tt, t, sizeof(int32_t) * n);
  tt[ilo] = chi;
  tt[ihi] = clo;
  double En = eval_energy(mdl, mode, n, x, tt, cell, P, mu, has_mu, NULL);
  int acc = (En < emax) && has_pair;
  if (acc) {
    memcpy(t, tt, sizeof(int32_t) * n);
    *energy = En;
  }
  free(tt);
  return acc;
}

static double round_energy(double e, int mode) {
  return mode == JRO_REF32 ? (double)(float)e : e;
}

/* Minimum-distance predicate (constraints/min_distance.py:25-47, MIC of
 * backends/geometry.py:18-69): periodic iff |det(cell)| > 1e-10, fractional
 * f = x . inv(cell), df = f_i - f_j - rint(f_i - f_j), delta = df . cell
 * (the pair-MIC FMA order; plain products in REF32), else the raw
 * difference; violated when sqrt(|delta|^2) < dmin[t_i][t_j], i != j. */
int32_t jro_min_distance_ok(const JroMoves* mv, int32_t S, int32_t n, const float* x,
                            const int32_t* t, const float* cell, int32_t mode) {
  const int periodic = fabsf(jro_det3(cell)) > 1e-10f;
  float inv[9];
  if (periodic) jro_inv_cell(cell, inv);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      float dd[3];
      if (periodic) {
        float fa[3], fb[3], df[3];
        for (int k = 0; k < 3; ++k) {
          if (mode == JRO_REF32) {
            fa[k] = x[3 * i] * inv[k] + x[3 * i + 1] * inv[3 + k] + x[3 * i + 2] * inv[6 + k];
            fb[k] = x[3 * j] * inv[k] + x[3 * j + 1] * inv[3 + k] + x[3 * j + 2] * inv[6 + k];
          } else {
            fa[k] = fmaf(x[3 * i + 2], inv[6 + k], fmaf(x[3 * i + 1], inv[3 + k], x[3 * i] * inv[k]));
            fb[k] = fmaf(x[3 * j + 2], inv[6 + k], fmaf(x[3 * j + 1], inv[3 + k], x[3 * j] * inv[k]));
          }
          df[k] = fa[k] - fb[k];
          df[k] = df[k] - rintf(df[k]);
        }
        for (int k = 0; k < 3; ++k)
          dd[k] = mode == JRO_REF32
                      ? df[0] * cell[k] + df[1] * cell[3 + k] + df[2] * cell[6 + k]
                      : fmaf(df[2], cell[6 + k], fmaf(df[1], cell[3 + k], df[0] * cell[k]));
      } else {
        for (int k = 0; k < 3; ++k) dd[k] = x[3 * i + k] - x[3 * j + k];
      }
      const float r2 = mode == JRO_REF32 ? dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]
                                         : fmaf(dd[2], dd[2], fmaf(dd[1], dd[1], dd[0] * dd[0]));
      if (sqrtf(r2) < mv->dmin[t[i] * S + t[j]]) return 0;
    }
  return 1;
}

int32_t jro_move_trial(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                       int32_t move_idx, const uint32_t key[2], float step,
                       double emax, int32_t n, float* x, float* d, int32_t* t,
                       float* cell, double* energy, float P, const float* mu,
                       int32_t has_mu, int32_t* reason_out) {
  int reason = 0, acc = 0;
  const int gated = mv->gate[move_idx] != 0;
  float* xs = NULL;
  int32_t* ts = NULL;
  float cs[9];
  double es = *energy;
  if (gated) {
    xs = (float*)malloc(sizeof(float) * 3 * n);
    ts = (int32_t*)malloc(sizeof(int32_t) * n);
    memcpy(xs, x, sizeof(float) * 3 * n);
    memcpy(ts, t, sizeof(int32_t) * n);
    memcpy(cs, cell, sizeof(cs));
  }
  switch (mv->type[move_idx]) {
    case JRO_MOVE_GALILEAN:
      acc = move_galilean(mdl, mode, key, step, mv->n_reflect[move_idx],
                          mv->perturb_angle[move_idx], emax, n, x, d, t, cell,
                          energy, P, mu, has_mu);
      break;
    case JRO_MOVE_VOLUME:
      acc = move_volume(mdl, mv, mode, key, step, emax, n, x, t, cell, energy,
                        P, mu, has_mu, &reason);
      break;
    case JRO_MOVE_MORPH:
      acc = move_morph(mdl, mode, key, emax, n, x, t, cell, energy, P, mu, has_mu);
      break;
    case JRO_MOVE_SWAP:
      acc = move_swap(mdl, mode, key, emax, n, x, t, cell, energy, P, mu, has_mu);
      reason = acc ? 0 : 1;
      break;
    case JRO_MOVE_SHEAR:
      acc = move_shear(mdl, mv, mode, key, step, emax, n, x, t, cell, energy, P, mu, has_mu,
                       &reason);
      break;
    case JRO_MOVE_STRETCH:
      acc = move_stretch(mdl, mv, mode, key, step, emax, n, x, t, cell, energy, P, mu, has_mu,
                         &reason);
      break;
  }
  *energy = round_energy(*energy, mode);
  if (gated) {
    /* mwg.py _wrap: an accepted violating move is undone (positions, cell,
     * types, energy; the direction is kept) with reject reason 4 */
    if (acc && !jro_min_distance_ok(mv, mdl->n_species, n, x, t, cell, mode)) {
      memcpy(x, xs, sizeof(float) * 3 * n);
      memcpy(t, ts, sizeof(int32_t) * n);
      memcpy(cell, cs, sizeof(cs));
      *energy = es;
      acc = 0;
      reason = 4;
    }
    free(xs);
    free(ts);
  }
  if (reason_out) *reason_out = reason;
  return acc;
}

/* build_mwg.step_fn (sampling/mwg.py:227-257) + _wrap (mwg.py:108-150). */
int32_t jro_mwg_step(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                     const uint32_t step_key[2], const uint32_t move_key[2],
                     double emax, int32_t n, float* x, float* d, int32_t* t,
                     float* cell, double* energy, const float* step_sizes,
                     int32_t* n_acc, int32_t* n_prop, float P, const float* mu,
                     int32_t has_mu, int32_t* move_idx_out, int32_t* reason_out,
                     int32_t* n_evals_out, int32_t* n_grad_out) {
  int idx = jro_choice(move_key, mv->cum_probs, mv->n_moves);
  int reason = 0;
  int acc = jro_move_trial(mdl, mv, mode, idx, step_key, step_sizes[idx], emax,
                           n, x, d, t, cell, energy, P, mu, has_mu, &reason);
  n_prop[idx] += 1;
  n_acc[idx] += acc;
  *move_idx_out = idx;
  *reason_out = reason;
  int ne = 1, ng = 0;
  if (mv->type[idx] == JRO_MOVE_GALILEAN) { ne = mv->n_reflect[idx]; ng = ne; }
  *n_evals_out = ne;
  *n_grad_out = ng;
  return acc;
}

/* ------------------------------------------------------------------ */
/* ns_step (sampling/nested_sampling.py:391-686)                        */
/* ------------------------------------------------------------------ */

static double logaddexp(double a, double b) {
  double amax = a > b ? a : b;
  double delta = a - b;
  if (isnan(delta)) return a + b;
  return amax + log1p(exp(-fabs(delta)));
}

static void copy_walker(JroReplica* r, int dst, int src, int M) {
  const int N = r->n_atoms;
  memcpy(r->positions + (size_t)dst * 3 * N, r->positions + (size_t)src * 3 * N, sizeof(float) * 3 * N);
  memcpy(r->direction + (size_t)dst * 3 * N, r->direction + (size_t)src * 3 * N, sizeof(float) * 3 * N);
  memcpy(r->types + (size_t)dst * N, r->types + (size_t)src * N, sizeof(int32_t) * N);
  memcpy(r->cell + (size_t)dst * 9, r->cell + (size_t)src * 9, sizeof(float) * 9);
  memcpy(r->step_sizes + (size_t)dst * M, r->step_sizes + (size_t)src * M, sizeof(float) * M);
  r->energy[dst] = r->energy[src];
}

/* jax.random.permutation of an array (jax/_src/random.py _shuffle, a
 * published algorithm): num_rounds = ceil(3 ln(max(1,n)) / ln(2^32 - 1))
 * rounds, each splitting the key (key, subkey = split(key)) and stably
 * sorting the array by 32-bit random_bits(subkey, 32, (n,)). */
static void jax_shuffle(const uint32_t key_in[2], int32_t* x, int n) {
  uint32_t key[2] = {key_in[0], key_in[1]};
  const int rounds = (int)ceil(3.0 * log((double)(n > 1 ? n : 1)) / log(4294967295.0));
  uint32_t* u = (uint32_t*)malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
  int32_t* y = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  for (int r = 0; r < rounds; ++r) {
    uint32_t nk[2], sub[2];
    jro_split(key, 0, nk);
    jro_split(key, 1, sub);
    key[0] = nk[0];
    key[1] = nk[1];
    for (int m = 0; m < n; ++m) u[m] = jro_bits32(sub, (uint32_t)m);
    for (int m = 0; m < n; ++m) {  /* stable: rank by (u, position) */
      int pos = 0;
      for (int q = 0; q < n; ++q)
        if (u[q] < u[m] || (u[q] == u[m] && q < m)) ++pos;
      y[pos] = x[m];
    }
    memcpy(x, y, sizeof(int32_t) * n);
  }
  free(u);
  free(y);
}

/* lexsort((-noise, -E)) order key: energies descending (NaN last, as in
 * XLA's float sort), then noise descending, then index ascending. */
static int cull_before(const double* E, const float* nz, int j, int k) {
  const int nj = isnan(E[j]), nk = isnan(E[k]);
  if (nj != nk) return nk;
  if (!nj && E[j] != E[k]) return E[j] > E[k];
  if (nz[j] != nz[k]) return nz[j] > nz[k];
  return j < k;
}

static double logsumexp_d(const double* v, int n) {
  double amax = -INFINITY;
  for (int i = 0; i < n; ++i)
    if (v[i] > amax || isnan(v[i])) amax = v[i];
  if (!isfinite(amax)) amax = 0.0;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += exp(v[i] - amax);
  return log(s) + amax;
}

void jro_ns_step_n(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                   JroReplica* rep, int32_t T, int32_t n_cull, int32_t n_extra,
                   const uint32_t* move_key_in, double log_alpha,
                   const double* w_offsets, JroIterInfo* info, int32_t* worst_out,
                   int32_t* clone_out, double* dead_E_out, float* dead_x,
                   int32_t* dead_t, float* dead_c) {
  const int K = rep->n_walkers, N = rep->n_atoms, M = mv->n_moves;
  uint32_t key[2] = {rep->rng_key[0], rep->rng_key[1]};
  uint32_t k_a[2], k_worst[2], k_next[2], k_clone[2], k_extra[2], k_mcmc[2], k_moves[2];
  jro_split(key, 0, k_a);
  jro_split(key, 1, k_worst);
  jro_split(k_a, 0, k_next);
  jro_split(k_a, 1, k_clone);
  jro_split(k_a, 2, k_extra);
  jro_split(k_a, 3, k_mcmc);
  jro_split(k_a, 4, k_moves);
  uint32_t move_key[2];
  if (move_key_in) { move_key[0] = move_key_in[0]; move_key[1] = move_key_in[1]; }
  else { move_key[0] = k_moves[0]; move_key[1] = k_moves[1]; }
  const int W = n_cull + n_extra;
  int* worst = (int*)malloc(sizeof(int) * n_cull);
  int* clone = (int*)malloc(sizeof(int) * n_cull);
  int* walk = (int*)malloc(sizeof(int) * W);
  double emax;
  if (n_cull == 1) {
    /* _find_worst_walker (nested_sampling.py:86-109): jnp.max propagates NaN */
    emax = rep->energy[0];
    int any_nan = 0;
    for (int k = 0; k < K; ++k) {
      if (isnan(rep->energy[k])) any_nan = 1;
      if (rep->energy[k] > emax) emax = rep->energy[k];
    }
    if (any_nan) emax = NAN;
    int w0 = 0;
    float best = -INFINITY;
    int found = 0;
    for (int k = 0; k < K; ++k) {
      if (rep->energy[k] == emax) {
        float nz = jro_uniform(jro_bits32(k_worst, (uint32_t)k), 0.0f, 1.0f);
        if (!found || nz > best) { best = nz; w0 = k; found = 1; }
      }
    }
    /* clone (nested_sampling.py:182-183) */
    int c0 = jro_randint(k_clone, 0, K - 1);
    if (c0 >= w0) c0 += 1;
    worst[0] = w0;
    clone[0] = c0;
    walk[0] = w0;
    /* extras (nested_sampling.py:112-133): stable argsort of -noise */
    if (n_extra > 0) {
      float* nz = (float*)malloc(sizeof(float) * K);
      for (int k = 0; k < K; ++k) nz[k] = jro_uniform(jro_bits32(k_extra, (uint32_t)k), 0.0f, 1.0f);
      nz[w0] = -INFINITY;
      nz[c0] = -INFINITY;
      char* used = (char*)calloc(K, 1);
      for (int e = 0; e < n_extra; ++e) {
        int bi = -1;
        for (int k = 0; k < K; ++k)
          if (!used[k] && (bi < 0 || nz[k] > nz[bi])) bi = k;
        used[bi] = 1;
        walk[1 + e] = bi;
      }
      free(used);
      free(nz);
    }
  } else {
    /* _select_culls n_cull > 1 (nested_sampling.py:195-212): order =
     * lexsort((-noise, -E)); worst = order[:n_cull]; survivors =
     * permutation(key_clone, order[n_cull:]); clone = survivors[:n_cull];
     * extras = survivors[n_cull:n_cull + n_extra]. */
    float* nz = (float*)malloc(sizeof(float) * K);
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * K);
    for (int k = 0; k < K; ++k) nz[k] = jro_uniform(jro_bits32(k_worst, (uint32_t)k), 0.0f, 1.0f);
    for (int k = 0; k < K; ++k) {
      int r = 0;
      for (int j = 0; j < K; ++j)
        if (j != k && cull_before(rep->energy, nz, j, k)) ++r;
      order[r] = k;
    }
    for (int c = 0; c < n_cull; ++c) worst[c] = order[c];
    emax = rep->energy[worst[n_cull - 1]];
    jax_shuffle(k_clone, order + n_cull, K - n_cull);
    for (int c = 0; c < n_cull; ++c) {
      clone[c] = order[n_cull + c];
      walk[c] = worst[c];
    }
    for (int e = 0; e < n_extra; ++e) walk[n_cull + e] = order[2 * n_cull + e];
    free(nz);
    free(order);
  }
  /* dead walkers + evidence (nested_sampling.py:486-501) */
  double* lw = (double*)malloc(sizeof(double) * n_cull);
  for (int c = 0; c < n_cull; ++c) {
    const int wc = worst[c];
    const double dE = rep->energy[wc];
    if (dead_E_out) dead_E_out[c] = dE;
    if (dead_x) memcpy(dead_x + (size_t)c * 3 * N, rep->positions + (size_t)wc * 3 * N, sizeof(float) * 3 * N);
    if (dead_t) memcpy(dead_t + (size_t)c * N, rep->types + (size_t)wc * N, sizeof(int32_t) * N);
    if (dead_c) memcpy(dead_c + (size_t)c * 9, rep->cell + (size_t)wc * 9, sizeof(float) * 9);
    lw[c] = (double)(*rep->iteration) * log_alpha + w_offsets[c] - dE;
  }
  const double dead_E0 = rep->energy[worst[0]];
  *rep->log_evidence = n_cull == 1 ? logaddexp(*rep->log_evidence, lw[0])
                                   : logaddexp(*rep->log_evidence, logsumexp_d(lw, n_cull));
  free(lw);
  /* clones into the culled slots, counters reset (nested_sampling.py:504-518) */
  for (int c = 0; c < n_cull; ++c) {
    copy_walker(rep, worst[c], clone[c], M);
    for (int m = 0; m < M; ++m) {
      rep->n_acc[(size_t)worst[c] * M + m] = 0;
      rep->n_prop[(size_t)worst[c] * M + m] = 0;
    }
  }
  memset(info, 0, sizeof(*info));
  info->worst_idx = worst[0];
  info->clone_idx = clone[0];
  info->emax = emax;
  info->dead_energy = dead_E0;
  if (worst_out) memcpy(worst_out, worst, sizeof(int) * n_cull);
  if (clone_out) memcpy(clone_out, clone, sizeof(int) * n_cull);
  /* walk W chains of T steps (nested_sampling.py:524-628) */
  for (int w = 0; w < W; ++w) {
    uint32_t ck[2];
    jro_split(k_mcmc, (uint32_t)w, ck);
    const int s = walk[w];
    float* x = rep->positions + (size_t)s * 3 * N;
    float* d = rep->direction + (size_t)s * 3 * N;
    int32_t* t = rep->types + (size_t)s * N;
    float* c = rep->cell + (size_t)s * 9;
    for (int step = 0; step < T; ++step) {
      uint32_t sk[2], mk[2];
      jro_split(ck, (uint32_t)step, sk);
      jro_split(move_key, (uint32_t)step, mk);
      int midx, reason, ne, ng;
      int acc = jro_mwg_step(mdl, mv, mode, sk, mk, emax, N, x, d, t, c,
                             &rep->energy[s], rep->step_sizes + (size_t)s * M,
                             rep->n_acc + (size_t)s * M, rep->n_prop + (size_t)s * M,
                             rep->pressure, rep->mu, rep->has_mu, &midx, &reason,
                             &ne, &ng);
      info->n_acc[midx] += acc;
      info->n_prop[midx] += 1;
      int col = acc ? 0 : (reason > 1 ? reason : 1);
      if (col < 4) info->rr[midx * 4 + col] += 1;  /* reason 4 is dropped */
      info->n_evals[midx] += ne;
      info->n_grad[midx] += ng;
      info->total_accepted += acc;
    }
  }
  free(worst);
  free(clone);
  free(walk);
  *rep->emax = emax;
  *rep->iteration += 1;
  rep->rng_key[0] = k_next[0];
  rep->rng_key[1] = k_next[1];
}

void jro_ns_step(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                 JroReplica* rep, int32_t T, int32_t n_extra,
                 const uint32_t* move_key_in, double log_alpha, double w_offset,
                 JroIterInfo* info, float* dead_x, int32_t* dead_t,
                 float* dead_c) {
  jro_ns_step_n(mdl, mv, mode, rep, T, 1, n_extra, move_key_in, log_alpha, &w_offset, info,
                NULL, NULL, NULL, dead_x, dead_t, dead_c);
}

/* _one_walk (init/burn_in.py:48-127) for one run: walker k takes walklength
 * MWG steps under the fixed contour emax with chain keys
 * split(split(run_key, K)[k], walklength) and the shared move schedule
 * split(move_key, walklength); its own step sizes, counters advanced. */
void jro_walk_population(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                         JroReplica* rep, int32_t walklength, const uint32_t run_key[2],
                         const uint32_t move_key[2], double emax) {
  const int K = rep->n_walkers, N = rep->n_atoms, M = mv->n_moves;
  for (int k = 0; k < K; ++k) {
    uint32_t ck[2];
    jro_split(run_key, (uint32_t)k, ck);
    float* x = rep->positions + (size_t)k * 3 * N;
    float* d = rep->direction + (size_t)k * 3 * N;
    int32_t* t = rep->types + (size_t)k * N;
    float* c = rep->cell + (size_t)k * 9;
    for (int step = 0; step < walklength; ++step) {
      uint32_t sk[2], mk[2];
      jro_split(ck, (uint32_t)step, sk);
      jro_split(move_key, (uint32_t)step, mk);
      int midx, reason, ne, ng;
      jro_mwg_step(mdl, mv, mode, sk, mk, emax, N, x, d, t, c, &rep->energy[k],
                   rep->step_sizes + (size_t)k * M, rep->n_acc + (size_t)k * M,
                   rep->n_prop + (size_t)k * M, rep->pressure, rep->mu, rep->has_mu,
                   &midx, &reason, &ne, &ng);
    }
  }
}

typedef struct {
  const JroModel* mdl; const JroMoves* mv; int32_t mode; JroReplica* reps;
  int32_t n_reps, T, n_extra; const uint32_t* mk; double log_alpha, w_offset;
  JroIterInfo* infos; int32_t stride, first;
} BatchArg;

static void* batch_worker(void* p) {
  BatchArg* a = (BatchArg*)p;
  for (int r = a->first; r < a->n_reps; r += a->stride)
    jro_ns_step(a->mdl, a->mv, a->mode, &a->reps[r], a->T, a->n_extra, a->mk,
                a->log_alpha, a->w_offset, &a->infos[r], NULL, NULL, NULL);
  return NULL;
}

/* Replicas are independent within one iteration: one pthread per slice. */
void jro_ns_step_batched(const JroModel* mdl, const JroMoves* mv, int32_t mode,
                         JroReplica* reps, int32_t n_reps, int32_t T,
                         int32_t n_extra, int32_t shared_move_key,
                         double log_alpha, double w_offset, JroIterInfo* infos,
                         int32_t n_threads) {
  uint32_t mk[2];
  if (shared_move_key) jro_fold_in(reps[0].rng_key, 1u, mk);
  int nt = n_threads > 0 ? n_threads : 1;
  if (nt > n_reps) nt = n_reps;
  if (nt > 256) nt = 256;
  pthread_t th[256];
  BatchArg args[256];
  for (int i = 0; i < nt; ++i) {
    BatchArg a = {mdl, mv, mode, reps, n_reps, T, n_extra,
                  shared_move_key ? mk : NULL, log_alpha, w_offset, infos, nt, i};
    args[i] = a;
  }
  for (int i = 1; i < nt; ++i) pthread_create(&th[i], NULL, batch_worker, &args[i]);
  batch_worker(&args[0]);
  for (int i = 1; i < nt; ++i) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------ */
/* Pressure / semi-grand replica exchange                              */
/* (sampling/moves/replica_exchange.py:318-436, EnsembleSwap :120-156) */
/* ------------------------------------------------------------------ */

static double ens_energy(const JroReplica* r, const float* cell,
                         const int32_t* t, int n, int S, int mode) {
  int32_t counts[JRO_MAX_SPECIES] = {0};
  for (int i = 0; i < n; ++i) counts[t[i]]++;
  float V = fabsf(jro_det3(cell));
  if (mode == JRO_REF32) {
    float e = r->pressure * V;
    if (r->has_mu) {
      float dot = 0.0f;
      for (int s = 0; s < S; ++s) dot = dot + r->mu[s] * (float)counts[s];
      e = e - dot;
    }
    return (double)e;
  }
  double e = (double)r->pressure * (double)V;
  if (r->has_mu) {
    double dot = 0.0;
    for (int s = 0; s < S; ++s) dot += (double)r->mu[s] * (double)counts[s];
    e = e - dot;
  }
  return e;
}

static double rebase(double E, const JroReplica* from, const JroReplica* to,
                     const float* cell, const int32_t* t, int n, int S, int mode) {
  double u = E - ens_energy(from, cell, t, n, S, mode);
  if (mode == JRO_REF32) u = (double)(float)u;
  double out = u + ens_energy(to, cell, t, n, S, mode);
  if (mode == JRO_REF32) out = (double)(float)out;
  return out;
}

static void swap_slot(JroReplica* a, int wa, JroReplica* b, int wb, double Ea,
                      double Eb) {
  const int N = a->n_atoms;
  float tx[3 * 1024];
  int32_t tt[1024];
  float tc[9];
  /* positions */
  memcpy(tx, a->positions + (size_t)wa * 3 * N, sizeof(float) * 3 * N);
  memcpy(a->positions + (size_t)wa * 3 * N, b->positions + (size_t)wb * 3 * N, sizeof(float) * 3 * N);
  memcpy(b->positions + (size_t)wb * 3 * N, tx, sizeof(float) * 3 * N);
  memcpy(tx, a->direction + (size_t)wa * 3 * N, sizeof(float) * 3 * N);
  memcpy(a->direction + (size_t)wa * 3 * N, b->direction + (size_t)wb * 3 * N, sizeof(float) * 3 * N);
  memcpy(b->direction + (size_t)wb * 3 * N, tx, sizeof(float) * 3 * N);
  memcpy(tt, a->types + (size_t)wa * N, sizeof(int32_t) * N);
  memcpy(a->types + (size_t)wa * N, b->types + (size_t)wb * N, sizeof(int32_t) * N);
  memcpy(b->types + (size_t)wb * N, tt, sizeof(int32_t) * N);
  memcpy(tc, a->cell + (size_t)wa * 9, sizeof(tc));
  memcpy(a->cell + (size_t)wa * 9, b->cell + (size_t)wb * 9, sizeof(tc));
  memcpy(b->cell + (size_t)wb * 9, tc, sizeof(tc));
  a->energy[wa] = Ea;
  b->energy[wb] = Eb;
}

void jro_re_step(JroReplica* reps, int32_t R, const uint32_t key[2],
                 int32_t n_cycles, int32_t mode, int32_t* acc_pp,
                 int32_t* att_pp) {
  if (R < 2) return;
  const int K = reps[0].n_walkers;
  const int n_even = (R - 1 + 1) / 2;       /* len(range(0, R-1, 2)) */
  const int n_odd = (R - 1) / 2;            /* len(range(1, R-1, 2)) */
  const int max_pairs = n_even > n_odd ? n_even : n_odd;
  for (int p = 0; p < R - 1; ++p) { acc_pp[p] = 0; att_pp[p] = 0; }
  for (int cyc = 0; cyc < n_cycles; ++cyc) {
    uint32_t ck[2];
    jro_split(key, (uint32_t)cyc, ck);
    for (int phase = 0; phase < 2; ++phase) {
      uint32_t pk[2];
      jro_split(ck, (uint32_t)phase, pk);
      const int n_valid = phase == 0 ? n_even : n_odd;
      for (int slot = 0; slot < max_pairs; ++slot) {
        uint32_t sk[2], k1[2], k2[2];
        jro_split(pk, (uint32_t)slot, sk);
        jro_split(sk, 0, k1);
        jro_split(sk, 1, k2);
        const int valid = slot < n_valid;
        const int ri = valid ? phase + 2 * slot : 0;
        const int rj = valid ? ri + 1 : 0;
        int wi = jro_randint(k1, 0, K);
        int wj = jro_randint(k2, 0, K);
        if (!valid) continue; /* padding entries never swap */
        JroReplica* A = &reps[ri];
        JroReplica* B = &reps[rj];
        const int N = A->n_atoms;
        int S = JRO_MAX_SPECIES;
        /* into_i = walker_j rebased into run i; into_j symmetric */
        double into_i = rebase(B->energy[wj], B, A, B->cell + (size_t)wj * 9,
                               B->types + (size_t)wj * N, N, S, mode);
        double into_j = rebase(A->energy[wi], A, B, A->cell + (size_t)wi * 9,
                               A->types + (size_t)wi * N, N, S, mode);
        int do_swap = (into_i < *A->emax) && (into_j < *B->emax);
        if (do_swap) swap_slot(A, wi, B, wj, into_i, into_j);
        acc_pp[ri] += do_swap;
        att_pp[ri] += 1;
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* Synthetic uniform-gas initial walkers                               */
/* ------------------------------------------------------------------ */
void jro_init_walkers(const uint32_t key[2], int32_t K, int32_t N, float v_hi,
                      float* positions, float* cell) {
  for (int k = 0; k < K; ++k) {
    uint32_t wk[2], kv[2], kp[2];
    jro_split(key, (uint32_t)k, wk);
    jro_split(wk, 0, kv);
    jro_split(wk, 1, kp);
    float u = jro_uniform(jro_bits32(kv, 0), 0.0f, 1.0f);
    float V = v_hi * (1.0f - u);
    float L = (float)pow((double)V, (double)(1.0f / 3.0f));
    float* c = cell + (size_t)k * 9;
    memset(c, 0, 9 * sizeof(float));
    c[0] = c[4] = c[8] = L;
    for (int i = 0; i < 3 * N; ++i) {
      float f = jro_uniform(jro_bits32(kp, (uint32_t)i), 0.0f, 1.0f);
      positions[(size_t)k * 3 * N + i] = f * L;
    }
  }
}
