// jr_sur.cu -- training kernels of the learned surrogate (jr_sur.cuh).
//
//   sur_descriptor_kernel  descriptors of a batch of configurations, one
//                          thread per atom summing its neighbours in
//                          ascending order (deterministic)
//   sur_train_kernel       fused forward + backward of the 16-64-64-1 network
//                          on the tensor cores (tcgen05.mma, bfloat16
//                          operands in shared memory, float32 accumulators in
//                          tensor memory), persistent CTAs over 128-row tiles
//                          (two 64-atom configurations per tile); the weight
//                          gradients accumulate in tensor memory across the
//                          CTA's tiles and leave as one partial per CTA
//   sur_adam_kernel        sums the partials in CTA order and takes an Adam
//                          step on the float32 master parameters
#include <cuda_runtime.h>

#include <string>

#include "../../include/jaxrens_b200.h"
#include "jr_host.cuh"
#include "jr_sur.cuh"

namespace jr {

// ------------------------------------------------------------ descriptors --

// One configuration per group of n threads (thread = atom i): D[i][k] over
// the neighbours j ascending, minimum image through the cell inverse.
__global__ void __launch_bounds__(128)
sur_descriptor_kernel(int n_configs, int n, const float* __restrict__ pos,
                      const float* __restrict__ cell, float* __restrict__ D) {
  const int per_block = blockDim.x / n;
  const int local = threadIdx.x / n, i = threadIdx.x % n;
  const int b = blockIdx.x * per_block + local;
  if (local >= per_block || b >= n_configs) return;
  const float* h = cell + (size_t)b * 9;
  // inverse of the cell (double adjugate), rows are lattice vectors
  double a[9], cof[9];
  for (int q = 0; q < 9; ++q) a[q] = h[q];
  cof[0] = a[4] * a[8] - a[5] * a[7];
  cof[1] = a[5] * a[6] - a[3] * a[8];
  cof[2] = a[3] * a[7] - a[4] * a[6];
  cof[3] = a[2] * a[7] - a[1] * a[8];
  cof[4] = a[0] * a[8] - a[2] * a[6];
  cof[5] = a[1] * a[6] - a[0] * a[7];
  cof[6] = a[1] * a[5] - a[2] * a[4];
  cof[7] = a[2] * a[3] - a[0] * a[5];
  cof[8] = a[0] * a[4] - a[1] * a[3];
  const double det = a[0] * cof[0] + a[1] * cof[1] + a[2] * cof[2];
  float inv[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) inv[r * 3 + c] = (float)(cof[c * 3 + r] / det);
  const float* x = pos + (size_t)b * n * 3;
  const float xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  float acc[kSurBasis];
#pragma unroll
  for (int k = 0; k < kSurBasis; ++k) acc[k] = 0.0f;
  for (int j = 0; j < n; ++j) {
    if (j == i) continue;
    float d[3] = {x[3 * j] - xi, x[3 * j + 1] - yi, x[3 * j + 2] - zi};
    float f[3];
    for (int q = 0; q < 3; ++q) f[q] = rintf(d[0] * inv[q] + d[1] * inv[3 + q] + d[2] * inv[6 + q]);
    for (int q = 0; q < 3; ++q) d[q] -= f[0] * h[q] + f[1] * h[3 + q] + f[2] * h[6 + q];
    const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (!(r2 < kSurRc * kSurRc)) continue;
    const float r = sqrtf(r2);
    float fc, dfc;
    sur_cutoff(r, fc, dfc);
#pragma unroll
    for (int k = 0; k < kSurBasis; ++k) {
      float phi, dphi;
      sur_basis(r, fc, dfc, k, phi, dphi);
      acc[k] += phi;
    }
  }
  float* out = D + ((size_t)b * n + i) * kSurBasis;
#pragma unroll
  for (int k = 0; k < kSurBasis; ++k) out[k] = acc[k];
}

// ------------------------------------------------- tensor-core primitives --

// Element index (bfloat16 units) of (row, col) in the K-major core-matrix
// layout of a tile with kdim columns: 8 x 8 cores of 128 contiguous bytes,
// [row group][column group][row][column].
__device__ __forceinline__ int core_idx(int row, int col, int kdim) {
  return (((row >> 3) * (kdim >> 3) + (col >> 3)) << 6) + ((row & 7) << 3) + (col & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all in 16-byte units), descriptor version 1.  For a
// K-major operand the leading offset steps between the two 8-element K
// chunks of an instruction and the stride offset between 8-row groups; for
// an MN-major operand the leading offset steps between 8-row K groups and
// the stride offset between 8-element MN chunks.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: bfloat16 A and B, float32 D, A/B
// K-major (0) or MN-major (1), shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                     int accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

// Bounded wait on an mbarrier phase.  Returns false (the caller flags an
// error and stops) if the phase does not complete within the limit.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < (1l << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive float32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// --------------------------------------------------------------- training --

constexpr int kTrainThreads = 128;  // one warpgroup: tensor-memory lanes 0..127 = tile rows
constexpr int kTmemCols = 256;
// tensor-memory columns of the accumulators
constexpr int kColZ = 0;      // Z1, then G1pre       (M=128, N=64)
constexpr int kColZ2 = 64;    // Z2                   (M=128, N=64)
constexpr int kColDW2 = 128;  // sum H1^T G2          (M=64,  N=64)
constexpr int kColDW1 = 192;  // sum G1^T X  (dW1^T)  (M=64,  N=16)
constexpr int kColDW3 = 208;  // sum H2^T E, col 0    (M=64,  N=16)
constexpr int kColDB2 = 224;  // sum G2^T E, col 1
constexpr int kColDB1 = 240;  // sum G1^T E, col 1
static_assert(kColDW3 == kColDW1 + 16 && kColDB1 == kColDB2 + 16, "epilogue reads pairs");
// shared-memory operand tiles (bytes from the 1024-aligned dynamic base)
constexpr int kSmX = 0, kSmE = 4096, kSmH1 = 8192, kSmH2 = 24576, kSmG2 = 40960, kSmG1 = 57344;
constexpr int kSmW1t = 73728, kSmW2t = 75776, kSmW2 = 83968, kSmBytes = 92160;

struct SurTrainArgs {
  const float* D;          // [*][64][16]
  const double* U;         // [*]
  const int32_t* idx;      // [n_batch]
  int n_batch;
  const float* params;     // [kSurParams]
  float in_scale[kSurBasis], in_shift[kSurBasis];
  float out_scale, out_shift;
  float* grad_part;        // [gridDim.x][kSurParams]
  float* loss_part;        // [gridDim.x]
  int* error;              // set to 1 if a tensor-core wait gave up
};

__global__ void __launch_bounds__(kTrainThreads, 1) sur_train_kernel(const SurTrainArgs A) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ float b1s[kSurHidden], b2s[kSurHidden], w3s[kSurHidden];
  __shared__ float cfg_sum[2][2];  // [configuration of the tile][warp of its half]
  __shared__ float red2[2][2];
  __shared__ int abort_flag;
  uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + kSmX);
  uint16_t* Es = reinterpret_cast<uint16_t*>(sm + kSmE);
  uint16_t* H1s = reinterpret_cast<uint16_t*>(sm + kSmH1);
  uint16_t* H2s = reinterpret_cast<uint16_t*>(sm + kSmH2);
  uint16_t* G2s = reinterpret_cast<uint16_t*>(sm + kSmG2);
  uint16_t* G1s = reinterpret_cast<uint16_t*>(sm + kSmG1);
  uint16_t* W1t = reinterpret_cast<uint16_t*>(sm + kSmW1t);
  uint16_t* W2t = reinterpret_cast<uint16_t*>(sm + kSmW2t);
  uint16_t* W2k = reinterpret_cast<uint16_t*>(sm + kSmW2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float* P = A.params;
  // weights into the K-major operand layouts
  for (int q = tid; q < kSurBasis * kSurHidden; q += kTrainThreads) {
    const int d = q / kSurHidden, h = q % kSurHidden;
    W1t[core_idx(h, d, kSurBasis)] = sur_bf16(P[kSurOffW1 + q]);  // B of x W1: [h][d]
  }
  for (int q = tid; q < kSurHidden * kSurHidden; q += kTrainThreads) {
    const int i = q / kSurHidden, o = q % kSurHidden;
    const uint16_t v = sur_bf16(P[kSurOffW2 + q]);
    W2t[core_idx(o, i, kSurHidden)] = v;  // B of h1 W2: [o][i]
    W2k[core_idx(i, o, kSurHidden)] = v;  // B of g2 W2^T: [i][o]
  }
  for (int q = tid; q < kSurHidden; q += kTrainThreads) {
    b1s[q] = P[kSurOffB1 + q];
    b2s[q] = P[kSurOffB2 + q];
    w3s[q] = P[kSurOffW3 + q];
  }
  const float b3 = P[kSurOffB3];
  if (tid == 0) {
    abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t mb = smem_u32(&mbar);
  const uint32_t sX = smem_u32(Xs), sE = smem_u32(Es), sH1 = smem_u32(H1s), sH2 = smem_u32(H2s);
  const uint32_t sG2 = smem_u32(G2s), sG1 = smem_u32(G1s);
  const uint32_t sW1t = smem_u32(W1t), sW2t = smem_u32(W2t), sW2k = smem_u32(W2k);
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  uint32_t phase = 0;
  bool ok = true;
  float loss = 0.0f, db3 = 0.0f;
  const int n_tiles = (A.n_batch + 1) / 2;
  int first = 1;
  // Thread 0 waits (bounded) for the committed products; the CTA barrier
  // then hands the verdict and the accumulators to every thread.
  auto wait_mma = [&]() {
    if (tid == 0 && !mbar_wait(mb, phase)) abort_flag = 1;
    phase ^= 1u;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    ok = abort_flag == 0;
  };
  for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
    // ---- X tile: row r = atom (r % 64) of configuration 2t + r / 64 ----
    const int c = tid >> 6;
    const bool valid = 2 * t + c < A.n_batch;
    const int cfg = valid ? A.idx[2 * t + c] : 0;
    const float* drow = A.D + ((size_t)cfg * 64 + (tid & 63)) * kSurBasis;
#pragma unroll
    for (int f = 0; f < kSurBasis; ++f) {
      const float xv = valid ? drow[f] * A.in_scale[f] + A.in_shift[f] : 0.0f;
      Xs[core_idx(tid, f, kSurBasis)] = sur_bf16(xv);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- Z1 = X W1 (M=128, N=64, K=16) ----
    if (tid == 0) {
      umma(tmem + kColZ, umma_desc(sX, 128, 256), umma_desc(sW1t, 128, 256),
           umma_idesc(128, 64, 0, 0), 0);
      umma_commit(mb);
    }
    wait_mma();
    if (!ok) break;
    float z1[kSurHidden];
    tmem_ld32(tmem + lane_base + kColZ, z1);
    tmem_ld32(tmem + lane_base + kColZ + 32, z1 + 32);
#pragma unroll
    for (int h = 0; h < kSurHidden; h += 2) {
      z1[h] += b1s[h];
      z1[h + 1] += b1s[h + 1];
      const uint32_t pk = sur_pack_bf16(sur_silu(z1[h]), sur_silu(z1[h + 1]));
      *reinterpret_cast<uint32_t*>(H1s + core_idx(tid, h, kSurHidden)) = pk;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- Z2 = H1 W2 (M=128, N=64, K=64: four k-steps of 16) ----
    if (tid == 0) {
      for (int s = 0; s < 4; ++s)
        umma(tmem + kColZ2, umma_desc(sH1 + 256 * s, 128, 1024),
             umma_desc(sW2t + 256 * s, 128, 1024), umma_idesc(128, 64, 0, 0), s > 0);
      umma_commit(mb);
    }
    wait_mma();
    if (!ok) break;
    float z2[kSurHidden];
    tmem_ld32(tmem + lane_base + kColZ2, z2);
    tmem_ld32(tmem + lane_base + kColZ2 + 32, z2 + 32);
    float e = b3;
#pragma unroll
    for (int h = 0; h < kSurHidden; h += 2) {
      z2[h] += b2s[h];
      z2[h + 1] += b2s[h + 1];
      const float a0 = sur_silu(z2[h]), a1 = sur_silu(z2[h + 1]);
      e = fmaf(a0, w3s[h], e);
      e = fmaf(a1, w3s[h + 1], e);
      *reinterpret_cast<uint32_t*>(H2s + core_idx(tid, h, kSurHidden)) = sur_pack_bf16(a0, a1);
    }
    // ---- per-configuration energies (rows 0..63, 64..127), loss gradient ----
    float es = e;
    for (int off = 16; off > 0; off >>= 1) es += __shfl_xor_sync(0xffffffffu, es, off);
    if (lane == 0) cfg_sum[warp >> 1][warp & 1] = es;
    __syncthreads();
    const float Epred = (cfg_sum[c][0] + cfg_sum[c][1]) * A.out_scale + 64.0f * A.out_shift;
    const float target = valid ? (float)A.U[cfg] : Epred;
    const float err = (Epred - target) / 64.0f;
    const float de = valid ? (2.0f * err / 64.0f / (float)A.n_batch) * A.out_scale : 0.0f;
    if (tid == 0 || tid == 64) {
      loss += valid ? err * err / (float)A.n_batch : 0.0f;
      db3 += 64.0f * de;
    }
#pragma unroll
    for (int h = 0; h < kSurHidden; h += 2) {
      const float g0 = de * w3s[h] * sur_dsilu(z2[h]);
      const float g1 = de * w3s[h + 1] * sur_dsilu(z2[h + 1]);
      *reinterpret_cast<uint32_t*>(G2s + core_idx(tid, h, kSurHidden)) = sur_pack_bf16(g0, g1);
    }
    // E: column 0 = de, column 1 = 1 (valid rows), the rest 0
#pragma unroll
    for (int f = 0; f < kSurBasis; f += 2) {
      const float v0 = f == 0 ? de : 0.0f;
      const float v1 = f == 0 ? (valid ? 1.0f : 0.0f) : 0.0f;
      *reinterpret_cast<uint32_t*>(Es + core_idx(tid, f, kSurBasis)) = sur_pack_bf16(v0, v1);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- G1pre = G2 W2^T; dW2 += H1^T G2; dW3 += H2^T E; db2 += G2^T E ----
    if (tid == 0) {
      for (int s = 0; s < 4; ++s)
        umma(tmem + kColZ, umma_desc(sG2 + 256 * s, 128, 1024),
             umma_desc(sW2k + 256 * s, 128, 1024), umma_idesc(128, 64, 0, 0), s > 0);
      for (int s = 0; s < 8; ++s) {
        const int acc = (first == 0) || (s > 0);
        // K = 16 tile rows per step: row groups 2s, 2s + 1
        umma(tmem + kColDW2, umma_desc(sH1 + 2048 * s, 1024, 128),
             umma_desc(sG2 + 2048 * s, 1024, 128), umma_idesc(64, 64, 1, 1), acc);
        umma(tmem + kColDW3, umma_desc(sH2 + 2048 * s, 1024, 128),
             umma_desc(sE + 512 * s, 256, 128), umma_idesc(64, 16, 1, 1), acc);
        umma(tmem + kColDB2, umma_desc(sG2 + 2048 * s, 1024, 128),
             umma_desc(sE + 512 * s, 256, 128), umma_idesc(64, 16, 1, 1), acc);
      }
      umma_commit(mb);
    }
    wait_mma();
    if (!ok) break;
    float g1p[kSurHidden];
    tmem_ld32(tmem + lane_base + kColZ, g1p);
    tmem_ld32(tmem + lane_base + kColZ + 32, g1p + 32);
#pragma unroll
    for (int h = 0; h < kSurHidden; h += 2) {
      const float g0 = g1p[h] * sur_dsilu(z1[h]);
      const float g1 = g1p[h + 1] * sur_dsilu(z1[h + 1]);
      *reinterpret_cast<uint32_t*>(G1s + core_idx(tid, h, kSurHidden)) = sur_pack_bf16(g0, g1);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- dW1^T += G1^T X; db1 += G1^T E ----
    if (tid == 0) {
      for (int s = 0; s < 8; ++s) {
        const int acc = (first == 0) || (s > 0);
        umma(tmem + kColDW1, umma_desc(sG1 + 2048 * s, 1024, 128),
             umma_desc(sX + 512 * s, 256, 128), umma_idesc(64, 16, 1, 1), acc);
        umma(tmem + kColDB1, umma_desc(sG1 + 2048 * s, 1024, 128),
             umma_desc(sE + 512 * s, 256, 128), umma_idesc(64, 16, 1, 1), acc);
      }
      umma_commit(mb);
    }
    wait_mma();  // the next tile overwrites X, E and G1
    first = 0;
  }
  __syncthreads();
  // ---- this CTA's gradient partial: an M=64 accumulator holds row m in
  // tensor-memory lane 32 (m / 16) + m % 16, i.e. lanes 0..15 of each warp ----
  float* gp = A.grad_part + (size_t)blockIdx.x * kSurParams;
  const bool has_tiles = blockIdx.x < n_tiles;
  const bool good = ok && abort_flag == 0;
  if (good && has_tiles) {
    float v[64];
    const int m = 16 * warp + lane;  // feature row of the M=64 accumulators
    tmem_ld32(tmem + lane_base + kColDW2, v);
    tmem_ld32(tmem + lane_base + kColDW2 + 32, v + 32);
    if (lane < 16)
      for (int o = 0; o < kSurHidden; ++o) gp[kSurOffW2 + m * kSurHidden + o] = v[o];
    tmem_ld32(tmem + lane_base + kColDW1, v);  // dW1^T (16 columns), then dW3 (column 0)
    if (lane < 16) {
      for (int d = 0; d < kSurBasis; ++d) gp[kSurOffW1 + d * kSurHidden + m] = v[d];
      gp[kSurOffW3 + m] = v[16];
    }
    tmem_ld32(tmem + lane_base + kColDB2, v);  // db2 (column 1), db1 (column 16 + 1)
    if (lane < 16) {
      gp[kSurOffB2 + m] = v[1];
      gp[kSurOffB1 + m] = v[17];
    }
  } else {
    for (int q = tid; q < kSurParams; q += kTrainThreads) gp[q] = 0.0f;
  }
  // loss and db3: threads 0 and 64 hold the partial sums
  if (tid == 0 || tid == 64) {
    red2[tid >> 6][0] = loss;
    red2[tid >> 6][1] = db3;
  }
  __syncthreads();
  if (tid == 0) {
    A.loss_part[blockIdx.x] = red2[0][0] + red2[1][0];
    if (good && has_tiles) gp[kSurOffB3] = red2[0][1] + red2[1][1];
    if (!good) {
      atomicExch(A.error, 1);
      // products may still be in flight: wait once more (bounded) before
      // the tensor memory is released
      mbar_wait(mb, phase);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
}

// Sum of the CTA partials (in CTA order) and one Adam step; thread 0 also
// sums the loss partials.
__global__ void sur_adam_kernel(int n_part, const float* __restrict__ grad_part,
                                const float* __restrict__ loss_part, float* params, float* m,
                                float* v, int step, float lr, float* loss_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) {
    float l = 0.0f;
    for (int b = 0; b < n_part; ++b) l += loss_part[b];
    *loss_out = l;
  }
  if (j >= kSurParams) return;
  float g = 0.0f;
  for (int b = 0; b < n_part; ++b) g += grad_part[(size_t)b * kSurParams + j];
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float mj = b1 * m[j] + (1.0f - b1) * g;
  const float vj = b2 * v[j] + (1.0f - b2) * g * g;
  m[j] = mj;
  v[j] = vj;
  const float mh = mj / (1.0f - powf(b1, (float)step));
  const float vh = vj / (1.0f - powf(b2, (float)step));
  params[j] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace jr

// ================================================================ host ====

namespace {
constexpr int kTrainGridMax = 148;

int train_grid(int n_batch) {
  const int tiles = (n_batch + 1) / 2;
  return tiles < kTrainGridMax ? (tiles > 0 ? tiles : 1) : kTrainGridMax;
}
}  // namespace

extern "C" {

int jr_sur_descriptors(int32_t n_configs, int32_t n_atoms, const float* positions,
                       const float* cell, float* descriptors, void* stream) {
  if (n_configs < 1 || n_atoms < 1 || n_atoms > 128 || !positions || !cell || !descriptors)
    return jrh::fail(JR_ERR_PARAM, "jr_sur_descriptors: invalid arguments");
  const int per_block = 128 / n_atoms;
  jr::sur_descriptor_kernel<<<(n_configs + per_block - 1) / per_block, per_block * n_atoms, 0,
                              (cudaStream_t)stream>>>(n_configs, n_atoms, positions, cell,
                                                      descriptors);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return jrh::cuda_fail(e, "sur_descriptor launch");
  return JR_OK;
}

// Workspace: [int32 error flag, padded to 256 bytes][gradient partials
// grid x JR_SUR_PARAMS][loss partials grid] (float32).
size_t jr_sur_train_workspace_size(int32_t n_batch, int32_t n_atoms) {
  (void)n_atoms;
  const size_t g = (size_t)train_grid(n_batch);
  return 256 + ((g * jr::kSurParams + g) * sizeof(float) + 255) / 256 * 256;
}

int jr_sur_train_step(const JrSurrogate* sur, const float* descriptors, const double* energy_u,
                      const int32_t* batch_idx, int32_t n_batch, int32_t n_atoms, float* params,
                      float* adam_m, float* adam_v, int32_t step, float lr, float* loss,
                      void* workspace, size_t workspace_bytes, void* stream) {
  if (!sur || !descriptors || !energy_u || !batch_idx || !params || !adam_m || !adam_v || !loss)
    return jrh::fail(JR_ERR_PARAM, "jr_sur_train_step: null argument");
  if (n_atoms != 64)
    return jrh::fail(JR_ERR_UNSUPPORTED, "jr_sur_train_step: the training tiles hold two "
                                         "64-atom configurations (n_atoms must be 64)");
  if (n_batch < 1 || step < 1) return jrh::fail(JR_ERR_PARAM, "jr_sur_train_step: n_batch, step");
  if (!workspace || workspace_bytes < jr_sur_train_workspace_size(n_batch, n_atoms))
    return jrh::fail(JR_ERR_WORKSPACE, "jr_sur_train_step: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = train_grid(n_batch);
  int* err = reinterpret_cast<int*>(workspace);
  float* gp = reinterpret_cast<float*>(reinterpret_cast<char*>(workspace) + 256);
  float* lp = gp + (size_t)grid * jr::kSurParams;
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e != cudaSuccess) return jrh::cuda_fail(e, "jr_sur_train_step: error flag");
  jr::SurTrainArgs A;
  A.D = descriptors;
  A.U = energy_u;
  A.idx = batch_idx;
  A.n_batch = n_batch;
  A.params = params;
  for (int k = 0; k < jr::kSurBasis; ++k) {
    A.in_scale[k] = sur->in_scale[k];
    A.in_shift[k] = sur->in_shift[k];
  }
  A.out_scale = sur->out_scale;
  A.out_shift = sur->out_shift;
  A.grad_part = gp;
  A.loss_part = lp;
  A.error = err;
  e = jrh::ensure_attrs(reinterpret_cast<const void*>(jr::sur_train_kernel), jr::kSmBytes, false);
  if (e != cudaSuccess) return jrh::cuda_fail(e, "sur_train attributes");
  jr::sur_train_kernel<<<grid, jr::kTrainThreads, jr::kSmBytes, s>>>(A);
  e = cudaGetLastError();
  if (e != cudaSuccess) return jrh::cuda_fail(e, "sur_train launch");
  jr::sur_adam_kernel<<<(jr::kSurParams + 255) / 256, 256, 0, s>>>(grid, gp, lp, params, adam_m,
                                                                   adam_v, step, lr, loss);
  e = cudaGetLastError();
  if (e != cudaSuccess) return jrh::cuda_fail(e, "sur_adam launch");
  return JR_OK;
}

}  // extern "C"
