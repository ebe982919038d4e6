// Device helpers of the tcgen05 network (5th-generation tensor cores,
// accumulators in tensor memory), shared by the batched forward and the
// learned move, sm_100a. One CTA of 128 threads evaluates 128 rows: row r is
// thread r and tensor-memory lane r. Layers: tcgen05.mma kind::f16 (BF16
// operands in shared memory, canonical K-major core-matrix layout, FP32
// accumulators), M = 128, N = 64 / 64 / 16, K = 16 / 64 / 64 in 16-wide
// slices; thread 0 issues and commits to an mbarrier, every thread waits
// (bounded), reads its row with tcgen05.ld, adds the bias, applies
// hard-swish, rounds to BF16 and writes the next layer's A operand.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tet_mlp.cuh"

namespace pyro {
// Hard-swish of a packed pair of BF16 values in BF16x2 arithmetic, for the
// learned move's networks (their hidden activations are BF16 MMA operands
// anyway): five paired operations per two activations instead of five per
// one. The batched forward and the training keep the FP32 activation.
__device__ __forceinline__ uint32_t hswish_bf16x2(uint32_t v) {
  const __nv_bfloat162 x = *reinterpret_cast<const __nv_bfloat162*>(&v);
  const __nv_bfloat162 three = __float2bfloat162_rn(3.0f), zero = __float2bfloat162_rn(0.0f),
                       six = __float2bfloat162_rn(6.0f), sixth = __float2bfloat162_rn(1.0f / 6.0f);
  const __nv_bfloat162 t = __hmin2(__hmax2(__hadd2(x, three), zero), six);
  __nv_bfloat162 y = __hmul2(__hmul2(x, t), sixth);
  return *reinterpret_cast<uint32_t*>(&y);
}

namespace umma {

constexpr int kURows = 128;
constexpr int kUBias = kImgTotal - kImgU1;                       // core-matrix weights (bytes)
constexpr int kUA0 = kUBias + (2 * kMlpHidden + kMlpOut) * 4;   // + biases
constexpr int kUA1 = kUA0 + kURows * kMlpIn * 2;                // + A0: 128 x 16 bf16
constexpr int kUBar = kUA1 + kURows * kMlpHidden * 2;           // + A1: 128 x 64 bf16
constexpr int kUSmem = kUBar + 16;                              // + mbarrier, tensor-memory address
constexpr int kUCols = 128;                                     // tensor-memory columns held
static_assert(kUA0 % 16 == 0 && kUA1 % 16 == 0 && kUBar % 8 == 0, "alignment");
static_assert((kImgB1 % 16) == 0 && ((2 * kMlpHidden + kMlpOut) * 4) % 16 == 0, "bias copy");
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance
// between the two 8-element K chunks of a 16-wide slice, sbo = between 8-row
// groups; version 1 (tcgen05).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kURows >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                     uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
      : "memory");
}

// Bounded wait for the mbarrier phase `parity`; false if it ran out.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// Generic-proxy shared-memory writes made visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// 16 consecutive FP32 columns of this warp's 32 lanes (one row per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float hswish_u(float x) {
  return x * fminf(fmaxf(x + 3.0f, 0.0f), 6.0f) * (1.0f / 6.0f);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Row `r` of an M x K operand in the core-matrix layout: K/8 chunks of 16 B.
// kPacked: hidden activations x + bias, rounded to BF16 pairs and activated
// by hswish_bf16x2 (the learned move's network); else x as given.
template <bool kPacked>
__device__ __forceinline__ void store_hidden(unsigned char* base, int r, const float* x,
                                             const float* bias) {
  constexpr int K = kMlpHidden;
  for (int c = 0; c < K / 8; ++c) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = 8 * c + 2 * q;
      w[q] = kPacked ? hswish_bf16x2(pack2(x[j] + bias[j], x[j + 1] + bias[j + 1]))
                     : pack2(hswish_u(x[j] + bias[j]), hswish_u(x[j + 1] + bias[j + 1]));
    }
    *reinterpret_cast<uint4*>(base + (r / 8) * (K / 8) * 128 + c * 128 + (r % 8) * 16) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__device__ __forceinline__ void store_row(unsigned char* base, int r, int K, const float* x) {
  for (int c = 0; c < K / 8; ++c) {
    uint4 q;
    q.x = pack2(x[8 * c + 0], x[8 * c + 1]);
    q.y = pack2(x[8 * c + 2], x[8 * c + 3]);
    q.z = pack2(x[8 * c + 4], x[8 * c + 5]);
    q.w = pack2(x[8 * c + 6], x[8 * c + 7]);
    *reinterpret_cast<uint4*>(base + (r / 8) * (K / 8) * 128 + c * 128 + (r % 8) * 16) = q;
  }
}


// Starts the 16-byte asynchronous copies of the core-matrix weights and the
// biases into shared memory (completed by cp.async.wait_all).
__device__ __forceinline__ void stage_network(unsigned char* smem, const unsigned char* image) {
  for (int i = threadIdx.x * 16; i < kUBias; i += kURows * 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem + i)),
                 "l"(image + kImgU1 + i)
                 : "memory");
  for (int i = threadIdx.x * 16; i < (2 * kMlpHidden + kMlpOut) * 4; i += kURows * 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem + kUBias + i)),
                 "l"(image + kImgB1 + i)
                 : "memory");
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Tensor memory (warp 0) and the mbarrier (thread 0); the address is read
// after the next CTA barrier.
__device__ __forceinline__ void setup(unsigned char* smem) {
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kUBar + 8);
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(tslot)),
                 "r"(kUCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(smem + kUBar))
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
}

// After the A0 rows and the weight copies are written: makes them visible to
// the tensor cores and returns the tensor-memory address.
__device__ __forceinline__ uint32_t ready(unsigned char* smem) {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return *reinterpret_cast<const uint32_t*>(smem + kUBar + 8);
}

// The three layers for the CTA's 128 rows (A0 in place); on success o[16]
// holds this thread's outputs (bias added). Returns false (for every thread)
// if a wait ran out; *parity is the mbarrier phase still expected then.
// kPacked: hidden activations in BF16x2 arithmetic (store_hidden), as the
// mma.sync forms of the learned move evaluate them.
template <bool kPacked = false>
__device__ __forceinline__ bool network(unsigned char* smem, uint32_t tmem, float* o,
                                        uint32_t* parity_io) {
  const float* bias = reinterpret_cast<const float*>(smem + kUBias);
  unsigned char* a1 = smem + kUA1;
  const uint32_t bar = smem_addr(smem + kUBar);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t a0s = smem_addr(smem + kUA0), a1s = smem_addr(a1), ws = smem_addr(smem);
  uint32_t parity = *parity_io;
  float x[kMlpHidden];
  bool ok;
  // layer 1: columns [0, 64) = A0 (128 x 16) . W1
  if (tid == 0) {
    umma(tmem, umma_desc(a0s, 128, 256), umma_desc(ws, 128, 256), umma_idesc(kMlpHidden), 0u);
    umma_commit(bar);
  }
  ok = bar_wait(bar, parity);
  if (ok) parity ^= 1u;
  ok = __syncthreads_and(ok);
  if (ok) {
    fence_after_sync();
#pragma unroll
    for (int c = 0; c < kMlpHidden / 16; ++c) tmem_ld16(lane_base + 16 * c, x + 16 * c);
    store_hidden<kPacked>(a1, tid, x, bias);
    fence_async_smem();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  // layer 2: columns [64, 128) = A1 (128 x 64) . W2, four K slices
  if (ok) {
    if (tid == 0) {
      for (int kk = 0; kk < 4; ++kk)
        umma(tmem + 64, umma_desc(a1s + kk * 256, 128, 1024),
             umma_desc(ws + (kImgU2 - kImgU1) + kk * 256, 128, 1024), umma_idesc(kMlpHidden),
             kk > 0 ? 1u : 0u);
      umma_commit(bar);
    }
    ok = bar_wait(bar, parity);
    if (ok) parity ^= 1u;
  }
  ok = __syncthreads_and(ok);
  if (ok) {
    fence_after_sync();
#pragma unroll
    for (int c = 0; c < kMlpHidden / 16; ++c) tmem_ld16(lane_base + 64 + 16 * c, x + 16 * c);
    // layer 2's reads of A1 completed with its commit
    store_hidden<kPacked>(a1, tid, x, bias + kMlpHidden);
    fence_async_smem();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  // layer 3: columns [0, 16) = A1 (128 x 64) . W3
  if (ok) {
    if (tid == 0) {
      for (int kk = 0; kk < 4; ++kk)
        umma(tmem, umma_desc(a1s + kk * 256, 128, 1024),
             umma_desc(ws + (kImgU3 - kImgU1) + kk * 256, 128, 1024), umma_idesc(kMlpOut),
             kk > 0 ? 1u : 0u);
      umma_commit(bar);
    }
    ok = bar_wait(bar, parity);
    if (ok) parity ^= 1u;
  }
  ok = __syncthreads_and(ok);
  if (ok) {
    fence_after_sync();
    tmem_ld16(lane_base, x);
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) o[j] = x[j] + bias[2 * kMlpHidden + j];
  }
  *parity_io = parity;
  return ok;
}

// Releases the tensor memory; after a failed wait, first gives the MMA in
// flight (bounded) time to complete.
__device__ __forceinline__ void teardown(unsigned char* smem, uint32_t tmem, bool ok,
                                         uint32_t parity) {
  if (!ok && threadIdx.x == 0) bar_wait(smem_addr(smem + kUBar), parity);
  fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kUCols)
                 : "memory");
  }
}

}  // namespace umma
}  // namespace pyro
