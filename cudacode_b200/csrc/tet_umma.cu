// Batched forward of the learned proposal's network on the 5th-generation
// tensor cores (tet_umma.cuh), 128 feature rows per CTA; the arithmetic is
// the same network as the mma.sync kernels (BF16 rounding points of inputs,
// weights and hidden activations; FP32 accumulation), so both agree with the
// oracle's FP64 restatement within the same tolerance.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tet_umma.cuh"

namespace pyro {
namespace {

using namespace umma;

__global__ void __launch_bounds__(kURows) umma_forward_kernel(const float* __restrict__ features,
                                                              int n,
                                                              const unsigned char* __restrict__ image,
                                                              float* __restrict__ out, int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  stage_network(smem, image);
  setup(smem);
  const int tid = threadIdx.x;
  const long long row = (long long)blockIdx.x * kURows + tid;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = row < n ? features[row * kMlpIn + i] : 0.0f;
  store_row(smem + kUA0, tid, kMlpIn, x);
  const uint32_t tmem = ready(smem);
  uint32_t parity = 0;
  float o[kMlpOut];
  const bool ok = network(smem, tmem, o, &parity);
  if (ok && row < n) {
    float4* dst = reinterpret_cast<float4*>(out + row * kMlpOut);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  teardown(smem, tmem, ok, parity);
}

}  // namespace

cudaError_t launch_umma_forward(const float* features, int n, const unsigned char* image,
                                float* out, int* err, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (n + kURows - 1) / kURows;
  umma_forward_kernel<<<blocks, kURows, kUSmem, st>>>(features, n, image, out, err);
  return cudaGetLastError();
}

}  // namespace pyro
