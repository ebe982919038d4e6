// Prints the first n outputs of cuRAND's Philox4x32-10 generator for
// (seed, subsequence), one uint4 per line: the library reference the
// engine's own Philox is compared with (tests/test_curand_philox.py).
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdio>
#include <cstdlib>

__global__ void draw(unsigned long long seed, unsigned long long subsequence, int n, uint4* out) {
  curandStatePhilox4_32_10_t st;
  curand_init(seed, subsequence, 0, &st);
  for (int i = 0; i < n; ++i) out[i] = curand4(&st);
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  const unsigned long long seed = std::strtoull(argv[1], nullptr, 10);
  const unsigned long long sub = std::strtoull(argv[2], nullptr, 10);
  const int n = std::atoi(argv[3]);
  if (n < 1 || n > 4096) return 2;
  uint4* d = nullptr;
  if (cudaMalloc(&d, sizeof(uint4) * n) != cudaSuccess) return 1;
  draw<<<1, 1>>>(seed, sub, n, d);
  uint4* h = new uint4[n];
  if (cudaMemcpy(h, d, sizeof(uint4) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  for (int i = 0; i < n; ++i) std::printf("%u %u %u %u\n", h[i].x, h[i].y, h[i].z, h[i].w);
  delete[] h;
  cudaFree(d);
  return 0;
}
