// FP64 energy and magnetisation of spins that live in the caller's device
// memory, computed without allocating anything on the device.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or
// arena that owns all device memory, or a host framework that forbids
// allocation once its buffers are sized (allocations there fail or would
// break its accounting), or a context whose creation itself would allocate.
// For them this file provides pyro_observables_noalloc(). The per-block FP64
// partial sums it needs live in a file-scope static device array of fixed
// size (kNoallocPartials double4 = 2 MiB) that every GPU loading the library
// holds until the process exits. The caller passes the spins and the output
// buffers; the function allocates nothing and calls no allocating routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/pyro.h"
#include "lattice.h"

namespace pyro {
namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocSitesPerThread = 8;
constexpr int kNoallocSitesPerBlock = kNoallocThreads * kNoallocSitesPerThread;
constexpr int kNoallocPartials = PYRO_NOALLOC_MAX_PARTIALS;
constexpr int kMaxDevices = 64;

// Shared scratch of every call on this device: one (E, Mx, My, Mz) partial
// per block. Each call writes every slot it later reads, so nothing has to
// start at zero; calls that overlap on the GPU race on it.
static __device__ __align__(256) double4 g_noalloc_partials[kNoallocPartials];

struct StaticSys {
  int L, L3, shells;
  double J[4];
};

std::mutex g_setup_mu;
double4* g_partials_addr[kMaxDevices] = {};
NbrTable g_tab;
bool g_tab_ready = false;

__device__ __forceinline__ int wrap_l(int v, int L) {
  v = v < 0 ? v + L : v;
  return v >= L ? v - L : v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kNoallocThreads)
    noalloc_partials_kernel(const float4* __restrict__ spins, const StaticSys sys,
                            int blocks_per_rep, const NbrTable tab, double4* partials) {
  const int rep = blockIdx.x / blocks_per_rep;
  const int chunk = blockIdx.x - rep * blocks_per_rep;
  const int L = sys.L, L3 = sys.L3, n = 16 * L3;
  const float4* rep_base = spins + (long long)rep * n;
  const int shell_begin[5] = {0, 6, 18, 24, 30};
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  const int first = chunk * kNoallocSitesPerBlock;
  for (int k = 0; k < kNoallocSitesPerThread; ++k) {
    const int i = first + k * kNoallocThreads + threadIdx.x;
    if (i >= n) break;
    const int s = i / L3;
    const int cell = i - s * L3;
    const int x = cell % L, yz = cell / L, y = yz % L, z = yz / L;
    const float4 sv = __ldg(rep_base + i);
    double hx = 0.0, hy = 0.0, hz = 0.0;
    for (int sh = 0; sh < 4; ++sh) {
      if (!(sys.shells & (1 << sh))) continue;
      double ax = 0.0, ay = 0.0, az = 0.0;
      for (int q = shell_begin[sh]; q < shell_begin[sh + 1]; ++q) {
        const NbrEntry en = tab.e[s][q];
        const int idx = (wrap_l(z + en.dz, L) * L + wrap_l(y + en.dy, L)) * L +
                        wrap_l(x + en.dx, L) + en.t * L3;
        const float4 v = __ldg(rep_base + idx);
        ax += v.x;
        ay += v.y;
        az += v.z;
      }
      hx += sys.J[sh] * ax;
      hy += sys.J[sh] * ay;
      hz += sys.J[sh] * az;
    }
    e += (double)sv.x * hx + (double)sv.y * hy + (double)sv.z * hz;
    mx += sv.x;
    my += sv.y;
    mz += sv.z;
  }
  __shared__ double red[4][kNoallocThreads / 32];
  e = warp_sum_d(e);
  mx = warp_sum_d(mx);
  my = warp_sum_d(my);
  mz = warp_sum_d(mz);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][w] = e;
    red[1][w] = mx;
    red[2][w] = my;
    red[3][w] = mz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double4 o = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int q = 0; q < kNoallocThreads / 32; ++q) {
      o.x += red[0][q];
      o.y += red[1][q];
      o.z += red[2][q];
      o.w += red[3][q];
    }
    partials[blockIdx.x] = o;
  }
}

// One warp per replica sums its partials in a fixed order.
__global__ void noalloc_finalise_kernel(const double4* __restrict__ partials, int blocks_per_rep,
                                        int n_rep, double* energy, double* mag) {
  const int rep = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (rep >= n_rep) return;
  const double4* pp = partials + (long long)rep * blocks_per_rep;
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  for (int b = lane; b < blocks_per_rep; b += 32) {
    const double4 v = pp[b];
    e += v.x;
    mx += v.y;
    my += v.z;
    mz += v.w;
  }
  e = warp_sum_d(e);
  mx = warp_sum_d(mx);
  my = warp_sum_d(my);
  mz = warp_sum_d(mz);
  if (lane == 0) {
    energy[rep] = 0.5 * e;
    if (mag) {
      mag[3 * rep + 0] = mx;
      mag[3 * rep + 1] = my;
      mag[3 * rep + 2] = mz;
    }
  }
}

// Once per device, with that device current: the device address of the
// static scratch (its name in host code is only a host-side stand-in).
int setup_current_device(double4** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fprintf(stderr, "pyro_observables_noalloc: cudaGetDevice: %s\n", cudaGetErrorString(e));
    return PYRO_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    fprintf(stderr, "pyro_observables_noalloc: device %d beyond the supported %d\n", dev,
            kMaxDevices);
    return PYRO_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_tab_ready) {
    if (!build_neighbour_table(&g_tab)) return PYRO_ERR_STATE;
    g_tab_ready = true;
  }
  if (!g_partials_addr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
    if (e != cudaSuccess || !ptr) {
      fprintf(stderr, "pyro_observables_noalloc: cudaGetSymbolAddress: %s\n",
              cudaGetErrorString(e));
      return PYRO_ERR_CUDA;
    }
    g_partials_addr[dev] = (double4*)ptr;
  }
  *out = g_partials_addr[dev];
  return PYRO_OK;
}

}  // namespace
}  // namespace pyro

extern "C" int pyro_observables_noalloc(const float* dev_spins_xyzw, int L, int n_replicas,
                                        double J1, double J2, double J3, double J3b,
                                        double* dev_energy, double* dev_magnetisation3,
                                        void* cuda_stream) {
  using namespace pyro;
  if (!dev_spins_xyzw || !dev_energy || L < 2 || L > 256 || n_replicas < 1) {
    fprintf(stderr, "pyro_observables_noalloc: need spins and energy pointers, 2 <= L <= 256, "
                    "n_replicas >= 1\n");
    return PYRO_ERR_ARG;
  }
  // The kernels read the spins as float4 and write doubles: a misaligned
  // caller pointer would fault the GPU, so it is refused here, before any
  // CUDA call.
  if (((uintptr_t)dev_spins_xyzw & 15u) || ((uintptr_t)dev_energy & 7u) ||
      ((uintptr_t)dev_magnetisation3 & 7u)) {
    fprintf(stderr, "pyro_observables_noalloc: spins must be 16-byte aligned and the energy "
                    "and magnetisation buffers 8-byte aligned\n");
    return PYRO_ERR_ARG;
  }
  const long long sites = 16ll * L * L * L;
  const long long blocks_per_rep = (sites + kNoallocSitesPerBlock - 1) / kNoallocSitesPerBlock;
  const long long blocks = blocks_per_rep * n_replicas;
  if (blocks > kNoallocPartials) {
    fprintf(stderr,
            "pyro_observables_noalloc: %d replicas of L=%d need %lld partial sums; the static "
            "scratch holds %d (at most %lld sites in total)\n",
            n_replicas, L, blocks, kNoallocPartials,
            (long long)kNoallocPartials * kNoallocSitesPerBlock);
    return PYRO_ERR_ARG;
  }
  double4* partials = nullptr;
  int rc = setup_current_device(&partials);
  if (rc != PYRO_OK) return rc;
  StaticSys sys;
  sys.L = L;
  sys.L3 = L * L * L;
  sys.J[0] = J1;
  sys.J[1] = J2;
  sys.J[2] = J3;
  sys.J[3] = J3b;
  sys.shells = (J1 != 0.0 ? 1 : 0) | (J2 != 0.0 ? 2 : 0) | (J3 != 0.0 ? 4 : 0) |
               (J3b != 0.0 ? 8 : 0);
  cudaStream_t st = (cudaStream_t)cuda_stream;
  noalloc_partials_kernel<<<(int)blocks, kNoallocThreads, 0, st>>>(
      (const float4*)dev_spins_xyzw, sys, (int)blocks_per_rep, g_tab, partials);
  const int fin_threads = 256;
  const int fin_blocks = (n_replicas * 32 + fin_threads - 1) / fin_threads;
  noalloc_finalise_kernel<<<fin_blocks, fin_threads, 0, st>>>(
      partials, (int)blocks_per_rep, n_replicas, dev_energy, dev_magnetisation3);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "pyro_observables_noalloc: launch: %s\n", cudaGetErrorString(e));
    return PYRO_ERR_CUDA;
  }
  return PYRO_OK;
}
