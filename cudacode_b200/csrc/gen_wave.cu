// The work-queue cycle kernel of 16-colour systems (isotropic J1 plus J2 /
// J3 shells): all sweeps of a cycle of every such system, in one launch,
// instead of one launch per colour pass (the batched configuration: 256
// systems of uneven L, 16 colour passes per sweep).
//
// A work item is colour pass k (site k mod 16 of the cubic cell) of one
// 256-cell chunk of one (system, replica). The kernel is persistent (as many
// CTAs as are resident at once); a CTA takes the next ticket of an atomic
// counter as its item, so items are taken in ticket order by running CTAs;
// it waits until the previous pass is complete on every chunk that holds a
// neighbour of its cells (progress counters, acquire loads, bounded), runs
// the updates of the per-pass kernel (far_update.cuh: same neighbour order,
// same arithmetic, neighbours read through L1 after the acquire), and
// releases its chunk's counter. Item order, dependency and wait bounds are those of the
// nearest-neighbour work-queue kernel (j1_kernels.cu), with units of
// (system, replica) from many systems in one queue.
//
// Replaces, for the batched further-neighbour systems the reference does not
// have, the per-colour launches of its driver loop (Pyrochlore.cu:74-133).
#include <cuda_runtime.h>

#include <algorithm>

#include "far_update.cuh"
#include "gen_wave.cuh"

namespace pyro {
namespace {

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// After the CTA's barrier: make its stores visible at GPU scope, then count
// the chunk's pass as complete.
__device__ __forceinline__ void release_add(unsigned int* p, unsigned int v) {
  asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v)
               : "memory");
}

template <int S>
__device__ __forceinline__ int item_site(const PassParams& p, const SysDev& sd, int rep, int cell,
                                         unsigned long long sweep, int tslot, bool metro) {
  return metro ? far::site_update<S, true, false>(p, sd, rep, cell, sweep, tslot)
               : far::site_update<S, false, false>(p, sd, rep, cell, sweep, tslot);
}

// One item of the CTA (every thread calls it): returns true when the queue
// is empty or a wait gave up (the CTA ends).
__device__ __forceinline__ bool gen_wave_item(const GenWaveParams& w, int* s_info) {
  if (threadIdx.x == 0) {
    const int item = (int)atomicAdd(w.queue, 1u);
    s_info[0] = item < w.n_items ? item : -1;
    if (item < w.n_items) {
      const int passes = 16 * (w.n_metro + w.n_or);
      int lo = 0, hi = w.n_groups - 1;  // the last group starting at or before the item
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (passes * w.groups[mid].chunk_prefix <= item) lo = mid;
        else hi = mid - 1;
      }
      const GenWaveGroup G = w.groups[lo];
      const int local = item - passes * G.chunk_prefix;
      const int k = local / G.chunks;
      const int b = local - k * G.chunks;
      const int ulo = w.chunk_unit[G.chunk_prefix + b];  // the unit holding chunk b
      const GenWaveUnit U = w.units[ulo];
      const int j = b - U.chunk_begin;
      s_info[1] = ulo;
      s_info[2] = k;
      s_info[3] = (int)(((long long)j + (long long)U.dep * k) % U.n_chunks);
    }
  }
  __syncthreads();
  const int item = s_info[0];
  if (item < 0) return true;
  const int u = s_info[1], k = s_info[2], q = s_info[3];
  const GenWaveUnit U = w.units[u];
  // Wait until pass k - 1 is complete on every chunk holding a neighbour.
  int failed = 0;
  if (k > 0) {
    const int nq = U.n_chunks;
    const int n_dep = 2 * U.dep + 1 >= nq ? nq : 2 * U.dep + 1;
    const unsigned int* row = w.progress + U.prog_off;
    for (int d = threadIdx.x; d < n_dep; d += blockDim.x) {
      int qq = n_dep == nq ? d : q - U.dep + d;
      qq = qq < 0 ? qq + nq : (qq >= nq ? qq - nq : qq);
      unsigned int polls = 0;
      while (ld_acquire(row + qq) < (unsigned int)k) {
        if (++polls >= w.spin_limit || *(volatile int*)w.status) {
          failed = 1;
          break;
        }
        __nanosleep(64);
      }
    }
  }
  if (__syncthreads_or(failed)) {
    if (threadIdx.x == 0) atomicExch(w.status, 1);
    return true;
  }
  const SysDev& sd = w.pass.sys[U.sys];
  const int sweep_idx = k >> 4;
  const bool metro = sweep_idx < w.n_metro;
  const unsigned long long sweep =
      (w.pass.sweep_ctr ? *w.pass.sweep_ctr : 0ull) + w.pass.sweep_off + sweep_idx;
  int tslot = 0;
  if (metro) tslot = w.pass.temp_of_rep[sd.temp_base + sd.rep_global + U.rep];
  const int cell = q * kPassThreads + threadIdx.x;
  int acc = 0;
  if (cell < sd.L3) {
    const PassParams& p = w.pass;
    switch (k & 15) {
#define PYRO_GEN_SITE(S) \
  case S:                \
    acc = item_site<S>(p, sd, U.rep, cell, sweep, tslot, metro); \
    break;
      PYRO_GEN_SITE(0) PYRO_GEN_SITE(1) PYRO_GEN_SITE(2) PYRO_GEN_SITE(3) PYRO_GEN_SITE(4)
      PYRO_GEN_SITE(5) PYRO_GEN_SITE(6) PYRO_GEN_SITE(7) PYRO_GEN_SITE(8) PYRO_GEN_SITE(9)
      PYRO_GEN_SITE(10) PYRO_GEN_SITE(11) PYRO_GEN_SITE(12) PYRO_GEN_SITE(13) PYRO_GEN_SITE(14)
      default:
        acc = item_site<15>(p, sd, U.rep, cell, sweep, tslot, metro);
        break;
#undef PYRO_GEN_SITE
    }
  }
  if (metro) {
    const int n = __syncthreads_count(acc);
    if (threadIdx.x == 0 && n > 0)
      atomicAdd(w.pass.accepted + sd.temp_base + tslot, (unsigned long long)n);
  }
  __syncthreads();  // every store of the item is issued
  if (threadIdx.x == 0 && item != w.stall_item) release_add(w.progress + U.prog_off + q, 1u);
  return false;
}

// Persistent: each CTA takes items until the queue is empty.
__global__ void __launch_bounds__(kPassThreads) gen_wave_kernel(const GenWaveParams w) {
  __shared__ int s_info[4];  // item (or -1), unit, pass, chunk
  for (;;) {
    if (gen_wave_item(w, s_info)) return;
    __syncthreads();  // s_info is rewritten by the next item
  }
}

}  // namespace

cudaError_t launch_gen_wave(const GenWaveParams& p, cudaStream_t st) {
  if (p.n_items <= 0) return cudaSuccess;
  // as many CTAs as fit on the device at once
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gen_wave_kernel, kPassThreads, 0);
  if (e != cudaSuccess) return e;
  const int resident = std::max(1, sms * per_sm);
  gen_wave_kernel<<<std::min(p.n_items, resident), kPassThreads, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace pyro
