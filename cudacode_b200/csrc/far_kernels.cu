// Colour passes of the 16-colour schedule (J1 plus J2 / J3 couplings) with
// compile-time neighbour offsets, for sm_100a.
//
// With further-neighbour couplings a colour class is one site s of the cubic
// cell, so in a pass every thread of every system updates the same site s:
// the 30 neighbour offsets of s (6 J1, 12 J2, 6 J3a, 6 J3b, canonical order)
// are template constants (far_neighbour), each neighbour address three
// integer adds of per-thread row offsets. Blocks map to (system, replica,
// 256-cell chunk) through the same segment lists as the generic kernel, so
// one launch covers all systems of a pass (or of a replica group). The
// arithmetic is the generic kernel's, bit for bit.
//
// Replaces, for the further-neighbour Hamiltonian that the reference does not
// have, the role of MCMultipleTemperaturesPerSystem (Pyrochlore.cu:829-885)
// and OverRelaxationByPiStep (975-1007).
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "far_kernels.cuh"
#include "far_update.cuh"

namespace pyro {
namespace {

template <typename Seg>
__device__ __forceinline__ int find_seg(const Seg* segs, int nseg, int block) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].block_begin <= block) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int S, bool kMetro>
__global__ void __launch_bounds__(kFarThreads) far_pass_kernel(const PassParams p) {
  // may overlap the drain of the previous kernel (programmatic dependent
  // launch): wait for it before any global access
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int seg_i = find_seg(p.segs, p.nseg, blockIdx.x);
  const PassSeg sg = p.segs[seg_i];
  const SysDev& sd = p.sys[sg.sys];
  const int rel = blockIdx.x - sg.block_begin;
  const int rep_in_seg = rel / sg.blocks_per_rep;
  const int rep = sg.rep_begin + rep_in_seg;
  const int cell = (rel - rep_in_seg * sg.blocks_per_rep) * kFarThreads + threadIdx.x;
  int accepted = 0;
  int tslot = 0;
  if (kMetro) tslot = p.temp_of_rep[sd.temp_base + sd.rep_global + rep];
  if (cell < sd.L3) {
    const unsigned long long sweep = (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off;
    accepted = far::site_update<S, kMetro>(p, sd, rep, cell, sweep, tslot);
  }
  if (kMetro) {
    const int n = __syncthreads_count(accepted);
    if (threadIdx.x == 0 && n > 0) atomicAdd(p.accepted + sd.temp_base + tslot, (unsigned long long)n);
  }
}

template <typename Kernel>
void launch_far_kernel(Kernel k, int n_blocks, const PassParams& p, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n_blocks, 1, 1);
  cfg.blockDim = dim3(kFarThreads, 1, 1);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, p);  // errors are read back with cudaGetLastError
}

template <bool kMetro>
void launch_far(const PassParams& p, int site, int n_blocks, cudaStream_t st) {
  switch (site) {
#define PYRO_FAR(S) \
  case S:           \
    launch_far_kernel(far_pass_kernel<S, kMetro>, n_blocks, p, st); \
    break;
    PYRO_FAR(0) PYRO_FAR(1) PYRO_FAR(2) PYRO_FAR(3) PYRO_FAR(4) PYRO_FAR(5) PYRO_FAR(6)
    PYRO_FAR(7) PYRO_FAR(8) PYRO_FAR(9) PYRO_FAR(10) PYRO_FAR(11) PYRO_FAR(12) PYRO_FAR(13)
    PYRO_FAR(14) PYRO_FAR(15)
#undef PYRO_FAR
    default:
      break;
  }
}

}  // namespace

void launch_far_pass(const PassParams& p, int site, int n_blocks, bool metro, cudaStream_t st) {
  if (n_blocks <= 0) return;
  if (metro) launch_far<true>(p, site, n_blocks, st);
  else launch_far<false>(p, site, n_blocks, st);
}

}  // namespace pyro
