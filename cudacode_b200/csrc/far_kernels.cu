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

namespace pyro {
namespace {

struct Frame3 {
  int zo[3], yo[3], xo[3];
};

__device__ __forceinline__ Frame3 frame_of(int cell, int L, float rcpL) {
  int q = (int)((float)cell * rcpL);
  int r = cell - q * L;
  if (r < 0) { --q; r += L; } else if (r >= L) { ++q; r -= L; }
  int q2 = (int)((float)q * rcpL);
  int r2 = q - q2 * L;
  if (r2 < 0) { --q2; r2 += L; } else if (r2 >= L) { ++q2; r2 -= L; }
  const int x = r, y = r2, z = q2, L2 = L * L;
  Frame3 f;
  f.xo[0] = x == 0 ? L - 1 : x - 1;
  f.xo[1] = x;
  f.xo[2] = x == L - 1 ? 0 : x + 1;
  f.yo[0] = (y == 0 ? L - 1 : y - 1) * L;
  f.yo[1] = y * L;
  f.yo[2] = (y == L - 1 ? 0 : y + 1) * L;
  f.zo[0] = (z == 0 ? L - 1 : z - 1) * L2;
  f.zo[1] = z * L2;
  f.zo[2] = (z == L - 1 ? 0 : z + 1) * L2;
  return f;
}

template <int S, int K>
__device__ __forceinline__ float4 nb(const float4* __restrict__ rep, const Frame3& f, int L3) {
  constexpr NbrEntry e = far_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  return __ldg(rep + f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3);
}

// Sum of neighbours K0..K1-1 of site S in canonical order (first value, then
// left-to-right adds), as shell_sum of the generic kernel.
template <int S, int K, int K1>
__device__ __forceinline__ void add_rest(const float4* __restrict__ rep, const Frame3& f, int L3,
                                         float3& a) {
  if constexpr (K < K1) {
    const float4 v = nb<S, K>(rep, f, L3);
    a.x = a.x + v.x;
    a.y = a.y + v.y;
    a.z = a.z + v.z;
    add_rest<S, K + 1, K1>(rep, f, L3, a);
  }
}

template <int S, int K0, int K1>
__device__ __forceinline__ float3 shell_sum_c(const float4* __restrict__ rep, const Frame3& f,
                                              int L3) {
  const float4 v0 = nb<S, K0>(rep, f, L3);
  float3 a = make_float3(v0.x, v0.y, v0.z);
  add_rest<S, K0 + 1, K1>(rep, f, L3, a);
  return a;
}

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
  const int L3 = sd.L3;
  int accepted = 0;
  int tslot = 0;
  if (kMetro) tslot = p.temp_of_rep[sd.temp_base + sd.rep_global + rep];
  if (cell < L3) {
    const Frame3 fr = frame_of(cell, sd.L, sd.rcpL);
    float4* rb = p.spins + sd.spin_off + (long long)rep * 16 * L3;
    const int own = S * L3 + cell;
    const float3 a1 = shell_sum_c<S, 0, 6>(rb, fr, L3);
    pyro_vec3 h;
    h.x = sd.J1 * a1.x;
    h.y = sd.J1 * a1.y;
    h.z = sd.J1 * a1.z;
    if (sd.shells & 2) {
      const float3 a = shell_sum_c<S, 6, 18>(rb, fr, L3);
      h.x = fmaf(sd.J2, a.x, h.x);
      h.y = fmaf(sd.J2, a.y, h.y);
      h.z = fmaf(sd.J2, a.z, h.z);
    }
    if (sd.shells & 4) {
      const float3 a = shell_sum_c<S, 18, 24>(rb, fr, L3);
      h.x = fmaf(sd.J3a, a.x, h.x);
      h.y = fmaf(sd.J3a, a.y, h.y);
      h.z = fmaf(sd.J3a, a.z, h.z);
    }
    if (sd.shells & 8) {
      const float3 a = shell_sum_c<S, 24, 30>(rb, fr, L3);
      h.x = fmaf(sd.J3b, a.x, h.x);
      h.y = fmaf(sd.J3b, a.y, h.y);
      h.z = fmaf(sd.J3b, a.z, h.z);
    }
    const float4 sv = rb[own];
    pyro_vec3 sp;
    sp.x = sv.x;
    sp.y = sv.y;
    sp.z = sv.z;
    const unsigned long long sweep = (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off;
    pyro_vec3 out;
    if (kMetro) {
      const float beta = p.beta[sd.temp_base + tslot];
      const float cosmax = p.cosmax[sd.temp_base + tslot];
      uint32_t r[4];
      pyro_philox((uint32_t)own, (uint32_t)(sd.rep_key + rep), (uint32_t)sweep, PYRO_PURPOSE_METRO,
                  p.seed_lo, p.seed_hi, r);
      const pyro_vec3 prop = pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
      accepted = pyro_metropolis_accept(pyro_delta_e(h, sp, prop), beta, pyro_uniform(r[2]));
      out = accepted ? prop : sp;
    } else {
      out = pyro_overrelax(sp, h);
    }
    if (p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0)
      out = pyro_renormalise(out);
    rb[own] = make_float4(out.x, out.y, out.z, 0.0f);
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
