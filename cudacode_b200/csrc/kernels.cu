// Colour-pass sweeps, spin initialisation, FP64 observables and the replica
// exchange, for sm_100a.
//
// A colour pass updates every site of one colour class of every replica in
// the launch. No two sites of a class interact, so a pass reads the other
// classes and rewrites its own in place, and its result does not depend on
// the order in which CTAs run. One thread owns one site; a CTA never spans
// two replicas, so per-replica values (beta, cone width, acceptance) are
// CTA-uniform. Spins are float4 (16 B), planes of L^3 cells per site of the
// cubic cell, so a warp reads 32 consecutive cells: 512 contiguous bytes for
// its own spin and for each neighbour.
//
// Reference kernels replaced: MCMultipleTemperaturesPerSystem
// (Pyrochlore.cu:829-885), OverRelaxationByPiStep (975-1007), the local field
// CalculateLocalExchangeField (210-275) with the periodic neighbour decode of
// TotalEnergy (468-523; the GPU decode CalculateNeighbor3D, Math.cu:988-1009,
// swaps the y/z offsets and is not followed), TotalEnergyGPU (344-389),
// MagnetizationGPU (277-342), Generate3DVectorList (Math.cu:132-143) and the
// host swap TrySwapingTemperatures (MonteCarlo.cu:105-172).
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "kernels.cuh"

namespace pyro {

namespace {

template <typename Seg>
__device__ __forceinline__ int find_segment(const Seg* segs, int nseg, int block) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].block_begin <= block) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int wrap(int v, int L) {
  v = v < 0 ? v + L : v;
  return v >= L ? v - L : v;
}

struct Acc3 {
  float x, y, z;
};

// Sum of the neighbours of one shell, in table order.
__device__ __forceinline__ Acc3 shell_sum(const float4* __restrict__ rep, const NbrTable& tab,
                                          int s, int first, int last, int x, int y, int z, int L,
                                          int L3) {
  Acc3 a;
  {
    const NbrEntry e = tab.e[s][first];
    const int idx = (wrap(z + e.dz, L) * L + wrap(y + e.dy, L)) * L + wrap(x + e.dx, L) + e.t * L3;
    const float4 v = __ldg(rep + idx);
    a.x = v.x;
    a.y = v.y;
    a.z = v.z;
  }
#pragma unroll 6
  for (int k = first + 1; k < last; ++k) {
    const NbrEntry e = tab.e[s][k];
    const int idx = (wrap(z + e.dz, L) * L + wrap(y + e.dy, L)) * L + wrap(x + e.dx, L) + e.t * L3;
    const float4 v = __ldg(rep + idx);
    a.x = a.x + v.x;
    a.y = a.y + v.y;
    a.z = a.z + v.z;
  }
  return a;
}

// Nearest-neighbour field of site s with bond matrices (anisotropic
// exchange), minus the site's Zeeman field: sum over the six neighbours in
// table order of A[b][b_k] S_k (pyro_matvec_add), then - f[b].
__device__ __forceinline__ pyro_vec3 exch_field(const float4* __restrict__ rep, const NbrTable& tab,
                                                const ExchangeDev& X, int s, int x, int y, int z,
                                                int L, int L3) {
  const int b = s & 3;
  pyro_vec3 h;
  h.x = h.y = h.z = 0.0f;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const NbrEntry e = tab.e[s][k];
    const int idx = (wrap(z + e.dz, L) * L + wrap(y + e.dy, L)) * L + wrap(x + e.dx, L) + e.t * L3;
    const float4 v = __ldg(rep + idx);
    h = pyro_matvec_add(h, X.A[4 * b + (e.t & 3)], v.x, v.y, v.z);
  }
  h.x = h.x - X.f[b][0];
  h.y = h.y - X.f[b][1];
  h.z = h.z - X.f[b][2];
  return h;
}

template <bool kJ1Only, bool kMetro>
__global__ void __launch_bounds__(kPassThreads) colour_pass_kernel(const PassParams p,
                                                                   const NbrTable tab) {
  // may overlap the drain of the previous kernel (programmatic dependent
  // launch): wait for it before any global access
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int seg_i = find_segment(p.segs, p.nseg, blockIdx.x);
  const PassSeg sg = p.segs[seg_i];
  const SysDev& sd = p.sys[sg.sys];
  const int rel = blockIdx.x - sg.block_begin;
  const int rep_in_seg = rel / sg.blocks_per_rep;
  const int rep = sg.rep_begin + rep_in_seg;
  const int u = (rel - rep_in_seg * sg.blocks_per_rep) * kPassThreads + threadIdx.x;
  const bool active = u < sd.units_per_colour;
  const int L = sd.L, L3 = sd.L3;

  int accepted = 0;
  if (active) {
    const int k = u / L3;
    const int cell = u - k * L3;
    const int s = colour_site(sd.n_colours, sg.colour, k);
    const int x = cell % L;
    const int yz = cell / L;
    const int y = yz % L;
    const int z = yz / L;
    float4* rep_base = p.spins + sd.spin_off + (long long)rep * 16 * L3;
    const int own = s * L3 + cell;
    const float4 sv = rep_base[own];

    pyro_vec3 h;
    if (!kJ1Only && sd.exch >= 0) {
      h = exch_field(rep_base, tab, p.exch[sd.exch], s, x, y, z, L, L3);
    } else {
      const Acc3 a1 = shell_sum(rep_base, tab, s, 0, 6, x, y, z, L, L3);
      h.x = sd.J1 * a1.x;
      h.y = sd.J1 * a1.y;
      h.z = sd.J1 * a1.z;
    }
    if (!kJ1Only) {
      if (sd.shells & 2) {
        const Acc3 a = shell_sum(rep_base, tab, s, 6, 18, x, y, z, L, L3);
        h.x = fmaf(sd.J2, a.x, h.x);
        h.y = fmaf(sd.J2, a.y, h.y);
        h.z = fmaf(sd.J2, a.z, h.z);
      }
      if (sd.shells & 4) {
        const Acc3 a = shell_sum(rep_base, tab, s, 18, 24, x, y, z, L, L3);
        h.x = fmaf(sd.J3a, a.x, h.x);
        h.y = fmaf(sd.J3a, a.y, h.y);
        h.z = fmaf(sd.J3a, a.z, h.z);
      }
      if (sd.shells & 8) {
        const Acc3 a = shell_sum(rep_base, tab, s, 24, 30, x, y, z, L, L3);
        h.x = fmaf(sd.J3b, a.x, h.x);
        h.y = fmaf(sd.J3b, a.y, h.y);
        h.z = fmaf(sd.J3b, a.z, h.z);
      }
    }

    pyro_vec3 sp;
    sp.x = sv.x;
    sp.y = sv.y;
    sp.z = sv.z;
    const unsigned long long sweep = (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off;
    pyro_vec3 out;
    if (kMetro) {
      const int g = sd.rep_global + rep;
      const int t = p.temp_of_rep[sd.temp_base + g];
      const float beta = p.beta[sd.temp_base + t];
      const float cosmax = p.cosmax[sd.temp_base + t];
      uint32_t r[4];
      pyro_philox((uint32_t)own, (uint32_t)(sd.rep_key + rep), (uint32_t)sweep, PYRO_PURPOSE_METRO,
                  p.seed_lo, p.seed_hi, r);
      const pyro_vec3 prop = pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
      const float dE = pyro_delta_e(h, sp, prop);
      accepted = pyro_metropolis_accept(dE, beta, pyro_uniform(r[2]));
      out = accepted ? prop : sp;
    } else {
      out = pyro_overrelax(sp, h);
    }
    if (p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0)
      out = pyro_renormalise(out);
    rep_base[own] = make_float4(out.x, out.y, out.z, 0.0f);
  }
  if (kMetro) {
    const int n_acc = __syncthreads_count(accepted);
    if (threadIdx.x == 0 && n_acc > 0) {
      const int g = sd.rep_global + rep;
      const int t = p.temp_of_rep[sd.temp_base + g];
      atomicAdd(p.accepted + sd.temp_base + t, (unsigned long long)n_acc);
    }
  }
}

__global__ void init_random_kernel(float4* spins, const SysDev* sys, int n_sys, long long total,
                                   uint32_t seed_lo, uint32_t seed_hi) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int si = 0;
    while (si + 1 < n_sys && sys[si + 1].spin_off <= i) ++si;
    const SysDev& sd = sys[si];
    const long long rel = i - sd.spin_off;
    const long long per_rep = 16ll * sd.L3;
    const int rep = (int)(rel / per_rep);
    const int site = (int)(rel - rep * per_rep);
    uint32_t r[4];
    pyro_philox((uint32_t)site, (uint32_t)(sd.rep_key + rep), 0u, PYRO_PURPOSE_INIT, seed_lo, seed_hi,
                r);
    const pyro_vec3 v = pyro_sphere_point(pyro_uniform(r[0]), pyro_uniform(r[1]));
    spins[i] = make_float4(v.x, v.y, v.z, 0.0f);
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// FP64 energy E = 1/2 sum_i S_i . h_i and magnetisation sum_i S_i (with
// bond matrices: E = 1/2 sum_i S_i . (sum_k A S_k) - sum_i f . S_i; the
// partials hold twice the energy, halved by the finalise kernel).
__global__ void __launch_bounds__(kObsThreads) observables_kernel(const ObsParams p,
                                                                  const NbrTable tab) {
  const int seg_i = find_segment(p.segs, p.nseg, blockIdx.x);
  const ObsSeg sg = p.segs[seg_i];
  const SysDev& sd = p.sys[sg.sys];
  const int rel = blockIdx.x - sg.block_begin;
  const int rep = rel / sg.blocks_per_rep;
  const int chunk = rel - rep * sg.blocks_per_rep;
  const int L = sd.L, L3 = sd.L3, n = 16 * L3;
  const float4* rep_base = p.spins + sd.spin_off + (long long)rep * n;
  const double Js[4] = {sd.J64[0], sd.J64[1], sd.J64[2], sd.J64[3]};
  const int shell_begin[5] = {0, 6, 18, 24, 30};

  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  const int first = chunk * kObsThreads * kObsSitesPerThread;
  for (int k = 0; k < kObsSitesPerThread; ++k) {
    const int i = first + k * kObsThreads + threadIdx.x;
    if (i >= n) break;
    const int s = i / L3;
    const int cell = i - s * L3;
    const int x = cell % L, yz = cell / L, y = yz % L, z = yz / L;
    const float4 sv = __ldg(rep_base + i);
    double hx = 0.0, hy = 0.0, hz = 0.0;
    if (sd.exch >= 0) {
      const ExchangeDev& X = p.exch[sd.exch];
      const int b = s & 3;
      for (int q = 0; q < 6; ++q) {
        const NbrEntry en = tab.e[s][q];
        const int idx =
            (wrap(z + en.dz, L) * L + wrap(y + en.dy, L)) * L + wrap(x + en.dx, L) + en.t * L3;
        const float4 v = __ldg(rep_base + idx);
        const double* m = X.A64[4 * b + (en.t & 3)];
        hx += m[0] * v.x + m[1] * v.y + m[2] * v.z;
        hy += m[3] * v.x + m[4] * v.y + m[5] * v.z;
        hz += m[6] * v.x + m[7] * v.y + m[8] * v.z;
      }
      hx -= 2.0 * X.f64[b][0];
      hy -= 2.0 * X.f64[b][1];
      hz -= 2.0 * X.f64[b][2];
    }
    for (int sh = 0; sh < 4; ++sh) {
      if (!(sd.shells & (1 << sh))) continue;
      if (sh == 0 && sd.exch >= 0) continue;
      double ax = 0.0, ay = 0.0, az = 0.0;
      for (int q = shell_begin[sh]; q < shell_begin[sh + 1]; ++q) {
        const NbrEntry en = tab.e[s][q];
        const int idx =
            (wrap(z + en.dz, L) * L + wrap(y + en.dy, L)) * L + wrap(x + en.dx, L) + en.t * L3;
        const float4 v = __ldg(rep_base + idx);
        ax += v.x;
        ay += v.y;
        az += v.z;
      }
      hx += Js[sh] * ax;
      hy += Js[sh] * ay;
      hz += Js[sh] * az;
    }
    e += (double)sv.x * hx + (double)sv.y * hy + (double)sv.z * hz;
    mx += sv.x;
    my += sv.y;
    mz += sv.z;
  }
  __shared__ double red[4][kObsThreads / 32];
  e = warp_sum(e);
  mx = warp_sum(mx);
  my = warp_sum(my);
  mz = warp_sum(mz);
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
    for (int q = 0; q < kObsThreads / 32; ++q) {
      o.x += red[0][q];
      o.y += red[1][q];
      o.z += red[2][q];
      o.w += red[3][q];
    }
    p.partials[sg.partial_begin + (blockIdx.x - sg.block_begin)] = o;
  }
}

// One warp per replica: fixed-order sum of its partials.
// One warp sums the partials of replica r of system si in a fixed order and
// writes its FP64 energy and magnetisation.
__device__ __forceinline__ void finalise_replica(const double4* __restrict__ partials,
                                                 const ObsSeg& sg, const SysDev& sd, int r,
                                                 double* energy, double* mag) {
  const int lane = threadIdx.x & 31;
  const double4* pp = partials + sg.block_begin + (long long)r * sg.blocks_per_rep;
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  for (int b = lane; b < sg.blocks_per_rep; b += 32) {
    const double4 v = pp[b];
    e += v.x;
    mx += v.y;
    my += v.z;
    mz += v.w;
  }
  e = warp_sum(e);
  mx = warp_sum(mx);
  my = warp_sum(my);
  mz = warp_sum(mz);
  if (lane == 0) {
    const int gi = sd.rep_ctx_base + r;
    energy[gi] = 0.5 * e;
    mag[3 * gi + 0] = mx;
    mag[3 * gi + 1] = my;
    mag[3 * gi + 2] = mz;
  }
}

__global__ void obs_finalise_kernel(const double4* __restrict__ partials, const ObsSeg* segs,
                                    const SysDev* sys, int total_reps, const int* rep_sys,
                                    const int* rep_local, double* energy, double* mag) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= total_reps) return;
  const int si = rep_sys[wid];
  finalise_replica(partials, segs[si], sys[si], rep_local[wid], energy, mag);
}

// One block per system. Pairs (t, t+1) with t % 2 == parity exchange
// temperature labels with probability min(1, exp((b_t - b_t+1)(E_t - E_t+1))).
__global__ void exchange_kernel(const ExchangeParams p) {
  const int si = p.sys_first + blockIdx.x;
  const SysDev& sd = p.sys[si];
  const int nT = sd.n_temp;
  const unsigned long long count = p.swap_count[si];
  __shared__ int n_acc;
  if (threadIdx.x == 0) n_acc = 0;
  if (p.partials) {
    const ObsSeg sg = p.obs_segs[si];
    for (int r = threadIdx.x >> 5; r < sd.n_rep; r += blockDim.x >> 5)
      finalise_replica(p.partials, sg, sd, r, p.energy_out, p.mag_out);
  }
  __syncthreads();
  if (p.history) {
    const unsigned long long slot = *p.history_count % (unsigned long long)p.history_cap;
    for (int t = threadIdx.x; t < nT; t += blockDim.x) {
      const int g = p.rep_of_temp[sd.temp_base + t];
      const double e = p.energy_is_global ? p.energy[g] : p.energy[sd.rep_ctx_base + g];
      p.history[slot * p.total_temps + sd.temp_base + t] = e;
    }
  }
  __syncthreads();
  if (p.do_swap) {
    const int parity = p.parity >= 0 ? p.parity : (int)(count & 1ull);
    for (int t = 2 * threadIdx.x + parity; t + 1 < nT; t += 2 * blockDim.x) {
      const int ga = p.rep_of_temp[sd.temp_base + t];
      const int gb = p.rep_of_temp[sd.temp_base + t + 1];
      const double ea = p.energy_is_global ? p.energy[ga] : p.energy[sd.rep_ctx_base + ga];
      const double eb = p.energy_is_global ? p.energy[gb] : p.energy[sd.rep_ctx_base + gb];
      uint32_t r[4];
      pyro_philox((uint32_t)t, (uint32_t)count, (uint32_t)sd.swap_key, PYRO_PURPOSE_SWAP, p.seed_lo,
                  p.seed_hi, r);
      const double u = pyro_uniform53(r[0], r[1]);
      const int acc =
          pyro_swap_accept(p.beta64[sd.temp_base + t], p.beta64[sd.temp_base + t + 1], ea, eb, u);
      p.swap_try[sd.temp_base + t] += 1ull;
      if (acc) {
        p.rep_of_temp[sd.temp_base + t] = gb;
        p.rep_of_temp[sd.temp_base + t + 1] = ga;
        p.temp_of_rep[sd.temp_base + ga] = t + 1;
        p.temp_of_rep[sd.temp_base + gb] = t;
        p.swap_acc[sd.temp_base + t] += 1ull;
        atomicAdd(&n_acc, 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (p.do_swap) {
      p.swap_count[si] = count + 1ull;
      if (p.last_accepted) p.last_accepted[si] = n_acc;
    }
  }
  // The last block to run cannot be known without a grid sync; block 0 of
  // the launch owns the context-wide counters (each launch covers all systems).
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (p.history) *p.history_count += 1ull;
    if (p.sweep_ctr) *p.sweep_ctr += p.sweep_advance;
  }
}

__global__ void advance_kernel(unsigned long long* ctr, unsigned long long by) { *ctr += by; }

__global__ void check_spins_kernel(const float4* spins, long long n, float tol,
                                   unsigned long long* first_bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 v = spins[i];
    const float n2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const bool ok = isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && fabsf(n2 - 1.0f) <= tol;
    if (!ok) atomicMin(first_bad, (unsigned long long)i);
  }
}

}  // namespace

namespace {
template <typename Kernel>
void launch_pass_kernel(Kernel k, int n_blocks, const PassParams& p, const NbrTable& tab,
                        cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n_blocks, 1, 1);
  cfg.blockDim = dim3(kPassThreads, 1, 1);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, p, tab);  // errors are read back with cudaGetLastError
}
}  // namespace

void launch_colour_pass(const PassParams& p, const NbrTable& tab, int n_blocks, bool metro,
                        bool j1_only, cudaStream_t st) {
  if (n_blocks <= 0) return;
  if (metro) {
    if (j1_only) launch_pass_kernel(colour_pass_kernel<true, true>, n_blocks, p, tab, st);
    else launch_pass_kernel(colour_pass_kernel<false, true>, n_blocks, p, tab, st);
  } else {
    if (j1_only) launch_pass_kernel(colour_pass_kernel<true, false>, n_blocks, p, tab, st);
    else launch_pass_kernel(colour_pass_kernel<false, false>, n_blocks, p, tab, st);
  }
}

void launch_init_random(float4* spins, const SysDev* sys_host, const SysDev* sys_dev, int n_sys,
                        uint32_t seed_lo, uint32_t seed_hi, cudaStream_t st) {
  const SysDev& last = sys_host[n_sys - 1];
  const long long total = last.spin_off + (long long)last.n_rep * 16 * last.L3;
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  init_random_kernel<<<(int)blocks, 256, 0, st>>>(spins, sys_dev, n_sys, total, seed_lo, seed_hi);
}

void launch_observables(const ObsParams& p, const NbrTable& tab, int n_blocks, cudaStream_t st) {
  observables_kernel<<<n_blocks, kObsThreads, 0, st>>>(p, tab);
}

void launch_obs_finalise(const double4* partials, const ObsSeg* segs, int nseg, const SysDev* sys,
                         int total_reps, const int* rep_sys, const int* rep_local,
                         double* energy_rep, double* mag_rep, cudaStream_t st) {
  (void)nseg;
  const int threads = 256;
  const int blocks = (total_reps * 32 + threads - 1) / threads;
  obs_finalise_kernel<<<blocks, threads, 0, st>>>(partials, segs, sys, total_reps, rep_sys,
                                                   rep_local, energy_rep, mag_rep);
}

void launch_exchange(const ExchangeParams& p, int n_sys, int max_pairs, cudaStream_t st) {
  int threads = p.partials ? 512 : 32;  // finalising: a warp per replica, 16 at a time
  while (threads < max_pairs && threads < 1024) threads *= 2;
  exchange_kernel<<<n_sys, threads, 0, st>>>(p);
}

void launch_advance(unsigned long long* ctr, unsigned long long by, cudaStream_t st) {
  advance_kernel<<<1, 1, 0, st>>>(ctr, by);
}

void launch_check_spins(const float4* spins, long long n, float tol, unsigned long long* first_bad,
                        cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  check_spins_kernel<<<(int)blocks, 256, 0, st>>>(spins, n, tol, first_bad);
}

}  // namespace pyro
