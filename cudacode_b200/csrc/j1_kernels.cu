// Nearest-neighbour (J1-only) kernels: the 4-colour schedule of the
// pyrochlore Heisenberg model, specialised for sm_100a.
//
// One thread owns one cubic cell of one replica and, in the pass of colour b,
// updates the four sites {b, 4+b, 8+b, 12+b} of that cell (one per FCC
// corner; none of them are neighbours). The 24 neighbour offsets are
// compile-time constants (j1_neighbour), so a neighbour address is three
// integer adds of precomputed row offsets; the periodic wrap is computed once
// per thread. The arithmetic of each update is exactly that of the generic
// colour pass (same neighbour order, same pyro_math.h functions), so both
// kernels and the host oracle agree bit for bit.
//
// Replaces MCMultipleTemperaturesPerSystem (Pyrochlore.cu:829-885, one thread
// per cell, 4 sites of a bond-free group) and OverRelaxationByPiStep
// (975-1007); the observables kernel replaces TotalEnergyGPU (344-389) and
// MagnetizationGPU (277-342) by sums over tetrahedra.
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "j1_kernels.cuh"

namespace pyro {
namespace {

struct CellFrame {
  int zo[3], yo[3], xo[3];  // offsets of the rows/columns at -1, 0, +1
};

// cell -> (x, y, z) with a float reciprocal and one correction step
// (exact for cell < 2^24, i.e. L <= 256).
__device__ __forceinline__ void decode_cell(int cell, int L, float rcpL, int* x, int* y, int* z) {
  int q = (int)((float)cell * rcpL);
  int r = cell - q * L;
  if (r < 0) { --q; r += L; } else if (r >= L) { ++q; r -= L; }
  *x = r;
  int q2 = (int)((float)q * rcpL);
  int r2 = q - q2 * L;
  if (r2 < 0) { --q2; r2 += L; } else if (r2 >= L) { ++q2; r2 -= L; }
  *y = r2;
  *z = q2;
}

__device__ __forceinline__ CellFrame make_frame(int x, int y, int z, int L) {
  CellFrame f;
  const int L2 = L * L;
  const int xm = x == 0 ? L - 1 : x - 1, xp = x == L - 1 ? 0 : x + 1;
  const int ym = y == 0 ? L - 1 : y - 1, yp = y == L - 1 ? 0 : y + 1;
  const int zm = z == 0 ? L - 1 : z - 1, zp = z == L - 1 ? 0 : z + 1;
  f.xo[0] = xm;
  f.xo[1] = x;
  f.xo[2] = xp;
  f.yo[0] = ym * L;
  f.yo[1] = y * L;
  f.yo[2] = yp * L;
  f.zo[0] = zm * L2;
  f.zo[1] = z * L2;
  f.zo[2] = zp * L2;
  return f;
}

template <int S, int K>
__device__ __forceinline__ float4 load_neighbour(const float4* __restrict__ rep, const CellFrame& f,
                                                 int L3) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  return __ldg(rep + f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3);
}

// Sum of the 6 nearest neighbours of site S, in canonical order.
template <int S>
__device__ __forceinline__ pyro_vec3 j1_sum(const float4* __restrict__ rep, const CellFrame& f,
                                            int L3) {
  const float4 n0 = load_neighbour<S, 0>(rep, f, L3);
  const float4 n1 = load_neighbour<S, 1>(rep, f, L3);
  const float4 n2 = load_neighbour<S, 2>(rep, f, L3);
  const float4 n3 = load_neighbour<S, 3>(rep, f, L3);
  const float4 n4 = load_neighbour<S, 4>(rep, f, L3);
  const float4 n5 = load_neighbour<S, 5>(rep, f, L3);
  pyro_vec3 a;
  a.x = ((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x;
  a.y = ((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y;
  a.z = ((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z;
  return a;
}

template <int S, bool kMetro>
__device__ __forceinline__ int update_site(float4* __restrict__ rep, const CellFrame& f, int cell,
                                           int L3, float J1, float beta, float cosmax, uint32_t rkey,
                                           uint32_t sweep32, bool renorm, uint32_t seed_lo,
                                           uint32_t seed_hi) {
  const int own = S * L3 + cell;
  const float4 sv = rep[own];
  const pyro_vec3 a = j1_sum<S>(rep, f, L3);
  pyro_vec3 h;
  h.x = J1 * a.x;
  h.y = J1 * a.y;
  h.z = J1 * a.z;
  pyro_vec3 sp;
  sp.x = sv.x;
  sp.y = sv.y;
  sp.z = sv.z;
  pyro_vec3 out;
  int acc = 0;
  if (kMetro) {
    uint32_t r[4];
    pyro_philox((uint32_t)own, rkey, sweep32, PYRO_PURPOSE_METRO, seed_lo, seed_hi, r);
    const pyro_vec3 prop = pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
    const float dE = pyro_delta_e(h, sp, prop);
    acc = pyro_metropolis_accept(dE, beta, pyro_uniform(r[2]));
    out = acc ? prop : sp;
  } else {
    out = pyro_overrelax(sp, h);
  }
  if (renorm) out = pyro_renormalise(out);
  rep[own] = make_float4(out.x, out.y, out.z, 0.0f);
  return acc;
}

template <int B, bool kMetro>
__global__ void __launch_bounds__(kJ1Threads) j1_pass_kernel(const J1PassParams p) {
  const int rep = blockIdx.y;
  const int cell = blockIdx.x * kJ1Threads + threadIdx.x;
  const int g = p.rep_global + rep;
  float beta = 0.0f, cosmax = 0.0f;
  int t = 0;
  if (kMetro) {
    t = p.temp_of_rep[p.temp_base + g];
    beta = p.beta[p.temp_base + t];
    cosmax = p.cosmax[p.temp_base + t];
  }
  int acc = 0;
  if (cell < p.L3) {
    int x, y, z;
    decode_cell(cell, p.L, p.rcpL, &x, &y, &z);
    const CellFrame f = make_frame(x, y, z, p.L);
    float4* rb = p.spins + (long long)rep * 16 * p.L3;
    const unsigned long long sweep = (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off;
    const bool renorm =
        p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0;
    const uint32_t rkey = (uint32_t)(p.rep_key + rep);
    const uint32_t sw = (uint32_t)sweep;
    acc += update_site<B, kMetro>(rb, f, cell, p.L3, p.J1, beta, cosmax, rkey, sw, renorm,
                                  p.seed_lo, p.seed_hi);
    acc += update_site<4 + B, kMetro>(rb, f, cell, p.L3, p.J1, beta, cosmax, rkey, sw, renorm,
                                      p.seed_lo, p.seed_hi);
    acc += update_site<8 + B, kMetro>(rb, f, cell, p.L3, p.J1, beta, cosmax, rkey, sw, renorm,
                                      p.seed_lo, p.seed_hi);
    acc += update_site<12 + B, kMetro>(rb, f, cell, p.L3, p.J1, beta, cosmax, rkey, sw, renorm,
                                       p.seed_lo, p.seed_hi);
  }
  if (kMetro) {
    // Block-wide count of accepted moves: one atomic per CTA.
    __shared__ int warp_acc[kJ1Threads / 32];
    int v = acc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_acc[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
#pragma unroll
      for (int w = 0; w < kJ1Threads / 32; ++w) s += warp_acc[w];
      if (s > 0) atomicAdd(p.accepted + p.temp_base + t, (unsigned long long)s);
    }
  }
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Down-tetrahedron partners of the sublattice-0 site 4F of a cell.
template <int F>
__device__ __forceinline__ void down_partners(const float4* __restrict__ rep, const CellFrame& f,
                                              int L3, float4* d1, float4* d2, float4* d3) {
  constexpr int S0 = 4 * F;
  constexpr int k1 = j1_down_index(S0, 0), k2 = j1_down_index(S0, 1), k3 = j1_down_index(S0, 2);
  static_assert(k1 >= 0 && k2 >= 0 && k3 >= 0, "three down-tetrahedron partners");
  *d1 = load_neighbour<S0, k1>(rep, f, L3);
  *d2 = load_neighbour<S0, k2>(rep, f, L3);
  *d3 = load_neighbour<S0, k3>(rep, f, L3);
}

// E_tet = J1 * sum_{i<j in tet} S_i.S_j = J1/2 (|sum S|^2 - sum |S|^2), FP64.
__device__ __forceinline__ double tet_energy(float4 a, float4 b, float4 c, float4 d) {
  const double mx = (double)a.x + b.x + c.x + d.x;
  const double my = (double)a.y + b.y + c.y + d.y;
  const double mz = (double)a.z + b.z + c.z + d.z;
  const double n2 = (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z +
                    (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z +
                    (double)c.x * c.x + (double)c.y * c.y + (double)c.z * c.z +
                    (double)d.x * d.x + (double)d.y * d.y + (double)d.z * d.z;
  return 0.5 * (mx * mx + my * my + mz * mz - n2);
}

template <int F>
__device__ __forceinline__ void cell_corner(const float4* __restrict__ rep, const CellFrame& f,
                                            int cell, int L3, double* e, double* mx, double* my,
                                            double* mz) {
  const float4 s0 = __ldg(rep + (4 * F + 0) * L3 + cell);
  const float4 s1 = __ldg(rep + (4 * F + 1) * L3 + cell);
  const float4 s2 = __ldg(rep + (4 * F + 2) * L3 + cell);
  const float4 s3 = __ldg(rep + (4 * F + 3) * L3 + cell);
  float4 d1, d2, d3;
  down_partners<F>(rep, f, L3, &d1, &d2, &d3);
  *e += tet_energy(s0, s1, s2, s3) + tet_energy(s0, d1, d2, d3);
  *mx += (double)s0.x + s1.x + s2.x + s3.x;
  *my += (double)s0.y + s1.y + s2.y + s3.y;
  *mz += (double)s0.z + s1.z + s2.z + s3.z;
}

// Each cell owns its 4 up-tetrahedra and the 4 down-tetrahedra that contain
// its sublattice-0 sites: every bond is counted exactly once.
__global__ void __launch_bounds__(kJ1Threads) j1_observables_kernel(const J1ObsParams p) {
  const int rep = blockIdx.y;
  const int cell = blockIdx.x * kJ1Threads + threadIdx.x;
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  if (cell < p.L3) {
    int x, y, z;
    decode_cell(cell, p.L, p.rcpL, &x, &y, &z);
    const CellFrame f = make_frame(x, y, z, p.L);
    const float4* rb = p.spins + (long long)rep * 16 * p.L3;
    cell_corner<0>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    cell_corner<1>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    cell_corner<2>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    cell_corner<3>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    e *= p.J1;
  }
  __shared__ double red[4][kJ1Threads / 32];
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
    for (int q = 0; q < kJ1Threads / 32; ++q) {
      o.x += red[0][q];
      o.y += red[1][q];
      o.z += red[2][q];
      o.w += red[3][q];
    }
    // E is accumulated per tetrahedron (each bond once); the finalise step
    // halves the site sum of the generic kernel, so store 2 E here.
    o.x *= 2.0;
    p.partials[p.partial_begin + (long long)rep * gridDim.x + blockIdx.x] = o;
  }
}

}  // namespace

void launch_j1_pass(const J1PassParams& p, int colour, bool metro, cudaStream_t st) {
  const dim3 grid((p.L3 + kJ1Threads - 1) / kJ1Threads, p.n_rep);
#define PYRO_J1_CASE(B)                                                          \
  case B:                                                                        \
    if (metro) j1_pass_kernel<B, true><<<grid, kJ1Threads, 0, st>>>(p);          \
    else j1_pass_kernel<B, false><<<grid, kJ1Threads, 0, st>>>(p);               \
    break;
  switch (colour) {
    PYRO_J1_CASE(0)
    PYRO_J1_CASE(1)
    PYRO_J1_CASE(2)
    PYRO_J1_CASE(3)
    default:
      break;
  }
#undef PYRO_J1_CASE
}

void launch_j1_observables(const J1ObsParams& p, cudaStream_t st) {
  const dim3 grid((p.L3 + kJ1Threads - 1) / kJ1Threads, p.n_rep);
  j1_observables_kernel<<<grid, kJ1Threads, 0, st>>>(p);
}

}  // namespace pyro
