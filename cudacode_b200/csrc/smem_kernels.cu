// Small lattices resident in shared memory, for sm_100a.
//
// For L <= 8 a replica (16 L^3 float4, at most 128 KiB) fits in one CTA's
// shared memory. One CTA per replica then runs many whole cycles (Metropolis
// and over-relaxation sweeps, every colour pass separated by __syncthreads,
// and the FP64 energy after each cycle) in a single launch: no kernel launch
// and no HBM round trip per pass, which is what bounds the per-pass kernels
// at these sizes. The updates are exactly those of the other kernels (same
// neighbour order, same pyro_math.h arithmetic, same Philox counters), so the
// results are bit-identical.
//
// Replaces the reference's special 4x4x4 shared-memory kernel MCKernel4x4x4
// (Pyrochlore.cu:713-827), which loaded the wrong cells across blocks.
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "smem_kernels.cuh"

namespace pyro {
namespace {

__device__ __forceinline__ int wrap_s(int v, int L) {
  v = v < 0 ? v + L : v;
  return v >= L ? v - L : v;
}

__device__ __forceinline__ float3 shell_sum_smem(const float4* lat, const NbrTable& tab, int s,
                                                 int first, int last, int x, int y, int z, int L,
                                                 int L3) {
  float3 a;
  {
    const NbrEntry e = tab.e[s][first];
    const float4 v =
        lat[(wrap_s(z + e.dz, L) * L + wrap_s(y + e.dy, L)) * L + wrap_s(x + e.dx, L) + e.t * L3];
    a = make_float3(v.x, v.y, v.z);
  }
  for (int k = first + 1; k < last; ++k) {
    const NbrEntry e = tab.e[s][k];
    const float4 v =
        lat[(wrap_s(z + e.dz, L) * L + wrap_s(y + e.dy, L)) * L + wrap_s(x + e.dx, L) + e.t * L3];
    a.x = a.x + v.x;
    a.y = a.y + v.y;
    a.z = a.z + v.z;
  }
  return a;
}

// Nearest-neighbour field with bond matrices minus the Zeeman field, in the
// arithmetic of the per-pass kernels (pyro_matvec_add in table order).
__device__ __forceinline__ pyro_vec3 exch_field_smem(const float4* lat, const NbrTable& tab,
                                                     const ExchangeDev& X, int s, int x, int y,
                                                     int z, int L, int L3) {
  const int b = s & 3;
  pyro_vec3 h;
  h.x = h.y = h.z = 0.0f;
  for (int k = 0; k < 6; ++k) {
    const NbrEntry e = tab.e[s][k];
    const float4 v =
        lat[(wrap_s(z + e.dz, L) * L + wrap_s(y + e.dy, L)) * L + wrap_s(x + e.dx, L) + e.t * L3];
    h = pyro_matvec_add(h, X.A[4 * b + (e.t & 3)], v.x, v.y, v.z);
  }
  h.x = h.x - X.f[b][0];
  h.y = h.y - X.f[b][1];
  h.z = h.z - X.f[b][2];
  return h;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  __syncthreads();
  return s;
}

// This thread's share of twice the FP64 energy of the replica in shared
// memory: sum over its sites of S_i . h_i (bonds counted from both ends;
// with bond matrices, minus twice the Zeeman term).
__device__ double energy2_share(const float4* lat, const NbrTable& tab, const SysDev& sd,
                                const ExchangeDev* exch, int L, int L3, int n) {
  double e = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int s = i / L3, cell = i - s * L3;
    const int x = cell % L, yz = cell / L, y = yz % L, z = yz / L;
    const float4 sv = lat[i];
    const int sb[5] = {0, 6, 18, 24, 30};
    if (sd.exch >= 0) {  // twice the bond energy of this site minus twice its Zeeman term
      const ExchangeDev& X = exch[sd.exch];
      const int b = s & 3;
      double hx = -2.0 * X.f64[b][0], hy = -2.0 * X.f64[b][1], hz = -2.0 * X.f64[b][2];
      for (int q = 0; q < 6; ++q) {
        const NbrEntry en = tab.e[s][q];
        const float4 v = lat[(wrap_s(z + en.dz, L) * L + wrap_s(y + en.dy, L)) * L +
                             wrap_s(x + en.dx, L) + en.t * L3];
        const double* m = X.A64[4 * b + (en.t & 3)];
        hx += m[0] * v.x + m[1] * v.y + m[2] * v.z;
        hy += m[3] * v.x + m[4] * v.y + m[5] * v.z;
        hz += m[6] * v.x + m[7] * v.y + m[8] * v.z;
      }
      e += (double)sv.x * hx + (double)sv.y * hy + (double)sv.z * hz;
    }
    for (int sh = 0; sh < 4; ++sh) {
      if (!(sd.shells & (1 << sh))) continue;
      if (sh == 0 && sd.exch >= 0) continue;
      double ax = 0.0, ay = 0.0, az = 0.0;
      for (int q = sb[sh]; q < sb[sh + 1]; ++q) {
        const NbrEntry en = tab.e[s][q];
        const float4 v = lat[(wrap_s(z + en.dz, L) * L + wrap_s(y + en.dy, L)) * L +
                             wrap_s(x + en.dx, L) + en.t * L3];
        ax += v.x;
        ay += v.y;
        az += v.z;
      }
      e += sd.J64[sh] * ((double)sv.x * ax + (double)sv.y * ay + (double)sv.z * az);
    }
  }
  return e;
}

// Isotropic J1-only systems: the colour pass with L and the neighbour
// offsets as compile-time constants (periodic wraps by selects, cell decode
// by constant division). Same arithmetic as the generic pass.
template <int L, int S, int K>
__device__ __forceinline__ int j1_nbr(int x, int y, int z) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  const int xx = e.dx == 0 ? x : (e.dx > 0 ? (x == L - 1 ? 0 : x + 1) : (x == 0 ? L - 1 : x - 1));
  const int yy = e.dy == 0 ? y : (e.dy > 0 ? (y == L - 1 ? 0 : y + 1) : (y == 0 ? L - 1 : y - 1));
  const int zz = e.dz == 0 ? z : (e.dz > 0 ? (z == L - 1 ? 0 : z + 1) : (z == 0 ? L - 1 : z - 1));
  return (zz * L + yy) * L + xx + e.t * L * L * L;
}

template <int L, int S, bool kMetro>
__device__ __forceinline__ int j1_site_smem(float4* lat, int cell, float J1, float beta,
                                            float cosmax, uint32_t rkey, uint32_t sweep32,
                                            bool renorm, uint32_t seed_lo, uint32_t seed_hi) {
  constexpr int L3 = L * L * L;
  const int x = cell % L, y = (cell / L) % L, z = cell / (L * L);
  const float4 n0 = lat[j1_nbr<L, S, 0>(x, y, z)], n1 = lat[j1_nbr<L, S, 1>(x, y, z)],
               n2 = lat[j1_nbr<L, S, 2>(x, y, z)], n3 = lat[j1_nbr<L, S, 3>(x, y, z)],
               n4 = lat[j1_nbr<L, S, 4>(x, y, z)], n5 = lat[j1_nbr<L, S, 5>(x, y, z)];
  pyro_vec3 h;
  h.x = J1 * (((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x);
  h.y = J1 * (((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y);
  h.z = J1 * (((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z);
  const int own = S * L3 + cell;
  const float4 sv = lat[own];
  pyro_vec3 sp;
  sp.x = sv.x;
  sp.y = sv.y;
  sp.z = sv.z;
  pyro_vec3 out;
  int a = 0;
  if (kMetro) {
    uint32_t r[4];
    pyro_philox((uint32_t)own, rkey, sweep32, PYRO_PURPOSE_METRO, seed_lo, seed_hi, r);
    const pyro_vec3 prop = pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
    a = pyro_metropolis_accept(pyro_delta_e(h, sp, prop), beta, pyro_uniform(r[2]));
    out = a ? prop : sp;
  } else {
    out = pyro_overrelax(sp, h);
  }
  if (renorm) out = pyro_renormalise(out);
  lat[own] = make_float4(out.x, out.y, out.z, 0.0f);
  return a;
}

// Colour B of the 4-colour schedule: sites B, 4+B, 8+B, 12+B of every cell.
template <int L, int B, bool kMetro>
__device__ __forceinline__ unsigned long long j1_pass_smem(float4* lat, float J1, float beta,
                                                           float cosmax, uint32_t rkey,
                                                           uint32_t sweep32, bool renorm,
                                                           uint32_t seed_lo, uint32_t seed_hi) {
  constexpr int L3 = L * L * L;
  unsigned long long acc = 0;
  for (int u = threadIdx.x; u < 4 * L3; u += blockDim.x) {
    const int k = u / L3, cell = u - k * L3;
    switch (k) {
      case 0: acc += j1_site_smem<L, B, kMetro>(lat, cell, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi); break;
      case 1: acc += j1_site_smem<L, 4 + B, kMetro>(lat, cell, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi); break;
      case 2: acc += j1_site_smem<L, 8 + B, kMetro>(lat, cell, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi); break;
      default: acc += j1_site_smem<L, 12 + B, kMetro>(lat, cell, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi); break;
    }
  }
  return acc;
}

// Twice the FP64 energy of an isotropic J1-only replica of fixed L from its
// tetrahedra (this thread's share): every bond lies in exactly one
// tetrahedron, and a tetrahedron's bonds sum to (|sum S|^2 - sum |S|^2) / 2.
// Each cell holds its four up-tetrahedra (sites 4F..4F+3) and the four down-
// tetrahedra through its sublattice-0 sites 4F. Same value as energy2_share
// up to FP64 rounding, from 8 tetrahedra per cell instead of 6 neighbours
// per site.
__device__ __forceinline__ double tet_pairs(float4 a, float4 b, float4 c, float4 d) {
  const double mx = (double)a.x + b.x + c.x + d.x;
  const double my = (double)a.y + b.y + c.y + d.y;
  const double mz = (double)a.z + b.z + c.z + d.z;
  const double n2 = (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z +
                    (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z +
                    (double)c.x * c.x + (double)c.y * c.y + (double)c.z * c.z +
                    (double)d.x * d.x + (double)d.y * d.y + (double)d.z * d.z;
  return mx * mx + my * my + mz * mz - n2;  // twice the sum of the pair products
}

template <int L, int F>
__device__ __forceinline__ double j1_cell_corner2(const float4* lat, int cell, int x, int y, int z) {
  constexpr int L3 = L * L * L, S = 4 * F;
  const float4 s0 = lat[S * L3 + cell], s1 = lat[(S + 1) * L3 + cell],
               s2 = lat[(S + 2) * L3 + cell], s3 = lat[(S + 3) * L3 + cell];
  const float4 d1 = lat[j1_nbr<L, S, j1_down_index(S, 0)>(x, y, z)];
  const float4 d2 = lat[j1_nbr<L, S, j1_down_index(S, 1)>(x, y, z)];
  const float4 d3 = lat[j1_nbr<L, S, j1_down_index(S, 2)>(x, y, z)];
  return tet_pairs(s0, s1, s2, s3) + tet_pairs(s0, d1, d2, d3);
}

template <int L>
__device__ double j1_energy2_share(const float4* lat, double J1) {
  constexpr int L3 = L * L * L;
  double e = 0.0;
  for (int cell = threadIdx.x; cell < L3; cell += blockDim.x) {
    const int x = cell % L, y = (cell / L) % L, z = cell / (L * L);
    e += j1_cell_corner2<L, 0>(lat, cell, x, y, z) + j1_cell_corner2<L, 1>(lat, cell, x, y, z) +
         j1_cell_corner2<L, 2>(lat, cell, x, y, z) + j1_cell_corner2<L, 3>(lat, cell, x, y, z);
  }
  return J1 * e;  // = sum over sites of S_i . h_i, as energy2_share
}

// Spin-independent part of a Metropolis update: the Philox words of the
// site and the cone geometry they give (cos, sin of the polar angle, the
// azimuth's cos and sin, the acceptance uniform), exactly as
// pyro_cone_proposal / pyro_metropolis_accept compute them.
struct MetroDraw {
  float ct, st, cp, sp, u3;
};

__device__ __forceinline__ MetroDraw metro_draw(uint32_t own, uint32_t rkey, uint32_t sweep32,
                                                float cosmax, uint32_t seed_lo,
                                                uint32_t seed_hi) {
  uint32_t r[4];
  pyro_philox(own, rkey, sweep32, PYRO_PURPOSE_METRO, seed_lo, seed_hi, r);
  MetroDraw d;
  d.ct = fmaf(-(1.0f - cosmax), pyro_uniform(r[0]), 1.0f);
  d.st = sqrtf(fmaxf(0.0f, fmaf(-d.ct, d.ct, 1.0f)));
  pyro_sincospif(2.0f * pyro_uniform(r[1]), &d.sp, &d.cp);
  d.u3 = pyro_uniform(r[2]);
  return d;
}

// Site S's Metropolis update from its precomputed draw.
template <int L, int S>
__device__ __forceinline__ int j1_metro_drawn(float4* lat, int cell, float J1, float beta,
                                              const MetroDraw& d, bool renorm) {
  constexpr int L3 = L * L * L;
  const int x = cell % L, y = (cell / L) % L, z = cell / (L * L);
  const float4 n0 = lat[j1_nbr<L, S, 0>(x, y, z)], n1 = lat[j1_nbr<L, S, 1>(x, y, z)],
               n2 = lat[j1_nbr<L, S, 2>(x, y, z)], n3 = lat[j1_nbr<L, S, 3>(x, y, z)],
               n4 = lat[j1_nbr<L, S, 4>(x, y, z)], n5 = lat[j1_nbr<L, S, 5>(x, y, z)];
  pyro_vec3 h;
  h.x = J1 * (((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x);
  h.y = J1 * (((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y);
  h.z = J1 * (((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z);
  const int own = S * L3 + cell;
  const float4 sv = lat[own];
  pyro_vec3 sp;
  sp.x = sv.x;
  sp.y = sv.y;
  sp.z = sv.z;
  const pyro_vec3 prop = pyro_about_axis(sp, d.ct, d.st, d.cp, d.sp);
  const int a = pyro_metropolis_accept(pyro_delta_e(h, sp, prop), beta, d.u3);
  pyro_vec3 out = a ? prop : sp;
  if (renorm) out = pyro_renormalise(out);
  lat[own] = make_float4(out.x, out.y, out.z, 0.0f);
  return a;
}

template <int L, int B>
__device__ __forceinline__ int j1_metro_pass_drawn(float4* lat, float J1, float beta,
                                                   const MetroDraw& d, bool renorm) {
  constexpr int L3 = L * L * L;
  const int u = threadIdx.x;
  if (u >= 4 * L3) return 0;
  const int k = u / L3, cell = u - k * L3;
  switch (k) {
    case 0: return j1_metro_drawn<L, B>(lat, cell, J1, beta, d, renorm);
    case 1: return j1_metro_drawn<L, 4 + B>(lat, cell, J1, beta, d, renorm);
    case 2: return j1_metro_drawn<L, 8 + B>(lat, cell, J1, beta, d, renorm);
    default: return j1_metro_drawn<L, 12 + B>(lat, cell, J1, beta, d, renorm);
  }
}

// Lattices whose colour classes have at most one site per thread
// (4 L^3 <= kSmemThreads): a thread's corner k and cell never change, so the
// shared-memory indices of its site's 6 neighbours and its own spin, for
// each of the 4 colours, are computed once per launch. The passes then run
// one code body per colour and no address arithmetic.
struct SiteIdx {
  int n[4][7];  // per colour b: neighbours 0..5 of site 4 k + b, then the site itself
};

template <int L, int S>
__device__ __forceinline__ void site_idx(int* out, int x, int y, int z, int cell) {
  out[0] = j1_nbr<L, S, 0>(x, y, z);
  out[1] = j1_nbr<L, S, 1>(x, y, z);
  out[2] = j1_nbr<L, S, 2>(x, y, z);
  out[3] = j1_nbr<L, S, 3>(x, y, z);
  out[4] = j1_nbr<L, S, 4>(x, y, z);
  out[5] = j1_nbr<L, S, 5>(x, y, z);
  out[6] = S * L * L * L + cell;
}

template <int L, int B>
__device__ __forceinline__ void colour_idx(int* out, int k, int x, int y, int z, int cell) {
  switch (k) {
    case 0: site_idx<L, B>(out, x, y, z, cell); break;
    case 1: site_idx<L, 4 + B>(out, x, y, z, cell); break;
    case 2: site_idx<L, 8 + B>(out, x, y, z, cell); break;
    default: site_idx<L, 12 + B>(out, x, y, z, cell); break;
  }
}

template <int L>
__device__ __forceinline__ SiteIdx make_site_idx(int k, int cell) {
  const int x = cell % L, y = (cell / L) % L, z = cell / (L * L);
  SiteIdx t;
  colour_idx<L, 0>(t.n[0], k, x, y, z, cell);
  colour_idx<L, 1>(t.n[1], k, x, y, z, cell);
  colour_idx<L, 2>(t.n[2], k, x, y, z, cell);
  colour_idx<L, 3>(t.n[3], k, x, y, z, cell);
  return t;
}

// One site update from precomputed indices (the arithmetic of
// j1_site_smem / j1_metro_drawn).
template <bool kMetro>
__device__ __forceinline__ int idx_update(float4* lat, const int* ix, float J1, float beta,
                                          const MetroDraw& d, bool renorm) {
  const float4 n0 = lat[ix[0]], n1 = lat[ix[1]], n2 = lat[ix[2]], n3 = lat[ix[3]],
               n4 = lat[ix[4]], n5 = lat[ix[5]];
  pyro_vec3 h;
  h.x = J1 * (((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x);
  h.y = J1 * (((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y);
  h.z = J1 * (((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z);
  const float4 sv = lat[ix[6]];
  pyro_vec3 sp;
  sp.x = sv.x;
  sp.y = sv.y;
  sp.z = sv.z;
  pyro_vec3 out;
  int a = 0;
  if (kMetro) {
    const pyro_vec3 prop = pyro_about_axis(sp, d.ct, d.st, d.cp, d.sp);
    a = pyro_metropolis_accept(pyro_delta_e(h, sp, prop), beta, d.u3);
    out = a ? prop : sp;
  } else {
    out = pyro_overrelax(sp, h);
  }
  if (renorm) out = pyro_renormalise(out);
  lat[ix[6]] = make_float4(out.x, out.y, out.z, 0.0f);
  return a;
}

// A sweep of a small lattice from precomputed indices (4 L^3 <= kSmemThreads).
template <int L, bool kMetro>
__device__ __forceinline__ unsigned long long idx_sweep(float4* lat, const SiteIdx& t, int k,
                                                        int cell, float J1, float beta,
                                                        float cosmax, uint32_t rkey,
                                                        uint32_t sweep32, bool renorm,
                                                        uint32_t seed_lo, uint32_t seed_hi) {
  constexpr int L3 = L * L * L;
  const bool active = threadIdx.x < 4 * L3;
  MetroDraw d[4];
  if (kMetro) {
#pragma unroll
    for (int b = 0; b < 4; ++b)
      d[b] = metro_draw((uint32_t)((4 * k + b) * L3 + cell), rkey, sweep32, cosmax, seed_lo,
                        seed_hi);
  }
  unsigned long long acc = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    if (active) acc += idx_update<kMetro>(lat, t.n[b], J1, beta, d[b], renorm);
    __syncthreads();
  }
  return acc;
}

template <int L, bool kMetro>
__device__ __forceinline__ unsigned long long j1_sweep_smem(float4* lat, float J1, float beta,
                                                            float cosmax, uint32_t rkey,
                                                            uint32_t sweep32, bool renorm,
                                                            uint32_t seed_lo, uint32_t seed_hi) {
  constexpr int L3 = L * L * L;
  if constexpr (kMetro && 4 * L3 <= kSmemThreads) {
    // one site per thread and colour: the four draws of the sweep do not
    // depend on the spins, so they are computed up front as four
    // independent chains, off the passes' critical path
    MetroDraw d[4];
    const int u = threadIdx.x < 4 * L3 ? threadIdx.x : 0;
    const int k = u / L3, cell = u - k * L3;
#pragma unroll
    for (int b = 0; b < 4; ++b)
      d[b] = metro_draw((uint32_t)((4 * k + b) * L3 + cell), rkey, sweep32, cosmax, seed_lo,
                        seed_hi);
    unsigned long long acc = 0;
    acc += j1_metro_pass_drawn<L, 0>(lat, J1, beta, d[0], renorm);
    __syncthreads();
    acc += j1_metro_pass_drawn<L, 1>(lat, J1, beta, d[1], renorm);
    __syncthreads();
    acc += j1_metro_pass_drawn<L, 2>(lat, J1, beta, d[2], renorm);
    __syncthreads();
    acc += j1_metro_pass_drawn<L, 3>(lat, J1, beta, d[3], renorm);
    __syncthreads();
    return acc;
  }
  unsigned long long acc = 0;
  acc += j1_pass_smem<L, 0, kMetro>(lat, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi);
  __syncthreads();
  acc += j1_pass_smem<L, 1, kMetro>(lat, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi);
  __syncthreads();
  acc += j1_pass_smem<L, 2, kMetro>(lat, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi);
  __syncthreads();
  acc += j1_pass_smem<L, 3, kMetro>(lat, J1, beta, cosmax, rkey, sweep32, renorm, seed_lo, seed_hi);
  __syncthreads();
  return acc;
}

// kL = 0: any system (neighbour table at run time); kL > 0: an isotropic
// J1-only system of that L (compile-time offsets).
template <int kL>
__global__ void __launch_bounds__(kSmemThreads) smem_cycles_kernel(const SmemCycleParams p,
                                                                   const NbrTable tab) {
  extern __shared__ float4 lat[];
  __shared__ double red[kSmemThreads / 32];
  const SysDev sd = p.sys;
  const int L = sd.L, L3 = sd.L3, n = 16 * L3;
  const int rep = blockIdx.x;
  float4* g = p.spins + (long long)rep * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) lat[i] = g[i];
  const int slot = p.temp_of_rep[sd.temp_base + sd.rep_global + rep];
  const float beta = p.beta[sd.temp_base + slot];
  const float cosmax = p.cosmax[sd.temp_base + slot];
  const uint32_t rkey = (uint32_t)(sd.rep_key + rep);
  const unsigned long long base = *p.sweep_ctr;
  const unsigned long long hist0 = p.history ? *p.history_count : 0ull;
  const int per_cycle = p.n_metro + p.n_or;
  __syncthreads();
  unsigned long long acc = 0;
  constexpr bool kIdx = kL > 0 && 4 * kL * kL * kL <= kSmemThreads;
  const int my_k = kIdx ? (int)threadIdx.x / (kL * kL * kL > 0 ? kL * kL * kL : 1) : 0;
  const int my_cell = kIdx ? (int)threadIdx.x - my_k * kL * kL * kL : 0;
  SiteIdx site_ix;
  if constexpr (kIdx) site_ix = make_site_idx<kL>(my_k < 4 ? my_k : 0, my_cell);
  for (int c = 0; c < p.n_cycles; ++c) {
    for (int k = 0; k < per_cycle; ++k) {
      const unsigned long long sweep = base + (unsigned long long)c * per_cycle + k;
      const bool metro = k < p.n_metro;
      const bool renorm =
          p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0;
      if constexpr (kIdx) {
        acc += metro ? idx_sweep<kL, true>(lat, site_ix, my_k, my_cell, sd.J1, beta, cosmax,
                                           rkey, (uint32_t)sweep, renorm, p.seed_lo, p.seed_hi)
                     : idx_sweep<kL, false>(lat, site_ix, my_k, my_cell, sd.J1, beta, cosmax,
                                            rkey, (uint32_t)sweep, renorm, p.seed_lo,
                                            p.seed_hi);
      } else if constexpr (kL > 0) {
        acc += metro ? j1_sweep_smem<kL, true>(lat, sd.J1, beta, cosmax, rkey, (uint32_t)sweep,
                                               renorm, p.seed_lo, p.seed_hi)
                     : j1_sweep_smem<kL, false>(lat, sd.J1, beta, cosmax, rkey, (uint32_t)sweep,
                                                renorm, p.seed_lo, p.seed_hi);
      } else {
        for (int colour = 0; colour < sd.n_colours; ++colour) {
          for (int u = threadIdx.x; u < sd.units_per_colour; u += blockDim.x) {
            const int kk = u / L3, cell = u - kk * L3;
            const int s = colour_site(sd.n_colours, colour, kk);
            const int x = cell % L, yz = cell / L, y = yz % L, z = yz / L;
            const int own = s * L3 + cell;
            pyro_vec3 h;
            if (sd.exch >= 0) {
              h = exch_field_smem(lat, tab, p.exch[sd.exch], s, x, y, z, L, L3);
            } else {
              const float3 a1 = shell_sum_smem(lat, tab, s, 0, 6, x, y, z, L, L3);
              h.x = sd.J1 * a1.x;
              h.y = sd.J1 * a1.y;
              h.z = sd.J1 * a1.z;
            }
            if (sd.shells & 2) {
              const float3 a = shell_sum_smem(lat, tab, s, 6, 18, x, y, z, L, L3);
              h.x = fmaf(sd.J2, a.x, h.x);
              h.y = fmaf(sd.J2, a.y, h.y);
              h.z = fmaf(sd.J2, a.z, h.z);
            }
            if (sd.shells & 4) {
              const float3 a = shell_sum_smem(lat, tab, s, 18, 24, x, y, z, L, L3);
              h.x = fmaf(sd.J3a, a.x, h.x);
              h.y = fmaf(sd.J3a, a.y, h.y);
              h.z = fmaf(sd.J3a, a.z, h.z);
            }
            if (sd.shells & 8) {
              const float3 a = shell_sum_smem(lat, tab, s, 24, 30, x, y, z, L, L3);
              h.x = fmaf(sd.J3b, a.x, h.x);
              h.y = fmaf(sd.J3b, a.y, h.y);
              h.z = fmaf(sd.J3b, a.z, h.z);
            }
            const float4 sv = lat[own];
            pyro_vec3 sp;
            sp.x = sv.x;
            sp.y = sv.y;
            sp.z = sv.z;
            pyro_vec3 out;
            if (metro) {
              uint32_t r[4];
              pyro_philox((uint32_t)own, rkey, (uint32_t)sweep, PYRO_PURPOSE_METRO, p.seed_lo,
                          p.seed_hi, r);
              const pyro_vec3 prop =
                  pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
              const int a = pyro_metropolis_accept(pyro_delta_e(h, sp, prop), beta, pyro_uniform(r[2]));
              acc += (unsigned long long)a;
              out = a ? prop : sp;
            } else {
              out = pyro_overrelax(sp, h);
            }
            if (renorm) out = pyro_renormalise(out);
            lat[own] = make_float4(out.x, out.y, out.z, 0.0f);
          }
          __syncthreads();
        }
      }
    }
    if (p.history) {
      // FP64 energy of the cycle's final state: E = 1/2 sum_i S_i . h_i
      double e;
      if constexpr (kL > 0) e = j1_energy2_share<kL>(lat, sd.J64[0]);
      else e = energy2_share(lat, tab, sd, p.exch, L, L3, n);
      const double tot = block_sum(e, red);
      if (threadIdx.x == 0) {
        const unsigned long long row = (hist0 + c) % (unsigned long long)p.history_cap;
        p.history[row * p.total_temps + sd.temp_base + slot] = 0.5 * tot;
      }
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) g[i] = lat[i];
  if (p.energy) {  // observables of the final state, as the per-pass path leaves them
    double e2;
    if constexpr (kL > 0) e2 = j1_energy2_share<kL>(lat, sd.J64[0]);
    else e2 = energy2_share(lat, tab, sd, p.exch, L, L3, n);
    const double e = block_sum(e2, red);
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      mx += lat[i].x;
      my += lat[i].y;
      mz += lat[i].z;
    }
    mx = block_sum(mx, red);
    my = block_sum(my, red);
    mz = block_sum(mz, red);
    if (threadIdx.x == 0) {
      const int gi = sd.rep_ctx_base + rep;
      p.energy[gi] = 0.5 * e;
      p.mag[3 * gi] = mx;
      p.mag[3 * gi + 1] = my;
      p.mag[3 * gi + 2] = mz;
    }
  }
  if (p.n_metro > 0) {
    const double a = block_sum((double)acc, red);
    if (threadIdx.x == 0 && a > 0.0)
      atomicAdd(p.accepted + sd.temp_base + slot, (unsigned long long)(a + 0.5));
  }
}

}  // namespace

size_t smem_cycle_bytes(int L) { return sizeof(float4) * 16 * (size_t)L * L * L; }

namespace {
template <int kL>
cudaError_t launch_smem(const SmemCycleParams& p, const NbrTable& tab, size_t bytes,
                        cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(smem_cycles_kernel<kL>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  smem_cycles_kernel<kL><<<p.sys.n_rep, kSmemThreads, bytes, st>>>(p, tab);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_smem_cycles(const SmemCycleParams& p, const NbrTable& tab, cudaStream_t st) {
  const size_t bytes = smem_cycle_bytes(p.sys.L);
  const SysDev& s = p.sys;
  if (s.n_colours == 4 && s.shells == 1 && s.exch < 0) {
    switch (s.L) {
      case 2: return launch_smem<2>(p, tab, bytes, st);
      case 3: return launch_smem<3>(p, tab, bytes, st);
      case 4: return launch_smem<4>(p, tab, bytes, st);
      case 5: return launch_smem<5>(p, tab, bytes, st);
      case 6: return launch_smem<6>(p, tab, bytes, st);
      case 7: return launch_smem<7>(p, tab, bytes, st);
      case 8: return launch_smem<8>(p, tab, bytes, st);
      default: break;
    }
  }
  return launch_smem<0>(p, tab, bytes, st);
}

}  // namespace pyro
