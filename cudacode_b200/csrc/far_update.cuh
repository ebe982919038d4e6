// The update of one site of a 16-colour system (J1 plus J2 / J3 shells)
// with compile-time neighbour offsets: shared by the per-pass kernel
// (far_kernels.cu) and the work-queue cycle kernel of such systems
// (gen_wave.cu).
//
// The 30 neighbour offsets of site S (6 J1, 12 J2, 6 J3a, 6 J3b, canonical
// order) are template constants (far_neighbour), each neighbour address
// three integer adds of per-thread row offsets; the shells are summed in
// canonical order, first value then left-to-right adds, as the generic
// table-driven kernel does, so the two agree bit for bit.
#pragma once
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "kernels.cuh"

namespace pyro {
namespace far {

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

template <int S, int K, bool kNc>
__device__ __forceinline__ float4 nb(const float4* __restrict__ rep, const Frame3& f, int L3) {
  constexpr NbrEntry e = far_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  const float4* a = rep + f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3;
  return kNc ? __ldg(a) : __ldca(a);
}

// Sum of neighbours K0..K1-1 of site S in canonical order (first value, then
// left-to-right adds), as shell_sum of the generic kernel.
template <int S, int K, int K1, bool kNc>
__device__ __forceinline__ void add_rest(const float4* __restrict__ rep, const Frame3& f, int L3,
                                         float3& a) {
  if constexpr (K < K1) {
    const float4 v = nb<S, K, kNc>(rep, f, L3);
    a.x = a.x + v.x;
    a.y = a.y + v.y;
    a.z = a.z + v.z;
    add_rest<S, K + 1, K1, kNc>(rep, f, L3, a);
  }
}

template <int S, int K0, int K1, bool kNc>
__device__ __forceinline__ float3 shell_sum_c(const float4* __restrict__ rep, const Frame3& f,
                                              int L3) {
  const float4 v0 = nb<S, K0, kNc>(rep, f, L3);
  float3 a = make_float3(v0.x, v0.y, v0.z);
  add_rest<S, K0 + 1, K1, kNc>(rep, f, L3, a);
  return a;
}

// Site S of `cell` of replica `rep` of system sd: field, Metropolis or
// over-relaxation, optional renormalisation, store. `sweep` is the sweep
// number (Philox counter word and renormalisation schedule), `tslot` the
// replica's temperature slot (Metropolis). Returns 1 if a Metropolis move was
// accepted. Neighbours are read through the read-only path when kNc, else
// through L1 with coherent loads (the work-queue kernel, whose neighbours
// may have been written by the same launch).
template <int S, bool kMetro, bool kNc = true>
__device__ __forceinline__ int site_update(const PassParams& p, const SysDev& sd, int rep,
                                           int cell, unsigned long long sweep, int tslot) {
  const int L3 = sd.L3;
  const Frame3 fr = frame_of(cell, sd.L, sd.rcpL);
  float4* rb = p.spins + sd.spin_off + (long long)rep * 16 * L3;
  const int own = S * L3 + cell;
  const float3 a1 = shell_sum_c<S, 0, 6, kNc>(rb, fr, L3);
  pyro_vec3 h;
  h.x = sd.J1 * a1.x;
  h.y = sd.J1 * a1.y;
  h.z = sd.J1 * a1.z;
  if (sd.shells & 2) {
    const float3 a = shell_sum_c<S, 6, 18, kNc>(rb, fr, L3);
    h.x = fmaf(sd.J2, a.x, h.x);
    h.y = fmaf(sd.J2, a.y, h.y);
    h.z = fmaf(sd.J2, a.z, h.z);
  }
  if (sd.shells & 4) {
    const float3 a = shell_sum_c<S, 18, 24, kNc>(rb, fr, L3);
    h.x = fmaf(sd.J3a, a.x, h.x);
    h.y = fmaf(sd.J3a, a.y, h.y);
    h.z = fmaf(sd.J3a, a.z, h.z);
  }
  if (sd.shells & 8) {
    const float3 a = shell_sum_c<S, 24, 30, kNc>(rb, fr, L3);
    h.x = fmaf(sd.J3b, a.x, h.x);
    h.y = fmaf(sd.J3b, a.y, h.y);
    h.z = fmaf(sd.J3b, a.z, h.z);
  }
  const float4 sv = rb[own];
  pyro_vec3 sp;
  sp.x = sv.x;
  sp.y = sv.y;
  sp.z = sv.z;
  int accepted = 0;
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
  return accepted;
}

}  // namespace far
}  // namespace pyro
