// Nearest-neighbour (J1-only) kernels: the 4-colour schedule of the
// pyrochlore Heisenberg model, specialised for sm_100a.
//
// Systems with bond matrices (anisotropic exchange and a Zeeman field) run
// the same per-pass kernels with the field of ExchangeDev: six
// pyro_matvec_add in canonical order, minus f, as the generic kernel.
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

#include <algorithm>

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

// Spin loads. Within one launch of a colour pass the neighbours read are
// never written, so the read-only path (ld.global.nc, kLdNc) is safe. The
// cluster-resident cycle kernel rewrites the lattice between passes of the
// same launch, so it reads through L2 only (ld.global.cg, kLdL2): an SM's L1
// may still hold lines from an earlier pass. The work-queue cycle kernel
// reads with ordinary coherent loads (ld.global.ca, kLdCoherent) after an
// acquire of the progress counters that its producers released: the memory
// model orders those loads after the producers' stores, so the SM's L1 can
// serve the reuse within a work item without returning stale lines.
constexpr int kLdNc = 0, kLdL2 = 1, kLdCoherent = 2;
template <int kLd>
__device__ __forceinline__ float4 load_spin(const float4* p) {
  if (kLd == kLdL2) return __ldcg(p);
  if (kLd == kLdCoherent) return __ldca(p);
  return __ldg(p);
}

template <int S, int K, int kLd = kLdNc>
__device__ __forceinline__ float4 load_neighbour(const float4* __restrict__ rep, const CellFrame& f,
                                                 int L3) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  return load_spin<kLd>(rep + f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3);
}

// Sum of the 6 nearest neighbours of site S, in canonical order.
template <int S, int kLd = kLdNc>
__device__ __forceinline__ pyro_vec3 j1_sum(const float4* __restrict__ rep, const CellFrame& f,
                                            int L3) {
  const float4 n0 = load_neighbour<S, 0, kLd>(rep, f, L3);
  const float4 n1 = load_neighbour<S, 1, kLd>(rep, f, L3);
  const float4 n2 = load_neighbour<S, 2, kLd>(rep, f, L3);
  const float4 n3 = load_neighbour<S, 3, kLd>(rep, f, L3);
  const float4 n4 = load_neighbour<S, 4, kLd>(rep, f, L3);
  const float4 n5 = load_neighbour<S, 5, kLd>(rep, f, L3);
  pyro_vec3 a;
  a.x = ((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x;
  a.y = ((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y;
  a.z = ((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z;
  return a;
}

// h + A[b][b_K] S_K for neighbour K of site S (b = S & 3): the matrix of
// the neighbour's sublattice among the three kept for b.
template <int S, int K, int kLd>
__device__ __forceinline__ pyro_vec3 exch_add(pyro_vec3 h, const float4* __restrict__ rep,
                                              const CellFrame& f, int L3, const J1PassParams& p) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  constexpr int b = S & 3, t = e.t & 3, slot = t < b ? t : t - 1;
  static_assert(t != b, "nearest neighbours are on other sublattices");
  const float4 v = load_neighbour<S, K, kLd>(rep, f, L3);
  return pyro_matvec_add(h, p.xa[b][slot], v.x, v.y, v.z);
}

// Own spin and local field of site S of `cell` (loads and field arithmetic).
template <int S, int kLd = kLdNc, bool kExch = false>
__device__ __forceinline__ void site_field(const float4* __restrict__ rep, const CellFrame& f,
                                           int cell, int L3, float J1, const J1PassParams& p,
                                           pyro_vec3* sp, pyro_vec3* h) {
  const int own = S * L3 + cell;
  const float4 sv = load_spin<kLd>(rep + own);
  if (kExch) {
    pyro_vec3 a;
    a.x = a.y = a.z = 0.0f;
    a = exch_add<S, 0, kLd>(a, rep, f, L3, p);
    a = exch_add<S, 1, kLd>(a, rep, f, L3, p);
    a = exch_add<S, 2, kLd>(a, rep, f, L3, p);
    a = exch_add<S, 3, kLd>(a, rep, f, L3, p);
    a = exch_add<S, 4, kLd>(a, rep, f, L3, p);
    a = exch_add<S, 5, kLd>(a, rep, f, L3, p);
    h->x = a.x - p.xf[S & 3][0];
    h->y = a.y - p.xf[S & 3][1];
    h->z = a.z - p.xf[S & 3][2];
  } else {
    const pyro_vec3 a = j1_sum<S, kLd>(rep, f, L3);
    h->x = J1 * a.x;
    h->y = J1 * a.y;
    h->z = J1 * a.z;
  }
  sp->x = sv.x;
  sp->y = sv.y;
  sp->z = sv.z;
}

// The update of site S given its spin and field: Metropolis (Philox, cone,
// exp) or over-relaxation, optional renormalisation, store. Returns 1 if a
// Metropolis move was accepted.
// `own` = S L3 + cell, the site's index in its replica (its Philox counter).
template <bool kMetro>
__device__ __forceinline__ float4 updated_spin(uint32_t own, pyro_vec3 sp, pyro_vec3 h,
                                               float beta, float cosmax, uint32_t rkey,
                                               uint32_t sweep32, bool renorm, uint32_t seed_lo,
                                               uint32_t seed_hi, int* acc) {
  pyro_vec3 out;
  if (kMetro) {
    uint32_t r[4];
    pyro_philox(own, rkey, sweep32, PYRO_PURPOSE_METRO, seed_lo, seed_hi, r);
    const pyro_vec3 prop = pyro_cone_proposal(sp, cosmax, pyro_uniform(r[0]), pyro_uniform(r[1]));
    const float dE = pyro_delta_e(h, sp, prop);
    *acc = pyro_metropolis_accept(dE, beta, pyro_uniform(r[2]));
    out = *acc ? prop : sp;
  } else {
    *acc = 0;
    out = pyro_overrelax(sp, h);
  }
  if (renorm) out = pyro_renormalise(out);
  return make_float4(out.x, out.y, out.z, 0.0f);
}

template <int S, bool kMetro>
__device__ __forceinline__ int site_update(float4* __restrict__ rep, int cell, int L3,
                                           pyro_vec3 sp, pyro_vec3 h, float beta, float cosmax,
                                           uint32_t rkey, uint32_t sweep32, bool renorm,
                                           uint32_t seed_lo, uint32_t seed_hi) {
  const int own = S * L3 + cell;
  int acc;
  rep[own] = updated_spin<kMetro>((uint32_t)own, sp, h, beta, cosmax, rkey, sweep32, renorm,
                                  seed_lo, seed_hi, &acc);
  return acc;
}

template <int S, bool kMetro, int kLd = kLdNc, bool kExch = false>
__device__ __forceinline__ int update_site(float4* __restrict__ rep, const CellFrame& f, int cell,
                                           int L3, float J1, float beta, float cosmax, uint32_t rkey,
                                           uint32_t sweep32, bool renorm, uint32_t seed_lo,
                                           uint32_t seed_hi, const J1PassParams& p) {
  pyro_vec3 sp, h;
  site_field<S, kLd, kExch>(rep, f, cell, L3, J1, p, &sp, &h);
  return site_update<S, kMetro>(rep, cell, L3, sp, h, beta, cosmax, rkey, sweep32, renorm, seed_lo,
                                seed_hi);
}

// ---------------------------------------------------------------------------
// Addressing with the lattice size fixed at compile time (L = 2^kLog2L,
// isotropic J1 systems with L = 16 or 32, which the per-pass launches pick
// by L). The thread's cell is decoded with shifts; the base pointer is its
// cell in site plane 8 of its replica, so the plane of a neighbour is a
// compile-time offset of at most 8 planes (8 L^3 x 16 B = 4 MiB at L = 32)
// that the load carries as an immediate; the wrapped offsets of the
// neighbouring columns, rows and planes are selected once per thread, so a
// neighbour cell costs one add and one pointer, shared by all loads from
// that cell (7 distinct cells per colour pass). The loads, their order and
// the update arithmetic are those of the run-time form: results are
// identical.
template <int kLog2L>
struct FixedCell {
  static constexpr int kL = 1 << kLog2L;
  static constexpr int kL3 = 1 << (3 * kLog2L);
  float4* mid;              // the thread's cell in site plane 8 of its replica
  int xo[3], yo[3], zo[3];  // cell offsets of the previous / same / next column, row, plane
};

template <int kLog2L>
__device__ __forceinline__ FixedCell<kLog2L> fixed_cell(float4* rb, int cell) {
  constexpr int L = FixedCell<kLog2L>::kL, L2 = L * L;
  const int x = cell & (L - 1), y = (cell >> kLog2L) & (L - 1), z = cell >> (2 * kLog2L);
  FixedCell<kLog2L> c;
  c.mid = rb + 8 * FixedCell<kLog2L>::kL3 + cell;
  c.xo[0] = x == 0 ? L - 1 : -1;
  c.xo[1] = 0;
  c.xo[2] = x == L - 1 ? 1 - L : 1;
  c.yo[0] = y == 0 ? (L - 1) * L : -L;
  c.yo[1] = 0;
  c.yo[2] = y == L - 1 ? (1 - L) * L : L;
  c.zo[0] = z == 0 ? (L - 1) * L2 : -L2;
  c.zo[1] = 0;
  c.zo[2] = z == L - 1 ? (1 - L) * L2 : L2;
  return c;
}

// Site s of the thread's cell (read-only path, or through L2 for the
// thread's own stores of the same launch).
template <int s, int kLog2L, int kLd = kLdNc>
__device__ __forceinline__ float4 fixed_own(const FixedCell<kLog2L>& c) {
  return load_spin<kLd>(c.mid + (s - 8) * FixedCell<kLog2L>::kL3);
}

template <int S, int K, int kLog2L, int kLd = kLdNc>
__device__ __forceinline__ float4 fixed_neighbour(const FixedCell<kLog2L>& c) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  static_assert(e.t >= 0, "neighbour table");
  const float4* pc = c.mid + (c.zo[e.dz + 1] + c.yo[e.dy + 1] + c.xo[e.dx + 1]);
  return load_spin<kLd>(pc + (e.t - 8) * FixedCell<kLog2L>::kL3);
}

// Spin and local field of site S (the arithmetic of site_field).
template <int S, int kLog2L, int kLd = kLdNc>
__device__ __forceinline__ void fixed_site_field(const FixedCell<kLog2L>& c, float J1,
                                                 pyro_vec3* sp, pyro_vec3* h) {
  const float4 sv = fixed_own<S, kLog2L, kLd>(c);
  const float4 n0 = fixed_neighbour<S, 0, kLog2L, kLd>(c);
  const float4 n1 = fixed_neighbour<S, 1, kLog2L, kLd>(c);
  const float4 n2 = fixed_neighbour<S, 2, kLog2L, kLd>(c);
  const float4 n3 = fixed_neighbour<S, 3, kLog2L, kLd>(c);
  const float4 n4 = fixed_neighbour<S, 4, kLog2L, kLd>(c);
  const float4 n5 = fixed_neighbour<S, 5, kLog2L, kLd>(c);
  h->x = J1 * (((((n0.x + n1.x) + n2.x) + n3.x) + n4.x) + n5.x);
  h->y = J1 * (((((n0.y + n1.y) + n2.y) + n3.y) + n4.y) + n5.y);
  h->z = J1 * (((((n0.z + n1.z) + n2.z) + n3.z) + n4.z) + n5.z);
  sp->x = sv.x;
  sp->y = sv.y;
  sp->z = sv.z;
}

template <int S, bool kMetro, int kLog2L>
__device__ __forceinline__ int fixed_site_update(const FixedCell<kLog2L>& c, int cell,
                                                 pyro_vec3 sp, pyro_vec3 h, float beta,
                                                 float cosmax, uint32_t rkey, uint32_t sweep32,
                                                 bool renorm, uint32_t seed_lo,
                                                 uint32_t seed_hi) {
  constexpr int L3 = FixedCell<kLog2L>::kL3;
  int acc;
  c.mid[(S - 8) * L3] = updated_spin<kMetro>((uint32_t)(S * L3 + cell), sp, h, beta, cosmax,
                                             rkey, sweep32, renorm, seed_lo, seed_hi, &acc);
  return acc;
}

// Sweep number, renormalisation flag and Philox replica word of a pass.
struct PassWords {
  uint32_t rkey, sw;
  bool renorm;
};
__device__ __forceinline__ PassWords pass_words(const J1PassParams& p, int rep,
                                                unsigned long long sweep_add = 0) {
  const unsigned long long sweep =
      (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off + sweep_add;
  PassWords w;
  w.renorm = p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0;
  w.rkey = (uint32_t)(p.rep_key + rep);
  w.sw = (uint32_t)sweep;
  return w;
}

// The four colour-B sites of a cell with fixed L: loads of all four before
// the first store (as cell_pass).
template <int B, bool kMetro, int kLog2L, int kLd = kLdNc>
__device__ __forceinline__ int fixed_cell_sites(const FixedCell<kLog2L>& c, int cell, float J1,
                                                float beta, float cosmax, const PassWords& w,
                                                uint32_t seed_lo, uint32_t seed_hi) {
  pyro_vec3 s0, h0, s1, h1, s2, h2, s3, h3;
  fixed_site_field<B, kLog2L, kLd>(c, J1, &s0, &h0);
  fixed_site_field<4 + B, kLog2L, kLd>(c, J1, &s1, &h1);
  fixed_site_field<8 + B, kLog2L, kLd>(c, J1, &s2, &h2);
  fixed_site_field<12 + B, kLog2L, kLd>(c, J1, &s3, &h3);
  int acc = 0;
  acc += fixed_site_update<B, kMetro, kLog2L>(c, cell, s0, h0, beta, cosmax, w.rkey, w.sw,
                                              w.renorm, seed_lo, seed_hi);
  acc += fixed_site_update<4 + B, kMetro, kLog2L>(c, cell, s1, h1, beta, cosmax, w.rkey, w.sw,
                                                  w.renorm, seed_lo, seed_hi);
  acc += fixed_site_update<8 + B, kMetro, kLog2L>(c, cell, s2, h2, beta, cosmax, w.rkey, w.sw,
                                                  w.renorm, seed_lo, seed_hi);
  acc += fixed_site_update<12 + B, kMetro, kLog2L>(c, cell, s3, h3, beta, cosmax, w.rkey, w.sw,
                                                   w.renorm, seed_lo, seed_hi);
  return acc;
}

// Cell form of a colour-B pass with fixed L (as cell_pass).
template <int B, bool kMetro, int kLog2L>
__device__ __forceinline__ int fixed_cell_pass(const J1PassParams& p, int rep, int cell,
                                               float beta, float cosmax) {
  const FixedCell<kLog2L> c =
      fixed_cell<kLog2L>(p.spins + (long long)rep * 16 * FixedCell<kLog2L>::kL3, cell);
  const PassWords w = pass_words(p, rep);
  return fixed_cell_sites<B, kMetro, kLog2L>(c, cell, p.J1, beta, cosmax, w, p.seed_lo,
                                             p.seed_hi);
}

template <int S, bool kMetro, int kLog2L>
__device__ __forceinline__ int fixed_update_site(const J1PassParams& p, int rep, int cell,
                                                 float beta, float cosmax) {
  const FixedCell<kLog2L> c =
      fixed_cell<kLog2L>(p.spins + (long long)rep * 16 * FixedCell<kLog2L>::kL3, cell);
  const PassWords w = pass_words(p, rep);
  pyro_vec3 sp, h;
  fixed_site_field<S, kLog2L>(c, p.J1, &sp, &h);
  return fixed_site_update<S, kMetro, kLog2L>(c, cell, sp, h, beta, cosmax, w.rkey, w.sw,
                                              w.renorm, p.seed_lo, p.seed_hi);
}

// Site form with fixed L (as site_item).
template <int B, bool kMetro, int kLog2L>
__device__ __forceinline__ int fixed_site_item(const J1PassParams& p, int rep, int f, int cell,
                                               float beta, float cosmax) {
  switch (f) {
    case 0:
      return fixed_update_site<B, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
    case 1:
      return fixed_update_site<4 + B, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
    case 2:
      return fixed_update_site<8 + B, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
    default:
      return fixed_update_site<12 + B, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
  }
}

// Start of a per-pass kernel: the grid this launch may overlap (programmatic
// dependent launch) must have completed and its writes be visible before any
// global load; then the next pass may begin launching.
__device__ __forceinline__ void pass_prologue() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// The four sites of colour B in `cell` of replica `rep` (cell form of a
// pass). Returns the number of accepted Metropolis moves.
template <int B, bool kMetro, bool kExch, int kLd = kLdNc>
__device__ __forceinline__ int cell_pass(const J1PassParams& p, int rep, int cell, float beta,
                                         float cosmax, unsigned long long sweep_add = 0) {
  int x, y, z;
  decode_cell(cell, p.L, p.rcpL, &x, &y, &z);
  const CellFrame f = make_frame(x, y, z, p.L);
  float4* rb = p.spins + (long long)rep * 16 * p.L3;
  const unsigned long long sweep =
      (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off + sweep_add;
  const bool renorm =
      p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0;
  const uint32_t rkey = (uint32_t)(p.rep_key + rep);
  const uint32_t sw = (uint32_t)sweep;
  // The four sites of the colour in this cell are not neighbours of each
  // other (nor of any site written in this pass), so all their loads are
  // issued before the first store: one memory round trip, not four.
  pyro_vec3 s0, h0, s1, h1, s2, h2, s3, h3;
  site_field<B, kLd, kExch>(rb, f, cell, p.L3, p.J1, p, &s0, &h0);
  site_field<4 + B, kLd, kExch>(rb, f, cell, p.L3, p.J1, p, &s1, &h1);
  site_field<8 + B, kLd, kExch>(rb, f, cell, p.L3, p.J1, p, &s2, &h2);
  site_field<12 + B, kLd, kExch>(rb, f, cell, p.L3, p.J1, p, &s3, &h3);
  int acc = 0;
  acc += site_update<B, kMetro>(rb, cell, p.L3, s0, h0, beta, cosmax, rkey, sw, renorm,
                                p.seed_lo, p.seed_hi);
  acc += site_update<4 + B, kMetro>(rb, cell, p.L3, s1, h1, beta, cosmax, rkey, sw, renorm,
                                    p.seed_lo, p.seed_hi);
  acc += site_update<8 + B, kMetro>(rb, cell, p.L3, s2, h2, beta, cosmax, rkey, sw, renorm,
                                    p.seed_lo, p.seed_hi);
  acc += site_update<12 + B, kMetro>(rb, cell, p.L3, s3, h3, beta, cosmax, rkey, sw, renorm,
                                     p.seed_lo, p.seed_hi);
  return acc;
}

// Block-wide count of accepted moves: one atomic per CTA. Every thread of
// the CTA calls it.
__device__ __forceinline__ void block_accept(const J1PassParams& p, int t, int acc) {
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

// The cell of this thread in a per-pass kernel's CTA (blockIdx.x: the CTA's
// chunk of the replica). Run-time L: kJ1Threads consecutive cells. Fixed L:
// a tile of L x kTy x 2 cells (x, y, z), so that the neighbours a thread
// reads in the previous plane, and in the rows next to its own, are mostly
// cells of the same CTA, whose spins the CTA loads anyway (L1 hits): at
// L = 32 a CTA of 32 x 4 x 2 cells reads 302 B per cell and pass from L2
// instead of 326 B for a CTA of 8 consecutive rows.
template <int kLog2L>
__device__ __forceinline__ int pass_cell() {
  if constexpr (kLog2L == 0) {
    return blockIdx.x * kJ1Threads + threadIdx.x;
  } else {
    constexpr int L = 1 << kLog2L, kTz = 2, kTy = kJ1Threads / (L * kTz), kTilesY = L / kTy;
    static_assert(L * kTy * kTz == kJ1Threads && L % kTy == 0 && L % kTz == 0, "tile");
    const int ty = blockIdx.x % kTilesY, tz = blockIdx.x / kTilesY;
    const int x = threadIdx.x & (L - 1);
    const int yy = (threadIdx.x >> kLog2L) % kTy;
    const int zz = threadIdx.x / (L * kTy);
    return ((tz * kTz + zz) * L + ty * kTy + yy) * L + x;
  }
}

// The cell of this thread in a fixed-L site-form CTA that holds all four
// corners: kJ1Threads / 4 cells per corner, a tile of L x kTy x 1 cells,
// the same tile for every corner group of the CTA.
template <int kLog2L>
__device__ __forceinline__ int corner_tile_cell() {
  constexpr int L = 1 << kLog2L, kCells = kJ1Threads / 4, kTy = kCells / L, kTilesY = L / kTy;
  static_assert(L * kTy == kCells && L % kTy == 0, "tile");
  const int t = threadIdx.x & (kCells - 1);
  const int ty = blockIdx.x % kTilesY, z = blockIdx.x / kTilesY;
  return (z * L + ty * kTy + (t >> kLog2L)) * L + (t & (L - 1));
}

// kLog2L > 0: the fixed-L addressing (isotropic J1 systems of L = 2^kLog2L).
template <int B, bool kMetro, bool kExch, int kLog2L = 0>
__global__ void __launch_bounds__(kJ1Threads) j1_pass_kernel(const J1PassParams p) {
  static_assert(kLog2L == 0 || !kExch, "fixed-L form is isotropic only");
  pass_prologue();
  const int rep = blockIdx.y;
  const int cell = pass_cell<kLog2L>();
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
    if constexpr (kLog2L > 0) acc = fixed_cell_pass<B, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
    else acc = cell_pass<B, kMetro, kExch>(p, rep, cell, beta, cosmax);
  }
  if (kMetro) block_accept(p, t, acc);
}

// Site 4 f + B of `cell` (site form of a pass). Returns 1 if a Metropolis
// move was accepted.
template <int B, bool kMetro, bool kExch, int kLd = kLdNc>
__device__ __forceinline__ int site_item(const J1PassParams& p, int rep, int f, int cell,
                                         float beta, float cosmax,
                                         unsigned long long sweep_add = 0) {
  int x, y, z;
  decode_cell(cell, p.L, p.rcpL, &x, &y, &z);
  const CellFrame fr = make_frame(x, y, z, p.L);
  float4* rb = p.spins + (long long)rep * 16 * p.L3;
  const unsigned long long sweep =
      (p.sweep_ctr ? *p.sweep_ctr : 0ull) + p.sweep_off + sweep_add;
  const bool renorm =
      p.renorm_every > 0 && ((sweep + 1) % (unsigned long long)p.renorm_every) == 0;
  const uint32_t rkey = (uint32_t)(p.rep_key + rep);
  const uint32_t sw = (uint32_t)sweep;
  switch (f) {
    case 0:
      return update_site<B, kMetro, kLd, kExch>(rb, fr, cell, p.L3, p.J1, beta, cosmax, rkey, sw,
                                                renorm, p.seed_lo, p.seed_hi, p);
    case 1:
      return update_site<4 + B, kMetro, kLd, kExch>(rb, fr, cell, p.L3, p.J1, beta, cosmax, rkey,
                                                    sw, renorm, p.seed_lo, p.seed_hi, p);
    case 2:
      return update_site<8 + B, kMetro, kLd, kExch>(rb, fr, cell, p.L3, p.J1, beta, cosmax, rkey,
                                                    sw, renorm, p.seed_lo, p.seed_hi, p);
    default:
      return update_site<12 + B, kMetro, kLd, kExch>(rb, fr, cell, p.L3, p.J1, beta, cosmax, rkey,
                                                     sw, renorm, p.seed_lo, p.seed_hi, p);
  }
}

// Same pass, one site per thread: blockIdx.y is the FCC corner f (so site
// S = 4 f + B is uniform in a CTA), blockIdx.z the replica. Fewer live
// registers than the cell-per-thread form, hence more warps in flight; the
// Metropolis pass (Philox, cone, exp) is latency-bound without them.
//
// With L fixed (kLog2L > 0) a CTA holds all four corners of a tile of
// kJ1Threads / 4 cells instead (corner f = warps 2f, 2f + 1; blockIdx.y = 0):
// its four corner groups together read every site plane of the tile's
// cells, so the neighbours one corner's sites read in the tile are spins
// another corner group has loaded (L1), which a CTA of one corner misses.
template <int B, bool kMetro, bool kExch, int kLog2L = 0>
__global__ void __launch_bounds__(kJ1Threads) j1_site_pass_kernel(const J1PassParams p) {
  static_assert(kLog2L == 0 || !kExch, "fixed-L form is isotropic only");
  pass_prologue();
  int f, cell;
  if constexpr (kLog2L > 0) {
    f = threadIdx.x / (kJ1Threads / 4);  // warp-uniform
    cell = corner_tile_cell<kLog2L>();
  } else {
    f = blockIdx.y;
    cell = pass_cell<0>();
  }
  const int rep = blockIdx.z;
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
    if constexpr (kLog2L > 0) acc = fixed_site_item<B, kMetro, kLog2L>(p, rep, f, cell, beta, cosmax);
    else acc = site_item<B, kMetro, kExch>(p, rep, f, cell, beta, cosmax);
  }
  if (kMetro) {
    const int n = __syncthreads_count(acc);
    if (threadIdx.x == 0 && n > 0)
      atomicAdd(p.accepted + p.temp_base + t, (unsigned long long)n);
  }
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Down-tetrahedron partners of the sublattice-0 site 4F of a cell.
template <int F, int kLd>
__device__ __forceinline__ void down_partners(const float4* __restrict__ rep, const CellFrame& f,
                                              int L3, float4* d1, float4* d2, float4* d3) {
  constexpr int S0 = 4 * F;
  constexpr int k1 = j1_down_index(S0, 0), k2 = j1_down_index(S0, 1), k3 = j1_down_index(S0, 2);
  static_assert(k1 >= 0 && k2 >= 0 && k3 >= 0, "three down-tetrahedron partners");
  *d1 = load_neighbour<S0, k1, kLd>(rep, f, L3);
  *d2 = load_neighbour<S0, k2, kLd>(rep, f, L3);
  *d3 = load_neighbour<S0, k3, kLd>(rep, f, L3);
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

template <int F, int kLd = kLdNc>
__device__ __forceinline__ void cell_corner(const float4* __restrict__ rep, const CellFrame& f,
                                            int cell, int L3, double* e, double* mx, double* my,
                                            double* mz) {
  const float4 s0 = load_spin<kLd>(rep + (4 * F + 0) * L3 + cell);
  const float4 s1 = load_spin<kLd>(rep + (4 * F + 1) * L3 + cell);
  const float4 s2 = load_spin<kLd>(rep + (4 * F + 2) * L3 + cell);
  const float4 s3 = load_spin<kLd>(rep + (4 * F + 3) * L3 + cell);
  float4 d1, d2, d3;
  down_partners<F, kLd>(rep, f, L3, &d1, &d2, &d3);
  *e += tet_energy(s0, s1, s2, s3) + tet_energy(s0, d1, d2, d3);
  *mx += (double)s0.x + s1.x + s2.x + s3.x;
  *my += (double)s0.y + s1.y + s2.y + s3.y;
  *mz += (double)s0.z + s1.z + s2.z + s3.z;
}

// Fixed-order CTA reduction of per-thread (E, M) terms; thread 0 returns
// (2 E, Mx, My, Mz). Every thread of the CTA calls it.
__device__ __forceinline__ double4 block_observables(double e, double mx, double my, double mz,
                                                     double (*red)[kJ1Threads / 32]) {
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
  double4 o = make_double4(0.0, 0.0, 0.0, 0.0);
  if (threadIdx.x == 0) {
    for (int q = 0; q < kJ1Threads / 32; ++q) {
      o.x += red[0][q];
      o.y += red[1][q];
      o.z += red[2][q];
      o.w += red[3][q];
    }
    o.x *= 2.0;
  }
  __syncthreads();
  return o;
}

// Energy (each bond once, by tetrahedra) and magnetisation of one chunk of
// kJ1Threads cells, reduced over the CTA in a fixed order; thread 0 returns
// (2 E, Mx, My, Mz) (the finalise step halves the site-sum convention of the
// generic kernel, hence 2 E). Every thread of the CTA must call it.
template <int kLd>
__device__ __forceinline__ double4 chunk_observables(const float4* __restrict__ rb, int cell,
                                                     int L, int L3, float rcpL, double J1,
                                                     double (*red)[kJ1Threads / 32]) {
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  if (cell < L3) {
    int x, y, z;
    decode_cell(cell, L, rcpL, &x, &y, &z);
    const CellFrame f = make_frame(x, y, z, L);
    // In the work-queue kernel (kLd == kLdCoherent) the corners run one
    // after another (a compiler barrier between them keeps 7 loads in
    // flight instead of 28), which bounds its register count; the sums are
    // the same in the same order.
    cell_corner<0, kLd>(rb, f, cell, L3, &e, &mx, &my, &mz);
    if (kLd == kLdCoherent) asm volatile("" ::: "memory");
    cell_corner<1, kLd>(rb, f, cell, L3, &e, &mx, &my, &mz);
    if (kLd == kLdCoherent) asm volatile("" ::: "memory");
    cell_corner<2, kLd>(rb, f, cell, L3, &e, &mx, &my, &mz);
    if (kLd == kLdCoherent) asm volatile("" ::: "memory");
    cell_corner<3, kLd>(rb, f, cell, L3, &e, &mx, &my, &mz);
    e *= J1;
  }
  return block_observables(e, mx, my, mz, red);
}

// Each cell owns its 4 up-tetrahedra and the 4 down-tetrahedra that contain
// its sublattice-0 sites: every bond is counted exactly once.
__global__ void __launch_bounds__(kJ1Threads) j1_observables_kernel(const J1ObsParams p) {
  pass_prologue();
  __shared__ double red[4][kJ1Threads / 32];
  const int rep = blockIdx.y;
  const int cell = blockIdx.x * kJ1Threads + threadIdx.x;
  const float4* rb = p.spins + (long long)rep * 16 * p.L3;
  const double4 o = chunk_observables<false>(rb, cell, p.L, p.L3, p.rcpL, p.J1, red);
  if (threadIdx.x == 0) p.partials[p.partial_begin + (long long)rep * gridDim.x + blockIdx.x] = o;
}

// The two tetrahedra of the sublattice-3 site S = 4F + 3 of `cell` after a
// colour-3 pass: the up-tetrahedron of corner F (sites 4F..4F + 3 of the
// cell) and S's down-tetrahedron. Every tetrahedron holds exactly one
// sublattice-3 site, so the cells' sums count each bond once; the up-
// tetrahedra of a cell cover its 16 sites once (magnetisation). The
// sublattice-3 spins are this thread's own stores of the pass, read back
// through L2; the others were not written by the pass.
template <int F, int kLd = kLdNc>
__device__ __forceinline__ void corner3_observables(const float4* __restrict__ rb,
                                                    const CellFrame& f, int cell, int L3,
                                                    double* e, double* mx, double* my,
                                                    double* mz) {
  constexpr int S = 4 * F + 3;
  constexpr int kOwn = kLd == kLdNc ? kLdL2 : kLd;  // this thread's own stores
  const float4 s0 = load_spin<kLd>(rb + (4 * F + 0) * L3 + cell);
  const float4 s1 = load_spin<kLd>(rb + (4 * F + 1) * L3 + cell);
  const float4 s2 = load_spin<kLd>(rb + (4 * F + 2) * L3 + cell);
  const float4 s3 = load_spin<kOwn>(rb + S * L3 + cell);
  const float4 d1 = load_neighbour<S, j1_down_index(S, 0), kLd>(rb, f, L3);
  const float4 d2 = load_neighbour<S, j1_down_index(S, 1), kLd>(rb, f, L3);
  const float4 d3 = load_neighbour<S, j1_down_index(S, 2), kLd>(rb, f, L3);
  *e += tet_energy(s0, s1, s2, s3) + tet_energy(s3, d1, d2, d3);
  *mx += (double)s0.x + s1.x + s2.x + s3.x;
  *my += (double)s0.y + s1.y + s2.y + s3.y;
  *mz += (double)s0.z + s1.z + s2.z + s3.z;
}

// Body of the fused last pass for one chunk of kJ1Threads cells: the colour-3
// updates of `cell` (cell form), the chunk's acceptance count, and the
// observables partial of the state it leaves, written to o.partials[slot].
// Every thread of the CTA calls it.
template <bool kMetro, int kLd>
__device__ __forceinline__ void last_item(const J1PassParams& p, const J1ObsParams& o, int rep,
                                          int cell, float beta, float cosmax, int t,
                                          unsigned long long sweep_add,
                                          double (*red)[kJ1Threads / 32], long long slot) {
  int acc = 0;
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  if (cell < p.L3) {
    acc = cell_pass<3, kMetro, false, kLd>(p, rep, cell, beta, cosmax, sweep_add);
    int x, y, z;
    decode_cell(cell, p.L, p.rcpL, &x, &y, &z);
    const CellFrame f = make_frame(x, y, z, p.L);
    const float4* rb = p.spins + (long long)rep * 16 * p.L3;
    corner3_observables<0, kLd>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    corner3_observables<1, kLd>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    corner3_observables<2, kLd>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    corner3_observables<3, kLd>(rb, f, cell, p.L3, &e, &mx, &my, &mz);
    e *= o.J1;
  }
  if (kMetro) block_accept(p, t, acc);
  const double4 r = block_observables(e, mx, my, mz, red);
  if (threadIdx.x == 0) o.partials[slot] = r;
}

// corner3_observables with the fixed-L addressing (same loads, same sums).
template <int F, int kLog2L>
__device__ __forceinline__ void fixed_corner3_observables(const FixedCell<kLog2L>& c, double* e,
                                                          double* mx, double* my, double* mz) {
  constexpr int S = 4 * F + 3;
  const float4 s0 = fixed_own<4 * F + 0, kLog2L>(c);
  const float4 s1 = fixed_own<4 * F + 1, kLog2L>(c);
  const float4 s2 = fixed_own<4 * F + 2, kLog2L>(c);
  const float4 s3 = fixed_own<S, kLog2L, kLdL2>(c);  // this thread's own store
  const float4 d1 = fixed_neighbour<S, j1_down_index(S, 0), kLog2L>(c);
  const float4 d2 = fixed_neighbour<S, j1_down_index(S, 1), kLog2L>(c);
  const float4 d3 = fixed_neighbour<S, j1_down_index(S, 2), kLog2L>(c);
  *e += tet_energy(s0, s1, s2, s3) + tet_energy(s3, d1, d2, d3);
  *mx += (double)s0.x + s1.x + s2.x + s3.x;
  *my += (double)s0.y + s1.y + s2.y + s3.y;
  *mz += (double)s0.z + s1.z + s2.z + s3.z;
}

// last_item with the fixed-L addressing.
template <bool kMetro, int kLog2L>
__device__ __forceinline__ void fixed_last_item(const J1PassParams& p, const J1ObsParams& o,
                                                int rep, int cell, float beta, float cosmax,
                                                int t, double (*red)[kJ1Threads / 32],
                                                long long slot) {
  int acc = 0;
  double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  if (cell < p.L3) {
    acc = fixed_cell_pass<3, kMetro, kLog2L>(p, rep, cell, beta, cosmax);
    const FixedCell<kLog2L> c =
        fixed_cell<kLog2L>(p.spins + (long long)rep * 16 * FixedCell<kLog2L>::kL3, cell);
    fixed_corner3_observables<0, kLog2L>(c, &e, &mx, &my, &mz);
    fixed_corner3_observables<1, kLog2L>(c, &e, &mx, &my, &mz);
    fixed_corner3_observables<2, kLog2L>(c, &e, &mx, &my, &mz);
    fixed_corner3_observables<3, kLog2L>(c, &e, &mx, &my, &mz);
    e *= o.J1;
  }
  if (kMetro) block_accept(p, t, acc);
  const double4 r = block_observables(e, mx, my, mz, red);
  if (threadIdx.x == 0) o.partials[slot] = r;
}

// The last pass of a cycle (colour 3, cell form, isotropic J1) fused with
// the FP64 energy and magnetisation partials of the state it leaves: the
// same updates as j1_pass_kernel<3, kMetro, false>, then each cell's eight
// tetrahedra from spins the pass just loaded (L1/L2), instead of a separate
// observables kernel reading the lattice again. Partials in the layout of
// j1_observables_kernel (one per CTA of kJ1Threads cells).
template <bool kMetro, int kLog2L = 0>
__global__ void __launch_bounds__(kJ1Threads) j1_last_pass_kernel(const J1PassParams p,
                                                                  const J1ObsParams o) {
  pass_prologue();
  __shared__ double red[4][kJ1Threads / 32];
  const int rep = blockIdx.y;
  const int cell = pass_cell<kLog2L>();
  const int g = p.rep_global + rep;
  float beta = 0.0f, cosmax = 0.0f;
  int t = 0;
  if (kMetro) {
    t = p.temp_of_rep[p.temp_base + g];
    beta = p.beta[p.temp_base + t];
    cosmax = p.cosmax[p.temp_base + t];
  }
  const long long slot = o.partial_begin + (long long)rep * gridDim.x + blockIdx.x;
  if constexpr (kLog2L > 0)
    fixed_last_item<kMetro, kLog2L>(p, o, rep, cell, beta, cosmax, t, red, slot);
  else
    last_item<kMetro, kLdNc>(p, o, rep, cell, beta, cosmax, t, 0ull, red, slot);
}

// One site update of the cluster kernel: site S of `cell`, neighbours read
// through L2. Returns 1 if a Metropolis move was accepted.
template <int S, bool kMetro>
__device__ __forceinline__ int cluster_site(float4* __restrict__ rb, int cell, int L, int L3,
                                            float rcpL, float J1, float beta, float cosmax,
                                            uint32_t rkey, uint32_t sw, bool renorm,
                                            uint32_t seed_lo, uint32_t seed_hi,
                                            const J1PassParams& pp) {
  int x, y, z;
  decode_cell(cell, L, rcpL, &x, &y, &z);
  const CellFrame f = make_frame(x, y, z, L);
  return update_site<S, kMetro, kLdL2>(rb, f, cell, L3, J1, beta, cosmax, rkey, sw, renorm,
                                      seed_lo, seed_hi, pp);
}

template <bool kMetro>
__device__ __forceinline__ int cluster_dispatch(int s, float4* __restrict__ rb, int cell, int L,
                                                int L3, float rcpL, float J1, float beta,
                                                float cosmax, uint32_t rkey, uint32_t sw,
                                                bool renorm, uint32_t seed_lo, uint32_t seed_hi,
                                                const J1PassParams& pp) {
  switch (s) {
#define PYRO_SITE(S) \
  case S:            \
    return cluster_site<S, kMetro>(rb, cell, L, L3, rcpL, J1, beta, cosmax, rkey, sw, renorm, \
                                   seed_lo, seed_hi, pp);
    PYRO_SITE(0) PYRO_SITE(1) PYRO_SITE(2) PYRO_SITE(3) PYRO_SITE(4) PYRO_SITE(5) PYRO_SITE(6)
    PYRO_SITE(7) PYRO_SITE(8) PYRO_SITE(9) PYRO_SITE(10) PYRO_SITE(11) PYRO_SITE(12)
    PYRO_SITE(13) PYRO_SITE(14) PYRO_SITE(15)
#undef PYRO_SITE
    default:
      return 0;
  }
}

__device__ __forceinline__ void cluster_barrier() {
  // Release our spin stores to the cluster and acquire everyone else's.
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// End of a cluster cycle: the replica's acceptance count (one atomic per CTA)
// and, when p.partials is set, the observables partials of the final state
// in the chunks and reduction order of j1_observables_kernel (thread group q
// of the CTA handles chunk oc). Every thread of the cluster calls it after
// the last pass's barrier.
__device__ __forceinline__ void cluster_cycle_tail(
    const J1CycleParams& p, int rep, int rank, int t, int acc,
    double (*red)[4][kJ1Threads / 32], int* warp_acc) {
  const int csize = p.cluster_size;
  const int L = p.pass.L, L3 = p.pass.L3;
  const float rcpL = p.pass.rcpL;
  const float4* rb = p.pass.spins + (long long)rep * 16 * L3;
  if (p.n_metro > 0) {
    int v = acc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_acc[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int w = 0; w < kJ1CycleThreads / 32; ++w) s += warp_acc[w];
      if (s > 0) atomicAdd(p.pass.accepted + p.pass.temp_base + t, (unsigned long long)s);
    }
  }
  if (p.partials) {
    constexpr int kGroups = kJ1CycleThreads / kJ1Threads;
    const int q = threadIdx.x / kJ1Threads;
    const int lt = threadIdx.x - q * kJ1Threads;
    const int n_obs = (L3 + kJ1Threads - 1) / kJ1Threads;
    for (int base_c = rank * kGroups; base_c < n_obs; base_c += csize * kGroups) {
      const int oc = base_c + q;
      const int cell = oc * kJ1Threads + lt;
      double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
      if (oc < n_obs && cell < L3) {
        int x, y, z;
        decode_cell(cell, L, rcpL, &x, &y, &z);
        const CellFrame f = make_frame(x, y, z, L);
        cell_corner<0, true>(rb, f, cell, L3, &e, &mx, &my, &mz);
        cell_corner<1, true>(rb, f, cell, L3, &e, &mx, &my, &mz);
        cell_corner<2, true>(rb, f, cell, L3, &e, &mx, &my, &mz);
        cell_corner<3, true>(rb, f, cell, L3, &e, &mx, &my, &mz);
        e *= p.J1_64;
      }
      e = warp_sum_d(e);
      mx = warp_sum_d(mx);
      my = warp_sum_d(my);
      mz = warp_sum_d(mz);
      const int w = lt >> 5, lane = lt & 31;
      if (lane == 0) {
        red[q][0][w] = e;
        red[q][1][w] = mx;
        red[q][2][w] = my;
        red[q][3][w] = mz;
      }
      __syncthreads();
      if (lt == 0 && oc < n_obs) {
        double4 o = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int ww = 0; ww < kJ1Threads / 32; ++ww) {
          o.x += red[q][0][ww];
          o.y += red[q][1][ww];
          o.z += red[q][2][ww];
          o.w += red[q][3][ww];
        }
        o.x *= 2.0;
        p.partials[p.partial_begin + (long long)rep * n_obs + oc] = o;
      }
      __syncthreads();
    }
  }
}

// A whole cycle for one replica per thread-block cluster: n_metro Metropolis
// then n_or over-relaxation sweeps, each sweep 4 colour passes separated by a
// cluster barrier, then (optionally) the observables partials of the final
// state. In a pass the 4 L^3 sites of the colour are split in chunks of
// kJ1CycleThreads over the CTAs of the cluster (chunk c to CTA c % cluster
// size), one site per thread per chunk, so a CTA keeps 32 warps of
// independent loads in flight. The replica's 16 L^3 float4 stay in L2 across
// the passes; HBM sees about one read and one write of the lattice per call.
// Results equal those of the per-pass kernels bit for bit.
__global__ void __launch_bounds__(kJ1CycleThreads, 1)
    j1_cycle_cluster_kernel(const J1CycleParams p) {
  __shared__ double red[kJ1CycleThreads / kJ1Threads][4][kJ1Threads / 32];
  __shared__ int warp_acc[kJ1CycleThreads / 32];
  const int csize = p.cluster_size;
  const int rep = blockIdx.x / csize;
  const int rank = blockIdx.x - rep * csize;
  const int g = p.pass.rep_global + rep;
  const int t = p.pass.temp_of_rep[p.pass.temp_base + g];
  const float beta = p.pass.beta[p.pass.temp_base + t];
  const float cosmax = p.pass.cosmax[p.pass.temp_base + t];
  const int L = p.pass.L, L3 = p.pass.L3;
  const float rcpL = p.pass.rcpL;
  float4* rb = p.pass.spins + (long long)rep * 16 * L3;
  const uint32_t rkey = (uint32_t)(p.pass.rep_key + rep);
  const unsigned long long base = (p.pass.sweep_ctr ? *p.pass.sweep_ctr : 0ull) + p.pass.sweep_off;
  const int items = 4 * L3;
  const int n_chunks = (items + kJ1CycleThreads - 1) / kJ1CycleThreads;
  int acc = 0;
  const int n_sweeps = p.n_metro + p.n_or;
  for (int k = 0; k < n_sweeps; ++k) {
    const unsigned long long sweep = base + (unsigned long long)k;
    const bool renorm = p.pass.renorm_every > 0 &&
                        ((sweep + 1) % (unsigned long long)p.pass.renorm_every) == 0;
    const uint32_t sw = (uint32_t)sweep;
    const bool metro = k < p.n_metro;
#pragma unroll 1
    for (int b = 0; b < 4; ++b) {
#pragma unroll 1
      for (int c = rank; c < n_chunks; c += csize) {
        const int item = c * kJ1CycleThreads + threadIdx.x;
        if (item < items) {
          const int fc = item / L3;
          const int cell = item - fc * L3;
          const int s = 4 * fc + b;
          if (metro)
            acc += cluster_dispatch<true>(s, rb, cell, L, L3, rcpL, p.pass.J1, beta, cosmax, rkey,
                                          sw, renorm, p.pass.seed_lo, p.pass.seed_hi, p.pass);
          else
            cluster_dispatch<false>(s, rb, cell, L, L3, rcpL, p.pass.J1, beta, cosmax, rkey, sw,
                                    renorm, p.pass.seed_lo, p.pass.seed_hi, p.pass);
        }
      }
      cluster_barrier();
    }
  }
  cluster_cycle_tail(p, rep, rank, t, acc, red, warp_acc);
}

// The four colour-b sites of one cell in a fixed-L cluster cycle: loads
// through L1 (coherent after the barrier's acquire), all four sites' loads
// before the first store.
template <bool kMetro, int kLog2L>
__device__ __forceinline__ int cluster_fixed_cell(int b, const FixedCell<kLog2L>& c, int cell,
                                                  float J1, float beta, float cosmax,
                                                  const PassWords& w, uint32_t seed_lo,
                                                  uint32_t seed_hi) {
  switch (b) {
    case 0:
      return fixed_cell_sites<0, kMetro, kLog2L, kLdCoherent>(c, cell, J1, beta, cosmax, w,
                                                              seed_lo, seed_hi);
    case 1:
      return fixed_cell_sites<1, kMetro, kLog2L, kLdCoherent>(c, cell, J1, beta, cosmax, w,
                                                              seed_lo, seed_hi);
    case 2:
      return fixed_cell_sites<2, kMetro, kLog2L, kLdCoherent>(c, cell, J1, beta, cosmax, w,
                                                              seed_lo, seed_hi);
    default:
      return fixed_cell_sites<3, kMetro, kLog2L, kLdCoherent>(c, cell, J1, beta, cosmax, w,
                                                              seed_lo, seed_hi);
  }
}

// The cluster cycle with L = 2^kLog2L fixed at compile time (isotropic J1,
// L = 16 or 32): every colour pass in the cell form (a thread updates the
// four sites of the colour in each of its cells, chunks of kJ1CycleThreads
// cells dealt to the CTAs of the cluster), the fixed-L addressing, and loads
// through L1: the cluster barrier between passes releases each CTA's stores
// and acquires the others', so the memory model orders the next pass's loads
// after them and the L1 serves the neighbour reuse within a pass. Same
// updates in the same order per site as the per-pass kernels.
template <int kLog2L>
__global__ void __launch_bounds__(kJ1CycleThreads, 1)
    j1_cycle_cluster_fixed_kernel(const J1CycleParams p) {
  __shared__ double red[kJ1CycleThreads / kJ1Threads][4][kJ1Threads / 32];
  __shared__ int warp_acc[kJ1CycleThreads / 32];
  constexpr int L3 = FixedCell<kLog2L>::kL3;
  const int csize = p.cluster_size;
  const int rep = blockIdx.x / csize;
  const int rank = blockIdx.x - rep * csize;
  const int g = p.pass.rep_global + rep;
  const int t = p.pass.temp_of_rep[p.pass.temp_base + g];
  const float beta = p.pass.beta[p.pass.temp_base + t];
  const float cosmax = p.pass.cosmax[p.pass.temp_base + t];
  float4* rb = p.pass.spins + (long long)rep * 16 * L3;
  const unsigned long long base =
      (p.pass.sweep_ctr ? *p.pass.sweep_ctr : 0ull) + p.pass.sweep_off;
  PassWords w;
  w.rkey = (uint32_t)(p.pass.rep_key + rep);
  int acc = 0;
  const int n_sweeps = p.n_metro + p.n_or;
  for (int k = 0; k < n_sweeps; ++k) {
    const unsigned long long sweep = base + (unsigned long long)k;
    w.renorm = p.pass.renorm_every > 0 &&
               ((sweep + 1) % (unsigned long long)p.pass.renorm_every) == 0;
    w.sw = (uint32_t)sweep;
    const bool metro = k < p.n_metro;
#pragma unroll 1
    for (int b = 0; b < 4; ++b) {
#pragma unroll 1
      for (int cell = rank * kJ1CycleThreads + threadIdx.x; cell < L3;
           cell += csize * kJ1CycleThreads) {
        const FixedCell<kLog2L> c = fixed_cell<kLog2L>(rb, cell);
        if (metro)
          acc += cluster_fixed_cell<true, kLog2L>(b, c, cell, p.pass.J1, beta, cosmax, w,
                                                  p.pass.seed_lo, p.pass.seed_hi);
        else
          cluster_fixed_cell<false, kLog2L>(b, c, cell, p.pass.J1, beta, cosmax, w,
                                            p.pass.seed_lo, p.pass.seed_hi);
      }
      cluster_barrier();
    }
  }
  cluster_cycle_tail(p, rep, rank, t, acc, red, warp_acc);
}


// ---------------------------------------------------------------------------
// Work-queue cycle kernel (see J1WaveParams in j1_kernels.cuh).

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Publishes this CTA's completed item: the stores of every thread of the
// CTA (ordered before this by the barrier that precedes the call) become
// visible before the count does (a release fence, then the add).
__device__ __forceinline__ void release_add_gpu(unsigned int* p, unsigned int v) {
  asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v)
               : "memory");
}

// One work item: colour B of pass k on chunk q of replica rep, sub-item f
// (FCC corner in the site form, unused in the cell form).
template <int B, bool kExch, bool kMetroSite, bool kOrSite, int kLd = kLdCoherent>
__device__ __forceinline__ void wave_item(const J1WaveParams& w, int rep, int q, int f,
                                          bool metro, unsigned long long sweep_add) {
  const J1PassParams& p = w.pass;
  const int cell = q * kJ1Threads + threadIdx.x;
  float beta = 0.0f, cosmax = 0.0f;
  int t = 0;
  if (metro) {
    t = p.temp_of_rep[p.temp_base + p.rep_global + rep];
    beta = p.beta[p.temp_base + t];
    cosmax = p.cosmax[p.temp_base + t];
  }
  int acc = 0;
  if (cell < p.L3) {
    if (metro) {
      if (kMetroSite)
        acc = site_item<B, true, kExch, kLd>(p, rep, f, cell, beta, cosmax, sweep_add);
      else
        acc = cell_pass<B, true, kExch, kLd>(p, rep, cell, beta, cosmax, sweep_add);
    } else {
      if (kOrSite)
        site_item<B, false, kExch, kLd>(p, rep, f, cell, beta, cosmax, sweep_add);
      else
        cell_pass<B, false, kExch, kLd>(p, rep, cell, beta, cosmax, sweep_add);
    }
  }
  if (metro) block_accept(p, t, acc);
}

// The observables item of the work-queue kernel, out of line: its FP64
// sums get their own register allocation instead of raising the kernel's.
__device__ __noinline__ void wave_observables(const float4* rb, int cell, int L, int L3,
                                              float rcpL, double J1,
                                              double (*red)[kJ1Threads / 32], double4* out) {
  const double4 o = chunk_observables<kLdCoherent>(rb, cell, L, L3, rcpL, J1, red);
  if (threadIdx.x == 0) *out = o;
}

// kForms: bit 0 the Metropolis passes in the site form, bit 1 the
// over-relaxation passes in the site form (else the cell form); the item
// numbering (J1WaveParams::sub_metro, sub_or) must match. Four resident
// CTAs per SM with both passes in the site form (64 registers), two with a
// cell-form pass (which needs more than 80 registers to run without
// spilling). One item per CTA: the grid has
// one CTA per item, and CTA c takes the c-th ticket of the queue, not item
// blockIdx.x, so items are taken in order by CTAs that are already running
// whatever order the hardware starts them in.
template <bool kExch, int kForms>
__global__ void __launch_bounds__(kJ1Threads, kForms == 3 ? 4 : 2)
    j1_wave_kernel(const J1WaveParams w) {
  constexpr bool kMetroSite = (kForms & 1) != 0, kOrSite = (kForms & 2) != 0;
  __shared__ int s_info[5];  // item (or -1), replica, pass, chunk, sub-item
  __shared__ unsigned int s_need;
  __shared__ double red[4][kJ1Threads / 32];
  const int nq = w.n_chunks;
  const int n_passes = 4 * (w.n_metro + w.n_or);  // colour passes; pass n_passes: observables
  if (threadIdx.x == 0) {
    // One thread takes the ticket and decodes it:
    // item -> (replica group g, pass k, position j, replica, sub-item f).
    // Items per chunk before pass k (cum) and of pass k (sub): the
    // Metropolis passes come first, then the over-relaxation passes, then
    // (with_obs) one observables item per chunk.
    const int item = (int)atomicAdd(w.queue, 1u);
    s_info[0] = item < w.n_items ? item : -1;
    if (item < w.n_items) {
      const int m_items = 4 * w.n_metro * w.sub_metro;
      const int c_items = m_items + 4 * w.n_or * w.sub_or;
      const int per_group = w.group * nq * (c_items + (w.with_obs ? 1 : 0));
      const int g = item / per_group;
      const int local = item - g * per_group;
      const int r0 = g * w.group;
      const int cnt = min(w.group, w.pass.n_rep - r0);
      const int per_unit = cnt * nq;
      const int u = local / per_unit;
      int k, cum, sub;
      if (u < m_items) {
        sub = w.sub_metro;
        k = u / sub;
        cum = k * sub;
      } else if (u < c_items) {
        sub = w.sub_or;
        k = 4 * w.n_metro + (u - m_items) / sub;
        cum = m_items + (k - 4 * w.n_metro) * sub;
      } else {
        sub = 1;
        k = n_passes;
        cum = c_items;
      }
      const int wi = local - per_unit * cum;
      const int tt = wi / sub;
      const int j = tt / cnt;
      s_info[1] = r0 + (tt - j * cnt);
      s_info[2] = k;
      s_info[3] = (int)(((long long)j + (long long)w.dep * k) % nq);
      s_info[4] = wi - tt * sub;  // FCC corner of a site-form pass
      s_need = (unsigned int)cum;
    }
  }
  __syncthreads();
  const int item = s_info[0];
  if (item < 0) return;
  const int rep = s_info[1], k = s_info[2], q = s_info[3], f = s_info[4];
  // Wait until pass k - 1 is complete on every chunk holding a neighbour.
  int failed = 0;
  if (k > 0) {
    const int n_dep = 2 * w.dep + 1 >= nq ? nq : 2 * w.dep + 1;
    const unsigned int need = s_need;
    const unsigned int* row = w.progress + (long long)rep * nq;
    for (int d = threadIdx.x; d < n_dep; d += blockDim.x) {
      int qq = n_dep == nq ? d : q - w.dep + d;
      qq = qq < 0 ? qq + nq : (qq >= nq ? qq - nq : qq);
      unsigned int polls = 0;
      while (ld_acquire_gpu(row + qq) < need) {
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
    return;
  }
  if (k == n_passes) {
    // the observables pass: partials of the state the last pass left, in
    // the layout and order of j1_observables_kernel
    const float4* rb = w.pass.spins + (long long)rep * 16 * w.pass.L3;
    wave_observables(rb, q * kJ1Threads + threadIdx.x, w.pass.L, w.pass.L3, w.pass.rcpL, w.obs.J1,
                     red, w.obs.partials + w.obs.partial_begin + (long long)rep * nq + q);
    return;  // nothing depends on it within the launch
  }
  const int sweep_idx = k >> 2;
  const bool metro = sweep_idx < w.n_metro;
  const unsigned long long sweep_add = (unsigned long long)sweep_idx;
  switch (k & 3) {
    case 0: wave_item<0, kExch, kMetroSite, kOrSite>(w, rep, q, f, metro, sweep_add); break;
    case 1: wave_item<1, kExch, kMetroSite, kOrSite>(w, rep, q, f, metro, sweep_add); break;
    case 2: wave_item<2, kExch, kMetroSite, kOrSite>(w, rep, q, f, metro, sweep_add); break;
    default: wave_item<3, kExch, kMetroSite, kOrSite>(w, rep, q, f, metro, sweep_add); break;
  }
  __syncthreads();  // every store of the item is issued
  if (threadIdx.x == 0 && item != w.stall_item)
    release_add_gpu(w.progress + (long long)rep * nq + q, 1u);
}

// Resident CTAs per SM of the skewed launches with both passes in the site
// form (their register bound).
#ifndef PYRO_SKEW_SITE_BLOCKS
#define PYRO_SKEW_SITE_BLOCKS 4
#endif
constexpr int kSkewSiteBlocks = PYRO_SKEW_SITE_BLOCKS;

// Skewed launches (see J1SkewParams): launch t runs pass t - stagger g of
// every replica group g that has one, all of them independent (different
// replicas); consecutive passes of a group are ordered by the stream. The
// CTA's item comes from blockIdx.x across the groups of the launch, group by
// group, then (replica, chunk, sub-item) as in the work-queue kernel. Within a
// launch nothing that an item reads is written (its own pass writes one
// colour, which no item of the launch reads), so the loads take the
// read-only path like the per-pass kernels'.
template <bool kExch, int kForms>
__global__ void __launch_bounds__(kJ1Threads, kForms == 3 ? kSkewSiteBlocks : 2)
    j1_skew_kernel(const J1SkewParams sp) {
  constexpr bool kMetroSite = (kForms & 1) != 0, kOrSite = (kForms & 2) != 0;
  pass_prologue();
  const J1WaveParams& w = sp.w;
  __shared__ int s_info[4];  // replica, pass, chunk, sub-item
  __shared__ double red[4][kJ1Threads / 32];
  const int nq = w.n_chunks;
  const int n_passes = 4 * (w.n_metro + w.n_or);
  if (threadIdx.x == 0) {
    int b = blockIdx.x;
    int g = skew_first_group(sp);
    for (;; ++g) {
      const int k = sp.t - sp.stagger * g;
      const int cnt = min(w.group, w.pass.n_rep - g * w.group);
      const int sub = skew_sub(w, k);
      const int items = cnt * nq * sub;
      if (b < items) {
        const int tt = b / sub;
        const int r = tt % cnt;
        s_info[0] = g * w.group + r;
        s_info[1] = k;
        s_info[2] = tt / cnt;
        s_info[3] = b - tt * sub;
        break;
      }
      b -= items;
    }
  }
  __syncthreads();
  const int rep = s_info[0], k = s_info[1], q = s_info[2], f = s_info[3];
  if (k == n_passes) {  // the group's observables, in the layout of j1_observables_kernel
    const float4* rb = w.pass.spins + (long long)rep * 16 * w.pass.L3;
    wave_observables(rb, q * kJ1Threads + threadIdx.x, w.pass.L, w.pass.L3, w.pass.rcpL, w.obs.J1,
                     red, w.obs.partials + w.obs.partial_begin + (long long)rep * nq + q);
    return;
  }
  const int sweep_idx = k >> 2;
  const bool metro = sweep_idx < w.n_metro;
  const unsigned long long sweep_add = (unsigned long long)sweep_idx;
  switch (k & 3) {
    case 0: wave_item<0, kExch, kMetroSite, kOrSite, kLdNc>(w, rep, q, f, metro, sweep_add); break;
    case 1: wave_item<1, kExch, kMetroSite, kOrSite, kLdNc>(w, rep, q, f, metro, sweep_add); break;
    case 2: wave_item<2, kExch, kMetroSite, kOrSite, kLdNc>(w, rep, q, f, metro, sweep_add); break;
    default: wave_item<3, kExch, kMetroSite, kOrSite, kLdNc>(w, rep, q, f, metro, sweep_add); break;
  }
}
}  // namespace

namespace {
template <typename Kernel>
void launch_pass(Kernel k, dim3 grid, const J1PassParams& p, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kJ1Threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, p);  // errors are read back with cudaGetLastError
}
}  // namespace

// log2 L of the fixed-L kernels for this pass (0: the run-time form).
int j1_fixed_log2(const J1PassParams& p) {
  if (p.exch || p.fixed_l == 0) return 0;
  if (p.L == 32) return 5;
  if (p.L == 16) return 4;
  return 0;
}

void launch_j1_pass(const J1PassParams& p, int colour, bool metro, bool site_per_thread,
                    cudaStream_t st) {
  const dim3 grid((p.L3 + kJ1Threads - 1) / kJ1Threads, p.n_rep);
  // site form: CTAs of one corner, or (fixed L) of all four corners of a tile
  const dim3 sgrid = j1_fixed_log2(p) > 0 ? dim3(4 * p.L3 / kJ1Threads, 1, p.n_rep)
                                          : dim3((p.L3 + kJ1Threads - 1) / kJ1Threads, 4, p.n_rep);
#define PYRO_J1_CASE(B, X, G)                                                         \
  case B:                                                                             \
    if (site_per_thread) {                                                            \
      if (metro) launch_pass(j1_site_pass_kernel<B, true, X, G>, sgrid, p, st);       \
      else launch_pass(j1_site_pass_kernel<B, false, X, G>, sgrid, p, st);            \
    } else {                                                                          \
      if (metro) launch_pass(j1_pass_kernel<B, true, X, G>, grid, p, st);             \
      else launch_pass(j1_pass_kernel<B, false, X, G>, grid, p, st);                  \
    }                                                                                 \
    break;
#define PYRO_J1_COLOURS(X, G) \
  switch (colour) {           \
    PYRO_J1_CASE(0, X, G)     \
    PYRO_J1_CASE(1, X, G)     \
    PYRO_J1_CASE(2, X, G)     \
    PYRO_J1_CASE(3, X, G)     \
    default:                  \
      break;                  \
  }
  const int lg = j1_fixed_log2(p);
  if (p.exch) {
    PYRO_J1_COLOURS(true, 0)
  } else if (lg == 5) {
    PYRO_J1_COLOURS(false, 5)
  } else if (lg == 4) {
    PYRO_J1_COLOURS(false, 4)
  } else {
    PYRO_J1_COLOURS(false, 0)
  }
#undef PYRO_J1_COLOURS
#undef PYRO_J1_CASE
}

void launch_j1_last_pass(const J1PassParams& p, const J1ObsParams& o, bool metro,
                         cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((p.L3 + kJ1Threads - 1) / kJ1Threads, p.n_rep);
  cfg.blockDim = dim3(kJ1Threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  const int lg = j1_fixed_log2(p);
  if (lg == 5) {
    if (metro) cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<true, 5>, p, o);
    else cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<false, 5>, p, o);
  } else if (lg == 4) {
    if (metro) cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<true, 4>, p, o);
    else cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<false, 4>, p, o);
  } else {
    if (metro) cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<true>, p, o);
    else cudaLaunchKernelEx(&cfg, j1_last_pass_kernel<false>, p, o);
  }
}

void launch_j1_observables(const J1ObsParams& p, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((p.L3 + kJ1Threads - 1) / kJ1Threads, p.n_rep);
  cfg.blockDim = dim3(kJ1Threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, j1_observables_kernel, p);  // errors are read back with cudaGetLastError
}

int j1_wave_dep(int L) {
  // A neighbour of a cell lies in the plane before or after it, at most
  // 2 L^2 - 1 cells away (modulo L^3); one chunk of slack covers the
  // partial last chunk when the distance wraps around.
  return (2 * L * L + kJ1Threads - 1) / kJ1Threads + 1;
}

namespace {
using WaveKernel = void (*)(const J1WaveParams);
WaveKernel wave_kernel(bool exch, int forms) {
  static const WaveKernel k[2][4] = {
      {j1_wave_kernel<false, 0>, j1_wave_kernel<false, 1>, j1_wave_kernel<false, 2>,
       j1_wave_kernel<false, 3>},
      {j1_wave_kernel<true, 0>, j1_wave_kernel<true, 1>, j1_wave_kernel<true, 2>,
       j1_wave_kernel<true, 3>}};
  return k[exch ? 1 : 0][forms & 3];
}
}  // namespace

cudaError_t launch_j1_wave(const J1WaveParams& p, int forms, cudaStream_t st) {
  wave_kernel(p.pass.exch != 0, forms)<<<p.n_items, kJ1Threads, 0, st>>>(p);
  return cudaGetLastError();
}

int j1_skew_items(const J1SkewParams& sp) {
  const J1WaveParams& w = sp.w;
  int total = 0;
  for (int g = skew_first_group(sp); g <= skew_last_group(sp); ++g) {
    const int cnt = std::min(w.group, w.pass.n_rep - g * w.group);
    total += cnt * w.n_chunks * skew_sub(w, sp.t - sp.stagger * g);
  }
  return total;
}

cudaError_t launch_j1_skew(const J1SkewParams& sp, int forms, cudaStream_t st) {
  using SkewKernel = void (*)(const J1SkewParams);
  static const SkewKernel k[2][4] = {
      {j1_skew_kernel<false, 0>, j1_skew_kernel<false, 1>, j1_skew_kernel<false, 2>,
       j1_skew_kernel<false, 3>},
      {j1_skew_kernel<true, 0>, j1_skew_kernel<true, 1>, j1_skew_kernel<true, 2>,
       j1_skew_kernel<true, 3>}};
  const int items = j1_skew_items(sp);
  if (items <= 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(items, 1, 1);
  cfg.blockDim = dim3(kJ1Threads, 1, 1);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = sp.w.pass.pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k[sp.w.pass.exch ? 1 : 0][forms & 3], sp);
}

namespace {
using CycleKernel = void (*)(const J1CycleParams);
CycleKernel cycle_kernel_for(int log2L) {
  if (log2L == 5) return j1_cycle_cluster_fixed_kernel<5>;
  if (log2L == 4) return j1_cycle_cluster_fixed_kernel<4>;
  return j1_cycle_cluster_kernel;
}

cudaError_t cycle_occupancy(void (*kern)(const J1CycleParams), int cluster_size, int* n) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cluster_size * 64, 1, 1);
  cfg.blockDim = dim3(kJ1CycleThreads, 1, 1);
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaOccupancyMaxActiveClusters(n, kern, &cfg);
}
}  // namespace

cudaError_t j1_cycle_prepare(int cluster_size, int* max_active_clusters) {
  *max_active_clusters = 0;
  int least = 1 << 30;
  for (int lg : {0, 4, 5}) {
    const CycleKernel kern = cycle_kernel_for(lg);
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cycle_occupancy(kern, cluster_size, &n);
    if (e != cudaSuccess) return e;
    least = std::min(least, n);
  }
  *max_active_clusters = least;
  return cudaSuccess;
}

cudaError_t launch_j1_cycle(const J1CycleParams& p, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.cluster_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(p.cluster_size * p.pass.n_rep, 1, 1);
  cfg.blockDim = dim3(kJ1CycleThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, cycle_kernel_for(j1_fixed_log2(p.pass)), p);
}

}  // namespace pyro
