// Pyrochlore geometry, colour schedules and the per-pass work description.
//
// Geometry (taillefu/cudacode Pyrochlore.cu:1339-1401, atom positions; 16-site
// conventional cubic cell = 4 FCC corners x 4-site basis, Pyrochlore.cu:29-30):
// site s = 4 f + b sits at F[f] + B[b], with the FCC corners
// F = (0,0,0), (1/2,1/2,0), (0,1/2,1/2), (1/2,0,1/2) and the basis B = F/2.
// b is the pyrochlore sublattice; {4f..4f+3} is one up-tetrahedron.
//
// The neighbour table is not copied from links16 (Pyrochlore.cu:152-167): it
// is generated from the positions by distance shell,
//   J1  : |r|^2 = 2/16  (6 neighbours)   J2 : 6/16 (12)
//   J3a : 8/16 through a shared neighbour (r = 2 x a J1 bond vector; 6)
//   J3b : 8/16 across a hexagon (the other 6),
// in the canonical order (shell, target site, dx, dy, dz). The oracle sums a
// site's neighbours in exactly this order, which the bit-exact parity needs.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PYRO_HOSTDEV __host__ __device__
#else
#define PYRO_HOSTDEV
#endif

namespace pyro {

constexpr int kSitesPerCell = 16;
constexpr int kMaxNbr = 30;
constexpr int kShellBegin[5] = {0, 6, 18, 24, 30};  // J1, J2, J3a, J3b, end

struct NbrEntry {
  int8_t dx, dy, dz, t;  // neighbour cell offset and its site in the cell
};


struct NbrTable {
  NbrEntry e[kSitesPerCell][kMaxNbr];
};

// Positions in units of a/4.
inline void site_pos4(int s, int p[3]) {
  static const int F[4][3] = {{0, 0, 0}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}};
  const int f = s >> 2, b = s & 3;
  for (int k = 0; k < 3; ++k) p[k] = F[f][k] + F[b][k] / 2;
}

// Builds the canonical table; returns false if a shell count is off.
bool build_neighbour_table(NbrTable* tab);

// Compile-time form of the J1 shell of the same table: the k-th (0..5)
// nearest neighbour of cubic-cell site s, in the canonical order (target
// site, dx, dy, dz). Enumerating the candidates in that order makes a sort
// unnecessary. Used by kernels that need the offsets as constants.
PYRO_HOSTDEV constexpr NbrEntry j1_neighbour(int s, int k) {
  const int F[4][3] = {{0, 0, 0}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}};
  int found = 0;
  for (int t = 0; t < kSitesPerCell; ++t)
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          const int vx = 4 * dx + F[t >> 2][0] + F[t & 3][0] / 2 - F[s >> 2][0] - F[s & 3][0] / 2;
          const int vy = 4 * dy + F[t >> 2][1] + F[t & 3][1] / 2 - F[s >> 2][1] - F[s & 3][1] / 2;
          const int vz = 4 * dz + F[t >> 2][2] + F[t & 3][2] / 2 - F[s >> 2][2] - F[s & 3][2] / 2;
          if (vx * vx + vy * vy + vz * vz == 2) {
            if (found == k) return NbrEntry{(int8_t)dx, (int8_t)dy, (int8_t)dz, (int8_t)t};
            ++found;
          }
        }
  return NbrEntry{0, 0, 0, -1};
}

// Compile-time form of the full canonical table (all four shells): entry k
// (0..29) of site s, enumerated in the order (shell, target site, dx, dy, dz)
// exactly as build_neighbour_table sorts it.
PYRO_HOSTDEV constexpr int site_at4(int x, int y, int z) {
  const int F[4][3] = {{0, 0, 0}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}};
  x &= 3;
  y &= 3;
  z &= 3;
  for (int t = 0; t < kSitesPerCell; ++t)
    if (F[t >> 2][0] + F[t & 3][0] / 2 == x && F[t >> 2][1] + F[t & 3][1] / 2 == y &&
        F[t >> 2][2] + F[t & 3][2] / 2 == z)
      return t;
  return -1;
}

PYRO_HOSTDEV constexpr NbrEntry far_neighbour(int s, int k) {
  const int F[4][3] = {{0, 0, 0}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}};
  const int px = F[s >> 2][0] + F[s & 3][0] / 2, py = F[s >> 2][1] + F[s & 3][1] / 2,
            pz = F[s >> 2][2] + F[s & 3][2] / 2;
  int found = 0;
  for (int shell = 0; shell < 4; ++shell)
    for (int t = 0; t < kSitesPerCell; ++t)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            const int vx = 4 * dx + F[t >> 2][0] + F[t & 3][0] / 2 - px;
            const int vy = 4 * dy + F[t >> 2][1] + F[t & 3][1] / 2 - py;
            const int vz = 4 * dz + F[t >> 2][2] + F[t & 3][2] / 2 - pz;
            const int r2 = vx * vx + vy * vy + vz * vz;
            int sh = -1;
            if (r2 == 2) sh = 0;
            else if (r2 == 6) sh = 1;
            else if (r2 == 8) {
              const bool even = vx % 2 == 0 && vy % 2 == 0 && vz % 2 == 0;
              sh = even && site_at4(px + vx / 2, py + vy / 2, pz + vz / 2) >= 0 ? 2 : 3;
            }
            if (sh != shell) continue;
            if (found == k) return NbrEntry{(int8_t)dx, (int8_t)dy, (int8_t)dz, (int8_t)t};
            ++found;
          }
  return NbrEntry{0, 0, 0, -1};
}

// Canonical index of the j-th (0..2) nearest neighbour of site s that is not
// in s's own up-tetrahedron (same cell, same FCC corner): its down-tetrahedron
// partners.
PYRO_HOSTDEV constexpr int j1_down_index(int s, int j) {
  int found = 0;
  for (int k = 0; k < 6; ++k) {
    const NbrEntry e = j1_neighbour(s, k);
    const bool up = e.dx == 0 && e.dy == 0 && e.dz == 0 && (e.t >> 2) == (s >> 2);
    if (!up) {
      if (found == j) return k;
      ++found;
    }
  }
  return -1;
}

// Work description of one colour pass over one (system, colour) pair.
struct PassSeg {
  int sys;             // system index
  int colour;          // colour class
  int blocks_per_rep;  // CTAs per replica
  int block_begin;     // first CTA of the segment in the launch
  int rep_begin;       // first replica of the system covered by the segment
};

// Per-system constants in device memory.
struct SysDev {
  int L, L3;
  int n_colours;       // 4 (J1 only) or 16
  int units_per_colour;  // sites per colour class per replica
  int n_rep;           // replicas held
  int rep_global;      // global replica id of replica 0 within the system's ladder
  int rep_key;         // Philox replica word of replica 0 (unique across systems)
  int swap_key;        // Philox word of the system's exchanges (its index, unique)
  int rep_ctx_base;    // index of replica 0 in the context-wide per-replica arrays
  int temp_base;       // offset of this system's temperature arrays
  int n_temp;          // ladder size
  long long spin_off;  // float4 offset of replica 0
  float rcpL;              // 1 / L (cell decode)
  float J1, J2, J3a, J3b;   // FP32 couplings of the update arithmetic
  double J64[4];           // the same couplings in FP64 for the observables
  int shells;          // bitmask of non-zero shells: 1 J1, 2 J2, 4 J3a, 8 J3b
  int exch;            // index of the system's bond matrices (ExchangeDev), -1: isotropic J1
};

// Bond-dependent nearest-neighbour exchange and Zeeman field of one system:
// H = sum_<ij> S_i^T A[b_i][b_j] S_j - sum_i f[b_i] . S_i, b the pyrochlore
// sublattice (site & 3). A[4 * bi + bj] is row-major; A[bj][bi] = A[bi][bj]^T.
// Replaces the isotropic J1 shell (further shells stay isotropic).
struct ExchangeDev {
  float A[16][9];
  float f[4][3];
  double A64[16][9];
  double f64[4][3];
};

// Sites of colour class c: for the 4-colour schedule colour b holds sites
// {b, 4+b, 8+b, 12+b} (the pyrochlore sublattices, Pyrochlore.cu:36-43
// groups {0,4,8,12}...{3,7,11,15}); for 16 colours colour c is site c.
PYRO_HOSTDEV inline int colour_site(int n_colours, int colour, int k) {
  return n_colours == 4 ? 4 * k + colour : colour;
}

}  // namespace pyro
