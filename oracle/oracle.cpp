// ORACLE — test infrastructure only. Nothing in the engine links or calls
// this file; tests/, the smoke check and the CPU-baseline leg of the
// benchmark use it as the checker.
//
// A plain C++/OpenMP restatement of the pyrochlore Heisenberg Monte Carlo of
// taillefu/cudacode with the engine's update order and Philox streams:
//   energy convention and periodic neighbour arithmetic  Pyrochlore.cu:468-523 (TotalEnergy)
//   site positions                                       Pyrochlore.cu:1339-1401
//   sublattice colour classes                            Pyrochlore.cu:36-43
//   sphere sampling                                      Math.cu:120-130
//   cone proposal                                        Math.cu:244-281
//   Metropolis rule                                      Math.cu:968-986
//   over-relaxation S -> 2(S.h)h/|h|^2 - S               Math.cu:220-242
//   replica exchange min(1, exp((b1-b2)(E1-E2)))         MonteCarlo.cu:105-172
//   cone-width adaptation                                MonteCarlo.cu:371-426
// Units: unit classical spins, H = J1 sum_<ij> S_i.S_j (+ J2, J3a, J3b shells),
// or, for the anisotropic model, H = sum_<ij> S_i^T A[b_i][b_j] S_j -
// sum_i f[b_i] . S_i (b the sublattice; CalculateLocalExchangeField
// Pyrochlore.cu:210-275 and TotalEnergy 468-523 with the bond matrices of
// couplings_const 169-184 and the site fields of InitializeMagneticField
// 414-450, their spin-1/2 factor folded into A and f).
// The reference's TotalEnergy equals this energy times S^2 = 1/4 when its
// J1 = J2 = J and J3 = J4 = 0 (couplings_const, Pyrochlore.cu:169-184).
//
// The reference itself cannot serve: its glue files (functions.h, reduce.cu,
// Device.cu, Measure.hpp, StructFactor.hpp, Utils.hpp) are absent and it needs
// MKL, GSL and popt, none of which exist here.
//
// Two precisions:
//  * float: every update uses the functions of include/pyro_math.h, so the
//    result is bit-identical to the CUDA kernels for any number of sweeps.
//  * double: spins, fields and updates in FP64 with libm functions and the
//    same Philox words; the "FP64 host run" for statistical comparisons.
//
// Geometry is derived independently of the engine's per-cell table: every
// site gets real-space coordinates (units a/4) and its neighbours are found by
// enumerating the displacement vectors of each distance shell and looking the
// target up by coordinates; they are then put in the canonical order (shell,
// target site of the cell, dx, dy, dz).
#include <omp.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/pyro_math.h"

namespace {

const int kShellBegin[5] = {0, 6, 18, 24, 30};

void pos4(int s, int p[3]) {
  // FCC corners F and basis F/2 of the 16-site cubic cell (Pyrochlore.cu:1339-1401).
  static const int F[4][3] = {{0, 0, 0}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}};
  for (int k = 0; k < 3; ++k) p[k] = F[s / 4][k] + F[s % 4][k] / 2;
}

// site-in-cell id from coordinates mod 4 (units a/4), or -1.
int site_at(int x, int y, int z) {
  x &= 3;
  y &= 3;
  z &= 3;
  for (int s = 0; s < 16; ++s) {
    int p[3];
    pos4(s, p);
    if (p[0] == x && p[1] == y && p[2] == z) return s;
  }
  return -1;
}

struct Nbr {
  int dx, dy, dz, t;
};

// nb[s][k], k in canonical order.
std::array<std::array<Nbr, 30>, 16> build_geometry() {
  std::array<std::array<Nbr, 30>, 16> nb;
  for (int s = 0; s < 16; ++s) {
    int p[3];
    pos4(s, p);
    struct C {
      int shell, t, dx, dy, dz;
    };
    std::vector<C> c;
    for (int vx = -3; vx <= 3; ++vx)
      for (int vy = -3; vy <= 3; ++vy)
        for (int vz = -3; vz <= 3; ++vz) {
          const int r2 = vx * vx + vy * vy + vz * vz;
          if (r2 != 2 && r2 != 6 && r2 != 8) continue;
          const int q[3] = {p[0] + vx, p[1] + vy, p[2] + vz};
          const int t = site_at(q[0], q[1], q[2]);
          if (t < 0) continue;
          int shell = r2 == 2 ? 0 : r2 == 6 ? 1 : 3;
          if (r2 == 8 && (vx % 2 == 0) && (vy % 2 == 0) && (vz % 2 == 0)) {
            // through a site: the midpoint is itself a site one J1 bond away
            if (site_at(p[0] + vx / 2, p[1] + vy / 2, p[2] + vz / 2) >= 0) shell = 2;
          }
          auto fdiv = [](int a) { return a >= 0 ? a / 4 : -((-a + 3) / 4); };
          c.push_back({shell, t, fdiv(q[0]), fdiv(q[1]), fdiv(q[2])});
        }
    std::sort(c.begin(), c.end(), [](const C& a, const C& b) {
      if (a.shell != b.shell) return a.shell < b.shell;
      if (a.t != b.t) return a.t < b.t;
      if (a.dx != b.dx) return a.dx < b.dx;
      if (a.dy != b.dy) return a.dy < b.dy;
      return a.dz < b.dz;
    });
    if (c.size() != 30) {
      fprintf(stderr, "oracle geometry: site %d has %zu neighbours\n", s, c.size());
      std::abort();
    }
    for (int k = 0; k < 30; ++k) nb[s][k] = {c[k].dx, c[k].dy, c[k].dz, c[k].t};
  }
  return nb;
}

struct Sys {
  int L, L3, R, off, nT, n_colours, temp_base, rep_key, shells;
  int swap_key;  // Philox word of the system's exchanges
  double J[4];
  bool exch = false;  // bond matrices replace the isotropic J1 shell
  float A[16][9] = {}, f[4][3] = {};
  double A64[16][9] = {}, f64[4][3] = {};
  std::vector<double> T;
  size_t spin_off;  // in spins
};

struct Oracle {
  bool fp64 = false;
  uint64_t seed = 0;
  int renorm_every = 0;
  std::array<std::array<Nbr, 30>, 16> nb;
  std::vector<Sys> sys;
  std::vector<float> s32;   // 4 per spin
  std::vector<double> s64;  // 4 per spin
  std::vector<int> temp_of_rep, rep_of_temp;  // [temp_base + g], [temp_base + t]
  std::vector<float> cosmax;
  std::vector<uint64_t> accepted, swap_acc, swap_try;
  std::vector<uint64_t> swap_count;
  uint64_t sweep = 0;
  uint64_t metro_since_reset = 0;
  int total_temps = 0;
};

inline int wrap(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

inline size_t nbr_index(const Sys& S, const Nbr& e, int x, int y, int z) {
  return (size_t)e.t * S.L3 +
         (size_t)((wrap(z + e.dz, S.L) * S.L + wrap(y + e.dy, S.L)) * S.L + wrap(x + e.dx, S.L));
}

// FP32 local field, summed in canonical order; identical arithmetic to the kernel.
pyro_vec3 field32(const Oracle& o, const Sys& S, const float* rep, int s, int x, int y, int z) {
  // The J1 shell is always summed (h = J1 * a1); further shells only when
  // their coupling is non-zero, each folded in with one fused multiply-add.
  const float Jf[4] = {(float)S.J[0], (float)S.J[1], (float)S.J[2], (float)S.J[3]};
  pyro_vec3 h = {0.f, 0.f, 0.f};
  for (int sh = 0; sh < 4; ++sh) {
    if (sh == 0 && S.exch) {
      // bond matrices: h = sum_k A[b][b_k] S_k (pyro_matvec_add), then - f[b]
      const int b = s & 3;
      for (int k = 0; k < 6; ++k) {
        const Nbr& e = o.nb[s][k];
        const float* v = rep + 4 * nbr_index(S, e, x, y, z);
        h = pyro_matvec_add(h, S.A[4 * b + (e.t & 3)], v[0], v[1], v[2]);
      }
      h.x = h.x - S.f[b][0];
      h.y = h.y - S.f[b][1];
      h.z = h.z - S.f[b][2];
      continue;
    }
    if (sh > 0 && !(S.shells & (1 << sh))) continue;
    const int k0 = kShellBegin[sh];
    const float* v0 = rep + 4 * nbr_index(S, o.nb[s][k0], x, y, z);
    float ax = v0[0], ay = v0[1], az = v0[2];
    for (int k = k0 + 1; k < kShellBegin[sh + 1]; ++k) {
      const float* v = rep + 4 * nbr_index(S, o.nb[s][k], x, y, z);
      ax = ax + v[0];
      ay = ay + v[1];
      az = az + v[2];
    }
    if (sh == 0) {
      h.x = Jf[0] * ax;
      h.y = Jf[0] * ay;
      h.z = Jf[0] * az;
    } else {
      h.x = fmaf(Jf[sh], ax, h.x);
      h.y = fmaf(Jf[sh], ay, h.y);
      h.z = fmaf(Jf[sh], az, h.z);
    }
  }
  return h;
}

struct V3d {
  double x, y, z;
};

// FP64 bond-matrix field minus the site field (anisotropic systems).
template <typename T>
V3d exch_field64(const Oracle& o, const Sys& S, const T* rep, int s, int x, int y, int z) {
  const int b = s & 3;
  V3d h = {-S.f64[b][0], -S.f64[b][1], -S.f64[b][2]};
  for (int k = 0; k < 6; ++k) {
    const Nbr& e = o.nb[s][k];
    const T* v = rep + 4 * nbr_index(S, e, x, y, z);
    const double* m = S.A64[4 * b + (e.t & 3)];
    h.x += m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    h.y += m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    h.z += m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
  }
  return h;
}

V3d field64(const Oracle& o, const Sys& S, const double* rep, int s, int x, int y, int z) {
  V3d h = {0, 0, 0};
  if (S.exch) h = exch_field64(o, S, rep, s, x, y, z);
  for (int sh = 0; sh < 4; ++sh) {
    if (!(S.shells & (1 << sh))) continue;
    if (sh == 0 && S.exch) continue;
    double ax = 0, ay = 0, az = 0;
    for (int k = kShellBegin[sh]; k < kShellBegin[sh + 1]; ++k) {
      const double* v = rep + 4 * nbr_index(S, o.nb[s][k], x, y, z);
      ax += v[0];
      ay += v[1];
      az += v[2];
    }
    h.x += S.J[sh] * ax;
    h.y += S.J[sh] * ay;
    h.z += S.J[sh] * az;
  }
  return h;
}

// FP64 field from FP32 spins (observables of the FP32 chain).
V3d field64f(const Oracle& o, const Sys& S, const float* rep, int s, int x, int y, int z) {
  V3d h = {0, 0, 0};
  if (S.exch) h = exch_field64(o, S, rep, s, x, y, z);
  for (int sh = 0; sh < 4; ++sh) {
    if (!(S.shells & (1 << sh))) continue;
    if (sh == 0 && S.exch) continue;
    double ax = 0, ay = 0, az = 0;
    for (int k = kShellBegin[sh]; k < kShellBegin[sh + 1]; ++k) {
      const float* v = rep + 4 * nbr_index(S, o.nb[s][k], x, y, z);
      ax += v[0];
      ay += v[1];
      az += v[2];
    }
    h.x += S.J[sh] * ax;
    h.y += S.J[sh] * ay;
    h.z += S.J[sh] * az;
  }
  return h;
}

int colour_site(int n_colours, int colour, int k) { return n_colours == 4 ? 4 * k + colour : colour; }

void sweep_one(Oracle& o, bool metro) {
  const uint64_t sweep = o.sweep;
  const bool renorm = o.renorm_every > 0 && ((sweep + 1) % (uint64_t)o.renorm_every) == 0;
  int max_col = 4;
  for (auto& S : o.sys) max_col = std::max(max_col, S.n_colours);
  for (int pass = 0; pass < max_col; ++pass) {
    for (size_t si = 0; si < o.sys.size(); ++si) {
      Sys& S = o.sys[si];
      int colour = -1;
      if (S.n_colours == max_col) colour = pass;
      else if (pass % 4 == 0) colour = pass / 4;
      if (colour < 0) continue;
      const int per_col = 16 * S.L3 / S.n_colours;
      const long long total = (long long)S.R * per_col;
      std::vector<uint64_t> acc_rep(S.R, 0);
#pragma omp parallel
      {
        std::vector<uint64_t> acc_local(S.R, 0);
#pragma omp for schedule(static)
        for (long long w = 0; w < total; ++w) {
          const int r = (int)(w / per_col);
          const int u = (int)(w - (long long)r * per_col);
          const int k = u / S.L3, cell = u - k * S.L3;
          const int s = colour_site(S.n_colours, colour, k);
          const int x = cell % S.L, y = (cell / S.L) % S.L, z = cell / (S.L * S.L);
          const size_t own = (size_t)s * S.L3 + cell;
          const int g = S.off + r;
          const int t = o.temp_of_rep[S.temp_base + g];
          uint32_t rr[4] = {0, 0, 0, 0};
          if (metro)
            pyro_philox((uint32_t)own, (uint32_t)(S.rep_key + r), (uint32_t)sweep, PYRO_PURPOSE_METRO,
                        (uint32_t)(o.seed & 0xffffffffu), (uint32_t)(o.seed >> 32), rr);
          if (!o.fp64) {
            float* rep = o.s32.data() + 4 * (S.spin_off + (size_t)r * 16 * S.L3);
            const pyro_vec3 h = field32(o, S, rep, s, x, y, z);
            pyro_vec3 sp = {rep[4 * own], rep[4 * own + 1], rep[4 * own + 2]};
            pyro_vec3 out;
            if (metro) {
              const float beta = (float)(1.0 / S.T[t]);
              const pyro_vec3 prop = pyro_cone_proposal(sp, o.cosmax[S.temp_base + t],
                                                        pyro_uniform(rr[0]), pyro_uniform(rr[1]));
              const float dE = pyro_delta_e(h, sp, prop);
              const int a = pyro_metropolis_accept(dE, beta, pyro_uniform(rr[2]));
              acc_local[r] += (uint64_t)a;
              out = a ? prop : sp;
            } else {
              out = pyro_overrelax(sp, h);
            }
            if (renorm) out = pyro_renormalise(out);
            rep[4 * own] = out.x;
            rep[4 * own + 1] = out.y;
            rep[4 * own + 2] = out.z;
            rep[4 * own + 3] = 0.0f;
          } else {
            double* rep = o.s64.data() + 4 * (S.spin_off + (size_t)r * 16 * S.L3);
            const V3d h = field64(o, S, rep, s, x, y, z);
            V3d sp = {rep[4 * own], rep[4 * own + 1], rep[4 * own + 2]};
            V3d out = sp;
            if (metro) {
              const double beta = 1.0 / S.T[t];
              const double c0 = o.cosmax[S.temp_base + t];
              const double u1 = pyro_uniform(rr[0]), u2 = pyro_uniform(rr[1]);
              const double ct = 1.0 - (1.0 - c0) * u1;
              const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
              const double ph = 2.0 * M_PI * u2;
              const double cp = std::cos(ph), spp = std::sin(ph);
              const double sgn = std::copysign(1.0, sp.z);
              const double aa = -1.0 / (sgn + sp.z);
              const double bb = sp.x * sp.y * aa;
              const V3d e1 = {1.0 + sgn * sp.x * sp.x * aa, sgn * bb, -sgn * sp.x};
              const V3d e2 = {bb, sgn + sp.y * sp.y * aa, -sp.y};
              const V3d prop = {st * cp * e1.x + st * spp * e2.x + ct * sp.x,
                                st * cp * e1.y + st * spp * e2.y + ct * sp.y,
                                st * cp * e1.z + st * spp * e2.z + ct * sp.z};
              const double dE =
                  h.x * (prop.x - sp.x) + h.y * (prop.y - sp.y) + h.z * (prop.z - sp.z);
              const int a = dE <= 0.0 || (double)pyro_uniform(rr[2]) < std::exp(-beta * dE);
              acc_local[r] += (uint64_t)a;
              out = a ? prop : sp;
            } else {
              const double hh = h.x * h.x + h.y * h.y + h.z * h.z;
              if (hh > 0.0) {
                const double k2 = 2.0 * (sp.x * h.x + sp.y * h.y + sp.z * h.z) / hh;
                out = {k2 * h.x - sp.x, k2 * h.y - sp.y, k2 * h.z - sp.z};
              }
            }
            if (renorm) {
              const double n = std::sqrt(out.x * out.x + out.y * out.y + out.z * out.z);
              out = {out.x / n, out.y / n, out.z / n};
            }
            rep[4 * own] = out.x;
            rep[4 * own + 1] = out.y;
            rep[4 * own + 2] = out.z;
            rep[4 * own + 3] = 0.0;
          }
        }
#pragma omp critical
        for (int r = 0; r < S.R; ++r) acc_rep[r] += acc_local[r];
      }
      if (metro)
        for (int r = 0; r < S.R; ++r)
          o.accepted[S.temp_base + o.temp_of_rep[S.temp_base + S.off + r]] += acc_rep[r];
    }
  }
  o.sweep += 1;
  if (metro) o.metro_since_reset += 1;
}

void observables(const Oracle& o, int si, std::vector<double>* E, std::vector<double>* M) {
  const Sys& S = o.sys[si];
  E->assign(S.R, 0.0);
  M->assign(3 * S.R, 0.0);
  for (int r = 0; r < S.R; ++r) {
    double e = 0, mx = 0, my = 0, mz = 0;
    const size_t base = S.spin_off + (size_t)r * 16 * S.L3;
#pragma omp parallel for reduction(+ : e, mx, my, mz) schedule(static)
    for (long long i = 0; i < 16ll * S.L3; ++i) {
      const int s = (int)(i / S.L3), cell = (int)(i % S.L3);
      const int x = cell % S.L, y = (cell / S.L) % S.L, z = cell / (S.L * S.L);
      double sx, sy, sz;
      V3d h;
      if (!o.fp64) {
        const float* rep = o.s32.data() + 4 * base;
        sx = rep[4 * i];
        sy = rep[4 * i + 1];
        sz = rep[4 * i + 2];
        h = field64f(o, S, rep, s, x, y, z);
      } else {
        const double* rep = o.s64.data() + 4 * base;
        sx = rep[4 * i];
        sy = rep[4 * i + 1];
        sz = rep[4 * i + 2];
        h = field64(o, S, rep, s, x, y, z);
      }
      e += sx * h.x + sy * h.y + sz * h.z;
      if (S.exch) {  // the site field enters E once, not halved like the bonds
        const int b = s & 3;
        e -= S.f64[b][0] * sx + S.f64[b][1] * sy + S.f64[b][2] * sz;
      }
      mx += sx;
      my += sy;
      mz += sz;
    }
    (*E)[r] = 0.5 * e;
    (*M)[3 * r] = mx;
    (*M)[3 * r + 1] = my;
    (*M)[3 * r + 2] = mz;
  }
}

// Replica exchange on one system given energies by global replica.
int exchange(Oracle& o, int si, const double* E_global, int parity) {
  Sys& S = o.sys[si];
  const uint64_t count = o.swap_count[si];
  if (parity < 0) parity = (int)(count & 1u);
  int n_acc = 0;
  for (int t = parity; t + 1 < S.nT; t += 2) {
    const int ga = o.rep_of_temp[S.temp_base + t], gb = o.rep_of_temp[S.temp_base + t + 1];
    uint32_t r[4];
    pyro_philox((uint32_t)t, (uint32_t)count, (uint32_t)S.swap_key, PYRO_PURPOSE_SWAP,
                (uint32_t)(o.seed & 0xffffffffu), (uint32_t)(o.seed >> 32), r);
    const double u = pyro_uniform53(r[0], r[1]);
    const int acc = pyro_swap_accept(1.0 / S.T[t], 1.0 / S.T[t + 1], E_global[ga], E_global[gb], u);
    o.swap_try[S.temp_base + t]++;
    if (acc) {
      o.rep_of_temp[S.temp_base + t] = gb;
      o.rep_of_temp[S.temp_base + t + 1] = ga;
      o.temp_of_rep[S.temp_base + ga] = t + 1;
      o.temp_of_rep[S.temp_base + gb] = t;
      o.swap_acc[S.temp_base + t]++;
      ++n_acc;
    }
  }
  o.swap_count[si] = count + 1;
  return n_acc;
}

}  // namespace

extern "C" {

void* orc_create(int n_sys, const int* L, const int* n_rep, const int* rep_off, const int* n_temp,
                 const double* temps_concat, const double* J4, uint64_t seed, int renorm_every,
                 int fp64) {
  Oracle* o = new Oracle();
  o->fp64 = fp64 != 0;
  o->seed = seed;
  o->renorm_every = renorm_every;
  o->nb = build_geometry();
  size_t spin_off = 0;
  int tb = 0;
  for (int i = 0; i < n_sys; ++i) {
    Sys S;
    S.L = L[i];
    S.L3 = L[i] * L[i] * L[i];
    S.R = n_rep[i];
    S.off = rep_off[i];
    S.nT = n_temp[i];
    for (int k = 0; k < 4; ++k) S.J[k] = J4[4 * i + k];
    S.shells = 0;
    for (int k = 0; k < 4; ++k)
      if (S.J[k] != 0.0) S.shells |= 1 << k;
    S.n_colours = (S.J[1] != 0.0 || S.J[2] != 0.0 || S.J[3] != 0.0) ? 16 : 4;
    S.T.assign(temps_concat + tb, temps_concat + tb + S.nT);
    S.temp_base = tb;
    S.rep_key = tb + S.off;
    S.swap_key = i;
    S.spin_off = spin_off;
    spin_off += (size_t)S.R * 16 * S.L3;
    for (int t = 0; t < S.nT; ++t) {
      o->temp_of_rep.push_back(t);
      o->rep_of_temp.push_back(t);
      o->cosmax.push_back(-1.0f);
      o->accepted.push_back(0);
      o->swap_acc.push_back(0);
      o->swap_try.push_back(0);
    }
    o->swap_count.push_back(0);
    tb += S.nT;
    o->sys.push_back(S);
  }
  o->total_temps = tb;
  if (o->fp64) o->s64.assign(4 * spin_off, 0.0);
  else o->s32.assign(4 * spin_off, 0.0f);
  return o;
}

void orc_destroy(void* p) { delete (Oracle*)p; }

// The engine's pyro_set_system_keys.
void orc_set_system_keys(void* p, int si, int key_base, int swap_key) {
  Sys& S = ((Oracle*)p)->sys[si];
  S.rep_key = key_base + S.off;
  S.swap_key = swap_key;
}

int orc_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

void orc_init_random(void* p) {
  Oracle& o = *(Oracle*)p;
  for (auto& S : o.sys) {
    const long long n = (long long)S.R * 16 * S.L3;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
      const int r = (int)(i / (16ll * S.L3));
      const int site = (int)(i % (16ll * S.L3));
      uint32_t rr[4];
      pyro_philox((uint32_t)site, (uint32_t)(S.rep_key + r), 0u, PYRO_PURPOSE_INIT,
                  (uint32_t)(o.seed & 0xffffffffu), (uint32_t)(o.seed >> 32), rr);
      const pyro_vec3 v = pyro_sphere_point(pyro_uniform(rr[0]), pyro_uniform(rr[1]));
      const size_t j = 4 * (S.spin_off + (size_t)i);
      if (o.fp64) {
        o.s64[j] = v.x;
        o.s64[j + 1] = v.y;
        o.s64[j + 2] = v.z;
        o.s64[j + 3] = 0.0;
      } else {
        o.s32[j] = v.x;
        o.s32[j + 1] = v.y;
        o.s32[j + 2] = v.z;
        o.s32[j + 3] = 0.0f;
      }
    }
  }
}

long long orc_n_spins(void* p, int si) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  return (long long)S.R * 16 * S.L3;
}

void orc_set_spins(void* p, int si, const float* xyzw) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  const size_t n = 4 * (size_t)S.R * 16 * S.L3;
  for (size_t i = 0; i < n; ++i) {
    if (o.fp64) o.s64[4 * S.spin_off + i] = xyzw[i];
    else o.s32[4 * S.spin_off + i] = xyzw[i];
  }
}

void orc_get_spins(void* p, int si, float* xyzw) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  const size_t n = 4 * (size_t)S.R * 16 * S.L3;
  for (size_t i = 0; i < n; ++i)
    xyzw[i] = o.fp64 ? (float)o.s64[4 * S.spin_off + i] : o.s32[4 * S.spin_off + i];
}

void orc_get_spins64(void* p, int si, double* xyzw) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  const size_t n = 4 * (size_t)S.R * 16 * S.L3;
  for (size_t i = 0; i < n; ++i)
    xyzw[i] = o.fp64 ? o.s64[4 * S.spin_off + i] : (double)o.s32[4 * S.spin_off + i];
}

void orc_metropolis_sweep(void* p, int n) {
  for (int i = 0; i < n; ++i) sweep_one(*(Oracle*)p, true);
}

void orc_overrelax_sweep(void* p, int n) {
  for (int i = 0; i < n; ++i) sweep_one(*(Oracle*)p, false);
}

// Order parameters of every replica of one system (FP64 sums over the
// lattice, 20 per replica): the irrep components of Measurement
// (Pyrochlore.cu:526-641) from the sublattice magnetisations, the quadrupole
// sums (_CudaQuadrupolarOrder, Math.cu:335-372), the monopole density
// (CudaCalculateMonopoleSquare, Math.cu:386-476) and sum |a_b . S| / sqrt 3
// (CudaCalculateAbsSz, Math.cu:478-510), a_b the reference's sublattice axes.
void orc_order_parameters(void* p, int si, double* out) {
  const Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  static const int ax[4][3] = {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}};
  // irrep rows as coefficient vectors per sublattice, and their normalisation
  static const int irrep[12][4][3] = {
      {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}},
      {{-2, 1, 1}, {2, -1, 1}, {-2, -1, -1}, {2, 1, -1}},
      {{0, -1, 1}, {0, 1, 1}, {0, 1, -1}, {0, -1, -1}},
      {{0, -1, 1}, {0, -1, -1}, {0, 1, -1}, {0, 1, 1}},
      {{1, 0, -1}, {1, 0, 1}, {-1, 0, -1}, {-1, 0, 1}},
      {{-1, 1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, -1, 0}},
      {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}},
      {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}},
      {{0, 0, 1}, {0, 0, 1}, {0, 0, 1}, {0, 0, 1}},
      {{0, -1, -1}, {0, -1, 1}, {0, 1, 1}, {0, 1, -1}},
      {{-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {1, 0, 1}},
      {{-1, -1, 0}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}}};
  for (int r = 0; r < S.R; ++r) {
    const size_t base = S.spin_off + (size_t)r * 16 * S.L3;
    double M[4][3] = {}, Q[6] = {}, mono = 0.0, absz = 0.0;
    for (int cell = 0; cell < S.L3; ++cell) {
      double cell_mono = 0.0;
      for (int t = 0; t < 4; ++t) {
        double charge = 0.0;
        for (int b = 0; b < 4; ++b) {
          const size_t i = base + (size_t)(4 * t + b) * S.L3 + cell;
          const double x = o.fp64 ? o.s64[4 * i] : o.s32[4 * i];
          const double y = o.fp64 ? o.s64[4 * i + 1] : o.s32[4 * i + 1];
          const double z = o.fp64 ? o.s64[4 * i + 2] : o.s32[4 * i + 2];
          M[b][0] += x;
          M[b][1] += y;
          M[b][2] += z;
          Q[0] += x * x - 1.0 / 3.0;
          Q[1] += x * y;
          Q[2] += x * z;
          Q[3] += y * y - 1.0 / 3.0;
          Q[4] += y * z;
          Q[5] += z * z - 1.0 / 3.0;
          const double pr = x * ax[b][0] + y * ax[b][1] + z * ax[b][2];
          charge += pr;
          absz += std::fabs(pr);
        }
        cell_mono += std::fabs(charge);
      }
      mono += 0.25 * cell_mono;
    }
    double* q = out + 20 * (size_t)r;
    for (int m = 0; m < 12; ++m) {
      const double norm = m == 0 ? 1.0 / std::sqrt(3.0)
                          : m == 1 ? 1.0 / std::sqrt(6.0)
                          : (m >= 6 && m <= 8) ? 1.0 : 1.0 / std::sqrt(2.0);
      double v = 0.0;
      for (int b = 0; b < 4; ++b)
        for (int k = 0; k < 3; ++k) v += irrep[m][b][k] * M[b][k];
      q[m] = norm * v;
    }
    for (int k = 0; k < 6; ++k) q[12 + k] = Q[k];
    q[18] = mono;
    q[19] = absz / std::sqrt(3.0);
  }
}

// Ising projection (CudaCalculateIsingConf, Math.cu:513-541): per cell, bit
// 4 t + b set where a_b . S < 0.
void orc_ising_configuration(void* p, int si, int r, int* out) {
  const Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  static const int ax[4][3] = {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}};
  const size_t base = S.spin_off + (size_t)r * 16 * S.L3;
  for (int cell = 0; cell < S.L3; ++cell) {
    int mask = 0;
    for (int s = 0; s < 16; ++s) {
      const size_t i = base + (size_t)s * S.L3 + cell;
      const double x = o.fp64 ? o.s64[4 * i] : o.s32[4 * i];
      const double y = o.fp64 ? o.s64[4 * i + 1] : o.s32[4 * i + 1];
      const double z = o.fp64 ? o.s64[4 * i + 2] : o.s32[4 * i + 2];
      if (x * ax[s & 3][0] + y * ax[s & 3][1] + z * ax[s & 3][2] < 0.0) mask |= 1 << s;
    }
    out[cell] = mask;
  }
}

// Bond matrices A[16][9] (row-major per sublattice pair) and site fields
// f[4][3] (null: none) of one system; A = null returns it to isotropic J1.
void orc_set_exchange(void* p, int si, const double* A144, const double* f12) {
  Oracle& o = *(Oracle*)p;
  Sys& S = o.sys[si];
  S.exch = A144 != nullptr;
  for (int q = 0; q < 144; ++q) {
    const int a = (q / 9) / 4, b = (q / 9) % 4;
    S.A64[q / 9][q % 9] = (A144 && a != b) ? A144[q] : 0.0;
    S.A[q / 9][q % 9] = (float)S.A64[q / 9][q % 9];
  }
  for (int q = 0; q < 12; ++q) {
    S.f64[q / 3][q % 3] = (A144 && f12) ? f12[q] : 0.0;
    S.f[q / 3][q % 3] = (float)S.f64[q / 3][q % 3];
  }
}

void orc_set_cone(void* p, int si, const float* c) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  for (int t = 0; t < S.nT; ++t) o.cosmax[S.temp_base + t] = c[t];
}

void orc_get_cone(void* p, int si, float* c) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  for (int t = 0; t < S.nT; ++t) c[t] = o.cosmax[S.temp_base + t];
}

void orc_get_acceptance(void* p, int si, uint64_t* acc, uint64_t* prop) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  for (int t = 0; t < S.nT; ++t) {
    acc[t] = o.accepted[S.temp_base + t];
    if (prop) prop[t] = (uint64_t)16 * S.L3 * o.metro_since_reset;
  }
}

void orc_reset_acceptance(void* p) {
  Oracle& o = *(Oracle*)p;
  std::fill(o.accepted.begin(), o.accepted.end(), 0);
  o.metro_since_reset = 0;
}

// Same adaptation rule as the engine's pyro_tune_cone.
void orc_tune_cone(void* p, double target, int iterations, int sweeps_per_iteration, int n_or) {
  Oracle& o = *(Oracle*)p;
  for (int it = 0; it < iterations; ++it) {
    orc_reset_acceptance(p);
    for (int k = 0; k < sweeps_per_iteration; ++k) {
      sweep_one(o, true);
      for (int j = 0; j < n_or; ++j) sweep_one(o, false);
    }
    bool done = true;
    for (auto& S : o.sys) {
      for (int t = 0; t < S.nT; ++t) {
        const double prop = (double)16 * S.L3 * o.metro_since_reset;
        const double ratio = prop > 0 ? (double)o.accepted[S.temp_base + t] / prop : target;
        if (std::fabs(ratio - target) > 0.02) done = false;
        double theta =
            std::acos(std::max(-1.0, std::min(1.0, (double)o.cosmax[S.temp_base + t])));
        const double f = std::max(0.5, std::min(2.0, ratio / target));
        theta = std::max(1e-4, std::min(M_PI, theta * f));
        float c = (float)std::cos(theta);
        if (c >= 1.0f) c = std::nextafter(1.0f, 0.0f);
        if (c < -1.0f) c = -1.0f;
        o.cosmax[S.temp_base + t] = c;
      }
    }
    if (done) break;
  }
  orc_reset_acceptance(p);
}

void orc_observables(void* p, int si, double* E, double* M3) {
  std::vector<double> e, m;
  observables(*(Oracle*)p, si, &e, &m);
  std::memcpy(E, e.data(), sizeof(double) * e.size());
  if (M3) std::memcpy(M3, m.data(), sizeof(double) * m.size());
}

// Unsharded exchange on every system, energies computed here.
int orc_pt_swap(void* p, int parity) {
  Oracle& o = *(Oracle*)p;
  int n = 0;
  for (size_t si = 0; si < o.sys.size(); ++si) {
    std::vector<double> e, m;
    observables(o, (int)si, &e, &m);
    n += exchange(o, (int)si, e.data(), parity);
  }
  return n;
}

int orc_pt_swap_global(void* p, int si, const double* E_all, int parity) {
  return exchange(*(Oracle*)p, si, E_all, parity);
}

// n_cycles of (n_metro M + n_or OR sweeps, energies, optional exchange of
// alternating parity). history (optional): [cycle][total_temps], E by slot.
void orc_cycle(void* p, int n_metro, int n_or, int do_swap, int n_cycles, double* history) {
  Oracle& o = *(Oracle*)p;
  for (int c = 0; c < n_cycles; ++c) {
    for (int i = 0; i < n_metro; ++i) sweep_one(o, true);
    for (int i = 0; i < n_or; ++i) sweep_one(o, false);
    for (size_t si = 0; si < o.sys.size(); ++si) {
      Sys& S = o.sys[si];
      std::vector<double> e, m;
      observables(o, (int)si, &e, &m);
      if (history)
        for (int t = 0; t < S.nT; ++t)
          history[(size_t)c * o.total_temps + S.temp_base + t] =
              e[o.rep_of_temp[S.temp_base + t] - S.off];
      if (do_swap) exchange(o, (int)si, e.data(), -1);
    }
  }
}

void orc_get_permutation(void* p, int si, int* rep_of_temp) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  for (int t = 0; t < S.nT; ++t) rep_of_temp[t] = o.rep_of_temp[S.temp_base + t];
}

void orc_get_swap_stats(void* p, int si, uint64_t* acc, uint64_t* tried) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  for (int t = 0; t < S.nT; ++t) {
    acc[t] = o.swap_acc[S.temp_base + t];
    tried[t] = o.swap_try[S.temp_base + t];
  }
}

uint64_t orc_sweep_count(void* p) { return ((Oracle*)p)->sweep; }

// Static structure factor by the direct sum over sites (Math.cu:721-741 sums
// |m_q|^2 over components after the FFT; positions Pyrochlore.cu:1339-1401):
// S(q) = (1/N) sum_a |sum_i S_i^a exp(-i q.r_i)|^2, q = (2 pi/L) stride (h,k,l),
// averaged over the chosen replicas; out[((h+G/2) G + (k+G/2)) G + (l+G/2)].
void orc_structure_factor(void* p, int si, int replica, int G, int stride, double* out) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  const int r0 = replica < 0 ? 0 : replica, r1 = replica < 0 ? S.R : replica + 1;
  const long long N = 16ll * S.L3;
  const long long G3 = (long long)G * G * G;
#pragma omp parallel for schedule(dynamic)
  for (long long q = 0; q < G3; ++q) {
    const int hi = (int)(q / (G * G)), ki = (int)((q / G) % G), li = (int)(q % G);
    const double th = 2.0 * M_PI * stride / S.L;
    const double qx = th * (hi - G / 2), qy = th * (ki - G / 2), qz = th * (li - G / 2);
    double acc = 0.0;
    for (int r = r0; r < r1; ++r) {
      double re[3] = {0, 0, 0}, im[3] = {0, 0, 0};
      for (long long i = 0; i < N; ++i) {
        const int s = (int)(i / S.L3), cell = (int)(i % S.L3);
        const int x = cell % S.L, y = (cell / S.L) % S.L, z = cell / (S.L * S.L);
        int p4[3];
        pos4(s, p4);
        const double ang = -(qx * (x + p4[0] / 4.0) + qy * (y + p4[1] / 4.0) + qz * (z + p4[2] / 4.0));
        const double c = std::cos(ang), sn = std::sin(ang);
        const size_t j = 4 * (S.spin_off + (size_t)r * N + (size_t)i);
        for (int a = 0; a < 3; ++a) {
          const double v = o.fp64 ? o.s64[j + a] : (double)o.s32[j + a];
          re[a] += v * c;
          im[a] += v * sn;
        }
      }
      for (int a = 0; a < 3; ++a) acc += re[a] * re[a] + im[a] * im[a];
    }
    out[q] = acc / ((double)N * (r1 - r0));
  }
}

// Geometry export: out[k*4 + {0,1,2,3}] = dx, dy, dz, t for k < 30.
void orc_neighbours(int s, int* out) {
  static const auto nb = build_geometry();
  for (int k = 0; k < 30; ++k) {
    out[4 * k] = nb[s][k].dx;
    out[4 * k + 1] = nb[s][k].dy;
    out[4 * k + 2] = nb[s][k].dz;
    out[4 * k + 3] = nb[s][k].t;
  }
}

// Elementary functions of the update contract, for tests on the host.
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  pyro_philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1], out);
}
float orc_expf(float x) { return pyro_expf(x); }
float orc_logf(float x) { return pyro_logf(x); }
void orc_sincospif(float a, float* s, float* c) { pyro_sincospif(a, s, c); }
double orc_exp64(double x) { return pyro_exp64(x); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Learned tetrahedron proposal (no counterpart in the reference): FP64 restatement of
// the network, its negative log-likelihood gradient and the tetrahedron features
// (the MH move itself is checked statistically, against the plain chain), with the
// engine's BF16 rounding points (inputs, weights, hidden activations and the
// backward activations are rounded to BF16 where the engine feeds them to
// the tensor cores; accumulation in FP64 here, FP32 there).
namespace {

const int kIn = 16, kH = 64, kOut = 16;
const int oW1 = 0, oB1 = oW1 + kIn * kH, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
          oB3 = oW3 + kH * kOut, kParams = oB3 + kOut;

bool g_bf16 = true;  // round where the engine rounds (tests may switch it off)

double bf16(double x) {
  if (!g_bf16) return x;
  float f = (float)x;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return f;  // inf / nan unchanged
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;  // round to nearest even
  u &= 0xffff0000u;
  memcpy(&f, &u, 4);
  return f;
}

// hard-swish x * clamp(x + 3, 0, 6) / 6 and its derivative
double hswish(double x) { return x * std::min(std::max(x + 3.0, 0.0), 6.0) / 6.0; }
double hswish_grad(double x) { return x <= -3.0 ? 0.0 : (x >= 3.0 ? 1.0 : x / 3.0 + 0.5); }

struct Fwd {
  double x[kIn], pre1[kH], h1[kH], pre2[kH], h2[kH], o[kOut];
};

void mlp_forward(const float* m, const float* feat, Fwd& f) {
  for (int i = 0; i < kIn; ++i) f.x[i] = bf16(feat[i]);
  for (int o = 0; o < kH; ++o) {
    double a = m[oB1 + o];
    for (int i = 0; i < kIn; ++i) a += f.x[i] * bf16(m[oW1 + i * kH + o]);
    f.pre1[o] = a;
    f.h1[o] = bf16(hswish(a));
  }
  for (int o = 0; o < kH; ++o) {
    double a = m[oB2 + o];
    for (int i = 0; i < kH; ++i) a += f.h1[i] * bf16(m[oW2 + i * kH + o]);
    f.pre2[o] = a;
    f.h2[o] = bf16(hswish(a));
  }
  for (int o = 0; o < kOut; ++o) {
    double a = m[oB3 + o];
    for (int i = 0; i < kH; ++i) a += f.h2[i] * bf16(m[oW3 + i * kOut + o]);
    f.o[o] = a;
  }
}

const double kZmin = -4.0, kZmax = 6.0;

// loss and d loss / d o for one sample (outputs o, target spins s[12]).
double nll(const double* o, const float* s, double* d) {
  double loss = 0.0;
  for (int k = 0; k < 4; ++k) {
    double n = std::sqrt(o[4 * k] * o[4 * k] + o[4 * k + 1] * o[4 * k + 1] + o[4 * k + 2] * o[4 * k + 2]);
    double mu[3] = {0, 0, 1};
    if (n > 1e-20) {
      mu[0] = o[4 * k] / n;
      mu[1] = o[4 * k + 1] / n;
      mu[2] = o[4 * k + 2] / n;
    } else {
      n = 1e-20;
    }
    const double lz = o[4 * k + 3];
    const double z = std::min(std::max(lz, kZmin), kZmax);
    const bool zin = lz > kZmin && lz < kZmax;
    const double kap = std::exp(z);
    const double m = mu[0] * s[3 * k] + mu[1] * s[3 * k + 1] + mu[2] * s[3 * k + 2];
    loss -= z - std::log(2.0 * M_PI) - std::log(-std::expm1(-2.0 * kap)) + kap * (m - 1.0);
    const double r = 2.0 * kap / std::expm1(2.0 * kap);
    d[4 * k + 3] = zin ? -(1.0 - r + kap * (m - 1.0)) : 0.0;
    for (int a = 0; a < 3; ++a) d[4 * k + a] = -kap * (s[3 * k + a] - m * mu[a]) / n;
  }
  return loss;
}

}  // namespace

extern "C" {

int orc_mlp_param_count() { return kParams; }
void orc_mlp_set_bf16(int on) { g_bf16 = on != 0; }

void orc_mlp_forward(const float* master, const float* feats, int n, double* out) {
#pragma omp parallel for schedule(static)
  for (int r = 0; r < n; ++r) {
    Fwd f;
    mlp_forward(master, feats + 16 * r, f);
    for (int o = 0; o < kOut; ++o) out[16 * r + o] = f.o[o];
  }
}

// Sum over samples of d NLL / d params (same layout as the weights) and the
// loss sum, with the engine's BF16 rounding points.
void orc_mlp_gradient(const float* master, const float* feats, const float* targets, int n,
                      double* grad, double* loss_sum) {
  std::vector<double> G(kParams, 0.0);
  double L = 0.0;
  for (int r = 0; r < n; ++r) {
    Fwd f;
    mlp_forward(master, feats + 16 * r, f);
    double d[kOut];
    L += nll(f.o, targets + 12 * r, d);
    double db[kOut];
    for (int o = 0; o < kOut; ++o) {
      G[oB3 + o] += d[o];
      db[o] = bf16(d[o]);
    }
    double da2[kH], da2b[kH];
    for (int i = 0; i < kH; ++i) {
      double a = 0.0;
      for (int o = 0; o < kOut; ++o) a += db[o] * bf16(master[oW3 + i * kOut + o]);
      da2[i] = a * hswish_grad(f.pre2[i]);
      G[oB2 + i] += da2[i];
      da2b[i] = bf16(da2[i]);
    }
    double da1b[kH];
    for (int i = 0; i < kH; ++i) {
      double a = 0.0;
      for (int o = 0; o < kH; ++o) a += da2b[o] * bf16(master[oW2 + i * kH + o]);
      const double v = a * hswish_grad(f.pre1[i]);
      G[oB1 + i] += v;
      da1b[i] = bf16(v);
    }
    for (int i = 0; i < kIn; ++i)
      for (int o = 0; o < kH; ++o) G[oW1 + i * kH + o] += f.x[i] * da1b[o];
    for (int i = 0; i < kH; ++i)
      for (int o = 0; o < kH; ++o) G[oW2 + i * kH + o] += f.h1[i] * da2b[o];
    for (int i = 0; i < kH; ++i)
      for (int o = 0; o < kOut; ++o) G[oW3 + i * kOut + o] += f.h2[i] * db[o];
  }
  memcpy(grad, G.data(), sizeof(double) * kParams);
  *loss_sum = L;
}

// Features of every up-tetrahedron of corner f of replica r (rows = cells):
// h_k / 3 (k = 0..3), log(beta) / 3, three zeros; and its four spins.
void orc_tet_features(void* p, int si, int r, int f, float* feats, float* spins) {
  Oracle& o = *(Oracle*)p;
  const Sys& S = o.sys[si];
  const size_t base = S.spin_off + (size_t)r * 16 * S.L3;
  const int t = o.temp_of_rep[S.temp_base + S.off + r];
  const double beta = 1.0 / S.T[t];
  for (int cell = 0; cell < S.L3; ++cell) {
    const int x = cell % S.L, y = (cell / S.L) % S.L, z = cell / (S.L * S.L);
    for (int k = 0; k < 4; ++k) {
      const int s = 4 * f + k;
      double h[3] = {0, 0, 0};
      for (int q = 0; q < 6; ++q) {
        const Nbr& e = o.nb[s][q];
        const bool up = e.dx == 0 && e.dy == 0 && e.dz == 0 && e.t / 4 == f;
        if (up) continue;
        const size_t j = base + nbr_index(S, e, x, y, z);
        for (int a = 0; a < 3; ++a) h[a] += o.fp64 ? o.s64[4 * j + a] : o.s32[4 * j + a];
      }
      for (int a = 0; a < 3; ++a) feats[16 * cell + 3 * k + a] = (float)(S.J[0] * h[a] / 3.0);
      const size_t own = base + (size_t)s * S.L3 + cell;
      for (int a = 0; a < 3; ++a)
        spins[12 * cell + 3 * k + a] = o.fp64 ? (float)o.s64[4 * own + a] : o.s32[4 * own + a];
    }
    feats[16 * cell + 12] = (float)(std::log(beta) / 3.0);
    feats[16 * cell + 13] = feats[16 * cell + 14] = feats[16 * cell + 15] = 0.0f;
  }
}


}  // extern "C"

// ---------------------------------------------------------------------------
// FP64 restatement of one learned tetrahedron move (the engine's tet_finish
// in cudacode_b200/csrc/tet_mlp.cu), checked against the engine's trace
// records (pyro_tet_trace_pass). From the record's spins s, fields h,
// network outputs o and proposal s', and the move's Philox words (recomputed
// here from seed, tetrahedron, replica key and counter):
//   * the vMF draws of sites 0-2 (mu = o_xyz / |o_xyz|, kappa = e^clamp(o_w))
//     and of site 3 (the network's fourth vMF, or its exact conditional
//     given the recorded s'_0..s'_2: natural parameter
//     -beta (J1 (s'_0 + s'_1 + s'_2) + h_3)) by Wood's (1994) inverse CDF,
//     w = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa, azimuth 2 pi v, in the
//     orthonormal frame of Duff et al. (2017);
//   * log q(S | S') - log q(S' | S): the network sites' kappa mu.(s - s'),
//     plus for the conditional site the difference of the two vMF log
//     densities with their normalisations log(2 sinh k / k);
//   * dE = E(S') - E(S) with E = J1 sum_{i<j} s_i.s_j + sum_k h_k.s_k;
//   * log r = -beta dE + log q ratio and the decision u < min(1, e^log r).
// The uniforms are formed from the Philox bits exactly as the engine forms
// them (23-bit mantissa fill); everything else is FP64 with libm.
namespace {

double tet_u(uint32_t r) {
  const uint32_t b = 0x3f800000u | (r >> 9);
  float f;
  memcpy(&f, &b, 4);
  return 2.0 - (double)f;
}

double tet_test_u(const uint32_t r[4]) {
  const uint32_t m = ((r[0] & 0x1ffu) << 14) | ((r[1] & 0x1ffu) << 5) | (r[2] & 0x1fu);
  const uint32_t b = 0x3f800000u | m;
  float f;
  memcpy(&f, &b, 4);
  return 2.0 - (double)f;
}

struct V3 {
  double x, y, z;
};
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

V3 vmf_draw64(V3 mu, double kappa, double u, double v) {
  double w = 1.0 + std::log(u + (1.0 - u) * std::exp(-2.0 * kappa)) / kappa;
  w = std::min(1.0, std::max(-1.0, w));
  const double st = std::sqrt(std::max(0.0, 1.0 - w * w));
  const double cp = std::cos(2.0 * M_PI * v), sp = std::sin(2.0 * M_PI * v);
  const double sgn = std::copysign(1.0, mu.z);
  const double a = -1.0 / (sgn + mu.z);
  const double b = mu.x * mu.y * a;
  const V3 e1 = {1.0 + sgn * mu.x * mu.x * a, sgn * b, -sgn * mu.x};
  const V3 e2 = {b, sgn + mu.y * mu.y * a, -mu.y};
  return {w * mu.x + st * (cp * e1.x + sp * e2.x), w * mu.y + st * (cp * e1.y + sp * e2.y),
          w * mu.z + st * (cp * e1.z + sp * e2.z)};
}

// log(2 sinh k / k): the vMF normaliser up to the constant log(2 pi).
double vmf_lognorm64(double k) { return k - std::log(k) + std::log1p(-std::exp(-2.0 * k)); }

void net_vmf(const float* o, V3* mu, double* kappa) {
  const double x = o[0], y = o[1], z = o[2];
  const double n2 = x * x + y * y + z * z;
  if (n2 > 1e-30) {
    const double n = std::sqrt(n2);
    *mu = {x / n, y / n, z / n};
  } else {
    *mu = {0.0, 0.0, 1.0};
  }
  *kappa = std::exp(std::min(std::max((double)o[3], -4.0), 6.0));
}

// Site 3's conditional given sites 0-2 (a0..a2) and its field h3.
void closure64(V3 a0, V3 a1, V3 a2, V3 h3, double beta, double J1, V3* mu, double* kappa) {
  const V3 f = {-beta * (J1 * (a0.x + a1.x + a2.x) + h3.x), -beta * (J1 * (a0.y + a1.y + a2.y) + h3.y),
                -beta * (J1 * (a0.z + a1.z + a2.z) + h3.z)};
  const double n2 = dot(f, f);
  double k = 0.0;
  if (n2 > 1e-30) {
    k = std::sqrt(n2);
    *mu = {f.x / k, f.y / k, f.z / k};
  } else {
    *mu = {0.0, 0.0, 1.0};
  }
  *kappa = std::max(k, (double)0.018315639f);  // the engine's floor, e^-4 in FP32
}

double tet_e64(const V3 s[4], const V3 h[4], double J1) {
  double b = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = i + 1; j < 4; ++j) b += dot(s[i], s[j]);
  double e = J1 * b;
  for (int k = 0; k < 4; ++k) e += dot(s[k], h[k]);
  return e;
}

}  // namespace

extern "C" {

// rec: n trace records of 56 floats; rep_key[i], cell[i]: the replica's
// Philox key and the cell of record i. out: n x 17 doubles per record:
// log r, test uniform, decision, log q ratio, dE, the FP64 draws (12).
void orc_tet_move_check(const float* rec, int n, const int* rep_key, const int* cell, int corner,
                        int L3, uint64_t seed, uint64_t sweep, double J1, int closure,
                        double* out) {
  const uint32_t seed_lo = (uint32_t)(seed & 0xffffffffu), seed_hi = (uint32_t)(seed >> 32);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const float* t = rec + (size_t)i * 56;
    V3 s[4], h[4], sn[4];
    for (int k = 0; k < 4; ++k) {
      s[k] = {t[3 * k], t[3 * k + 1], t[3 * k + 2]};
      h[k] = {t[12 + 3 * k], t[12 + 3 * k + 1], t[12 + 3 * k + 2]};
      sn[k] = {t[40 + 3 * k], t[40 + 3 * k + 1], t[40 + 3 * k + 2]};
    }
    const double beta = t[55];
    const uint32_t key_tet = (uint32_t)(corner * L3 + cell[i]);
    uint32_t r0[4], r1[4];
    pyro_philox(key_tet, (uint32_t)rep_key[i], (uint32_t)sweep, PYRO_PURPOSE_TET + 0, seed_lo,
                seed_hi, r0);
    pyro_philox(key_tet, (uint32_t)rep_key[i], (uint32_t)sweep, PYRO_PURPOSE_TET + 1, seed_lo,
                seed_hi, r1);
    const uint32_t ru[4] = {r0[0], r0[2], r1[0], r1[2]}, rv[4] = {r0[1], r0[3], r1[1], r1[3]};
    double* o = out + (size_t)i * 17;
    double log_q = 0.0;
    for (int k = 0; k < 3 + (closure ? 0 : 1); ++k) {
      V3 mu;
      double kap;
      net_vmf(t + 24 + 4 * k, &mu, &kap);
      const V3 d = vmf_draw64(mu, kap, tet_u(ru[k]), tet_u(rv[k]));
      o[5 + 3 * k] = d.x;
      o[5 + 3 * k + 1] = d.y;
      o[5 + 3 * k + 2] = d.z;
      log_q += kap * (dot(mu, s[k]) - dot(mu, sn[k]));
    }
    if (closure) {
      V3 mo, mn;
      double ko, kn;
      closure64(s[0], s[1], s[2], h[3], beta, J1, &mo, &ko);
      closure64(sn[0], sn[1], sn[2], h[3], beta, J1, &mn, &kn);
      const V3 d = vmf_draw64(mn, kn, tet_u(ru[3]), tet_u(rv[3]));
      o[14] = d.x;
      o[15] = d.y;
      o[16] = d.z;
      log_q += (ko * dot(mo, s[3]) - vmf_lognorm64(ko)) - (kn * dot(mn, sn[3]) - vmf_lognorm64(kn));
    }
    const double dE = tet_e64(sn, h, J1) - tet_e64(s, h, J1);
    const double log_r = -beta * dE + log_q;
    const double u = tet_test_u(r0);
    o[0] = log_r;
    o[1] = u;
    o[2] = (log_r >= 0.0 || u < std::exp(log_r)) ? 1.0 : 0.0;
    o[3] = log_q;
    o[4] = dE;
  }
}

}  // extern "C"
