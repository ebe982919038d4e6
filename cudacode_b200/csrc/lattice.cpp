// Neighbour table of the 16-site cubic cell, generated from the site
// positions by distance shell (see lattice.h for the conventions).
#include "lattice.h"

#include <algorithm>
#include <array>
#include <vector>

namespace pyro {

bool build_neighbour_table(NbrTable* tab) {
  for (int s = 0; s < kSitesPerCell; ++s) {
    int ps[3];
    site_pos4(s, ps);
    struct Cand {
      int shell, t, dx, dy, dz;
    };
    std::vector<Cand> c;
    std::vector<std::array<int, 3>> nn_vec;  // J1 bond vectors of s (units a/4)
    for (int pass = 0; pass < 2; ++pass) {
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz)
            for (int t = 0; t < kSitesPerCell; ++t) {
              int pt[3];
              site_pos4(t, pt);
              const int v[3] = {4 * dx + pt[0] - ps[0], 4 * dy + pt[1] - ps[1],
                                4 * dz + pt[2] - ps[2]};
              const int r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
              if (pass == 0) {
                if (r2 == 2) nn_vec.push_back({v[0], v[1], v[2]});
                continue;
              }
              int shell = -1;
              if (r2 == 2) shell = 0;
              else if (r2 == 6) shell = 1;
              else if (r2 == 8) {
                shell = 3;
                for (const auto& w : nn_vec)
                  if (v[0] == 2 * w[0] && v[1] == 2 * w[1] && v[2] == 2 * w[2]) shell = 2;
              }
              if (shell >= 0) c.push_back({shell, t, dx, dy, dz});
            }
    }
    std::sort(c.begin(), c.end(), [](const Cand& a, const Cand& b) {
      if (a.shell != b.shell) return a.shell < b.shell;
      if (a.t != b.t) return a.t < b.t;
      if (a.dx != b.dx) return a.dx < b.dx;
      if (a.dy != b.dy) return a.dy < b.dy;
      return a.dz < b.dz;
    });
    if ((int)c.size() != kMaxNbr) return false;
    for (int k = 0; k < kMaxNbr; ++k) {
      const int sh = c[k].shell;
      if (k < kShellBegin[sh] || k >= kShellBegin[sh + 1]) return false;
      tab->e[s][k] = NbrEntry{(int8_t)c[k].dx, (int8_t)c[k].dy, (int8_t)c[k].dz, (int8_t)c[k].t};
    }
  }
  return true;
}

}  // namespace pyro
