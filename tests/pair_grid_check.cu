// Randomised check of the derivative forms' neighbour search
// (pair_grid_plan, pair_grid_key and pair_grid_visit of mhd_pairgrid.cuh):
// for random particle sets -- 2-D and 3-D, periodic and open axes, boxes
// from a few reaches wide to many, smoothing lengths spread over a factor of
// several with a few large ones -- the pairs the grid walk reports for each
// particle, over all slices, are exactly those of a brute-force test of
// every pair with the same rule (r2 < (R h_i)^2 or r2 < (R h_j)^2 on the
// minimum-image displacement), each once.  Host code only; built and run by
// tests/test_pair_grid.py.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "mhd_pairgrid.cuh"

using mhd::DevParams;
using mhd::PairGrid;

template <int DIM>
static bool check(std::mt19937_64& g, int trials, long& pairs, long& cells_max) {
  std::uniform_real_distribution<double> U(0.0, 1.0);
  for (int trial = 0; trial < trials; trial++) {
    DevParams P{};
    P.dim = DIM;
    P.R = U(g) < 0.5 ? 2.0 : 3.0;
    for (int a = 0; a < 3; a++) {
      P.periodic[a] = a < DIM && U(g) < 0.7;
      P.lo[a] = -0.5 + 0.3 * (U(g) - 0.5);
      P.L[a] = a < DIM ? 0.3 + 1.7 * U(g) : 1.0;
      P.hi[a] = P.lo[a] + P.L[a];
      P.half[a] = 0.5 * P.L[a];
    }
    const int n = 20 + (int)(U(g) * (DIM == 3 ? 1500 : 900));
    const double hb = (DIM == 3 ? 0.03 : 0.02) * (0.3 + U(g));
    std::vector<double> x(n), y(n), z(n), h(n);
    for (int i = 0; i < n; i++) {
      // periodic axes: inside the box (the integrator wraps); open axes:
      // anywhere around it
      x[i] = P.lo[0] + P.L[0] * (P.periodic[0] ? U(g) : 1.4 * U(g) - 0.2);
      y[i] = P.lo[1] + P.L[1] * (P.periodic[1] ? U(g) : 1.4 * U(g) - 0.2);
      z[i] = DIM == 3 ? P.lo[2] + P.L[2] * (P.periodic[2] ? U(g) : 1.4 * U(g) - 0.2) : 0.0;
      h[i] = hb * (0.5 + 2.0 * U(g)) * (U(g) < 0.02 ? 3.0 : 1.0);
    }
    double lo[3], hi[3], hmax = 0.0;
    for (int a = 0; a < 3; a++) {
      lo[a] = 1e300;
      hi[a] = -1e300;
    }
    for (int i = 0; i < n; i++) {
      const double v[3] = {x[i], y[i], z[i]};
      for (int a = 0; a < 3; a++) {
        lo[a] = std::min(lo[a], v[a]);
        hi[a] = std::max(hi[a], v[a]);
      }
      hmax = std::max(hmax, h[i]);
    }
    const int cap = std::max(n, 64);
    const PairGrid G = mhd::pair_grid_plan(P, hmax, lo, hi, cap);
    const long ncells = (long)G.nc[0] * G.nc[1] * G.nc[2];
    if (ncells > cap) {
      std::printf("FAIL plan: %ld cells > cap %d\n", ncells, cap);
      return false;
    }
    cells_max = std::max(cells_max, ncells);
    std::vector<int> key(n), perm(n), cell_start(ncells + 1);
    for (int i = 0; i < n; i++) key[i] = mhd::pair_grid_key(G, x[i], y[i], z[i]);
    for (int i = 0; i < n; i++) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
    for (long c = 0, t = 0; c <= ncells; c++) {
      while (t < n && key[perm[t]] < c) t++;
      cell_start[c] = (int)t;
    }
    std::vector<double4> pos(n);
    for (int i = 0; i < n; i++) pos[i] = make_double4(x[i], y[i], z[i], h[i]);
    const int slices = 1 + (int)(U(g) * 4);
    for (int i = 0; i < n; i++) {
      std::vector<int> got;
      for (int sl = 0; sl < slices; sl++)
        mhd::pair_grid_visit<DIM>(G, cell_start.data(), perm.data(), pos.data(), P, i, sl, slices,
                                  [&](int j, double, double, double) { got.push_back(j); });
      std::vector<int> want;
      const double rhi2 = mhd::rh2_exact(P.R, h[i]);
      for (int j = 0; j < n; j++) {
        const double dx = mhd::min_image(x[i] - x[j], P.L[0], P.half[0], P.periodic[0]);
        const double dy = mhd::min_image(y[i] - y[j], P.L[1], P.half[1], P.periodic[1]);
        const double dz = DIM == 3 ? mhd::min_image(z[i] - z[j], P.L[2], P.half[2], P.periodic[2]) : 0.0;
        const double r2 = mhd::r2_exact(dx, dy, dz);
        if (r2 < rhi2 || r2 < mhd::rh2_exact(P.R, h[j])) want.push_back(j);
      }
      std::sort(got.begin(), got.end());
      if (got != want) {
        std::printf("FAIL dim %d trial %d particle %d: grid %zu pairs, brute force %zu (nc %d %d %d)\n", DIM,
                    trial, i, got.size(), want.size(), G.nc[0], G.nc[1], G.nc[2]);
        return false;
      }
      pairs += (long)want.size();
    }
  }
  return true;
}

int main() {
  std::mt19937_64 g(12345);
  long pairs = 0, cells_max = 0;
  if (!check<2>(g, 120, pairs, cells_max) || !check<3>(g, 60, pairs, cells_max)) return 1;
  std::printf("ok pairs %ld cells_max %ld\n", pairs, cells_max);
  return 0;
}
