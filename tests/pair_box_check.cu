// Randomised check of pair_boxes_apart, the test with which a warp of the
// derivative forms' all-pairs searches skips a staged tile of candidates:
// whenever it reports the warp's box and the tile's box apart, no pair
// between them may pass the neighbour test r2 < (R h_i)^2 or r2 < (R h_j)^2
// on the minimum-image displacement.  Host code only; built and run by
// tests/test_pair_box_skip.py.
#include <cstdio>
#include <random>

#include "mhd_common.cuh"

using mhd::PairBox;

static double min_image_host(double d, double L, int periodic) {
  if (periodic) {
    if (d > 0.5 * L) d -= L;
    if (d < -0.5 * L) d += L;
  }
  return d;
}

template <int DIM>
static int check(std::mt19937_64& g, int trials, long& apart, long& pairs_checked) {
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const int NW = 32, NT = 128;
  double xw[NW][3], hw[NW], xt[NT][3], ht[NT];
  for (int trial = 0; trial < trials; trial++) {
    double L[3];
    int per[3];
    for (int a = 0; a < 3; a++) {
      L[a] = 0.5 + 2.0 * U(g);
      per[a] = U(g) < 0.7;
    }
    const double R = U(g) < 0.5 ? 2.0 : 3.0;
    const double hb = 0.005 + 0.05 * U(g);
    const double spread = hb * (1.0 + 8.0 * U(g));
    double cw[3], ct[3];
    const bool near = U(g) < 0.5;
    for (int a = 0; a < 3; a++) {
      // centres a little outside the box too (positions between wraps)
      cw[a] = (1.2 * U(g) - 0.1) * L[a];
      ct[a] = (1.2 * U(g) - 0.1) * L[a];
      if (near) {
        // half the trials close to the reach, some across the periodic seam
        ct[a] = cw[a] + 2.0 * (U(g) - 0.5) * (spread + 2.0 * R * hb);
        if (per[a] && U(g) < 0.3) ct[a] += U(g) < 0.5 ? L[a] : -L[a];
      }
    }
    PairBox w{}, t{};
    for (int a = 0; a < 3; a++) {
      w.lo[a] = t.lo[a] = 1e300;
      w.hi[a] = t.hi[a] = -1e300;
    }
    w.h = t.h = 0.0;
    for (int k = 0; k < NW; k++) {
      for (int a = 0; a < 3; a++) {
        xw[k][a] = a < DIM ? cw[a] + spread * (U(g) - 0.5) : 0.0;
        w.lo[a] = xw[k][a] < w.lo[a] ? xw[k][a] : w.lo[a];
        w.hi[a] = xw[k][a] > w.hi[a] ? xw[k][a] : w.hi[a];
      }
      hw[k] = hb * (0.5 + U(g));
      w.h = hw[k] > w.h ? hw[k] : w.h;
    }
    for (int k = 0; k < NT; k++) {
      for (int a = 0; a < 3; a++) {
        xt[k][a] = a < DIM ? ct[a] + spread * (U(g) - 0.5) : 0.0;
        t.lo[a] = xt[k][a] < t.lo[a] ? xt[k][a] : t.lo[a];
        t.hi[a] = xt[k][a] > t.hi[a] ? xt[k][a] : t.hi[a];
      }
      ht[k] = hb * (0.5 + U(g));
      t.h = ht[k] > t.h ? ht[k] : t.h;
    }
    if (!mhd::pair_boxes_apart<DIM>(w, t, R, L, per)) continue;
    apart++;
    for (int i = 0; i < NW; i++)
      for (int j = 0; j < NT; j++) {
        double r2 = 0.0;
        for (int a = 0; a < DIM; a++) {
          const double d = min_image_host(xw[i][a] - xt[j][a], L[a], per[a]);
          r2 += d * d;
        }
        pairs_checked++;
        const double ri = R * hw[i], rj = R * ht[j];
        if (r2 < ri * ri || r2 < rj * rj) {
          std::printf("FAIL dim %d trial %d pair (%d, %d): r2 %.17g reach %.17g\n", DIM, trial, i, j, r2,
                      ri > rj ? ri : rj);
          return 1;
        }
      }
  }
  return 0;
}

int main() {
  std::mt19937_64 g(12345);
  long apart = 0, pairs = 0;
  const int trials = 20000;
  if (check<2>(g, trials, apart, pairs) || check<3>(g, trials, apart, pairs)) return 1;
  std::printf("ok trials %d apart %ld pairs %ld\n", 2 * trials, apart, pairs);
  return 0;
}
