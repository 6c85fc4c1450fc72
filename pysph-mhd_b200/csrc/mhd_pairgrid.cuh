// mhd_pairgrid.cuh -- the neighbour search of the derivative forms.
//
// The forward-mode and adjoint passes keep the caller's particle order (the
// tape and the checkpoints are indexed by it), so they do not sort the
// particles as the production path does.  Before each pair pass they build
// a uniform cell grid over the pass's positions and smoothing lengths --
// cells at least R h_max wide, so every pair of the symmetric rule
// r < R max(h_i, h_j) (PySPH's, src/application.py:63-78) lies within the
// 3^dim cells around either particle -- by a stable sort of the cell keys
// (the particle indices of a cell in ascending order), and walk it with an
// indirection through the sort's permutation.
#pragma once

#include "mhd_common.cuh"

namespace mhd {

struct Ctx;

// The grid of one pass (device memory).  An axis of fewer than three cells
// is scanned whole.
struct PairGrid {
  int nc[3];
  int whole[3];
  double lo[3];
  double inv_cs[3];
};

// Reduction targets of a build: order-mapped doubles.
struct PairGridRed {
  unsigned long long h_max;
  unsigned long long lo[3], hi[3];
};

// Device state of the derivative forms' search, kept in the context.
struct PairGridBufs {
  double4* pos = nullptr;         // {x, y, z, h} of the pass, caller order
  PairGrid* grid = nullptr;
  PairGridRed* red = nullptr;
  int* cell_start = nullptr;      // cap + 1 entries
  const int* perm = nullptr;      // sorted slot -> particle (the context's sort buffers)
  int cap = 0;                    // cells at most
};

__host__ __device__ __forceinline__ int pair_grid_coord(const PairGrid& g, int a, double v) {
  int c = (int)floor((v - g.lo[a]) * g.inv_cs[a]);
  return c < 0 ? 0 : (c >= g.nc[a] ? g.nc[a] - 1 : c);
}

// The plan: cells at least R h_max (1 + 1e-6) wide along each coordinate
// axis -- the periodic box on periodic axes, the particles' bounding box
// [lo, hi] otherwise -- at most `cap` cells in all (coarser cells stay
// valid).  The 1e-6 absorbs the rounding of the cell coordinates.
__host__ __device__ inline PairGrid pair_grid_plan(const DevParams& P, double h_max, const double* lo_b,
                                                   const double* hi_b, int cap) {
  const double cut = P.R * h_max * (1.0 + 1e-6);
  PairGrid G;
  double ext[3];
  for (int a = 0; a < 3; a++) {
    if (a >= P.dim) {
      G.nc[a] = 1;
      G.lo[a] = 0.0;
      ext[a] = 1.0;
      continue;
    }
    double lo, e;
    if (P.periodic[a]) {
      lo = P.lo[a];
      e = P.L[a];
    } else {
      lo = lo_b[a];
      e = (hi_b[a] - lo) * (1.0 + 1e-12) + 1e-300;
    }
    double nc = cut > 0.0 && isfinite(cut) && isfinite(e) ? floor(e / cut) : 1.0;
    nc = nc < 1.0 ? 1.0 : (nc > 65536.0 ? 65536.0 : nc);
    G.nc[a] = (int)nc;
    G.lo[a] = isfinite(lo) ? lo : 0.0;
    ext[a] = isfinite(e) && e > 0.0 ? e : 1.0;
  }
  while ((long long)G.nc[0] * G.nc[1] * G.nc[2] > cap) {
    int a = 0;
    for (int b = 1; b < 3; b++)
      if (G.nc[b] > G.nc[a]) a = b;
    const int shrunk = (int)(G.nc[a] * 0.8);
    G.nc[a] = shrunk > 1 ? shrunk : 1;
  }
  for (int a = 0; a < 3; a++) {
    G.inv_cs[a] = a < P.dim ? (double)G.nc[a] / ext[a] : 0.0;
    G.whole[a] = G.nc[a] < 3;
  }
  return G;
}

__host__ __device__ __forceinline__ int pair_grid_key(const PairGrid& g, double x, double y, double z) {
  return (pair_grid_coord(g, 2, z) * g.nc[1] + pair_grid_coord(g, 1, y)) * g.nc[0] + pair_grid_coord(g, 0, x);
}

// f(j, dx, dy, dz) for every j (i itself included) with r^2 < (R h_i)^2 or
// r^2 < (R h_j)^2 on the minimum-image FP64 displacement x_i - x_j, among
// the candidates whose sorted slot t has t % slices == slice (the passes
// split their pairs over `slices` partial sums added in slice order; a
// slice steps through its own slots only).  Order: the stencil's rows (z,
// then y), x ascending within a row, particle index ascending within a
// cell -- deterministic.
template <int DIM, class F>
__host__ __device__ inline void pair_grid_visit(const PairGrid& g, const int* __restrict__ cell_start,
                                       const int* __restrict__ perm, const double4* __restrict__ pos,
                                       const DevParams& P, int i, int slice, int slices, F&& f) {
  const double4 pi = pos[i];
  const double rhi2 = rh2_exact(P.R, pi.w);
  const int c[3] = {pair_grid_coord(g, 0, pi.x), pair_grid_coord(g, 1, pi.y),
                    DIM == 3 ? pair_grid_coord(g, 2, pi.z) : 0};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    lo[a] = g.whole[a] ? 0 : c[a] - 1;
    hi[a] = g.whole[a] ? g.nc[a] - 1 : c[a] + 1;
  }
  const int nx = g.nc[0], ny = g.nc[1], nz = g.nc[2];
  auto row = [&](int base, int xl, int xh) {
    // cells xl..xh of one row, contiguous in the sorted order
    const int ts = cell_start[base + xl], te = cell_start[base + xh + 1];
    for (int t = ts + ((slice - ts % slices) + slices) % slices; t < te; t += slices) {
      const int j = perm[t];
      const double4 q = pos[j];
      const double dx = min_image(pi.x - q.x, P.L[0], P.half[0], P.periodic[0]);
      const double dy = min_image(pi.y - q.y, P.L[1], P.half[1], P.periodic[1]);
      const double dz = DIM == 3 ? min_image(pi.z - q.z, P.L[2], P.half[2], P.periodic[2]) : 0.0;
      const double r2 = r2_exact(dx, dy, dz);
      if (r2 < rhi2 || r2 < rh2_exact(P.R, q.w)) f(j, dx, dy, dz);
    }
  };
  for (int zu = lo[2]; zu <= hi[2]; zu++) {
    int zc = zu;
    if (zc < 0 || zc >= nz) {
      if (!P.periodic[2]) continue;
      zc = zc < 0 ? zc + nz : zc - nz;
    }
    for (int yu = lo[1]; yu <= hi[1]; yu++) {
      int yc = yu;
      if (yc < 0 || yc >= ny) {
        if (!P.periodic[1]) continue;
        yc = yc < 0 ? yc + ny : yc - ny;
      }
      const int base = (zc * ny + yc) * nx;
      // x pieces: the part below 0 (wrapped), inside, above nx - 1 (wrapped)
      if (lo[0] < 0 && P.periodic[0]) row(base, lo[0] + nx, nx - 1);
      row(base, lo[0] < 0 ? 0 : lo[0], hi[0] >= nx ? nx - 1 : hi[0]);
      if (hi[0] >= nx && P.periodic[0]) row(base, 0, hi[0] - nx);
    }
  }
}

// Partial-sum slices of the derivative forms' pair passes: a small case is
// spread over 8 slices (grid y) so that it fills the GPU, a large one has
// enough particles for one.
inline int derivative_slices(int64_t n) { return n <= 65536 ? 8 : 1; }
// The largest slices(n) x n over n <= n_max: the particle records a
// partial-sum buffer needs per summed quantity.
inline size_t derivative_slice_records(int64_t n_max) {
  const int64_t small = n_max < 65536 ? n_max : 65536;
  return (size_t)(8 * small > n_max ? 8 * small : n_max);
}

// Builds bufs.grid and the cell table over bufs.pos[0, n) (after the
// caller filled bufs.pos); leaves bufs.perm.  Stream-ordered, no host
// synchronisation.
void build_pair_grid(Ctx* c, PairGridBufs& bufs, int n, cudaStream_t st);
// Allocates the buffers for up to n_max particles (set-up, not captured).
int alloc_pair_grid(PairGridBufs& bufs, int64_t n_max);
void free_pair_grid(PairGridBufs& bufs);

}  // namespace mhd
