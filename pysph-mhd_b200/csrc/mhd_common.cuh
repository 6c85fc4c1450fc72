// mhd_common.cuh -- device-side parameters, SPH kernels and neighbour-grid
// helpers shared by the sm_100a kernels of the SPMHD particle update.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "mhd_b200.h"

namespace mhd {

constexpr double kDensityTolerance = 1.0e-4;            // src/equations.py:6
constexpr double kCourantFactor = 0.3;                  // src/equations.py:7
constexpr double kForceFactor = 0.25;                   // src/equations.py:8
constexpr double kPairDistanceEpsilon = 1.0e-12;        // src/equations.py:9
constexpr double kInteractionDistanceEpsilon = 1.0e-8;  // src/equations.py:10
constexpr double kFloatTiny = 2.2250738585072014e-308;  // src/equations.py:11
constexpr double kMachineEps = 2.220446049250313e-16;   // src/equations.py:67
constexpr double kBigNumber = 1.0e29;                   // src/equations.py:574

// One instance's uniform cell grid and periodic box (a batch holds one per
// instance, indexed by the particle's instance; a single simulation is
// instance 0).  Cells along x are contiguous in the sorted particle order.
struct Grid {
  int nc[3];
  int ncells;
  int cell_base;  // first global cell key of the instance
  int sw;         // stencil half-width in cells: widths >= cut-off / sw
  int periodic[3];
  double lo[3];
  double inv_cs[3];
  double cs[3];
  double L[3];  // the instance's periodic box (lo .. lo + L on periodic axes)
  double half[3];
  double h_plan;  // largest h whose list cut-off the +-sw stencil covers
  double cut;     // search reach of a normal particle: R (1 + margin) h_plan (>= the planned cutoff)
  float csf[3];   // cell widths in FP32 (packed-position geometry)
  float h_bigf;   // particles with FP32 h above this are "big": they search an extended stencil
  // Fixed-point frame of the FP32 pair passes: a coordinate is stored as
  // u = (x - fx_lo) * fx_scale modulo 2^32 (uint32), so x_i - x_j is the
  // wrapped 32-bit difference times fx_len.  On a periodic axis the frame is
  // the box (2^32 units = L): the wrapped difference is the minimum image.
  // On an open axis it is four times the particles' extent, centred on them,
  // so no difference wraps.  Zero scale on axes beyond dim.
  double fx_lo[3];
  double fx_scale[3];
  float fx_len[3];
};

__device__ __forceinline__ const Grid& grid_of(const Grid* __restrict__ grids, const int* __restrict__ inst, int i) {
  return grids[inst ? inst[i] : 0];
}

// Compacted neighbour lists: entry k of particle i lives at
// idx[((i / 32) * cap + k) * 32 + i % 32], so the 32 lanes of a warp read
// entry k of their particles from one 128-byte line.  A list holds every j
// with r_ij < R * max(h_i, h_j) * (1 + margin) for the h it was built with;
// hlim[i] (slightly below h_i * (1 + margin)) is the largest h_i it stays
// valid for.
struct NbrList {
  const int* idx;
  const int* cnt;
  const double* hlim;
  int cap;
};

// Everything a kernel needs besides the grids, passed by value.
struct DevParams {
  int dim;
  int kernel;
  int iterate;
  int min_iter;
  int max_iter;
  int periodic[3];
  int fp32;  // pair arithmetic in FP32 (MHD_PRECISION_FP32)
  double L[3];
  double half[3];
  double lo[3];
  double hi[3];
  double R;  // kernel radius scale
  double hfact, gamma, gamma1, mu0, inv_mu0, av, ac, ar, clean_speed, clean_damp, clean_active;
  double c_cour, c_force, alpha_min, alpha_max, tf;
  double norm;  // kernel normalisation sigma_d
  // FP32 copies for the FP32 pair loops (kernel-parameter operands, no
  // conversion in the kernel)
  float Rf, normf, avf, acf, arf, inv_mu0f;
};

// Device-resident scalars of one context (status, pass counters, events).
struct DevScalars {
  int status;       // first device error, MHD_OK if none
  int relist;       // an h outgrew its neighbour list, or a list overflowed
  int list_max;     // longest neighbour list met by the last build
  int passes_done;  // density passes executed in the current group evaluation
  int loop_pass;    // captured runs: the pass the density loop's body runs next
  unsigned long long loop_iters;  // density-loop body iterations run (accumulating; each runs 2 kernels)
  unsigned int ticket;              // last-block counter of the dt reduction
  int events;                       // captured runs: bit 0 = density passes ran out before the group stopped
  int n_big;                        // big particles met by the last list build
  int n_app;                        // particles the last build's scatter pass appended entries to
  int n_reb;                        // particles whose lists the last build rebuilds (carried builds)
  unsigned long long n_pairs;       // force-pass neighbour pairs (accumulating)
  unsigned long long n_candidates;  // force-pass distance tests (accumulating)
  int n_unconverged[256 + 8];       // per density pass
  unsigned long long n_listed;      // particles whose lists were built or carried over (accumulating)
  unsigned long long n_rebuilt;     // of those, lists built afresh (accumulating)
};

// Device-resident scalars of one instance: its step clock and the
// reductions its grid is planned from (a single simulation uses entry 0).
struct InstScalars {
  double dt;       // step size in use (stage2 of the current step)
  double dt_next;  // next step size (min dt_adapt, clipped to tf)
  double t;        // time at the start of the current step
  double t_next;   // time at the start of the next step
  unsigned long long dt_min_bits;  // atomicMin target (order-mapped); reset to ~0 after use
  unsigned long long h_max_bits;   // order-mapped; reset to 0 after use
  unsigned long long lo_bits[3];   // bounding box, order-mapped; reset to ~0 / 0 after use
  unsigned long long hi_bits[3];
  unsigned long long h_sum;        // sum of h / h_max in 2^-32 units (exact, order-independent)
  int nc_cap[3];   // per-axis cell capacity (batched contexts)
  int cell_base;   // first global cell key of the instance
  int n;           // particles of the instance
  int pad;
};

// ------------------------------------------------------------ kernels (SPH)
// w(q) and dw/dq, unnormalised; forms and branch conditions follow PySPH's
// pysph.base.kernels (restated): cubic spline (Monaghan), quintic spline
// (Morris), Wendland C2/C4/C6, Gaussian, super-Gaussian.
template <int K, class T>
__device__ __forceinline__ void w_dw(T q, int dim, T& w, T& dw) {
  constexpr T c0 = 0, c1 = 1, c2 = 2, c3 = 3;
  if constexpr (K == MHD_KERNEL_CUBIC) {
    if (q > c2) {
      w = c0; dw = c0;
    } else if (q > c1) {
      const T t = c2 - q;
      w = (T)0.25 * t * t * t; dw = (T)-0.75 * t * t;
    } else {
      w = c1 - (T)1.5 * q * q * (c1 - (T)0.5 * q); dw = (T)-3.0 * q * (c1 - (T)0.75 * q);
    }
  } else if constexpr (K == MHD_KERNEL_QUINTIC) {
    if (q > c3) { w = c0; dw = c0; return; }
    const T t3 = c3 - q, t2 = c2 - q, t1 = c1 - q;
    const T t3s = t3 * t3, t2s = t2 * t2, t1s = t1 * t1;
    w = t3s * t3s * t3;
    dw = (T)-5.0 * t3s * t3s;
    if (q <= c2) {
      w -= (T)6.0 * t2s * t2s * t2;
      dw += (T)30.0 * t2s * t2s;
      if (q <= c1) {
        w += (T)15.0 * t1s * t1s * t1;
        dw -= (T)75.0 * t1s * t1s;
      }
    }
  } else if constexpr (K == MHD_KERNEL_WENDLAND_C2) {
    if (q >= c2) { w = c0; dw = c0; return; }
    const T s = c1 - (T)0.5 * q, s3 = s * s * s;
    w = s3 * s * (c2 * q + c1); dw = (T)-5.0 * q * s3;
  } else if constexpr (K == MHD_KERNEL_WENDLAND_C4) {
    if (q >= c2) { w = c0; dw = c0; return; }
    const T s = c1 - (T)0.5 * q, s2 = s * s, s5 = s2 * s2 * s;
    w = s5 * s * ((T)(35.0 / 12.0) * q * q + c3 * q + c1);
    dw = (T)(-14.0 / 3.0) * q * (c1 + (T)2.5 * q) * s5;
  } else if constexpr (K == MHD_KERNEL_WENDLAND_C6) {
    if (q >= c2) { w = c0; dw = c0; return; }
    const T s = c1 - (T)0.5 * q, s2 = s * s, s4 = s2 * s2, s7 = s4 * s2 * s;
    w = s7 * s * ((T)4.0 * q * q * q + (T)6.25 * q * q + (T)4.0 * q + c1);
    dw = (T)-5.5 * q * (c1 + (T)3.5 * q + (T)4.0 * q * q) * s7;
  } else if constexpr (K == MHD_KERNEL_GAUSSIAN) {
    if (q >= c3) { w = c0; dw = c0; return; }
    const T e = exp(-q * q);
    w = e; dw = -c2 * q * e;
  } else {
    if (q >= c3) { w = c0; dw = c0; return; }
    const T e = exp(-q * q), d2 = (T)0.5 * (T)dim;
    w = e * (d2 + c1 - q * q); dw = -c2 * q * e * (d2 + c2 - q * q);
  }
}

inline double radius_scale_of(int k) {
  return (k == MHD_KERNEL_QUINTIC || k == MHD_KERNEL_GAUSSIAN || k == MHD_KERNEL_SUPER_GAUSSIAN) ? 3.0 : 2.0;
}

double kernel_norm(int kernel, int dim);  // host, mhd_abi.cu

template <int DIM>
__device__ __forceinline__ double pow_dim(double a) {
  if constexpr (DIM == 2) return a * a;
  else return a * a * a;
}

// Minimum-image displacement along one periodic axis.
__host__ __device__ __forceinline__ double min_image(double d, double L, double half, int periodic) {
  if (periodic) {
    if (d > half) d = d - L;
    if (d < -half) d = d + L;
  }
  return d;
}

// Squared distance evaluated without FMA contraction, in the oracle's order
// ((dx*dx + dy*dy) + dz*dz), so neighbour sets are bit-identical to it.
// (Host code: compiled without contraction, as the oracle is.)
__host__ __device__ __forceinline__ double r2_exact(double dx, double dy, double dz) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
#else
  return (dx * dx + dy * dy) + dz * dz;
#endif
}

// (R*h)^2 without contraction.
__host__ __device__ __forceinline__ double rh2_exact(double R, double h) {
#ifdef __CUDA_ARCH__
  const double rh = __dmul_rn(R, h);
  return __dmul_rn(rh, rh);
#else
  const double rh = R * h;
  return rh * rh;
#endif
}

__device__ __forceinline__ unsigned long long dbl_order(double v) {
  // Monotone map of doubles to unsigned integers.
  unsigned long long b = __double_as_longlong(v);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ inline double dbl_unorder(unsigned long long b) {
  unsigned long long v = (b & 0x8000000000000000ULL) ? (b & 0x7fffffffffffffffULL) : ~b;
  double d;
  memcpy(&d, &v, sizeof d);
  return d;
}

// Products, quotients and sums rounded once each (no contraction), so the
// device planner reproduces the host planner bit for bit.
__host__ __device__ inline double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ inline double div_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
__host__ __device__ inline double add_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}

// What the grid plans of a context's instances share.
struct PlanSpec {
  int dim;
  int stencil;  // cells are >= cut-off / stencil wide
  int periodic[3];
  double lo[3];  // periodic box
  double L[3];
  double half[3];
  double R;
  double grid_margin;
  double list_margin;
  double cell_kappa;  // cells follow min(h_max, cell_kappa * h_mean)
};

// Uniform grid of one instance from its h_max, mean h and bounding box
// [lo, hi] (used on non-periodic axes).  The cells follow
// h_cell = min(h_max, cell_kappa * h_mean), not h_max, so that a few
// particles with a large h do not coarsen the grid for all: particles with h
// above h_plan (the largest h the +-stencil covers) are "big" and search an
// extended stencil of their own.  Cells are at least
// R * h_cell * grid_margin * (1 + list_margin) / stencil wide, at most
// 2047/2047/1023 (3-D) or 65535 (2-D) per axis (the packed cell-coordinate
// widths) and 2^24 in all, and at most nc_cap[a] per axis when nc_cap is
// given.  Fills everything but cell_base.  Returns MHD_OK or
// MHD_ERR_NONFINITE.
__host__ __device__ inline int plan_instance(const PlanSpec& S, int n, double hmax, double hmean,
                                             const double* lo_red, const double* hi_red, const int* nc_cap,
                                             Grid& g) {
  g = Grid{};
  if (n <= 0) hmax = hmean = 1.0;
  const double hk = mul_rn(S.cell_kappa, hmean);
  const double hcell = hk < hmax ? hk : hmax;
  const double cutoff = mul_rn(mul_rn(mul_rn(S.R, hcell), S.grid_margin), add_rn(1.0, S.list_margin));
  double extent[3];
  for (int a = 0; a < 3; a++) {
    g.periodic[a] = a < S.dim ? S.periodic[a] : 0;
    g.L[a] = S.L[a];
    g.half[a] = S.half[a];
    if (a >= S.dim) {
      g.nc[a] = 1;
      g.lo[a] = 0.0;
      extent[a] = 1.0;
      continue;
    }
    double lo, ext;
    if (S.periodic[a]) {
      lo = S.lo[a];
      ext = S.L[a];
    } else {
      lo = n > 0 ? lo_red[a] : 0.0;
      const double hi = n > 0 ? hi_red[a] : 1.0;
      ext = add_rn(mul_rn(add_rn(hi, -lo), 1.0 + 1e-12), 1e-300);
    }
    if (!isfinite(lo) || !isfinite(ext) || !isfinite(cutoff)) return MHD_ERR_NONFINITE;
    const double axis_max = S.dim == 3 ? (a == 2 ? 1023.0 : 2047.0) : 65535.0;
    const double ncd = floor(div_rn(mul_rn(ext, (double)S.stencil), cutoff));
    g.nc[a] = ncd < 1.0 ? 1 : (ncd > axis_max ? (int)axis_max : (int)ncd);
    g.lo[a] = lo;
    extent[a] = ext;
  }
  // Keep the table within 2^24 cells; coarser cells stay valid.
  const long long cap = 1LL << 24;
  while ((long long)g.nc[0] * g.nc[1] * g.nc[2] > cap) {
    int a = 0;
    for (int b = 1; b < 3; b++)
      if (g.nc[b] > g.nc[a]) a = b;
    const int shrunk = (int)mul_rn((double)g.nc[a], 0.8);
    g.nc[a] = shrunk > 1 ? shrunk : 1;
  }
  if (nc_cap)
    for (int a = 0; a < 3; a++) g.nc[a] = g.nc[a] < nc_cap[a] ? g.nc[a] : (nc_cap[a] > 1 ? nc_cap[a] : 1);
  // The stencil of +-stencil cells covers the cut-off on every axis with at
  // least 2*stencil+1 cells; smaller axes are scanned whole.
  double hplan = INFINITY;
  g.sw = S.stencil;
  for (int a = 0; a < 3; a++) {
    g.cs[a] = div_rn(extent[a], (double)g.nc[a]);
    g.csf[a] = (float)g.cs[a];
    g.inv_cs[a] = a < S.dim ? div_rn(1.0, g.cs[a]) : 0.0;
    const bool limits = a < S.dim && g.nc[a] >= 2 * g.sw + 1;
    if (limits) {
      const double hp = mul_rn(div_rn(mul_rn((double)g.sw, g.cs[a]), mul_rn(S.R, add_rn(1.0, S.list_margin))),
                               1.0 - 1e-9);
      hplan = hp < hplan ? hp : hplan;
    }
  }
  g.h_plan = hplan;
  g.h_bigf = hplan < 1e30 ? (float)mul_rn(hplan, 1.0 - 1e-5) : INFINITY;
  // A normal particle (h <= h_plan) reaches up to R (1 + margin) h_plan,
  // which the rounding of the cell count can put above the planned cutoff.
  g.cut = hplan < 1e30 ? mul_rn(mul_rn(S.R, add_rn(1.0, S.list_margin)), hplan) : cutoff;
  if (g.cut < cutoff) g.cut = cutoff;
  g.ncells = g.nc[0] * g.nc[1] * g.nc[2];
  for (int a = 0; a < 3; a++) {
    if (a >= S.dim) {
      g.fx_lo[a] = 0.0;
      g.fx_scale[a] = 0.0;
      g.fx_len[a] = 0.f;
      continue;
    }
    double span = S.periodic[a] ? S.L[a] : mul_rn(4.0, extent[a]);
    if (!(span > 1e-250)) span = 1e-250;  // a degenerate open axis (every particle on one coordinate)
    g.fx_lo[a] = S.periodic[a] ? S.lo[a] : add_rn(g.lo[a], -mul_rn(1.5, extent[a]));
    g.fx_scale[a] = div_rn(4294967296.0, span);
    g.fx_len[a] = (float)div_rn(span, 4294967296.0);
  }
  return MHD_OK;
}

// Fixed-point coordinate of x along axis a (see Grid::fx_lo).
__device__ __forceinline__ unsigned fixed_coord(const Grid& g, int a, double x) {
  return (unsigned)(unsigned long long)(long long)floor((x - g.fx_lo[a]) * g.fx_scale[a]);
}
// FP32 displacement from two fixed-point coordinates.
__device__ __forceinline__ float fixed_delta(const Grid& g, int a, unsigned ui, unsigned uj) {
  return __int2float_rn((int)(ui - uj)) * g.fx_len[a];
}

// Mean h from the fixed-point sum of h / h_max.
__host__ __device__ inline double mean_h(double hmax, unsigned long long h_sum, int n) {
  return n > 0 ? mul_rn(hmax, div_rn((double)h_sum, mul_rn((double)n, 4294967296.0))) : 1.0;
}

__device__ __forceinline__ void set_status(DevScalars* sc, int code) { atomicCAS(&sc->status, MHD_OK, code); }

// Cell coordinate of a position along axis a.
__device__ __forceinline__ int cell_coord(const Grid& g, int a, double x) {
  int c = (int)floor((x - g.lo[a]) * g.inv_cs[a]);
  c = c < 0 ? 0 : c;
  c = c >= g.nc[a] ? g.nc[a] - 1 : c;
  return c;
}

// Cell coordinates in one int: 11/11/10 bits in 3-D, 16/16 in 2-D.
template <int DIM>
__device__ __forceinline__ int pack_cell(int cx, int cy, int cz) {
  if constexpr (DIM == 3) return cx | (cy << 11) | (cz << 22);
  else return cx | (cy << 16);
}
template <int DIM>
__device__ __forceinline__ void unpack_cell(int c, int& cx, int& cy, int& cz) {
  if constexpr (DIM == 3) {
    cx = c & 2047;
    cy = (c >> 11) & 2047;
    cz = (c >> 22) & 1023;
  } else {
    cx = c & 65535;
    cy = (c >> 16) & 65535;
    cz = 0;
  }
}

// Cell offset ci - cj along an axis, wrapped to the nearest periodic image.
__device__ __forceinline__ int cell_delta(int d, int nc, int periodic) {
  if (periodic && nc >= 3) {
    if (d > nc / 2) d -= nc;
    else if (d < -(nc / 2)) d += nc;
  }
  return d;
}

// FP32 minimum-image displacement x_i - x_j from packed positions: the cell
// offset carries the large part exactly, the in-cell offsets the rest.  On a
// periodic axis with at least 2*sw+1 cells a pair of normal particles is at
// most sw cells apart and the wrapped cell offset selects its image; on an
// axis with fewer cells (scanned whole), or for a pair more than sw cells
// apart (a big particle's), the FP32 minimum image is taken as well.  The
// result is exactly antisymmetric in i and j.
__device__ __forceinline__ float fold_image(float d, float L) {
  const float hL = 0.5f * L;
  return d > hL ? d - L : (d < -hL ? d + L : d);
}

template <int DIM>
__device__ __forceinline__ void rel_dx(const Grid& G, const float4& pi, int ci, const float4& pj, int cj, float& dx,
                                       float& dy, float& dz) {
  int xi, yi, zi, xj, yj, zj;
  unpack_cell<DIM>(ci, xi, yi, zi);
  unpack_cell<DIM>(cj, xj, yj, zj);
  const int ex = cell_delta(xi - xj, G.nc[0], G.periodic[0]);
  const int ey = cell_delta(yi - yj, G.nc[1], G.periodic[1]);
  const int ez = DIM == 3 ? cell_delta(zi - zj, G.nc[2], G.periodic[2]) : 0;
  dx = (pi.x - pj.x) + (float)ex * G.csf[0];
  dy = (pi.y - pj.y) + (float)ey * G.csf[1];
  dz = DIM == 3 ? (pi.z - pj.z) + (float)ez * G.csf[2] : 0.f;
  const int whole = 2 * G.sw + 1;
  if (G.periodic[0] && (G.nc[0] < whole || abs(ex) > G.sw)) dx = fold_image(dx, (float)G.L[0]);
  if (G.periodic[1] && (G.nc[1] < whole || abs(ey) > G.sw)) dy = fold_image(dy, (float)G.L[1]);
  if (DIM == 3 && G.periodic[2] && (G.nc[2] < whole || abs(ez) > G.sw)) dz = fold_image(dz, (float)G.L[2]);
}

// Calls f(cx, cy, cz, jb, je) for every cell within `cut` of (xi, yi, zi),
// searching +-sw cells (cut <= sw cell widths): (cx, cy, cz) are unwrapped
// cell coordinates (their offset from the particle's own cell selects the
// periodic image), [jb, je) the cell's range in the sorted order.  Rows
// farther than `cut` are skipped and each row is trimmed to
// [x - cut, x + cut].  Axes with fewer than 2*sw+1 cells are scanned whole
// with their own coordinates (no image selection).
template <int DIM, class F>
__device__ __forceinline__ void for_each_cell_trimmed(const Grid& G, int sw, const int* __restrict__ cell_start,
                                                      double xi, double yi, double zi, double cut, F&& f) {
  const int whole = 2 * sw + 1;
  const int nx = G.nc[0], ny = G.nc[1], nz = G.nc[2];
  const int cy = cell_coord(G, 1, yi);
  const int cz = DIM == 3 ? cell_coord(G, 2, zi) : 0;
  int xl, xh;
  if (nx < whole) {
    xl = 0;
    xh = nx - 1;
  } else {
    xl = (int)floor((xi - cut - G.lo[0]) * G.inv_cs[0]);
    xh = (int)floor((xi + cut - G.lo[0]) * G.inv_cs[0]);
    if (!G.periodic[0]) {
      xl = xl < 0 ? 0 : xl;
      xh = xh >= nx ? nx - 1 : xh;
    }
    if (xh - xl >= nx) xh = xl + nx - 1;  // never visit a cell twice
  }
  const double cut2 = cut * cut;
  const bool zs = DIM == 3 && nz >= whole, ys = ny >= whole;
  const int zlo = DIM == 3 ? (zs ? cz - sw : 0) : 0, zhi = DIM == 3 ? (zs ? cz + sw : nz - 1) : 0;
  const int ylo = ys ? cy - sw : 0, yhi = ys ? cy + sw : ny - 1;
  for (int zu = zlo; zu <= zhi; zu++) {
    int zc = zu;
    double dzm = 0.0;
    if (zs) {
      const double c_lo = G.lo[2] + zu * G.cs[2], c_hi = c_lo + G.cs[2];
      dzm = zi < c_lo ? c_lo - zi : (zi > c_hi ? zi - c_hi : 0.0);
      if (dzm * dzm >= cut2) continue;
      if (zc < 0 || zc >= nz) {
        if (!G.periodic[2]) continue;
        zc = zc < 0 ? zc + nz : zc - nz;
      }
    }
    for (int yu = ylo; yu <= yhi; yu++) {
      int yc = yu;
      if (ys) {
        const double c_lo = G.lo[1] + yu * G.cs[1], c_hi = c_lo + G.cs[1];
        const double dym = yi < c_lo ? c_lo - yi : (yi > c_hi ? yi - c_hi : 0.0);
        if (dym * dym + dzm * dzm >= cut2) continue;
        if (yc < 0 || yc >= ny) {
          if (!G.periodic[1]) continue;
          yc = yc < 0 ? yc + ny : yc - ny;
        }
      }
      const int base = G.cell_base + (zc * ny + yc) * nx;
      int xw = xl < 0 ? xl + nx : xl;
      int jb = cell_start[base + xw];
      for (int xu = xl; xu <= xh; xu++) {
        const int next = xw + 1;
        const int je = cell_start[base + next];
        f(xu, yu, zu, jb, je);
        if (next == nx) {
          xw = 0;
          jb = cell_start[base];
        } else {
          xw = next;
          jb = je;
        }
      }
    }
  }
}

// The cells for_each_cell_trimmed visits, a stencil row at a time: calls
// f(yu, zu, jb, je, xoff) for every contiguous piece of a row's trimmed
// x-range, [jb, je) the particles of the piece in sorted order and xoff the
// offset that turns a particle's own cell x into its unwrapped coordinate
// (-nx, 0 or +nx; 0 on an axis scanned whole).  Pieces come in ascending
// unwrapped x, so a caller sees the particles in the order of
// for_each_cell_trimmed.  Where the x-range is not the whole axis, a row
// keeps only its cells within sqrt(cut^2 - dym^2 - dzm^2) of xi (dym, dzm
// the distances to the row's cell box): a subset of the full range in the
// same order, missing only particles farther than cut.
template <int DIM, class F>
__device__ __forceinline__ void for_each_row_trimmed(const Grid& G, int sw, const int* __restrict__ cell_start,
                                                     double xi, double yi, double zi, double cut, F&& f) {
  const int whole = 2 * sw + 1;
  const int nx = G.nc[0], ny = G.nc[1], nz = G.nc[2];
  const int cy = cell_coord(G, 1, yi);
  const int cz = DIM == 3 ? cell_coord(G, 2, zi) : 0;
  int xl0, xh0;
  bool xtrim = false;
  if (nx < whole) {
    xl0 = 0;
    xh0 = nx - 1;
  } else {
    xl0 = (int)floor((xi - cut - G.lo[0]) * G.inv_cs[0]);
    xh0 = (int)floor((xi + cut - G.lo[0]) * G.inv_cs[0]);
    if (!G.periodic[0]) {
      xl0 = xl0 < 0 ? 0 : xl0;
      xh0 = xh0 >= nx ? nx - 1 : xh0;
    }
    if (xh0 - xl0 >= nx) xh0 = xl0 + nx - 1;  // never visit a cell twice
    else xtrim = true;
  }
  const double cut2 = cut * cut;
  const bool zs = DIM == 3 && nz >= whole, ys = ny >= whole;
  const int zlo = DIM == 3 ? (zs ? cz - sw : 0) : 0, zhi = DIM == 3 ? (zs ? cz + sw : nz - 1) : 0;
  const int ylo = ys ? cy - sw : 0, yhi = ys ? cy + sw : ny - 1;
  for (int zu = zlo; zu <= zhi; zu++) {
    int zc = zu;
    double dzm = 0.0;
    if (zs) {
      const double c_lo = G.lo[2] + zu * G.cs[2], c_hi = c_lo + G.cs[2];
      dzm = zi < c_lo ? c_lo - zi : (zi > c_hi ? zi - c_hi : 0.0);
      if (dzm * dzm >= cut2) continue;
      if (zc < 0 || zc >= nz) {
        if (!G.periodic[2]) continue;
        zc = zc < 0 ? zc + nz : zc - nz;
      }
    }
    for (int yu = ylo; yu <= yhi; yu++) {
      int yc = yu;
      double dym = 0.0;
      if (ys) {
        const double c_lo = G.lo[1] + yu * G.cs[1], c_hi = c_lo + G.cs[1];
        dym = yi < c_lo ? c_lo - yi : (yi > c_hi ? yi - c_hi : 0.0);
        if (dym * dym + dzm * dzm >= cut2) continue;
        if (yc < 0 || yc >= ny) {
          if (!G.periodic[1]) continue;
          yc = yc < 0 ? yc + ny : yc - ny;
        }
      }
      const int base = G.cell_base + (zc * ny + yc) * nx;
      int xl = xl0, xh = xh0;
      if (xtrim) {
        const double wx = sqrt(cut2 - (dym * dym + dzm * dzm));
        const int a = (int)floor((xi - wx - G.lo[0]) * G.inv_cs[0]);
        const int b = (int)floor((xi + wx - G.lo[0]) * G.inv_cs[0]);
        xl = a > xl ? a : xl;
        xh = b < xh ? b : xh;
        if (xl > xh) continue;
      }
      // [xl, xh] in unwrapped cells: at most three pieces (below 0, inside,
      // above nx - 1)
      if (xl < 0) {
        const int a = xl + nx, b = (xh < 0 ? xh : -1) + nx;
        f(yu, zu, cell_start[base + a], cell_start[base + b + 1], -nx);
      }
      if (xh >= 0 && xl < nx) {
        const int a = xl < 0 ? 0 : xl, b = xh >= nx ? nx - 1 : xh;
        f(yu, zu, cell_start[base + a], cell_start[base + b + 1], 0);
      }
      if (xh >= nx) {
        const int a = (xl >= nx ? xl : nx) - nx, b = xh - nx;
        f(yu, zu, cell_start[base + a], cell_start[base + b + 1], nx);
      }
    }
  }
}

// The rows of for_each_row_trimmed's walk, restated one row at a time so
// that a warp can take one row per lane (warp_rows): rows yu in
// [ylo, yhi] (and zu in [zlo, zhi] in 3-D), each over the unwrapped x-range
// [xl0, xh0], trimmed per row when xtrim.
struct RowPlan {
  int ylo, yhi, zlo, zhi, xl0, xh0;
  bool xtrim, ys, zs;
  double cut2;
};

template <int DIM>
__device__ __forceinline__ RowPlan row_plan(const Grid& G, int sw, double xi, double yi, double zi, double cut) {
  RowPlan R;
  const int whole = 2 * sw + 1;
  const int nx = G.nc[0], ny = G.nc[1], nz = G.nc[2];
  const int cy = cell_coord(G, 1, yi);
  const int cz = DIM == 3 ? cell_coord(G, 2, zi) : 0;
  R.xtrim = false;
  if (nx < whole) {
    R.xl0 = 0;
    R.xh0 = nx - 1;
  } else {
    R.xl0 = (int)floor((xi - cut - G.lo[0]) * G.inv_cs[0]);
    R.xh0 = (int)floor((xi + cut - G.lo[0]) * G.inv_cs[0]);
    if (!G.periodic[0]) {
      R.xl0 = R.xl0 < 0 ? 0 : R.xl0;
      R.xh0 = R.xh0 >= nx ? nx - 1 : R.xh0;
    }
    if (R.xh0 - R.xl0 >= nx) R.xh0 = R.xl0 + nx - 1;
    else R.xtrim = true;
  }
  R.cut2 = cut * cut;
  R.zs = DIM == 3 && nz >= whole;
  R.ys = ny >= whole;
  R.zlo = DIM == 3 ? (R.zs ? cz - sw : 0) : 0;
  R.zhi = DIM == 3 ? (R.zs ? cz + sw : nz - 1) : 0;
  R.ylo = R.ys ? cy - sw : 0;
  R.yhi = R.ys ? cy + sw : ny - 1;
  return R;
}

// The pieces of row (yu, zu): [jb[p], je[p]) holds the particles of its
// cells below 0 (p = 0, x offset -nx), inside the grid (p = 1, offset 0) and
// above nx - 1 (p = 2, offset +nx); an absent piece is empty.  The cells and
// their order are for_each_row_trimmed's.
template <int DIM>
__device__ __forceinline__ void row_pieces(const Grid& G, const RowPlan& R, const int* __restrict__ cell_start,
                                           double xi, double yi, double zi, int yu, int zu, int (&jb)[3],
                                           int (&je)[3]) {
  jb[0] = je[0] = jb[1] = je[1] = jb[2] = je[2] = 0;
  const int nx = G.nc[0], ny = G.nc[1], nz = G.nc[2];
  int zc = zu;
  double dzm = 0.0;
  if (R.zs) {
    const double c_lo = G.lo[2] + zu * G.cs[2], c_hi = c_lo + G.cs[2];
    dzm = zi < c_lo ? c_lo - zi : (zi > c_hi ? zi - c_hi : 0.0);
    if (dzm * dzm >= R.cut2) return;
    if (zc < 0 || zc >= nz) {
      if (!G.periodic[2]) return;
      zc = zc < 0 ? zc + nz : zc - nz;
    }
  }
  int yc = yu;
  double dym = 0.0;
  if (R.ys) {
    const double c_lo = G.lo[1] + yu * G.cs[1], c_hi = c_lo + G.cs[1];
    dym = yi < c_lo ? c_lo - yi : (yi > c_hi ? yi - c_hi : 0.0);
    if (dym * dym + dzm * dzm >= R.cut2) return;
    if (yc < 0 || yc >= ny) {
      if (!G.periodic[1]) return;
      yc = yc < 0 ? yc + ny : yc - ny;
    }
  }
  const int base = G.cell_base + (zc * ny + yc) * nx;
  int xl = R.xl0, xh = R.xh0;
  if (R.xtrim) {
    const double wx = sqrt(R.cut2 - (dym * dym + dzm * dzm));
    const int a = (int)floor((xi - wx - G.lo[0]) * G.inv_cs[0]);
    const int b = (int)floor((xi + wx - G.lo[0]) * G.inv_cs[0]);
    xl = a > xl ? a : xl;
    xh = b < xh ? b : xh;
    if (xl > xh) return;
  }
  if (xl < 0) {
    const int a = xl + nx, b = (xh < 0 ? xh : -1) + nx;
    jb[0] = cell_start[base + a];
    je[0] = cell_start[base + b + 1];
  }
  if (xh >= 0 && xl < nx) {
    const int a = xl < 0 ? 0 : xl, b = xh >= nx ? nx - 1 : xh;
    jb[1] = cell_start[base + a];
    je[1] = cell_start[base + b + 1];
  }
  if (xh >= nx) {
    const int a = (xl >= nx ? xl : nx) - nx, b = xh - nx;
    jb[2] = cell_start[base + a];
    je[2] = cell_start[base + b + 1];
  }
}

// for_each_row_trimmed's walk for a whole warp searching from one point:
// the lanes look up 32 rows' pieces side by side (one row each, instead of
// every row in turn), a warp prefix sum lays the rows' particles end to
// end, and f(j, yu, zu, xoff) is called by every lane for 32 consecutive
// candidates at a time, in for_each_row_trimmed's order (j < 0 past the
// end; yu, zu the candidate's row and xoff its piece's offset, as
// for_each_row_trimmed passes them).  Must be called by all 32 lanes with
// the same arguments; f may use warp-wide operations.
template <int DIM, class F>
__device__ __forceinline__ void warp_rows(const Grid& G, int sw, const int* __restrict__ cell_start, double xi,
                                          double yi, double zi, double cut, F&& f) {
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const RowPlan R = row_plan<DIM>(G, sw, xi, yi, zi, cut);
  const int nyr = R.yhi - R.ylo + 1, nrows = nyr * (R.zhi - R.zlo + 1);
  const int nx = G.nc[0];
  for (int r0 = 0; r0 < nrows; r0 += 32) {
    const int r = r0 + lane;
    int jb[3] = {0, 0, 0}, je[3] = {0, 0, 0}, yu = 0, zu = 0;
    if (r < nrows) {
      zu = R.zlo + r / nyr;
      yu = R.ylo + r % nyr;
      row_pieces<DIM>(G, R, cell_start, xi, yi, zi, yu, zu, jb, je);
    }
    const int l0 = je[0] - jb[0], l1 = je[1] - jb[1], m = l0 + l1 + (je[2] - jb[2]);
    int incl = m;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int v = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += v;
    }
    const int excl = incl - m;
    const int total = __shfl_sync(kFull, incl, 31);
    for (int c0 = 0; c0 < total; c0 += 32) {
      const int c = c0 + lane;
      // the row lane owning candidate c: the last lane whose range starts at
      // or before c (a lane with no candidates never is)
      int L = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int e = __shfl_sync(kFull, excl, L + step);
        if (e <= c) L += step;
      }
      const int k = c - __shfl_sync(kFull, excl, L);
      const int a0 = __shfl_sync(kFull, l0, L), a1 = __shfl_sync(kFull, l1, L);
      const int b0 = __shfl_sync(kFull, jb[0], L), b1 = __shfl_sync(kFull, jb[1], L),
                b2 = __shfl_sync(kFull, jb[2], L);
      const int yr = __shfl_sync(kFull, yu, L), zr = __shfl_sync(kFull, zu, L);
      int j = -1, xoff = 0;
      if (c < total) {
        if (k < a0) {
          j = b0 + k;
          xoff = -nx;
        } else if (k < a0 + a1) {
          j = b1 + (k - a0);
        } else {
          j = b2 + (k - a0 - a1);
          xoff = nx;
        }
      }
      f(j, yr, zr, xoff);
    }
  }
}

}  // namespace mhd
