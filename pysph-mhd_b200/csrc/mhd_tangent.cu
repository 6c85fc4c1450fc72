// mhd_tangent.cu -- derivative form of the SPMHD step (forward mode, sm_100a).
//
// The literal PEC step of the reference -- MHDStep.initialize/stage1
// (src/integrator.py:12-65), the ten equation groups of
// MHDScheme.get_equations (src/scheme.py:66-81; src/equations.py) with a
// single density pass (density = "single"), MHDStep.stage2
// (src/integrator.py:68-82) -- written once over a scalar type and run on
// dual numbers: every state value carries its derivatives with respect to
// MHD_TANGENT_DIRS parameters.  The step size is a plain value (frozen: the
// adaptive rule's min() is not differentiated).  Neighbours come from the
// cell grid of mhd_pairgrid.cuh, built over each pass's positions and
// smoothing lengths, with the exact FP64 rule.  Compiled with
// --fmad=false: no contraction, the reference's expression order
// throughout.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <string>

#include "mhd_common.cuh"
#include "mhd_dual.cuh"
#include "mhd_internal.h"
#include "mhd_pairgrid.cuh"

namespace mhd {

using TD = Dual<MHD_TANGENT_DIRS>;
constexpr int kTile = 128;

#define TF(name) reinterpret_cast<TD*>(s.name)

// ------------------------------------------------------------- SPH kernels
// hfac, W, grad W, dW/dh as PySPH defines them (restated): sigma / h^dim,
// W = sigma w(q) / h^dim, grad W = sigma w'(q) / h^(dim+1) x_ij / r_ij
// (0 for r_ij <= 1e-12), dW/dh = -sigma / h^(dim+1) (w' q + dim w).
template <int DIM, class D>
__device__ inline D t_hfac(double norm, const D& h1) {
  return DIM == 2 ? norm * h1 * h1 : norm * h1 * h1 * h1;
}
template <int K, int DIM, class D>
__device__ inline D t_kern_w(double norm, const D& r, const D& h) {
  const D h1 = 1.0 / h, q = r * h1;
  D w, dw;
  w_dw<K, D>(q, DIM, w, dw);
  return w * t_hfac<DIM>(norm, h1);
}
template <int K, int DIM, class D>
__device__ inline void t_kern_grad(double norm, const D* xij, const D& r, const D& h, D* g) {
  const D h1 = 1.0 / h;
  D tmp(0.0);
  if (r > 1.0e-12) {
    const D q = r * h1;
    D w, dw;
    w_dw<K, D>(q, DIM, w, dw);
    tmp = t_hfac<DIM>(norm, h1) * dw * h1 / r;
  }
  g[0] = tmp * xij[0];
  g[1] = tmp * xij[1];
  g[2] = tmp * xij[2];
}
template <int K, int DIM, class D>
__device__ inline D t_kern_gradh(double norm, const D& r, const D& h) {
  const D h1 = 1.0 / h, q = r * h1;
  D w, dw;
  w_dw<K, D>(q, DIM, w, dw);
  return -(t_hfac<DIM>(norm, h1) * h1 * (dw * q + w * (double)DIM));
}

template <class D>
__device__ inline D pmax(const D& a, const D& b) { return b > a ? b : a; }
template <class D>
__device__ inline D pmin(const D& a, const D& b) { return b < a ? b : a; }

// ------------------------------------------------------- neighbour search
// Calls f(j) for every j with r2 < (R h_i)^2 or r2 < (R h_j)^2 on the
// minimum-image FP64 values, self included, among the particles of this
// block's slice (grid y): the cell grid of mhd_pairgrid.cuh over the pass's
// x and h.  Each pair kernel writes its partial sums per slice and a
// per-particle kernel adds them in slice order (deterministic).
constexpr int kTWidth = 24;  // partial records per particle and slice (the 24 CD moments at most)

struct TGrid {
  const PairGrid* g;
  const int* cell_start;
  const int* perm;
  const double4* pos;
  int slices;
};

__device__ inline TD& t_part(TD* part, int n, int q, int i) {
  return part[((size_t)blockIdx.y * kTWidth + q) * n + i];
}
__device__ inline TD t_slices_sum(const TD* part, int n, int q, int i, int slices) {
  TD v(0.0);
  for (int sl = 0; sl < slices; sl++) v = v + part[((size_t)sl * kTWidth + q) * n + i];
  return v;
}

template <int DIM, class F>
__device__ inline void t_pairs(const TGrid& tg, const DevParams& P, int i, int n, F&& f) {
  if (i >= n) return;
  pair_grid_visit<DIM>(*tg.g, tg.cell_start, tg.perm, tg.pos, P, i, (int)blockIdx.y, tg.slices,
                       [&](int j, double, double, double) { f(j); });
}

// {x, y, z, h} values of the current state for the grid build.
template <int DIM>
__global__ void __launch_bounds__(256) k_t_pack_pos(int n, MhdState s, double4* __restrict__ pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] = make_double4(TF(x)[i].v, TF(y)[i].v, DIM == 3 ? TF(z)[i].v : 0.0, TF(h)[i].v);
}

// Minimum-image x_i - x_j along one axis as a dual number: the image shift
// is decided on the values and is a constant.
__device__ inline TD image_diff(const TD& a, const TD& b, double L, double half, int periodic) {
  TD d = a - b;
  if (periodic) {
    if (d.v > half) d = d - L;
    if (d.v < -half) d = d + L;
  }
  return d;
}

template <int DIM>
__device__ inline void pair_geometry(const DevParams& P, const MhdState& s, int i, int j, TD* xij, TD& rij) {
  xij[0] = image_diff(TF(x)[i], TF(x)[j], P.L[0], P.half[0], P.periodic[0]);
  xij[1] = image_diff(TF(y)[i], TF(y)[j], P.L[1], P.half[1], P.periodic[1]);
  xij[2] = DIM == 3 ? image_diff(TF(z)[i], TF(z)[j], P.L[2], P.half[2], P.periodic[2]) : TD(0.0);
  rij = sqrt(xij[0] * xij[0] + xij[1] * xij[1] + xij[2] * xij[2]);
}

// ------------------------------------------ initialize + stage1 + wrap
// src/integrator.py:12-65 for every particle (stage1 only for itype 1), then
// the periodic wrap.
__device__ inline TD wrap_dual(TD x, double lo, double hi, double L) {
  if (x.v < lo) x = x + L;
  if (x.v > hi) x = x - L;
  return x;
}

__global__ void __launch_bounds__(256) k_t_predict(int n, DevParams P, MhdState s, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TD x0 = TF(x)[i], y0 = TF(y)[i], z0 = TF(z)[i];
  const TD u0 = TF(u)[i], v0 = TF(v)[i], w0 = TF(w)[i], e0 = TF(e)[i], h0 = TF(h)[i];
  const TD a10 = TF(alpha1)[i];
  const TD bx0 = TF(Bevolx)[i], by0 = TF(Bevoly)[i], bz0 = TF(Bevolz)[i], psi0 = TF(psi)[i];
  TF(h0)[i] = h0;
  TF(converged)[i] = TD(0.0);
  TF(omega)[i] = TD(1.0);
  TF(upred)[i] = u0;
  TF(vpred)[i] = v0;
  TF(wpred)[i] = w0;
  TF(epred)[i] = e0;
  TF(Bevolxpred)[i] = bx0;
  TF(Bevolypred)[i] = by0;
  TF(Bevolzpred)[i] = bz0;
  TF(psipred)[i] = psi0;
  if (s.itype[i] != 1) return;
  const double dtb2 = 0.5 * dt;
  const TD au = TF(au)[i], av = TF(av)[i], aw = TF(aw)[i];
  const TD u = u0 + dtb2 * au, v = v0 + dtb2 * av, w = w0 + dtb2 * aw;
  TF(u)[i] = u;
  TF(v)[i] = v;
  TF(w)[i] = w;
  TF(upred)[i] = u0 + dt * au;
  TF(vpred)[i] = v0 + dt * av;
  TF(wpred)[i] = w0 + dt * aw;
  TD x = x0 + dt * u, y = y0 + dt * v, z = z0;
  if (P.dim == 3) z = z0 + dt * w;
  if (P.periodic[0]) x = wrap_dual(x, P.lo[0], P.hi[0], P.L[0]);
  if (P.periodic[1]) y = wrap_dual(y, P.lo[1], P.hi[1], P.L[1]);
  if (P.dim == 3 && P.periodic[2]) z = wrap_dual(z, P.lo[2], P.hi[2], P.L[2]);
  TF(x)[i] = x;
  TF(y)[i] = y;
  TF(z)[i] = z;
  const TD ae = TF(ae)[i];
  TF(e)[i] = e0 + dtb2 * ae;
  TF(epred)[i] = e0 + dt * ae;
  const TD h = h0 + dt * TF(ah)[i];
  TF(h)[i] = h;
  const TD decay_rate = 0.1 * TF(cs)[i] / h;
  const TD aloc = TF(alphaloc)[i];
  TF(alpha1)[i] = a10 < aloc ? aloc : (a10 + dt * aloc * decay_rate) / (1.0 + dt * decay_rate);
  const TD abx = TF(aBevolx)[i], aby = TF(aBevoly)[i], abz = TF(aBevolz)[i], apsi = TF(apsi)[i];
  TF(Bevolx)[i] = bx0 + dtb2 * abx;
  TF(Bevoly)[i] = by0 + dtb2 * aby;
  TF(Bevolz)[i] = bz0 + dtb2 * abz;
  TF(psi)[i] = psi0 + dtb2 * apsi;
  TF(Bevolxpred)[i] = bx0 + dt * abx;
  TF(Bevolypred)[i] = by0 + dt * aby;
  TF(Bevolzpred)[i] = bz0 + dt * abz;
  TF(psipred)[i] = psi0 + dt * apsi;
}

// --------------------------------------------------------------- stage2
__global__ void __launch_bounds__(256) k_t_correct(int n, DevParams P, MhdState s, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || s.itype[i] != 1) return;
  const double dtb2 = 0.5 * dt;
  TF(u)[i] = TF(u)[i] + dtb2 * TF(au)[i];
  TF(v)[i] = TF(v)[i] + dtb2 * TF(av)[i];
  TF(w)[i] = TF(w)[i] + dtb2 * TF(aw)[i];
  const TD e = TF(e)[i] + dtb2 * TF(ae)[i];
  TF(e)[i] = e;
  const TD rho = TF(rho)[i];
  TF(p)[i] = P.gamma1 * rho * e;
  const TD bx = TF(Bevolx)[i] + dtb2 * TF(aBevolx)[i];
  const TD by = TF(Bevoly)[i] + dtb2 * TF(aBevoly)[i];
  const TD bz = TF(Bevolz)[i] + dtb2 * TF(aBevolz)[i];
  TF(Bevolx)[i] = bx;
  TF(Bevoly)[i] = by;
  TF(Bevolz)[i] = bz;
  TF(psi)[i] = TF(psi)[i] + dtb2 * TF(apsi)[i];
  TF(Bx)[i] = bx * rho;
  TF(By)[i] = by * rho;
  TF(Bz)[i] = bz * rho;
}

// src/application.py:99-108 (_sync_initial_mhd_state): Bevol = B / rho,
// psi = 0 and the predicted copies.
__global__ void __launch_bounds__(256) k_t_sync(int n, MhdState s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TD rho = TF(rho)[i];
  const TD bx = TF(Bx)[i] / rho, by = TF(By)[i] / rho, bz = TF(Bz)[i] / rho;
  TF(Bevolx)[i] = bx;
  TF(Bevoly)[i] = by;
  TF(Bevolz)[i] = bz;
  TF(psi)[i] = TD(0.0);
  TF(Bevolxpred)[i] = bx;
  TF(Bevolypred)[i] = by;
  TF(Bevolzpred)[i] = bz;
  TF(psipred)[i] = TD(0.0);
  TF(upred)[i] = TF(u)[i];
  TF(vpred)[i] = TF(v)[i];
  TF(wpred)[i] = TF(w)[i];
  TF(epred)[i] = TF(e)[i];
}

// ------------------------------------------------- G1 single density pass
// DensityIteration with iterate_only_once (src/equations.py:24-88): sums with
// h_i, Omega from the old h, then h = hfact (m / rho)^(1/dim).  The new h goes
// to h_new (other threads still read h).
template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_t_density_pair(int n, DevParams P, MhdState s, TD* __restrict__ part, TGrid tg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  TD rho(0.0), dwdh(0.0);
  const TD hi = i < n ? TF(h)[i] : TD(1.0);
  t_pairs<DIM>(tg, P, i, n, [&](int j) {
    TD xij[3], rij;
    pair_geometry<DIM>(P, s, i, j, xij, rij);
    const TD mj = TF(m)[j];
    rho += mj * t_kern_w<K, DIM>(P.norm, rij, hi);
    dwdh += mj * t_kern_gradh<K, DIM>(P.norm, rij, hi);
  });
  if (i >= n) return;
  t_part(part, n, 0, i) = rho;
  t_part(part, n, 1, i) = dwdh;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_t_density(int n, DevParams P, MhdState s, const TD* __restrict__ part,
                                                   TD* __restrict__ h_new, int slices) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TD hi = TF(h)[i];
  const TD rho = t_slices_sum(part, n, 0, i, slices), dwdh = t_slices_sum(part, n, 1, i, slices);
  TF(rho_sum)[i] = rho;
  if (TF(converged)[i].v == 1.0) {
    // already finalised in this group evaluation (the warm-up's second and
    // third RHS): post_loop skips it (src/equations.py:56), h and Omega stay
    h_new[i] = hi;
    return;
  }
  const double k = P.hfact;
  const TD mi = TF(m)[i];
  const TD hk = hi / k;
  const TD rhoi = mi / (DIM == 2 ? hk * hk : hk * hk * hk);
  const TD dhdrhoi = -hi / ((double)DIM * rhoi);
  const TD omegai = 1.0 - dhdrhoi * dwdh;
  TF(omega)[i] = 1.0 / omegai;
  TF(converged)[i] = TD(1.0);
  h_new[i] = k * pow(mi / rho, 1.0 / (double)DIM);
}

// G2, G3 and G5 (src/equations.py:109-118, 97-106, 474-485): the new h,
// rho = m / (h / hfact)^dim, EOS, B = Bevol_pred rho.
template <int DIM>
__global__ void __launch_bounds__(256) k_t_prologue(int n, DevParams P, MhdState s, const TD* __restrict__ h_new) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TD h = h_new[i];
  TF(h)[i] = h;
  const TD hk = h / P.hfact;
  const TD rho = TF(m)[i] / (DIM == 2 ? hk * hk : hk * hk * hk);
  TF(rho)[i] = rho;
  const TD p = P.gamma1 * rho * TF(epred)[i];
  TF(p)[i] = p;
  TF(cs)[i] = sqrt(P.gamma * p / rho);
  TF(Bx)[i] = TF(Bevolxpred)[i] * rho;
  TF(By)[i] = TF(Bevolypred)[i] * rho;
  TF(Bz)[i] = TF(Bevolzpred)[i] * rho;
}

// ----------------------------------------- G4 Cullen-Dehnen diagnostics
// src/equations.py:318-429 with the previous step's accelerations; the
// alpha clip [alpha_min, alpha_max] with alpha_max a dual number.
template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_t_cd_pair(int n, DevParams P, MhdState s, TD* __restrict__ part, TGrid tg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  TD r[6], vv[9], aa[9];
  for (int k = 0; k < 6; k++) r[k] = TD(0.0);
  for (int k = 0; k < 9; k++) vv[k] = aa[k] = TD(0.0);
  const bool act = i < n;
  const TD hi = act ? TF(h)[i] : TD(1.0);
  t_pairs<DIM>(tg, P, i, n, [&](int j) {
    TD xij[3], rij, dwi[3];
    pair_geometry<DIM>(P, s, i, j, xij, rij);
    t_kern_grad<K, DIM>(P.norm, xij, rij, hi, dwi);
    const TD mj = TF(m)[j];
    const TD run[3] = {mj * dwi[0], mj * dwi[1], mj * dwi[2]};
    const TD dv[3] = {TF(upred)[i] - TF(upred)[j], TF(vpred)[i] - TF(vpred)[j], TF(wpred)[i] - TF(wpred)[j]};
    const TD da[3] = {TF(au)[i] - TF(au)[j], TF(av)[i] - TF(av)[j], TF(aw)[i] - TF(aw)[j]};
    r[0] += -xij[0] * run[0];
    r[1] += -xij[0] * run[1];
    r[2] += -xij[0] * run[2];
    r[3] += -xij[1] * run[1];
    r[4] += -xij[1] * run[2];
    r[5] += -xij[2] * run[2];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        vv[3 * a + b] += dv[a] * run[b];
        aa[3 * a + b] += da[a] * run[b];
      }
  });
  if (!act) return;
  for (int k = 0; k < 6; k++) t_part(part, n, k, i) = r[k];
  for (int k = 0; k < 9; k++) {
    t_part(part, n, 6 + k, i) = vv[k];
    t_part(part, n, 15 + k, i) = aa[k];
  }
}

__global__ void __launch_bounds__(256) k_t_cd(int n, DevParams P, MhdState s, const TD* __restrict__ part,
                                              TD alpha_max, int slices) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TD hi = TF(h)[i];
  TD r[6], vv[9], aa[9];
  for (int k = 0; k < 6; k++) r[k] = t_slices_sum(part, n, k, i, slices);
  for (int k = 0; k < 9; k++) {
    vv[k] = t_slices_sum(part, n, 6 + k, i, slices);
    aa[k] = t_slices_sum(part, n, 15 + k, i, slices);
  }
  const TD rxx = r[0], rxy = r[1], rxz = r[2], ryy = r[3], ryz = r[4], rzz = r[5];
  const TD denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy;
  const TD termnorm = TF(omega)[i] / TF(rho)[i];
  TD div_a, g[9];  // g[3a+b] = d v_a / d x_b
  if (::fabs(denom.v) > kFloatTiny) {
    const TD dd = 1.0 / denom;
    const TD txx = ryy * rzz - ryz * ryz, txy = rxz * ryz - rzz * rxy, txz = rxy * ryz - rxz * ryy;
    const TD tyy = rzz * rxx - rxz * rxz, tyz = rxy * rxz - rxx * ryz, tzz = rxx * ryy - rxy * rxy;
    const TD gax = (aa[0] * txx + aa[1] * txy + aa[2] * txz) * dd;
    const TD gay = (aa[3] * txy + aa[4] * tyy + aa[5] * tyz) * dd;
    const TD gaz = (aa[6] * txz + aa[7] * tyz + aa[8] * tzz) * dd;
    div_a = -(gax + gay + gaz);
    for (int a = 0; a < 3; a++) {
      g[3 * a + 0] = -((vv[3 * a] * txx + vv[3 * a + 1] * txy + vv[3 * a + 2] * txz) * dd);
      g[3 * a + 1] = -((vv[3 * a] * txy + vv[3 * a + 1] * tyy + vv[3 * a + 2] * tyz) * dd);
      g[3 * a + 2] = -((vv[3 * a] * txz + vv[3 * a + 1] * tyz + vv[3 * a + 2] * tzz) * dd);
    }
  } else {
    div_a = -termnorm * (aa[0] + aa[4] + aa[8]);
    for (int k = 0; k < 9; k++) g[k] = -termnorm * vv[k];
  }
  const TD divvdt = div_a - (g[0] * g[0] + g[4] * g[4] + g[8] * g[8] +
                             2.0 * (g[1] * g[3] + g[2] * g[6] + g[5] * g[7]));
  const TD divv = g[0] + g[4] + g[8];
  const TD curlx = g[7] - g[5], curly = g[2] - g[6], curlz = g[3] - g[1];
  const TD compression = pmax(-divv, TD(0.0));
  const TD fac = compression * compression;
  const TD trace_s = curlx * curlx + curly * curly + curlz * curlz;
  const TD denominator = fac + trace_s;
  const TD xi = denominator > 0.0 ? fac / denominator : TD(1.0);
  const TD source = 10.0 * hi * hi * xi * pmax(-divvdt, TD(0.0));
  const TD cs = TF(cs)[i];
  const TD temp = cs * cs;
  TF(alphaloc)[i] = pmax(pmin(source / temp, alpha_max), TD(P.alpha_min));
  TF(divvdt)[i] = divvdt;
  TF(xilimiter)[i] = xi;
}

// ------------------------------------------------ G6-G10 force groups
// MHDAccelerations, SmoothingLengthRateFromForceDivergence,
// MagneticStressAccelerations, MagneticStateRates (src/equations.py:198-280,
// 133-140, 143-195, 488-567) in one neighbour loop with the accumulations
// of each group kept apart, then EnergyLimiter, DivBCorrection and
// AdaptiveTimestep (src/equations.py:588-624, 570-585).
// The i-side values of the force groups, shared by the pair and post-loop
// kernels (a macro, so that both read as the one loop they split).
#define T_FORCE_SIDE_I                                                                                        \
  const double beta = 2.0, mu0 = P.mu0;                                                                       \
  const TD hi = TF(h)[ii], rhoi = TF(rho)[ii], p_i = TF(p)[ii], omegai = TF(omega)[ii], csi = TF(cs)[ii];      \
  const TD bi[3] = {TF(Bx)[ii], TF(By)[ii], TF(Bz)[ii]};                                                       \
  const TD vi[3] = {TF(upred)[ii], TF(vpred)[ii], TF(wpred)[ii]};                                              \
  const TD epi = TF(epred)[ii], alphai = TF(alpha1)[ii], psii = TF(psipred)[ii];                               \
  const TD bi2 = bi[0] * bi[0] + bi[1] * bi[1] + bi[2] * bi[2];                                                \
  const TD vwave_i = sqrt(csi * csi + bi2 / (mu0 * rhoi));                                                     \
  const TD brhoi[3] = {bi[0] / rhoi, bi[1] / rhoi, bi[2] / rhoi};                                              \
  const TD bro2_i = (brhoi[0] * brhoi[0] + brhoi[1] * brhoi[1] + brhoi[2] * brhoi[2]) / mu0;                   \
  const TD rho_i2_inv = 1.0 / (rhoi * rhoi);                                                                   \
  const TD ch_i = P.clean_speed * vwave_i;

// Partial records of the force pair kernel: the 14 sums, dt_cfl and the
// index of the pair that set it (so that the slices' maxima combine to the
// first maximum in ascending j, as one loop over all pairs gives).
enum { TF_A6 = 0, TF_A8 = 3, TF_AE6 = 6, TF_AE9 = 7, TF_DIV = 8, TF_AB = 9, TF_DIVBS = 12, TF_DIVBD = 13,
       TF_DTCFL = 14, TF_JMAX = 15 };

template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_t_force_pair(int n, DevParams P, MhdState s, TD* __restrict__ part, TGrid tg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < n;
  TD a6[3] = {TD(0.0), TD(0.0), TD(0.0)}, a8[3] = {TD(0.0), TD(0.0), TD(0.0)};
  TD ae6(0.0), ae9(0.0), div(0.0), dtcfl(0.0), ab[3] = {TD(0.0), TD(0.0), TD(0.0)}, divbs(0.0), divbd(0.0);
  int jmax = INT_MAX;
  const int ii = act ? i : 0;
  T_FORCE_SIDE_I
  t_pairs<DIM>(tg, P, i, n, [&](int j) {
    TD xij[3], rij, dwi[3], dwj[3];
    pair_geometry<DIM>(P, s, i, j, xij, rij);
    t_kern_grad<K, DIM>(P.norm, xij, rij, hi, dwi);
    t_kern_grad<K, DIM>(P.norm, xij, rij, TF(h)[j], dwj);
    const TD mj = TF(m)[j], rhoj = TF(rho)[j], pj = TF(p)[j], omegaj = TF(omega)[j], csj = TF(cs)[j];
    const TD bj[3] = {TF(Bx)[j], TF(By)[j], TF(Bz)[j]};
    const TD dv[3] = {vi[0] - TF(upred)[j], vi[1] - TF(vpred)[j], vi[2] - TF(wpred)[j]};
    // ---- G6 MHDAccelerations (src/equations.py:217-275)
    {
      const TD rhoij = 0.5 * (rhoi + rhoj);
      const TD pibrhoi2 = p_i / (rhoi * rhoi), pjbrhoj2 = pj / (rhoj * rhoj);
      const TD bj2 = bj[0] * bj[0] + bj[1] * bj[1] + bj[2] * bj[2];
      const TD vwave_j = sqrt(csj * csj + bj2 / (mu0 * rhoj));
      TD run[3];
      if (rij < kInteractionDistanceEpsilon) {
        run[0] = run[1] = run[2] = TD(0.0);
      } else {
        run[0] = xij[0] / rij;
        run[1] = xij[1] / rij;
        run[2] = xij[2] / rij;
      }
      const TD dot = dv[0] * run[0] + dv[1] * run[1] + dv[2] * run[2];
      const TD grad_i = omegai * (run[0] * dwi[0] + run[1] * dwi[1] + run[2] * dwi[2]);
      const TD grad_j = omegaj * (run[0] * dwj[0] + run[1] * dwj[1] + run[2] * dwj[2]);
      div += mj * dot * grad_i;
      const TD pdiff = fabs(p_i - pj);
      const TD vsig2 = sqrt(pdiff / rhoij);
      TD c = vwave_i - beta * dot;
      c = pmax(c, vwave_j - beta * dot);
      c = pmax(c, TD(0.0));
      if (c > dtcfl || (c.v == dtcfl.v && j < jmax && jmax != INT_MAX)) {  // pmax, keeping the smallest j at the max
        dtcfl = c;
        jmax = j;
      }
      if (dot < 0.0) {
        const TD vav_i = pmax(alphai * vwave_i - beta * dot, TD(0.0));
        const TD vav_j = pmax(TF(alpha1)[j] * vwave_j - beta * dot, TD(0.0));
        const TD q_i = -0.5 / rhoi * vav_i * dot * P.av;
        const TD q_j = -0.5 / rhoj * vav_j * dot * P.av;
        for (int a = 0; a < 3; a++) a6[a] += -mj * (q_i * omegai * dwi[a] + q_j * omegaj * dwj[a]);
        ae6 += mj * q_i * dot * grad_i;
      }
      for (int a = 0; a < 3; a++) a6[a] += -mj * (pibrhoi2 * omegai * dwi[a] + pjbrhoj2 * omegaj * dwj[a]);
      const TD vdw = dv[0] * dwi[0] + dv[1] * dwi[1] + dv[2] * dwi[2];
      ae6 += mj * pibrhoi2 * omegai * vdw;
      const TD eij = epi - TF(epred)[j];
      ae6 += P.ac * vsig2 * eij * (0.5 * mj / rhoi * grad_i + 0.5 * mj / rhoj * grad_j);
    }
    // unit vector of the magnetic groups (src/equations.py:159-164, 513-518)
    TD run[3];
    if (rij > kPairDistanceEpsilon) {
      run[0] = xij[0] / rij;
      run[1] = xij[1] / rij;
      run[2] = xij[2] / rij;
    } else {
      run[0] = run[1] = run[2] = TD(0.0);
    }
    const TD grad_i = omegai * (run[0] * dwi[0] + run[1] * dwi[1] + run[2] * dwi[2]);
    const TD grad_j = omegaj * (run[0] * dwj[0] + run[1] * dwj[1] + run[2] * dwj[2]);
    // ---- G8 MagneticStressAccelerations (src/equations.py:149-195)
    {
      const TD brhoj[3] = {bj[0] / rhoj, bj[1] / rhoj, bj[2] / rhoj};
      const TD bro2_j = (brhoj[0] * brhoj[0] + brhoj[1] * brhoj[1] + brhoj[2] * brhoj[2]) / mu0;
      const TD gradp = mj * (0.5 * bro2_i * grad_i + 0.5 * bro2_j * grad_j);
      TD si[3][3], sj[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          si[a][b] = -mj * brhoi[a] * brhoi[b] / mu0;
          sj[a][b] = -mj * brhoj[a] * brhoj[b] / mu0;
        }
      for (int a = 0; a < 3; a++) {
        const TD proj = (si[a][0] * run[0] + si[a][1] * run[1] + si[a][2] * run[2]) * grad_i +
                        (sj[a][0] * run[0] + sj[a][1] * run[1] + sj[a][2] * run[2]) * grad_j;
        a8[a] += -run[a] * gradp - proj;
      }
    }
    // ---- G9 MagneticStateRates (src/equations.py:507-559)
    {
      const TD proj_bi = bi[0] * run[0] + bi[1] * run[1] + bi[2] * run[2];
      const TD proj_bj = bj[0] * run[0] + bj[1] * run[1] + bj[2] * run[2];
      const TD db[3] = {bi[0] - bj[0], bi[1] - bj[1], bi[2] - bj[2]};
      const TD proj_db = db[0] * run[0] + db[1] * run[1] + db[2] * run[2];
      const TD delta_b2 = db[0] * db[0] + db[1] * db[1] + db[2] * db[2];
      const TD rho_j2_inv = 1.0 / (rhoj * rhoj);
      const TD pgi = mj * rho_i2_inv * grad_i, pgj = mj * rho_j2_inv * grad_j;
      const TD d_brho = -(pgi * proj_bi);
      const TD projv = dv[0] * run[0] + dv[1] * run[1] + dv[2] * run[2];
      const TD dvt[3] = {dv[0] - projv * run[0], dv[1] - projv * run[1], dv[2] - projv * run[2]};
      const TD vsig_b = sqrt(dvt[0] * dvt[0] + dvt[1] * dvt[1] + dvt[2] * dvt[2]);
      const TD d_diss = 0.5 * (mj * rho_i2_inv * grad_i + mj * rho_j2_inv * grad_j) * vsig_b * P.ar;
      const TD bj2 = bj[0] * bj[0] + bj[1] * bj[1] + bj[2] * bj[2];
      const TD vwave_j = sqrt(csj * csj + bj2 / (mu0 * rhoj));
      const TD ch_j = P.clean_speed * vwave_j;
      const TD dpsi = pgi * psii * ch_i + pgj * TF(psipred)[j] * ch_j;
      for (int a = 0; a < 3; a++) ab[a] += d_brho * dv[a] + d_diss * db[a] - dpsi * run[a];
      ae9 += -0.5 * delta_b2 * d_diss / mu0;
      divbs += pgi * proj_bi + pgj * proj_bj;
      divbd += -mj * proj_db * grad_i;
    }
  });
  if (!act) return;
  for (int a = 0; a < 3; a++) {
    t_part(part, n, TF_A6 + a, i) = a6[a];
    t_part(part, n, TF_A8 + a, i) = a8[a];
    t_part(part, n, TF_AB + a, i) = ab[a];
  }
  t_part(part, n, TF_AE6, i) = ae6;
  t_part(part, n, TF_AE9, i) = ae9;
  t_part(part, n, TF_DIV, i) = div;
  t_part(part, n, TF_DIVBS, i) = divbs;
  t_part(part, n, TF_DIVBD, i) = divbd;
  t_part(part, n, TF_DTCFL, i) = dtcfl;
  t_part(part, n, TF_JMAX, i) = TD((double)jmax);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_t_force(int n, DevParams P, MhdState s, const TD* __restrict__ part,
                                                 int slices) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ii = i;
  T_FORCE_SIDE_I
  (void)beta;
  (void)omegai;
  (void)vi;
  (void)alphai;
  (void)bro2_i;
  (void)rho_i2_inv;
  TD a6[3], a8[3], ab[3];
  for (int a = 0; a < 3; a++) {
    a6[a] = t_slices_sum(part, n, TF_A6 + a, i, slices);
    a8[a] = t_slices_sum(part, n, TF_A8 + a, i, slices);
    ab[a] = t_slices_sum(part, n, TF_AB + a, i, slices);
  }
  const TD ae6 = t_slices_sum(part, n, TF_AE6, i, slices), ae9 = t_slices_sum(part, n, TF_AE9, i, slices);
  const TD div = t_slices_sum(part, n, TF_DIV, i, slices);
  const TD divbs = t_slices_sum(part, n, TF_DIVBS, i, slices), divbd = t_slices_sum(part, n, TF_DIVBD, i, slices);
  // the largest slice maximum; on a tie the one set by the smaller j
  TD dtcfl(0.0);
  double jbest = (double)INT_MAX;
  for (int sl = 0; sl < slices; sl++) {
    const TD v = part[((size_t)sl * kTWidth + TF_DTCFL) * n + i];
    const double jv = part[((size_t)sl * kTWidth + TF_JMAX) * n + i].v;
    if (v > dtcfl || (v.v == dtcfl.v && jv < jbest)) {
      dtcfl = v;
      jbest = jv;
    }
  }
  // G6 post (src/equations.py:278-280) and G7 (:133-140)
  const TD divv = -div / rhoi;
  TF(div)[i] = divv;
  TF(div_for_psi)[i] = divv;
  TF(ah)[i] = hi * divv * (1.0 / (double)DIM);
  // G9 post (src/equations.py:562-567)
  TF(aBevolx)[i] = ab[0];
  TF(aBevoly)[i] = ab[1];
  TF(aBevolz)[i] = ab[2];
  TF(divBdiff)[i] = divbd;
  TF(apsi)[i] = -ch_i * divbd / rhoi - P.clean_damp * psii * ch_i / hi - 0.5 * P.clean_active * psii * divv;
  dtcfl = pmax(dtcfl, vwave_i);
  dtcfl = pmax(dtcfl, ch_i);
  TF(dt_cfl)[i] = dtcfl;
  // G10: EnergyLimiter (src/equations.py:594-598)
  TD ae = ae6 + ae9;
  if (dtcfl > 0.0) {
    const TD dtc = P.c_cour * hi / dtcfl;
    if (epi + dtc * ae < 0.0 && epi > 0.0) ae = ae / (1.0 - dtc * ae / epi);
  }
  TF(ae)[i] = ae;
  // DivBCorrection (src/equations.py:607-624)
  TD frac(0.0);
  if (bi2 > 0.0) {
    const TD pbeta = 2.0 * mu0 * p_i / bi2;
    frac = pmax(TD(0.0), pmin(TD(1.0), (10.0 - pbeta) * 0.125));
  }
  TD acc[3];
  for (int a = 0; a < 3; a++) acc[a] = (a6[a] + a8[a]) + (-bi[a] * divbs * frac / mu0);
  TF(au)[i] = acc[0];
  TF(av)[i] = acc[1];
  TF(aw)[i] = acc[2];
  TF(divBsymm)[i] = rhoi * divbs;
  // AdaptiveTimestep (src/equations.py:578-585)
  TD dta(kBigNumber);
  if (dtcfl > 0.0) dta = P.c_cour * hi / dtcfl;
  const TD f2 = acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2];
  if (f2 > 0.0) dta = pmin(dta, P.c_force * sqrt(hi / sqrt(f2)));
  TF(dt_adapt)[i] = dta;
}

// --------------------------------------------------------- magnetic energy
// sum_i m_i |B_i|^2 / (2 mu0 rho_i): per-block partial sums, then one block
// adds the partials in order (deterministic).
__global__ void __launch_bounds__(256) k_t_energy_partial(int n, DevParams P, MhdState s, TD* __restrict__ part) {
  __shared__ double sh[MHD_TANGENT_DIRS + 1][256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  TD e(0.0);
  if (i < n) {
    const TD bx = TF(Bx)[i], by = TF(By)[i], bz = TF(Bz)[i];
    e = TF(m)[i] * (bx * bx + by * by + bz * bz) / (2.0 * P.mu0 * TF(rho)[i]);
  }
  sh[0][threadIdx.x] = e.v;
  for (int k = 0; k < MHD_TANGENT_DIRS; k++) sh[1 + k][threadIdx.x] = e.d[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k <= MHD_TANGENT_DIRS; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    TD r(sh[0][0]);
    for (int k = 0; k < MHD_TANGENT_DIRS; k++) r.d[k] = sh[1 + k][0];
    part[blockIdx.x] = r;
  }
}

__global__ void k_t_energy_final(int nb, const TD* __restrict__ part, TD* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  TD e(0.0);
  for (int b = 0; b < nb; b++) e = e + part[b];
  *out = e;
}

#undef TF

// ------------------------------------------------------------- launchers
// The grid of the current x and h for the next pair passes.
template <int DIM>
static TGrid t_grid(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  k_t_pack_pos<DIM><<<(n + 255) / 256, 256, 0, st>>>(n, *s, c->pgrid.pos);
  c->launches++;
  build_pair_grid(c, c->pgrid, n, st);
  return TGrid{c->pgrid.grid, c->pgrid.cell_start, c->pgrid.perm, c->pgrid.pos, derivative_slices(n)};
}

template <int K, int DIM>
static void t_rhs_launch(Ctx* c, MhdState* s, int n, TD amax, cudaStream_t st) {
  const int nb = (n + kTile - 1) / kTile, np = (n + 255) / 256;
  TD* h_new = reinterpret_cast<TD*>(c->tan_work);
  TD* part = h_new + c->n_max + 1024;  // slices * kTWidth records per particle
  TGrid tg = t_grid<DIM>(c, s, n, st);  // density pass: the h before it
  const dim3 sliced(nb, tg.slices);
  k_t_density_pair<K, DIM><<<sliced, kTile, 0, st>>>(n, c->P, *s, part, tg);
  k_t_density<DIM><<<np, 256, 0, st>>>(n, c->P, *s, part, h_new, tg.slices);
  k_t_prologue<DIM><<<np, 256, 0, st>>>(n, c->P, *s, h_new);
  tg = t_grid<DIM>(c, s, n, st);  // the later groups: the new h
  k_t_cd_pair<K, DIM><<<sliced, kTile, 0, st>>>(n, c->P, *s, part, tg);
  k_t_cd<<<np, 256, 0, st>>>(n, c->P, *s, part, amax, tg.slices);
  k_t_force_pair<K, DIM><<<sliced, kTile, 0, st>>>(n, c->P, *s, part, tg);
  k_t_force<DIM><<<np, 256, 0, st>>>(n, c->P, *s, part, tg.slices);
  c->launches += 7;
}

#define MHD_T_DISPATCH(...)                                                                                   \
  do {                                                                                                        \
    const int d3 = c->P.dim == 3;                                                                             \
    switch (c->P.kernel) {                                                                                    \
      case MHD_KERNEL_CUBIC: d3 ? t_rhs_launch<0, 3>(__VA_ARGS__) : t_rhs_launch<0, 2>(__VA_ARGS__); break;   \
      case MHD_KERNEL_QUINTIC: d3 ? t_rhs_launch<1, 3>(__VA_ARGS__) : t_rhs_launch<1, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C2: d3 ? t_rhs_launch<2, 3>(__VA_ARGS__) : t_rhs_launch<2, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C4: d3 ? t_rhs_launch<3, 3>(__VA_ARGS__) : t_rhs_launch<3, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C6: d3 ? t_rhs_launch<4, 3>(__VA_ARGS__) : t_rhs_launch<4, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_GAUSSIAN: d3 ? t_rhs_launch<5, 3>(__VA_ARGS__) : t_rhs_launch<5, 2>(__VA_ARGS__); break; \
      default: d3 ? t_rhs_launch<6, 3>(__VA_ARGS__) : t_rhs_launch<6, 2>(__VA_ARGS__); break;                 \
    }                                                                                                         \
  } while (0)

}  // namespace mhd

using namespace mhd;

namespace {

#define T_FAIL(code, msg) \
  do {                    \
    c->err = (msg);       \
    return (code);        \
  } while (0)
#define T_CK(call)                                                   \
  do {                                                               \
    cudaError_t e_ = (call);                                         \
    if (e_ != cudaSuccess) {                                         \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);   \
      return MHD_ERR_CUDA;                                           \
    }                                                                \
  } while (0)

const char* const kTangentFields[] = {
    "x", "y", "z", "u", "v", "w", "e", "h", "h0", "m", "rho", "rho_sum", "p", "cs", "omega", "converged",
    "upred", "vpred", "wpred", "epred", "Bevolx", "Bevoly", "Bevolz", "Bevolxpred", "Bevolypred", "Bevolzpred",
    "psi", "psipred", "alpha1", "alphaloc", "au", "av", "aw", "ae", "ah", "aBevolx", "aBevoly", "aBevolz", "apsi",
    "Bx", "By", "Bz", "div", "div_for_psi", "dt_cfl", "dt_adapt", "divBsymm", "divBdiff", "divvdt", "xilimiter"};

int check_tangent(Ctx* c, const MhdState* s, int64_t n) {
  if (!s) T_FAIL(MHD_ERR_INVALID, "state is null");
  if (n < 1 || n > c->n_max) T_FAIL(MHD_ERR_INVALID, "n must be in [1, n_max]");
  if (c->P.iterate) T_FAIL(MHD_ERR_INVALID, "the derivative form needs the single density pass (iterate = 0)");
  const double* const* f = reinterpret_cast<const double* const*>(s);
  for (const char* name : kTangentFields) {
    for (int k = 0; k < mhd_state_field_count(); k++)
      if (!strcmp(mhd_state_field_name(k), name) && !f[k])
        T_FAIL(MHD_ERR_INVALID, std::string("tangent state field ") + name + " is null");
  }
  if (!s->itype) T_FAIL(MHD_ERR_INVALID, "itype is null");
  if (!c->tan_work) {
    // new h (n_max + 1024 records), then the pair kernels' partial sums
    T_CK(cudaMalloc(&c->tan_work,
                    sizeof(TD) * ((size_t)c->n_max + 1024 + derivative_slice_records(c->n_max) * kTWidth)));
  }
  if (alloc_pair_grid(c->pgrid, c->n_max) != MHD_OK) T_FAIL(MHD_ERR_CUDA, "pair grid allocation failed");
  return MHD_OK;
}

TD dual_of(const double* a) {
  TD r(a ? a[0] : 0.0);
  for (int k = 0; k < MHD_TANGENT_DIRS; k++) r.d[k] = a ? a[1 + k] : 0.0;
  return r;
}

}  // namespace

extern "C" {

int mhd_tangent_dirs(void) { return MHD_TANGENT_DIRS; }

int mhd_tangent_sync(void* ctx, MhdState* s, int64_t n, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  int rc = check_tangent(c, s, n);
  if (rc != MHD_OK) return rc;
  k_t_sync<<<(int)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>((int)n, *s);
  c->launches++;
  T_CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_tangent_rhs(void* ctx, MhdState* s, int64_t n, const double* alpha_max, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  int rc = check_tangent(c, s, n);
  if (rc != MHD_OK) return rc;
  TD amax = alpha_max ? dual_of(alpha_max) : TD(c->P.alpha_max);
  MHD_T_DISPATCH(c, s, (int)n, amax, (cudaStream_t)stream);
  T_CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_tangent_step(void* ctx, MhdState* s, int64_t n, double dt, const double* alpha_max, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  int rc = check_tangent(c, s, n);
  if (rc != MHD_OK) return rc;
  if (!(dt >= 0.0) || !isfinite(dt)) T_FAIL(MHD_ERR_INVALID, "dt must be finite and >= 0");
  const cudaStream_t st = (cudaStream_t)stream;
  const int np = (int)((n + 255) / 256);
  k_t_predict<<<np, 256, 0, st>>>((int)n, c->P, *s, dt);
  TD amax = alpha_max ? dual_of(alpha_max) : TD(c->P.alpha_max);
  MHD_T_DISPATCH(c, s, (int)n, amax, st);
  k_t_correct<<<np, 256, 0, st>>>((int)n, c->P, *s, dt);
  c->launches += 2;
  T_CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_tangent_magnetic_energy(void* ctx, const MhdState* s, int64_t n, double* energy, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (!energy) T_FAIL(MHD_ERR_INVALID, "energy is null");
  int rc = check_tangent(c, s, n);
  if (rc != MHD_OK) return rc;
  const cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)((n + 255) / 256);
  TD* part = reinterpret_cast<TD*>(c->tan_work);  // the energy needs no h_new
  TD* out = part + nb;
  k_t_energy_partial<<<nb, 256, 0, st>>>((int)n, c->P, *s, part);
  k_t_energy_final<<<1, 32, 0, st>>>(nb, part, out);
  c->launches += 2;
  T_CK(cudaGetLastError());
  TD host;
  T_CK(cudaMemcpyAsync(&host, out, sizeof(TD), cudaMemcpyDeviceToHost, st));
  T_CK(cudaStreamSynchronize(st));
  energy[0] = host.v;
  for (int k = 0; k < MHD_TANGENT_DIRS; k++) energy[1 + k] = host.d[k];
  return MHD_OK;
}

}  // extern "C"
