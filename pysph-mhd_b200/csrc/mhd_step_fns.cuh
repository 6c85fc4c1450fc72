// mhd_step_fns.cuh -- the SPMHD step as pure functions over a scalar type.
//
// One restatement of the reference's equations for the derivative forms:
// instantiated on double (values), on Dual<N> for forward-mode tangents, and
// on Dual<k> seeded per input for the local Jacobians the adjoint contracts.
// Each function names the reference lines it follows.  Pair functions take
// the two particles' inputs and the minimum-image x_ij and accumulate into
// per-particle sums; post functions turn sums into outputs.
#pragma once

#include "mhd_common.cuh"
#include "mhd_dual.cuh"

namespace mhd {

template <class D>
__device__ inline D pmax(const D& a, const D& b) { return b > a ? b : a; }
template <class D>
__device__ inline D pmin(const D& a, const D& b) { return b < a ? b : a; }

// ---------------------------------------------------------- SPH kernels
// PySPH's kernel interface (restated): sigma / h^dim, W = sigma w(q) / h^dim,
// grad W = sigma w'(q) / h^(dim+1) x_ij / r_ij (0 for r_ij <= 1e-12),
// dW/dh = -sigma / h^(dim+1) (w' q + dim w).
template <int DIM, class D>
__device__ inline D f_hfac(double norm, const D& h1) {
  return DIM == 2 ? norm * h1 * h1 : norm * h1 * h1 * h1;
}
template <int K, int DIM, class D>
__device__ inline D f_kern_w(double norm, const D& r, const D& h) {
  const D h1 = 1.0 / h, q = r * h1;
  D w, dw;
  w_dw<K, D>(q, DIM, w, dw);
  return w * f_hfac<DIM>(norm, h1);
}
template <int K, int DIM, class D>
__device__ inline void f_kern_grad(double norm, const D* xij, const D& r, const D& h, D* g) {
  const D h1 = 1.0 / h;
  D tmp(0.0);
  if (r > 1.0e-12) {
    const D q = r * h1;
    D w, dw;
    w_dw<K, D>(q, DIM, w, dw);
    tmp = f_hfac<DIM>(norm, h1) * dw * h1 / r;
  }
  g[0] = tmp * xij[0];
  g[1] = tmp * xij[1];
  g[2] = tmp * xij[2];
}
template <int K, int DIM, class D>
__device__ inline D f_kern_gradh(double norm, const D& r, const D& h) {
  const D h1 = 1.0 / h, q = r * h1;
  D w, dw;
  w_dw<K, D>(q, DIM, w, dw);
  return -(f_hfac<DIM>(norm, h1) * h1 * (dw * q + w * (double)DIM));
}

template <class D>
__device__ inline D f_norm(const D* x) {
  return gsqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
}

// ------------------------------------------------- G1 density (one pass)
// Pair: rho += m_j W(r, h_i), dwdh += m_j dW/dh(r, h_i) (src/equations.py:38-50).
template <int K, int DIM, class D>
__device__ inline void f_density_pair(double norm, const D* xij, const D& hi, const D& mj, D& rho, D& dwdh) {
  const D r = f_norm(xij);
  rho += mj * f_kern_w<K, DIM>(norm, r, hi);
  dwdh += mj * f_kern_gradh<K, DIM>(norm, r, hi);
}
// Post of the single pass (src/equations.py:53-88 with iterate_only_once):
// Omega from the old h, then h = hfact (m / rho)^(1/dim).
template <int DIM, class D>
__device__ inline void f_density_post(double hfact, const D& hi, const D& mi, const D& rho, const D& dwdh,
                                      D& omega, D& hnew) {
  const D hk = hi / hfact;
  const D rhoi = mi / (DIM == 2 ? hk * hk : hk * hk * hk);
  const D dhdrhoi = -hi / ((double)DIM * rhoi);
  const D omegai = 1.0 - dhdrhoi * dwdh;
  omega = 1.0 / omegai;
  hnew = hfact * gpow(mi / rho, 1.0 / (double)DIM);
}

// G2, G3, G5 (src/equations.py:109-118, 97-106, 474-485).
template <int DIM, class D>
__device__ inline void f_prologue(const DevParams& P, const D& h, const D& m, const D& epred, const D* bevpred,
                                  D& rho, D& p, D& cs, D* b) {
  const D hk = h / P.hfact;
  rho = m / (DIM == 2 ? hk * hk : hk * hk * hk);
  p = P.gamma1 * rho * epred;
  cs = gsqrt(P.gamma * p / rho);
  for (int a = 0; a < 3; a++) b[a] = bevpred[a] * rho;
}

// ---------------------------------------- G4 Cullen-Dehnen diagnostics
// Pair (src/equations.py:318-354): r[6] = -x_a m grad_b W (upper triangle),
// vv[3a+b] = dv_a m grad_b W, aa[3a+b] = da_a m grad_b W, grad W at h_i.
template <int K, int DIM, class D>
__device__ inline void f_cd_pair(double norm, const D* xij, const D& hi, const D& mj, const D* dv, const D* da, D* r,
                                 D* vv, D* aa) {
  const D rij = f_norm(xij);
  D dwi[3];
  f_kern_grad<K, DIM>(norm, xij, rij, hi, dwi);
  const D run[3] = {mj * dwi[0], mj * dwi[1], mj * dwi[2]};
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
}
// Post (src/equations.py:357-429): velocity gradient (3x3 inverse, or the
// -Omega/rho fallback when |det| <= FLOAT_TINY), d(div v)/dt, the limiter xi
// and alpha_loc clipped to [alpha_min, alpha_max].
template <class D>
__device__ inline D f_cd_post(const D* r, const D* vv, const D* aa, const D& omega, const D& rho, const D& h,
                              const D& cs, const D& alpha_max, double alpha_min, D* divvdt_out = nullptr,
                              D* xi_out = nullptr) {
  const D rxx = r[0], rxy = r[1], rxz = r[2], ryy = r[3], ryz = r[4], rzz = r[5];
  const D denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy;
  const D termnorm = omega / rho;
  D div_a, g[9];
  if (::fabs(val(denom)) > kFloatTiny) {
    const D dd = 1.0 / denom;
    const D txx = ryy * rzz - ryz * ryz, txy = rxz * ryz - rzz * rxy, txz = rxy * ryz - rxz * ryy;
    const D tyy = rzz * rxx - rxz * rxz, tyz = rxy * rxz - rxx * ryz, tzz = rxx * ryy - rxy * rxy;
    const D gax = (aa[0] * txx + aa[1] * txy + aa[2] * txz) * dd;
    const D gay = (aa[3] * txy + aa[4] * tyy + aa[5] * tyz) * dd;
    const D gaz = (aa[6] * txz + aa[7] * tyz + aa[8] * tzz) * dd;
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
  const D divvdt = div_a - (g[0] * g[0] + g[4] * g[4] + g[8] * g[8] + 2.0 * (g[1] * g[3] + g[2] * g[6] + g[5] * g[7]));
  const D divv = g[0] + g[4] + g[8];
  const D curlx = g[7] - g[5], curly = g[2] - g[6], curlz = g[3] - g[1];
  const D compression = pmax(-divv, D(0.0));
  const D fac = compression * compression;
  const D trace_s = curlx * curlx + curly * curly + curlz * curlz;
  const D denominator = fac + trace_s;
  const D xi = denominator > 0.0 ? fac / denominator : D(1.0);
  const D source = 10.0 * h * h * xi * pmax(-divvdt, D(0.0));
  if (divvdt_out) *divvdt_out = divvdt;
  if (xi_out) *xi_out = xi;
  return pmax(pmin(source / (cs * cs), alpha_max), D(alpha_min));
}

// The vector-Jacobian product of f_cd_pair, written out by hand: weights w
// on its 24 sums (r 6, vv 9, aa 9) give g over (x_ij 3, h_i, dv 3, da 3);
// the kernel gradient's Jacobian comes from a 4-direction dual evaluation.
template <int K, int DIM>
__device__ inline void vjp_cd_pair(double norm, const double* x, double hi, double mj, const double* dv,
                                   const double* da, const double* w, double* g) {
  const double r = f_norm(x);
  double dwi[3];
  f_kern_grad<K, DIM>(norm, x, r, hi, dwi);
  const double run[3] = {mj * dwi[0], mj * dwi[1], mj * dwi[2]};
  double run_[3] = {}, x_[3] = {};
  // r[6] = -x_a run_b over (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
  const int ra[6] = {0, 0, 0, 1, 1, 2}, rb[6] = {0, 1, 2, 1, 2, 2};
  for (int q = 0; q < 6; q++) {
    run_[rb[q]] -= w[q] * x[ra[q]];
    x_[ra[q]] -= w[q] * run[rb[q]];
  }
  for (int a = 0; a < 3; a++) {
    double dv_ = 0.0, da_ = 0.0;
    for (int b = 0; b < 3; b++) {
      dv_ += w[6 + 3 * a + b] * run[b];
      da_ += w[15 + 3 * a + b] * run[b];
      run_[b] += w[6 + 3 * a + b] * dv[a] + w[15 + 3 * a + b] * da[a];
    }
    g[4 + a] = dv_;
    g[7 + a] = da_;
  }
  using D4 = Dual<4>;
  D4 xd[3];
  for (int a = 0; a < 3; a++) {
    xd[a] = D4(x[a]);
    xd[a].d[a] = 1.0;
  }
  D4 hd(hi);
  hd.d[3] = 1.0;
  D4 gd[3];
  f_kern_grad<K, DIM>(norm, xd, f_norm(xd), hd, gd);
  g[3] = 0.0;
  for (int a = 0; a < 3; a++) g[a] = x_[a];
  for (int b = 0; b < 3; b++) {
    const double dwi_ = mj * run_[b];
    for (int a = 0; a < 3; a++) g[a] += dwi_ * gd[b].d[a];
    g[3] += dwi_ * gd[b].d[3];
  }
}

// ------------------------------------------------- G6-G10 force groups
// The per-particle inputs of the force pair loop.
template <class D>
struct Side {
  D h, rho, p, omega, cs, b[3], v[3], e, alpha, psi;
};
constexpr int kSideDirs = 14;  // h rho p omega cs b3 v3 e alpha psi

template <class D>
struct FSums {
  D a6[3], a8[3], ae6, ae9, div, ab[3], divbs, divbd;
  D dtcfl;
  __device__ void zero() {
    for (int a = 0; a < 3; a++) a6[a] = a8[a] = ab[a] = D(0.0);
    ae6 = ae9 = div = divbs = divbd = dtcfl = D(0.0);
  }
};
constexpr int kFSumDirs = 14;  // a6 3, a8 3, ae6, ae9, div, ab 3, divbs, divbd (dtcfl is not differentiated)

// The differentiated sums in that order, as pointers into the struct.
template <class D>
__device__ inline void fsum_ptrs(FSums<D>& S, D** p) {
  p[0] = &S.a6[0];
  p[1] = &S.a6[1];
  p[2] = &S.a6[2];
  p[3] = &S.a8[0];
  p[4] = &S.a8[1];
  p[5] = &S.a8[2];
  p[6] = &S.ae6;
  p[7] = &S.ae9;
  p[8] = &S.div;
  p[9] = &S.ab[0];
  p[10] = &S.ab[1];
  p[11] = &S.ab[2];
  p[12] = &S.divbs;
  p[13] = &S.divbd;
}

// MHDAccelerations, MagneticStressAccelerations, MagneticStateRates pair
// terms (src/equations.py:217-275, 149-195, 507-559).
template <int K, int DIM, class D>
__device__ inline void f_force_pair(const DevParams& P, const Side<D>& I, const Side<D>& J, const D& mj, const D* xij,
                                    FSums<D>& S) {
  const double beta = 2.0, mu0 = P.mu0;
  const D rij = f_norm(xij);
  D dwi[3], dwj[3];
  f_kern_grad<K, DIM>(P.norm, xij, rij, I.h, dwi);
  f_kern_grad<K, DIM>(P.norm, xij, rij, J.h, dwj);
  const D dv[3] = {I.v[0] - J.v[0], I.v[1] - J.v[1], I.v[2] - J.v[2]};
  const D bi2 = I.b[0] * I.b[0] + I.b[1] * I.b[1] + I.b[2] * I.b[2];
  const D bj2 = J.b[0] * J.b[0] + J.b[1] * J.b[1] + J.b[2] * J.b[2];
  const D vwave_i = gsqrt(I.cs * I.cs + bi2 / (mu0 * I.rho));
  const D vwave_j = gsqrt(J.cs * J.cs + bj2 / (mu0 * J.rho));
  {  // G6
    const D rhoij = 0.5 * (I.rho + J.rho);
    const D pibrhoi2 = I.p / (I.rho * I.rho), pjbrhoj2 = J.p / (J.rho * J.rho);
    D run[3];
    if (rij < kInteractionDistanceEpsilon) {
      run[0] = run[1] = run[2] = D(0.0);
    } else {
      for (int a = 0; a < 3; a++) run[a] = xij[a] / rij;
    }
    const D dot = dv[0] * run[0] + dv[1] * run[1] + dv[2] * run[2];
    const D grad_i = I.omega * (run[0] * dwi[0] + run[1] * dwi[1] + run[2] * dwi[2]);
    const D grad_j = J.omega * (run[0] * dwj[0] + run[1] * dwj[1] + run[2] * dwj[2]);
    S.div += mj * dot * grad_i;
    const D vsig2 = gsqrt(gfabs(I.p - J.p) / rhoij);
    D c = vwave_i - beta * dot;
    c = pmax(c, vwave_j - beta * dot);
    c = pmax(c, D(0.0));
    S.dtcfl = pmax(S.dtcfl, c);
    if (dot < 0.0) {
      const D vav_i = pmax(I.alpha * vwave_i - beta * dot, D(0.0));
      const D vav_j = pmax(J.alpha * vwave_j - beta * dot, D(0.0));
      const D q_i = -0.5 / I.rho * vav_i * dot * P.av;
      const D q_j = -0.5 / J.rho * vav_j * dot * P.av;
      for (int a = 0; a < 3; a++) S.a6[a] += -mj * (q_i * I.omega * dwi[a] + q_j * J.omega * dwj[a]);
      S.ae6 += mj * q_i * dot * grad_i;
    }
    for (int a = 0; a < 3; a++) S.a6[a] += -mj * (pibrhoi2 * I.omega * dwi[a] + pjbrhoj2 * J.omega * dwj[a]);
    S.ae6 += mj * pibrhoi2 * I.omega * (dv[0] * dwi[0] + dv[1] * dwi[1] + dv[2] * dwi[2]);
    S.ae6 += P.ac * vsig2 * (I.e - J.e) * (0.5 * mj / I.rho * grad_i + 0.5 * mj / J.rho * grad_j);
  }
  D run[3];
  if (rij > kPairDistanceEpsilon) {
    for (int a = 0; a < 3; a++) run[a] = xij[a] / rij;
  } else {
    run[0] = run[1] = run[2] = D(0.0);
  }
  const D grad_i = I.omega * (run[0] * dwi[0] + run[1] * dwi[1] + run[2] * dwi[2]);
  const D grad_j = J.omega * (run[0] * dwj[0] + run[1] * dwj[1] + run[2] * dwj[2]);
  {  // G8
    const D brhoi[3] = {I.b[0] / I.rho, I.b[1] / I.rho, I.b[2] / I.rho};
    const D brhoj[3] = {J.b[0] / J.rho, J.b[1] / J.rho, J.b[2] / J.rho};
    const D bro2_i = (brhoi[0] * brhoi[0] + brhoi[1] * brhoi[1] + brhoi[2] * brhoi[2]) / mu0;
    const D bro2_j = (brhoj[0] * brhoj[0] + brhoj[1] * brhoj[1] + brhoj[2] * brhoj[2]) / mu0;
    const D gradp = mj * (0.5 * bro2_i * grad_i + 0.5 * bro2_j * grad_j);
    for (int a = 0; a < 3; a++) {
      D pi(0.0), pj(0.0);
      for (int b = 0; b < 3; b++) {
        pi += (-mj * brhoi[a] * brhoi[b] / mu0) * run[b];
        pj += (-mj * brhoj[a] * brhoj[b] / mu0) * run[b];
      }
      S.a8[a] += -run[a] * gradp - (pi * grad_i + pj * grad_j);
    }
  }
  {  // G9
    const D proj_bi = I.b[0] * run[0] + I.b[1] * run[1] + I.b[2] * run[2];
    const D proj_bj = J.b[0] * run[0] + J.b[1] * run[1] + J.b[2] * run[2];
    const D db[3] = {I.b[0] - J.b[0], I.b[1] - J.b[1], I.b[2] - J.b[2]};
    const D proj_db = db[0] * run[0] + db[1] * run[1] + db[2] * run[2];
    const D delta_b2 = db[0] * db[0] + db[1] * db[1] + db[2] * db[2];
    const D rho_i2_inv = 1.0 / (I.rho * I.rho), rho_j2_inv = 1.0 / (J.rho * J.rho);
    const D pgi = mj * rho_i2_inv * grad_i, pgj = mj * rho_j2_inv * grad_j;
    const D d_brho = -(pgi * proj_bi);
    const D projv = dv[0] * run[0] + dv[1] * run[1] + dv[2] * run[2];
    const D dvt[3] = {dv[0] - projv * run[0], dv[1] - projv * run[1], dv[2] - projv * run[2]};
    const D vsig_b = f_norm(dvt);
    const D d_diss = 0.5 * (mj * rho_i2_inv * grad_i + mj * rho_j2_inv * grad_j) * vsig_b * P.ar;
    const D dpsi = pgi * I.psi * (P.clean_speed * vwave_i) + pgj * J.psi * (P.clean_speed * vwave_j);
    for (int a = 0; a < 3; a++) S.ab[a] += d_brho * dv[a] + d_diss * db[a] - dpsi * run[a];
    S.ae9 += -0.5 * delta_b2 * d_diss / mu0;
    S.divbs += pgi * proj_bi + pgj * proj_bj;
    S.divbd += -mj * proj_db * grad_i;
  }
}

// The vector-Jacobian product of f_force_pair, written out by hand: given
// weights w on the 14 differentiated sums (fsum_ptrs order), the gradients
// of sum_q w_q S_q with respect to the i side (gI), the j side (gJ) and
// x_ij (gx), each in Side order (h rho p omega cs b3 v3 e alpha psi).  The
// kernel gradients' own Jacobians come from a 4-direction dual evaluation
// (x_ij and h).  Derivative conventions follow the dual numbers: sqrt and
// |.| have zero derivative at 0, max(a, b) passes a's derivative when a >= b.
template <int K, int DIM>
__device__ inline void vjp_force_pair(const DevParams& P, const Side<double>& I, const Side<double>& J, double mj,
                                      const double* x, const double* w, double* gI, double* gJ, double* gx) {
  const double beta = 2.0, mu0 = P.mu0, ch = P.clean_speed;
  const double wa6[3] = {w[0], w[1], w[2]}, wa8[3] = {w[3], w[4], w[5]};
  const double wae6 = w[6], wae9 = w[7], wdiv = w[8];
  const double wab[3] = {w[9], w[10], w[11]}, wdivbs = w[12], wdivbd = w[13];
  for (int d = 0; d < kSideDirs; d++) gI[d] = gJ[d] = 0.0;
  gx[0] = gx[1] = gx[2] = 0.0;
  // ---- forward values
  const double r = f_norm(x);
  double dwi[3], dwj[3];
  f_kern_grad<K, DIM>(P.norm, x, r, I.h, dwi);
  f_kern_grad<K, DIM>(P.norm, x, r, J.h, dwj);
  const double dv[3] = {I.v[0] - J.v[0], I.v[1] - J.v[1], I.v[2] - J.v[2]};
  const double bi2 = I.b[0] * I.b[0] + I.b[1] * I.b[1] + I.b[2] * I.b[2];
  const double bj2 = J.b[0] * J.b[0] + J.b[1] * J.b[1] + J.b[2] * J.b[2];
  const double si = I.cs * I.cs + bi2 / (mu0 * I.rho), sj = J.cs * J.cs + bj2 / (mu0 * J.rho);
  const double vwi = ::sqrt(si), vwj = ::sqrt(sj);
  const double rhoij = 0.5 * (I.rho + J.rho);
  const double pri = I.p / (I.rho * I.rho), prj = J.p / (J.rho * J.rho);
  const bool near6 = r < kInteractionDistanceEpsilon;
  double run6[3];
  for (int a = 0; a < 3; a++) run6[a] = near6 ? 0.0 : x[a] / r;
  const double dot = dv[0] * run6[0] + dv[1] * run6[1] + dv[2] * run6[2];
  const double gi6 = I.omega * (run6[0] * dwi[0] + run6[1] * dwi[1] + run6[2] * dwi[2]);
  const double gj6 = J.omega * (run6[0] * dwj[0] + run6[1] * dwj[1] + run6[2] * dwj[2]);
  const double dp = I.p - J.p;
  const double va = ::fabs(dp) / rhoij;
  const double vsig2 = ::sqrt(va);
  const bool av = dot < 0.0;
  const double ti = I.alpha * vwi - beta * dot, tj = J.alpha * vwj - beta * dot;
  const double vav_i = ti >= 0.0 ? ti : 0.0, vav_j = tj >= 0.0 ? tj : 0.0;
  const double q_i = -0.5 / I.rho * vav_i * dot * P.av, q_j = -0.5 / J.rho * vav_j * dot * P.av;
  const double de = I.e - J.e;
  const double tc = 0.5 * mj / I.rho * gi6 + 0.5 * mj / J.rho * gj6;
  const double udw = dv[0] * dwi[0] + dv[1] * dwi[1] + dv[2] * dwi[2];
  const bool far8 = r > kPairDistanceEpsilon;
  double run8[3];
  for (int a = 0; a < 3; a++) run8[a] = far8 ? x[a] / r : 0.0;
  const double gi = I.omega * (run8[0] * dwi[0] + run8[1] * dwi[1] + run8[2] * dwi[2]);
  const double gj = J.omega * (run8[0] * dwj[0] + run8[1] * dwj[1] + run8[2] * dwj[2]);
  const double bri[3] = {I.b[0] / I.rho, I.b[1] / I.rho, I.b[2] / I.rho};
  const double brj[3] = {J.b[0] / J.rho, J.b[1] / J.rho, J.b[2] / J.rho};
  const double bro2_i = (bri[0] * bri[0] + bri[1] * bri[1] + bri[2] * bri[2]) / mu0;
  const double bro2_j = (brj[0] * brj[0] + brj[1] * brj[1] + brj[2] * brj[2]) / mu0;
  const double gradp = mj * (0.5 * bro2_i * gi + 0.5 * bro2_j * gj);
  const double si8 = bri[0] * run8[0] + bri[1] * run8[1] + bri[2] * run8[2];
  const double sj8 = brj[0] * run8[0] + brj[1] * run8[1] + brj[2] * run8[2];
  const double cm = -mj / mu0;
  const double proj_bi = I.b[0] * run8[0] + I.b[1] * run8[1] + I.b[2] * run8[2];
  const double proj_bj = J.b[0] * run8[0] + J.b[1] * run8[1] + J.b[2] * run8[2];
  const double db[3] = {I.b[0] - J.b[0], I.b[1] - J.b[1], I.b[2] - J.b[2]};
  const double proj_db = db[0] * run8[0] + db[1] * run8[1] + db[2] * run8[2];
  const double delta_b2 = db[0] * db[0] + db[1] * db[1] + db[2] * db[2];
  const double ri2 = 1.0 / (I.rho * I.rho), rj2 = 1.0 / (J.rho * J.rho);
  const double pgi = mj * ri2 * gi, pgj = mj * rj2 * gj;
  const double d_brho = -(pgi * proj_bi);
  const double projv = dv[0] * run8[0] + dv[1] * run8[1] + dv[2] * run8[2];
  const double dvt[3] = {dv[0] - projv * run8[0], dv[1] - projv * run8[1], dv[2] - projv * run8[2]};
  const double vsig_b = f_norm(dvt);
  const double d_diss = 0.5 * (pgi + pgj) * vsig_b * P.ar;
  const double dpsi = pgi * I.psi * (ch * vwi) + pgj * J.psi * (ch * vwj);
  // ---- reverse
  double r_ = 0.0, dwi_[3] = {}, dwj_[3] = {}, dv_[3] = {}, run6_[3] = {}, run8_[3] = {};
  double vwi_ = 0.0, vwj_ = 0.0, gi_ = 0.0, gj_ = 0.0, gi6_ = 0.0, gj6_ = 0.0, dot_ = 0.0;
  double Ib_[3] = {}, Jb_[3] = {};
  // G9
  double proj_db_ = wdivbd * (-mj * gi);
  gi_ += wdivbd * (-mj * proj_db);
  double pgi_ = wdivbs * proj_bi, pgj_ = wdivbs * proj_bj;
  double proj_bi_ = wdivbs * pgi, proj_bj_ = wdivbs * pgj;
  double delta_b2_ = wae9 * (-0.5 * d_diss / mu0);
  double d_diss_ = wae9 * (-0.5 * delta_b2 / mu0);
  double d_brho_ = 0.0, dpsi_ = 0.0, db_[3] = {};
  for (int a = 0; a < 3; a++) {
    d_brho_ += wab[a] * dv[a];
    dv_[a] += wab[a] * d_brho;
    d_diss_ += wab[a] * db[a];
    db_[a] += wab[a] * d_diss;
    dpsi_ -= wab[a] * run8[a];
    run8_[a] -= wab[a] * dpsi;
  }
  pgi_ += dpsi_ * I.psi * ch * vwi;
  gI[13] += dpsi_ * pgi * ch * vwi;
  vwi_ += dpsi_ * pgi * I.psi * ch;
  pgj_ += dpsi_ * J.psi * ch * vwj;
  gJ[13] += dpsi_ * pgj * ch * vwj;
  vwj_ += dpsi_ * pgj * J.psi * ch;
  pgi_ += d_diss_ * 0.5 * vsig_b * P.ar;
  pgj_ += d_diss_ * 0.5 * vsig_b * P.ar;
  const double vsig_b_ = d_diss_ * 0.5 * (pgi + pgj) * P.ar;
  double dvt_[3];
  for (int a = 0; a < 3; a++) dvt_[a] = vsig_b > 0.0 ? vsig_b_ * dvt[a] / vsig_b : 0.0;
  double projv_ = 0.0;
  for (int a = 0; a < 3; a++) {
    dv_[a] += dvt_[a];
    projv_ -= dvt_[a] * run8[a];
    run8_[a] -= dvt_[a] * projv;
  }
  for (int a = 0; a < 3; a++) {
    dv_[a] += projv_ * run8[a];
    run8_[a] += projv_ * dv[a];
  }
  pgi_ -= d_brho_ * proj_bi;
  proj_bi_ -= d_brho_ * pgi;
  const double ri2_ = pgi_ * mj * gi, rj2_ = pgj_ * mj * gj;
  gi_ += pgi_ * mj * ri2;
  gj_ += pgj_ * mj * rj2;
  gI[1] += ri2_ * (-2.0 * ri2 / I.rho);
  gJ[1] += rj2_ * (-2.0 * rj2 / J.rho);
  for (int a = 0; a < 3; a++) {
    db_[a] += delta_b2_ * 2.0 * db[a] + proj_db_ * run8[a];
    run8_[a] += proj_db_ * db[a] + proj_bi_ * I.b[a] + proj_bj_ * J.b[a];
    Ib_[a] += db_[a] + proj_bi_ * run8[a];
    Jb_[a] += -db_[a] + proj_bj_ * run8[a];
  }
  // G8
  double gradp_ = 0.0, si8_ = 0.0, sj8_ = 0.0, bri_[3] = {}, brj_[3] = {};
  for (int a = 0; a < 3; a++) {
    const double pia = cm * bri[a] * si8, pja = cm * brj[a] * sj8;
    run8_[a] -= wa8[a] * gradp;
    gradp_ -= wa8[a] * run8[a];
    const double pia_ = -wa8[a] * gi, pja_ = -wa8[a] * gj;
    gi_ -= wa8[a] * pia;
    gj_ -= wa8[a] * pja;
    bri_[a] += pia_ * cm * si8;
    si8_ += pia_ * cm * bri[a];
    brj_[a] += pja_ * cm * sj8;
    sj8_ += pja_ * cm * brj[a];
  }
  for (int b = 0; b < 3; b++) {
    bri_[b] += si8_ * run8[b];
    run8_[b] += si8_ * bri[b] + sj8_ * brj[b];
    brj_[b] += sj8_ * run8[b];
  }
  const double bro2_i_ = gradp_ * 0.5 * mj * gi, bro2_j_ = gradp_ * 0.5 * mj * gj;
  gi_ += gradp_ * 0.5 * mj * bro2_i;
  gj_ += gradp_ * 0.5 * mj * bro2_j;
  for (int a = 0; a < 3; a++) {
    bri_[a] += bro2_i_ * 2.0 * bri[a] / mu0;
    brj_[a] += bro2_j_ * 2.0 * brj[a] / mu0;
    Ib_[a] += bri_[a] / I.rho;
    gI[1] -= bri_[a] * bri[a] / I.rho;
    Jb_[a] += brj_[a] / J.rho;
    gJ[1] -= brj_[a] * brj[a] / J.rho;
  }
  // gi, gj (run8 path)
  gI[3] += gi_ * (run8[0] * dwi[0] + run8[1] * dwi[1] + run8[2] * dwi[2]);
  gJ[3] += gj_ * (run8[0] * dwj[0] + run8[1] * dwj[1] + run8[2] * dwj[2]);
  for (int a = 0; a < 3; a++) {
    run8_[a] += gi_ * I.omega * dwi[a] + gj_ * J.omega * dwj[a];
    dwi_[a] += gi_ * I.omega * run8[a];
    dwj_[a] += gj_ * J.omega * run8[a];
  }
  if (far8)
    for (int a = 0; a < 3; a++) {
      gx[a] += run8_[a] / r;
      r_ -= run8_[a] * x[a] / (r * r);
    }
  // G6: conduction, pressure, viscosity, divergence
  {
    const double T_ = wae6 * P.ac * vsig2 * de;
    const double vsig2_ = wae6 * P.ac * de * tc;
    gI[11] += wae6 * P.ac * vsig2 * tc;
    gJ[11] -= wae6 * P.ac * vsig2 * tc;
    gI[1] -= T_ * 0.5 * mj * gi6 / (I.rho * I.rho);
    gi6_ += T_ * 0.5 * mj / I.rho;
    gJ[1] -= T_ * 0.5 * mj * gj6 / (J.rho * J.rho);
    gj6_ += T_ * 0.5 * mj / J.rho;
    const double va_ = va > 0.0 ? vsig2_ * 0.5 / vsig2 : 0.0;
    const double sgn = dp > 0.0 ? 1.0 : (dp < 0.0 ? -1.0 : 0.0);
    gI[2] += va_ * sgn / rhoij;
    gJ[2] -= va_ * sgn / rhoij;
    const double rhoij_ = -va_ * va / rhoij;
    gI[1] += 0.5 * rhoij_;
    gJ[1] += 0.5 * rhoij_;
  }
  double pri_ = wae6 * mj * I.omega * udw;
  gI[3] += wae6 * mj * pri * udw;
  {
    const double udw_ = wae6 * mj * pri * I.omega;
    for (int a = 0; a < 3; a++) {
      dv_[a] += udw_ * dwi[a];
      dwi_[a] += udw_ * dv[a];
    }
  }
  double prj_ = 0.0;
  for (int a = 0; a < 3; a++) {
    pri_ -= wa6[a] * mj * I.omega * dwi[a];
    gI[3] -= wa6[a] * mj * pri * dwi[a];
    dwi_[a] -= wa6[a] * mj * pri * I.omega;
    prj_ -= wa6[a] * mj * J.omega * dwj[a];
    gJ[3] -= wa6[a] * mj * prj * dwj[a];
    dwj_[a] -= wa6[a] * mj * prj * J.omega;
  }
  if (av) {
    double q_i_ = wae6 * mj * dot * gi6;
    dot_ += wae6 * mj * q_i * gi6;
    gi6_ += wae6 * mj * q_i * dot;
    double q_j_ = 0.0;
    for (int a = 0; a < 3; a++) {
      q_i_ -= wa6[a] * mj * I.omega * dwi[a];
      gI[3] -= wa6[a] * mj * q_i * dwi[a];
      dwi_[a] -= wa6[a] * mj * q_i * I.omega;
      q_j_ -= wa6[a] * mj * J.omega * dwj[a];
      gJ[3] -= wa6[a] * mj * q_j * dwj[a];
      dwj_[a] -= wa6[a] * mj * q_j * J.omega;
    }
    gI[1] += q_i_ * 0.5 / (I.rho * I.rho) * vav_i * dot * P.av;
    gJ[1] += q_j_ * 0.5 / (J.rho * J.rho) * vav_j * dot * P.av;
    const double vav_i_ = q_i_ * (-0.5 / I.rho * dot * P.av), vav_j_ = q_j_ * (-0.5 / J.rho * dot * P.av);
    dot_ += q_i_ * (-0.5 / I.rho * vav_i * P.av) + q_j_ * (-0.5 / J.rho * vav_j * P.av);
    if (ti >= 0.0) {
      gI[12] += vav_i_ * vwi;
      vwi_ += vav_i_ * I.alpha;
      dot_ -= beta * vav_i_;
    }
    if (tj >= 0.0) {
      gJ[12] += vav_j_ * vwj;
      vwj_ += vav_j_ * J.alpha;
      dot_ -= beta * vav_j_;
    }
  }
  dot_ += wdiv * mj * gi6;
  gi6_ += wdiv * mj * dot;
  gI[3] += gi6_ * (run6[0] * dwi[0] + run6[1] * dwi[1] + run6[2] * dwi[2]);
  gJ[3] += gj6_ * (run6[0] * dwj[0] + run6[1] * dwj[1] + run6[2] * dwj[2]);
  for (int a = 0; a < 3; a++) {
    run6_[a] += gi6_ * I.omega * dwi[a] + gj6_ * J.omega * dwj[a] + dot_ * dv[a];
    dwi_[a] += gi6_ * I.omega * run6[a];
    dwj_[a] += gj6_ * J.omega * run6[a];
    dv_[a] += dot_ * run6[a];
  }
  if (!near6)
    for (int a = 0; a < 3; a++) {
      gx[a] += run6_[a] / r;
      r_ -= run6_[a] * x[a] / (r * r);
    }
  gI[2] += pri_ / (I.rho * I.rho);
  gI[1] -= pri_ * 2.0 * I.p / (I.rho * I.rho * I.rho);
  gJ[2] += prj_ / (J.rho * J.rho);
  gJ[1] -= prj_ * 2.0 * J.p / (J.rho * J.rho * J.rho);
  // wave speeds
  {
    const double si_ = si > 0.0 ? vwi_ * 0.5 / vwi : 0.0, sj_ = sj > 0.0 ? vwj_ * 0.5 / vwj : 0.0;
    gI[4] += si_ * 2.0 * I.cs;
    gJ[4] += sj_ * 2.0 * J.cs;
    const double bi2_ = si_ / (mu0 * I.rho), bj2_ = sj_ / (mu0 * J.rho);
    gI[1] -= si_ * bi2 / (mu0 * I.rho * I.rho);
    gJ[1] -= sj_ * bj2 / (mu0 * J.rho * J.rho);
    for (int a = 0; a < 3; a++) {
      Ib_[a] += bi2_ * 2.0 * I.b[a];
      Jb_[a] += bj2_ * 2.0 * J.b[a];
    }
  }
  for (int a = 0; a < 3; a++) {
    gI[5 + a] += Ib_[a];
    gJ[5 + a] += Jb_[a];
    gI[8 + a] += dv_[a];
    gJ[8 + a] -= dv_[a];
  }
  // kernel gradients: Jacobians in x_ij and h from a dual evaluation
  {
    using D4 = Dual<4>;
    D4 xd[3];
    for (int a = 0; a < 3; a++) {
      xd[a] = D4(x[a]);
      xd[a].d[a] = 1.0;
    }
    const D4 rd = f_norm(xd);
    D4 hi(I.h), hj(J.h);
    hi.d[3] = 1.0;
    hj.d[3] = 1.0;
    D4 gdi[3], gdj[3];
    f_kern_grad<K, DIM>(P.norm, xd, rd, hi, gdi);
    f_kern_grad<K, DIM>(P.norm, xd, rd, hj, gdj);
    for (int a = 0; a < 3; a++) {
      for (int b = 0; b < 3; b++) gx[b] += dwi_[a] * gdi[a].d[b] + dwj_[a] * gdj[a].d[b];
      gI[0] += dwi_[a] * gdi[a].d[3];
      gJ[0] += dwj_[a] * gdj[a].d[3];
    }
  }
  if (r > 0.0)
    for (int a = 0; a < 3; a++) gx[a] += r_ * x[a] / r;
}

// Outputs of the force groups' post loops and G10.
template <class D>
struct FOut {
  D au[3], ae, ah, ab[3], apsi, div, divbs, dtcfl, dta;
};
constexpr int kFOutDirs = 9;  // au 3, ae, ah, ab 3, apsi (the rest is not differentiated)

// G6 post (:278-280), G7 (:133-140), G9 post (:562-567), EnergyLimiter
// (:594-598), DivBCorrection (:607-624), AdaptiveTimestep (:578-585).
template <int DIM, class D>
__device__ inline void f_force_post(const DevParams& P, const Side<D>& I, const FSums<D>& S, FOut<D>& o) {
  const double mu0 = P.mu0;
  const D bi2 = I.b[0] * I.b[0] + I.b[1] * I.b[1] + I.b[2] * I.b[2];
  const D vwave = gsqrt(I.cs * I.cs + bi2 / (mu0 * I.rho));
  const D ch = P.clean_speed * vwave;
  const D divv = -S.div / I.rho;
  o.div = divv;
  o.ah = I.h * divv * (1.0 / (double)DIM);
  for (int a = 0; a < 3; a++) o.ab[a] = S.ab[a];
  o.apsi = -ch * S.divbd / I.rho - P.clean_damp * I.psi * ch / I.h - 0.5 * P.clean_active * I.psi * divv;
  D dtcfl = pmax(S.dtcfl, vwave);
  dtcfl = pmax(dtcfl, ch);
  o.dtcfl = dtcfl;
  D ae = S.ae6 + S.ae9;
  if (dtcfl > 0.0) {
    const D dtc = P.c_cour * I.h / dtcfl;
    if (I.e + dtc * ae < 0.0 && I.e > 0.0) ae = ae / (1.0 - dtc * ae / I.e);
  }
  o.ae = ae;
  D frac(0.0);
  if (bi2 > 0.0) {
    const D pbeta = 2.0 * mu0 * I.p / bi2;
    frac = pmax(D(0.0), pmin(D(1.0), (10.0 - pbeta) * 0.125));
  }
  for (int a = 0; a < 3; a++) o.au[a] = (S.a6[a] + S.a8[a]) + (-I.b[a] * S.divbs * frac / mu0);
  o.divbs = I.rho * S.divbs;
  D dta(kBigNumber);
  if (dtcfl > 0.0) dta = P.c_cour * I.h / dtcfl;
  const D f2 = o.au[0] * o.au[0] + o.au[1] * o.au[1] + o.au[2] * o.au[2];
  if (f2 > 0.0) dta = pmin(dta, P.c_force * gsqrt(I.h / gsqrt(f2)));
  o.dta = dta;
}

// -------------------------------------------------- integrator stages
// The state the literal PEC step carries from one step to the next.
template <class D>
struct StepState {
  D x[3], v[3], e, h, alpha1, bev[3], psi, a[3], ae, ah, aloc, cs, abev[3], apsi;
};
constexpr int kStateDirs = 24;

// What initialize + stage1 + wrap produce (src/integrator.py:12-65).
template <class D>
struct Predicted {
  D x[3], vhalf[3], vpred[3], ehalf, epred, h, alpha1, bhalf[3], bpred[3], psihalf, psipred;
};

template <class D>
__device__ inline D f_wrap(D x, double lo, double hi, double L) {
  if (x < lo) x = x + L;
  if (x > hi) x = x - L;
  return x;
}

template <class D>
__device__ inline void f_predict(const DevParams& P, const StepState<D>& s, bool fluid, double dt, Predicted<D>& o) {
  for (int a = 0; a < 3; a++) {
    o.x[a] = s.x[a];
    o.vhalf[a] = o.vpred[a] = s.v[a];
    o.bhalf[a] = o.bpred[a] = s.bev[a];
  }
  o.ehalf = o.epred = s.e;
  o.h = s.h;
  o.alpha1 = s.alpha1;
  o.psihalf = o.psipred = s.psi;
  if (!fluid) return;
  const double dtb2 = 0.5 * dt;
  for (int a = 0; a < 3; a++) {
    o.vhalf[a] = s.v[a] + dtb2 * s.a[a];
    o.vpred[a] = s.v[a] + dt * s.a[a];
  }
  for (int a = 0; a < P.dim; a++) {
    o.x[a] = s.x[a] + dt * o.vhalf[a];
    if (P.periodic[a]) o.x[a] = f_wrap(o.x[a], P.lo[a], P.hi[a], P.L[a]);
  }
  o.ehalf = s.e + dtb2 * s.ae;
  o.epred = s.e + dt * s.ae;
  o.h = s.h + dt * s.ah;
  const D decay_rate = 0.1 * s.cs / o.h;
  o.alpha1 = s.alpha1 < s.aloc ? s.aloc : (s.alpha1 + dt * s.aloc * decay_rate) / (1.0 + dt * decay_rate);
  for (int a = 0; a < 3; a++) {
    o.bhalf[a] = s.bev[a] + dtb2 * s.abev[a];
    o.bpred[a] = s.bev[a] + dt * s.abev[a];
  }
  o.psihalf = s.psi + dtb2 * s.apsi;
  o.psipred = s.psi + dt * s.apsi;
}

}  // namespace mhd
