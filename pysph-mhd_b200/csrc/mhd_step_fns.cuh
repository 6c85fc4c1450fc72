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
