// mhd_pairs.cu -- FP64 neighbour passes of the SPMHD right-hand side (sm_100a).
//
// k_density_pass: one pass of DensityIteration (src/equations.py:14-94) --
//   pair sums rho = sum m W(h_i), dwdh = sum m dW/dh(h_i), then the Newton
//   update of h with the [0.8h, 1.2h] clip and the convergence test, one
//   thread per particle of the cell-sorted order, h read from one buffer and
//   written to another (Jacobi semantics of PySPH's post_loop).
// k_force_prologue: DensityFromSmoothingLength, IdealGasEOS and
//   MagneticStateReconstruction (src/equations.py:109-118, 97-106, 474-485)
//   plus the per-particle factors the pair loop reuses.
// k_force_pass: CullenDehnenAlphaDiagnostics, MHDAccelerations,
//   MagneticStressAccelerations and MagneticStateRates as one neighbour loop
//   (src/equations.py:318-354, 217-275, 149-195, 507-559) with the per-particle
//   epilogue of their post_loops, SmoothingLengthRateFromForceDivergence,
//   EnergyLimiter, DivBCorrection and AdaptiveTimestep
//   (src/equations.py:357-429, 278-280, 133-140, 562-567, 588-624, 570-585).
//   Gather formulation: each thread writes only its own particle, no atomics.
#include <cuda_runtime.h>

#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

// ------------------------------------------------------------ density pass
template <int K, int DIM>
__global__ void __launch_bounds__(128) k_density_pass(int n, int pass, DevParams P, NbrList L,
                                                      const double* __restrict__ x, const double* __restrict__ y,
                                                      const double* __restrict__ z, const double* __restrict__ m,
                                                      const double* __restrict__ h_in, double* __restrict__ h_out,
                                                      const double* __restrict__ h0, double* __restrict__ rho_sum,
                                                      double* __restrict__ omega, double* __restrict__ converged,
                                                      DevScalars* sc) {
  // Stop when the iterated group already stopped after pass `pass` (1-based
  // count), or when the neighbour lists no longer cover the current h.
  if (sc->relist) return;
  if (pass > 0) {
    const bool stop = !P.iterate || pass >= P.max_iter || (pass >= P.min_iter && sc->n_unconverged[pass - 1] == 0);
    if (stop) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&sc->passes_done, pass + 1);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double hi = h_in[i];
  if (converged[i] == 1.0) {
    // Already finalised: its h is frozen; a re-summation would only refresh
    // the unconsumed rho_sum diagnostic (src/equations.py:117).
    h_out[i] = hi;
    return;
  }
  const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
  const double h1 = 1.0 / hi;
  const double fac = hfac<DIM>(P.norm, h1);
  const double rhi2 = rh2_exact(P.R, hi);
  constexpr bool compact = K <= MHD_KERNEL_WENDLAND_C6;
  double rs = 0.0, ds = 0.0;
  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  for (int k = 0; k < cnt; k++) {
    const int j = row[k * 32];
    const double dx = min_image(xi - x[j], P.L[0], P.half[0], P.periodic[0]);
    const double dy = min_image(yi - y[j], P.L[1], P.half[1], P.periodic[1]);
    const double dz = DIM == 3 ? min_image(zi - z[j], P.L[2], P.half[2], P.periodic[2]) : 0.0;
    const double r2 = r2_exact(dx, dy, dz);
    // For compact kernels a pair admitted only by R*h_j has W(h_i) = 0 and
    // dW/dh(h_i) = 0, so the h_i test alone gives the same sums.
    bool nb = r2 < rhi2;
    if (!compact && !nb) nb = r2 < rh2_exact(P.R, h_in[j]);
    if (nb) {
      const double r = sqrt(r2);
      const double q = r * h1;
      double w, dw;
      w_dw<K>(q, DIM, w, dw);
      const double mj = m[j];
      rs += mj * (w * fac);
      ds += mj * (-fac * h1 * (dw * q + w * (double)DIM));
    }
  }
  // post_loop (src/equations.py:53-86)
  const double mi = m[i];
  const double rhoi = mi / pow_dim<DIM>(hi / P.hfact);
  const double dhdrhoi = -hi / ((double)DIM * rhoi);
  const double omegai = 1.0 - dhdrhoi * ds;
  omega[i] = 1.0 / omegai;
  const double func = rhoi - rs;
  const double dfdh1 = omegai > 0.0 ? dhdrhoi / omegai : dhdrhoi / fabs(omegai + kMachineEps);
  double hnew = hi - func * dfdh1;
  if (hnew > 1.2 * hi) hnew = 1.2 * hi;
  else if (hnew < 0.8 * hi) hnew = 0.8 * hi;
  const double diff = fabs(hnew - hi) / h0[i];
  const bool finalize = ((diff < kDensityTolerance) && (omegai > 0.0) && (hi > 0.0)) || !P.iterate;
  double hout;
  if (!finalize) {
    hout = hnew;
    converged[i] = 0.0;
    atomicAdd(&sc->n_unconverged[pass], 1);
  } else {
    hout = P.hfact * pow(mi / rs, 1.0 / (double)DIM);
    converged[i] = 1.0;
  }
  h_out[i] = hout;
  rho_sum[i] = rs;
  // The lists hold every j within R * max(h_i, h_j) of the h they were built
  // with, enlarged by the list margin; a larger h needs new lists.
  if (!(hout <= L.hlim[i])) atomicExch(&sc->relist, 1);
}

// ------------------------------------------------------- neighbour lists
// One thread per particle scans the 3^DIM cells around it (uniform work per
// candidate, only the append is predicated) and appends every j within the
// margin-enlarged symmetric radius.  Counts beyond `cap` are recorded, not
// stored, and flag a rebuild with a larger capacity.
template <int DIM>
__global__ void __launch_bounds__(128) k_build_lists(int n, DevParams P, Grid G, const int* __restrict__ cell_start,
                                                     const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ z, const double* __restrict__ h,
                                                     double grow, int cap, int* __restrict__ idx,
                                                     int* __restrict__ cnt_out, double* __restrict__ hlim,
                                                     DevScalars* sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
  const double hg = h[i] * grow;
  const double rhi = P.R * hg, rhi2 = rhi * rhi;
  int* __restrict__ row = idx + (size_t)(i >> 5) * cap * 32 + (i & 31);
  int cnt = 0;
  for_each_candidate<DIM>(G, P, cell_start, xi, yi, zi, [&](int j) {
    const double dx = min_image(xi - x[j], P.L[0], P.half[0], P.periodic[0]);
    const double dy = min_image(yi - y[j], P.L[1], P.half[1], P.periodic[1]);
    const double dz = DIM == 3 ? min_image(zi - z[j], P.L[2], P.half[2], P.periodic[2]) : 0.0;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double rhj = P.R * h[j] * grow;
    if (r2 < rhi2 || r2 < rhj * rhj) {
      if (cnt < cap) row[cnt * 32] = j;
      cnt++;
    }
  });
  cnt_out[i] = cnt < cap ? cnt : cap;
  hlim[i] = hg;
  if (cnt > cap) {
    atomicMax(&sc->list_max, cnt);
    atomicExch(&sc->relist, 1);
  }
}

void launch_build_lists(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  TimedScope ts(c, MHD_TIMING_CELLS, st);
  const double grow = 1.0 + c->list_margin;
  if (c->P.dim == 3)
    k_build_lists<3><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->grid, c->cell_start, s->x, s->y, s->z, s->h, grow,
                                                     c->list_cap, c->nbr_idx, c->nbr_cnt, c->nbr_hlim, c->d_sc);
  else
    k_build_lists<2><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->grid, c->cell_start, s->x, s->y, s->z, s->h, grow,
                                                     c->list_cap, c->nbr_idx, c->nbr_cnt, c->nbr_hlim, c->d_sc);
  c->launches++;
}

// ------------------------------------------------------------ force pass
struct ForceArgs {
  // inputs (cell-sorted order)
  const double *x, *y, *z, *h, *m, *rho, *omega, *p, *epred, *upred, *vpred, *wpred, *Bx, *By, *Bz, *alpha1,
      *au_prev, *av_prev, *aw_prev;
  const double *inv_h, *inv_rho, *vwave, *psich, *psipred, *cs;
  // outputs
  double *au, *av, *aw, *ae, *ah, *div, *div_for_psi, *dt_cfl, *dt_adapt, *aBx, *aBy, *aBz, *apsi, *divBsymm,
      *divBdiff, *alphaloc;
  // optional diagnostics (may be null)
  double *xilimiter, *divvdt;
  double* cd[24];   // rxx rxy rxz ryy ryz rzz vxx..vzz axx..azz
  double* dvdx[9];  // xx xy xz yx yy yz zx zy zz
};

// Prologue: G2 (rho from h), G3 (EOS), G5 (B from B/rho), per-particle factors.
template <int DIM>
__global__ void __launch_bounds__(256) k_force_prologue(int n, DevParams P, MhdState s, double* __restrict__ inv_h,
                                                        double* __restrict__ inv_rho, double* __restrict__ vwave,
                                                        double* __restrict__ psich) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h = s.h[i];
  const double rho = s.m[i] / pow_dim<DIM>(h / P.hfact);
  const double p = P.gamma1 * rho * s.epred[i];
  const double cs = sqrt(P.gamma * p / rho);
  const double bx = s.Bevolxpred[i] * rho, by = s.Bevolypred[i] * rho, bz = s.Bevolzpred[i] * rho;
  s.rho[i] = rho;
  s.p[i] = p;
  s.cs[i] = cs;
  s.Bx[i] = bx;
  s.By[i] = by;
  s.Bz[i] = bz;
  s.Bxpred[i] = bx;
  s.Bypred[i] = by;
  s.Bzpred[i] = bz;
  const double vw = sqrt(cs * cs + (bx * bx + by * by + bz * bz) / (P.mu0 * rho));
  inv_h[i] = 1.0 / h;
  inv_rho[i] = 1.0 / rho;
  vwave[i] = vw;
  psich[i] = s.psipred[i] * (P.clean_speed * vw);
}

template <int K, int DIM>
__global__ void __launch_bounds__(128) k_force_pass(int n, DevParams P, NbrList L, ForceArgs a, DevScalars* sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = a.x[i], yi = a.y[i], zi = DIM == 3 ? a.z[i] : 0.0;
  const double hi = a.h[i], h1i = a.inv_h[i];
  const double faci = hfac<DIM>(P.norm, h1i);
  const double rhi2 = rh2_exact(P.R, hi);
  const double rhoi = a.rho[i], irhoi = a.inv_rho[i], omegai = a.omega[i];
  const double p_i = a.p[i];
  const double pibrhoi2 = p_i * irhoi * irhoi;
  const double vwi = a.vwave[i], alphai = a.alpha1[i], epi = a.epred[i];
  const double ui = a.upred[i], vi = a.vpred[i], wi = a.wpred[i];
  const double aui = a.au_prev[i], avi = a.av_prev[i], awi = a.aw_prev[i];
  const double bxi = a.Bx[i], byi = a.By[i], bzi = a.Bz[i];
  const double brxi = bxi * irhoi, bryi = byi * irhoi, brzi = bzi * irhoi;
  const double bro2i = (brxi * brxi + bryi * bryi + brzi * brzi) * P.inv_mu0;
  const double rhoi2inv = irhoi * irhoi;
  const double psichi = a.psich[i];
  const double beta = 2.0;

  // Cullen-Dehnen moments (src/equations.py:329-354)
  double rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
  double vxx = 0, vxy = 0, vxz = 0, vyx = 0, vyy = 0, vyz = 0, vzx = 0, vzy = 0, vzz = 0;
  double axx = 0, axy = 0, axz = 0, ayx = 0, ayy = 0, ayz = 0, azx = 0, azy = 0, azz = 0;
  // MHDAccelerations + MagneticStressAccelerations + MagneticStateRates
  double fx = 0, fy = 0, fz = 0, fe = 0, fdiv = 0, dtc = 0;
  double bx_r = 0, by_r = 0, bz_r = 0, dbs = 0, dbd = 0;
  unsigned npair = 0, ncand = 0;

  auto pair = [&](int j) {
    ncand++;
    const double dx = min_image(xi - a.x[j], P.L[0], P.half[0], P.periodic[0]);
    const double dy = min_image(yi - a.y[j], P.L[1], P.half[1], P.periodic[1]);
    const double dz = DIM == 3 ? min_image(zi - a.z[j], P.L[2], P.half[2], P.periodic[2]) : 0.0;
    const double r2 = r2_exact(dx, dy, dz);
    if (!(r2 < rhi2 || r2 < rh2_exact(P.R, a.h[j]))) return;
    npair++;
    const double r = sqrt(r2);
    const double h1j = a.inv_h[j];
    // DWI = ti * XIJ, DWJ = tj * XIJ (kernel gradient, zero at r <= 1e-12)
    double ti = 0.0, tj = 0.0, inv_r = 0.0;
    if (r > kPairDistanceEpsilon) {
      inv_r = 1.0 / r;
      double w, dw;
      w_dw<K>(r * h1i, DIM, w, dw);
      ti = faci * dw * h1i * inv_r;
      w_dw<K>(r * h1j, DIM, w, dw);
      tj = hfac<DIM>(P.norm, h1j) * dw * h1j * inv_r;
    }
    const double mj = a.m[j];
    const double dvx = ui - a.upred[j], dvy = vi - a.vpred[j], dvz = wi - a.wpred[j];

    // ---- CullenDehnenAlphaDiagnostics.loop
    {
      const double c = mj * ti;
      const double cx = c * dx, cy = c * dy, cz = c * dz;
      const double dax = aui - a.au_prev[j], day = avi - a.av_prev[j], daz = awi - a.aw_prev[j];
      if (DIM == 3) {
        rxx -= dx * cx; rxy -= dx * cy; rxz -= dx * cz;
        ryy -= dy * cy; ryz -= dy * cz; rzz -= dz * cz;
        vxz += dvx * cz; vyz += dvy * cz; vzz += dvz * cz;
        axy += dax * cy; axz += dax * cz; ayx += day * cx; ayz += day * cz; azx += daz * cx; azy += daz * cy;
        azz += daz * cz;
      }
      vxx += dvx * cx; vxy += dvx * cy;
      vyx += dvy * cx; vyy += dvy * cy;
      vzx += dvz * cx; vzy += dvz * cy;
      axx += dax * cx; ayy += day * cy;
    }
    const double rhoj = a.rho[j], irhoj = a.inv_rho[j], omegaj = a.omega[j];
    const double vwj = a.vwave[j];
    // ---- MHDAccelerations.loop (r-hat is zero below 1e-8 here)
    {
      const double inv_r6 = r < kInteractionDistanceEpsilon ? 0.0 : inv_r;
      const double dot = (dvx * dx + dvy * dy + dvz * dz) * inv_r6;
      const double g6 = r < kInteractionDistanceEpsilon ? 0.0 : r;
      const double grad_i = omegai * ti * g6;
      const double grad_j = omegaj * tj * g6;
      fdiv += mj * dot * grad_i;
      const double pj = a.p[j];
      const double vsig2 = sqrt(fabs(p_i - pj) / (0.5 * (rhoi + rhoj)));
      double c = vwi - beta * dot;
      c = fmax(c, vwj - beta * dot);
      c = fmax(c, 0.0);
      dtc = fmax(dtc, c);
      double fcoef = pibrhoi2 * omegai * ti + pj * irhoj * irhoj * omegaj * tj;
      if (dot < 0.0) {
        const double vsigav_i = fmax(alphai * vwi - beta * dot, 0.0);
        const double vsigav_j = fmax(a.alpha1[j] * vwj - beta * dot, 0.0);
        const double qi = -0.5 * irhoi * vsigav_i * dot * P.av;
        const double qj = -0.5 * irhoj * vsigav_j * dot * P.av;
        fcoef += qi * omegai * ti + qj * omegaj * tj;
        fe += mj * qi * dot * grad_i;
      }
      fx -= mj * fcoef * dx;
      fy -= mj * fcoef * dy;
      fz -= mj * fcoef * dz;
      fe += mj * pibrhoi2 * omegai * ti * (dvx * dx + dvy * dy + dvz * dz);
      const double eij = epi - a.epred[j];
      fe += P.ac * vsig2 * eij * (0.5 * mj * irhoi * grad_i + 0.5 * mj * irhoj * grad_j);
    }
    // ---- MagneticStressAccelerations.loop and MagneticStateRates.loop
    {
      const double rux = dx * inv_r, ruy = dy * inv_r, ruz = dz * inv_r;
      const double g8 = r > kPairDistanceEpsilon ? r : 0.0;
      const double grad_i = omegai * ti * g8;
      const double grad_j = omegaj * tj * g8;
      const double bxj = a.Bx[j], byj = a.By[j], bzj = a.Bz[j];
      const double brxj = bxj * irhoj, bryj = byj * irhoj, brzj = bzj * irhoj;
      const double bro2j = (brxj * brxj + bryj * bryj + brzj * brzj) * P.inv_mu0;
      const double gradp = mj * (0.5 * bro2i * grad_i + 0.5 * bro2j * grad_j);
      const double si = (brxi * rux + bryi * ruy + brzi * ruz) * grad_i;
      const double sj = (brxj * rux + bryj * ruy + brzj * ruz) * grad_j;
      const double ms = -mj * P.inv_mu0;
      fx += -rux * gradp - ms * (brxi * si + brxj * sj);
      fy += -ruy * gradp - ms * (bryi * si + bryj * sj);
      fz += -ruz * gradp - ms * (brzi * si + brzj * sj);

      const double proj_bi = bxi * rux + byi * ruy + bzi * ruz;
      const double proj_bj = bxj * rux + byj * ruy + bzj * ruz;
      const double dbx = bxi - bxj, dby = byi - byj, dbz = bzi - bzj;
      const double proj_db = dbx * rux + dby * ruy + dbz * ruz;
      const double delta_b2 = dbx * dbx + dby * dby + dbz * dbz;
      const double pmi = mj * rhoi2inv * grad_i;
      const double pmj = mj * irhoj * irhoj * grad_j;
      const double d_brho = -(pmi * proj_bi);
      const double projv = dvx * rux + dvy * ruy + dvz * ruz;
      const double tx = dvx - projv * rux, ty = dvy - projv * ruy, tz = dvz - projv * ruz;
      const double vsig_b = sqrt(tx * tx + ty * ty + tz * tz);
      const double diss = 0.5 * (pmi + pmj) * vsig_b * P.ar;
      const double dpsi = pmi * psichi + pmj * a.psich[j];
      bx_r += d_brho * dvx + diss * dbx - dpsi * rux;
      by_r += d_brho * dvy + diss * dby - dpsi * ruy;
      bz_r += d_brho * dvz + diss * dbz - dpsi * ruz;
      fe += -0.5 * delta_b2 * diss * P.inv_mu0;
      dbs += pmi * proj_bi + pmj * proj_bj;
      dbd += -mj * proj_db * grad_i;
    }
  };
  {
    const int cnt = L.cnt[i];
    const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
    for (int k = 0; k < cnt; k++) pair(row[k * 32]);
  }

  // ---- CullenDehnenAlphaDiagnostics.post_loop (src/equations.py:357-429)
  const double termnorm = omegai * irhoi;
  double div_a, dvxdx, dvxdy, dvxdz, dvydx, dvydy, dvydz, dvzdx, dvzdy, dvzdz;
  const double denom =
      DIM == 3 ? rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy : 0.0;
  double tm[6] = {0, 0, 0, 0, 0, 0};
  bool full = fabs(denom) > kFloatTiny;
  if (full) {
    const double dd = 1.0 / denom;
    tm[0] = (ryy * rzz - ryz * ryz) * dd;
    tm[1] = (rxz * ryz - rzz * rxy) * dd;
    tm[2] = (rxy * ryz - rxz * ryy) * dd;
    tm[3] = (rzz * rxx - rxz * rxz) * dd;
    tm[4] = (rxy * rxz - rxx * ryz) * dd;
    tm[5] = (rxx * ryy - rxy * rxy) * dd;
    div_a = -((axx * tm[0] + axy * tm[1] + axz * tm[2]) + (ayx * tm[1] + ayy * tm[3] + ayz * tm[4]) +
              (azx * tm[2] + azy * tm[4] + azz * tm[5]));
    dvxdx = -(vxx * tm[0] + vxy * tm[1] + vxz * tm[2]);
    dvxdy = -(vxx * tm[1] + vxy * tm[3] + vxz * tm[4]);
    dvxdz = -(vxx * tm[2] + vxy * tm[4] + vxz * tm[5]);
    dvydx = -(vyx * tm[0] + vyy * tm[1] + vyz * tm[2]);
    dvydy = -(vyx * tm[1] + vyy * tm[3] + vyz * tm[4]);
    dvydz = -(vyx * tm[2] + vyy * tm[4] + vyz * tm[5]);
    dvzdx = -(vzx * tm[0] + vzy * tm[1] + vzz * tm[2]);
    dvzdy = -(vzx * tm[1] + vzy * tm[3] + vzz * tm[4]);
    dvzdz = -(vzx * tm[2] + vzy * tm[4] + vzz * tm[5]);
  } else {
    div_a = -termnorm * (axx + ayy + azz);
    dvxdx = -termnorm * vxx; dvxdy = -termnorm * vxy; dvxdz = -termnorm * vxz;
    dvydx = -termnorm * vyx; dvydy = -termnorm * vyy; dvydz = -termnorm * vyz;
    dvzdx = -termnorm * vzx; dvzdy = -termnorm * vzy; dvzdz = -termnorm * vzz;
  }
  const double divvdt =
      div_a - (dvxdx * dvxdx + dvydy * dvydy + dvzdz * dvzdz + 2.0 * (dvxdy * dvydx + dvxdz * dvzdx + dvydz * dvzdy));
  const double divv = dvxdx + dvydy + dvzdz;
  const double curlx = dvzdy - dvydz, curly = dvxdz - dvzdx, curlz = dvydx - dvxdy;
  const double compression = fmax(-divv, 0.0);
  const double fac = compression * compression;
  const double denominator = fac + (curlx * curlx + curly * curly + curlz * curlz);
  const double xil = denominator > 0.0 ? fac / denominator : 1.0;
  const double source = 10.0 * hi * hi * xil * fmax(-divvdt, 0.0);
  const double csi = a.cs[i];
  // alpha clip: reference literal [0, 1] (src/equations.py:428); alpha_min/max extend it
  a.alphaloc[i] = fmax(fmin(source / (csi * csi), P.alpha_max), P.alpha_min);
  if (a.xilimiter) a.xilimiter[i] = xil;
  if (a.divvdt) a.divvdt[i] = divvdt;
  if (a.cd[0]) {
    const double v[24] = {rxx, rxy, rxz, ryy, ryz, rzz, vxx, vxy, vxz, vyx, vyy, vyz,
                          vzx, vzy, vzz, axx, axy, axz, ayx, ayy, ayz, azx, azy, azz};
#pragma unroll
    for (int k = 0; k < 24; k++)
      if (a.cd[k]) a.cd[k][i] = v[k];
  }
  if (a.dvdx[0]) {
    const double v[9] = {dvxdx, dvxdy, dvxdz, dvydx, dvydy, dvydz, dvzdx, dvzdy, dvzdz};
#pragma unroll
    for (int k = 0; k < 9; k++)
      if (a.dvdx[k]) a.dvdx[k][i] = v[k];
  }

  // ---- MHDAccelerations.post_loop, SmoothingLengthRateFromForceDivergence
  const double divi = -fdiv * irhoi;
  // ---- MagneticStateRates.post_loop
  const double chi = P.clean_speed * vwi;
  const double psipi = a.psipred[i];
  const double apsi = -chi * dbd * irhoi - P.clean_damp * psipi * chi * h1i - 0.5 * P.clean_active * psipi * divi;
  dtc = fmax(dtc, vwi);
  dtc = fmax(dtc, chi);
  // ---- EnergyLimiter
  if (dtc > 0.0) {
    const double dtcour = P.c_cour * hi / dtc;
    if (epi + dtcour * fe < 0.0 && epi > 0.0) fe /= 1.0 - dtcour * fe / epi;
  }
  // ---- DivBCorrection
  {
    const double b2 = bxi * bxi + byi * byi + bzi * bzi;
    double frac = 0.0;
    if (b2 > 0.0) {
      const double betap = 2.0 * P.mu0 * p_i / b2;
      frac = fmax(0.0, fmin(1.0, (10.0 - betap) * 0.125));
    }
    const double cf = dbs * frac * P.inv_mu0;
    fx -= bxi * cf;
    fy -= byi * cf;
    fz -= bzi * cf;
  }
  // ---- AdaptiveTimestep
  double dta = kBigNumber;
  if (dtc > 0.0) dta = P.c_cour * hi / dtc;
  const double f2 = fx * fx + fy * fy + fz * fz;
  if (f2 > 0.0) dta = fmin(dta, P.c_force * sqrt(hi / sqrt(f2)));

  a.au[i] = fx;
  a.av[i] = fy;
  a.aw[i] = fz;
  a.ae[i] = fe;
  a.ah[i] = hi * divi * (1.0 / (double)DIM);
  a.div[i] = divi;
  a.div_for_psi[i] = divi;
  a.dt_cfl[i] = dtc;
  a.dt_adapt[i] = dta;
  a.aBx[i] = bx_r;
  a.aBy[i] = by_r;
  a.aBz[i] = bz_r;
  a.apsi[i] = apsi;
  a.divBsymm[i] = rhoi * dbs;
  a.divBdiff[i] = dbd;
  const unsigned mask = __activemask();
  const unsigned sp = __reduce_add_sync(mask, npair), sc_ = __reduce_add_sync(mask, ncand);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) {
    atomicAdd(&sc->n_pairs, (unsigned long long)sp);
    atomicAdd(&sc->n_candidates, (unsigned long long)sc_);
  }
}

// ------------------------------------------------------------- dispatch
template <int K, int DIM>
static void density_launch(Ctx* c, MhdState* s, int n, int pass, const double* h_in, double* h_out, cudaStream_t st) {
  k_density_pass<K, DIM><<<(n + 127) / 128, 128, 0, st>>>(n, pass, c->P, c->lists(), s->x, s->y, s->z, s->m, h_in,
                                                          h_out, s->h0, s->rho_sum, s->omega, s->converged, c->d_sc);
}

template <int K, int DIM>
static void force_launch(Ctx* c, const ForceArgs& a, int n, cudaStream_t st) {
  k_force_pass<K, DIM><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->lists(), a, c->d_sc);
}

#define MHD_DISPATCH(FN, ...)                                                   \
  do {                                                                          \
    const int d3 = c->P.dim == 3;                                               \
    switch (c->P.kernel) {                                                      \
      case MHD_KERNEL_CUBIC: d3 ? FN<0, 3>(__VA_ARGS__) : FN<0, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_QUINTIC: d3 ? FN<1, 3>(__VA_ARGS__) : FN<1, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C2: d3 ? FN<2, 3>(__VA_ARGS__) : FN<2, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C4: d3 ? FN<3, 3>(__VA_ARGS__) : FN<3, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_WENDLAND_C6: d3 ? FN<4, 3>(__VA_ARGS__) : FN<4, 2>(__VA_ARGS__); break; \
      case MHD_KERNEL_GAUSSIAN: d3 ? FN<5, 3>(__VA_ARGS__) : FN<5, 2>(__VA_ARGS__); break; \
      default: d3 ? FN<6, 3>(__VA_ARGS__) : FN<6, 2>(__VA_ARGS__); break;       \
    }                                                                           \
  } while (0)

void launch_density_pass(Ctx* c, MhdState* s, int n, int pass, const double* h_in, double* h_out, cudaStream_t st) {
  if (n <= 0) return;
  TimedScope ts(c, MHD_TIMING_DENSITY, st);
  MHD_DISPATCH(density_launch, c, s, n, pass, h_in, h_out, st);
  c->launches++;
}

void launch_force_prologue(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  TimedScope ts(c, MHD_TIMING_PROLOGUE, st);
  if (c->P.dim == 3)
    k_force_prologue<3><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->inv_h, c->inv_rho, c->vwave, c->psich);
  else
    k_force_prologue<2><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->inv_h, c->inv_rho, c->vwave, c->psich);
  c->launches++;
}

void launch_force_pass(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  ForceArgs a;
  a.x = s->x; a.y = s->y; a.z = s->z; a.h = s->h; a.m = s->m; a.rho = s->rho; a.omega = s->omega; a.p = s->p;
  a.epred = s->epred; a.upred = s->upred; a.vpred = s->vpred; a.wpred = s->wpred;
  a.Bx = s->Bxpred; a.By = s->Bypred; a.Bz = s->Bzpred; a.alpha1 = s->alpha1;
  a.au_prev = c->au_prev; a.av_prev = c->av_prev; a.aw_prev = c->aw_prev;
  a.inv_h = c->inv_h; a.inv_rho = c->inv_rho; a.vwave = c->vwave; a.psich = c->psich; a.psipred = s->psipred;
  a.cs = s->cs;
  a.au = s->au; a.av = s->av; a.aw = s->aw; a.ae = s->ae; a.ah = s->ah; a.div = s->div;
  a.div_for_psi = s->div_for_psi; a.dt_cfl = s->dt_cfl; a.dt_adapt = s->dt_adapt;
  a.aBx = s->aBevolx; a.aBy = s->aBevoly; a.aBz = s->aBevolz; a.apsi = s->apsi; a.divBsymm = s->divBsymm;
  a.divBdiff = s->divBdiff; a.alphaloc = s->alphaloc;
  a.xilimiter = s->xilimiter; a.divvdt = s->divvdt;
  double* cd[24] = {s->cd_rxx, s->cd_rxy, s->cd_rxz, s->cd_ryy, s->cd_ryz, s->cd_rzz, s->cd_vxx, s->cd_vxy,
                    s->cd_vxz, s->cd_vyx, s->cd_vyy, s->cd_vyz, s->cd_vzx, s->cd_vzy, s->cd_vzz, s->cd_axx,
                    s->cd_axy, s->cd_axz, s->cd_ayx, s->cd_ayy, s->cd_ayz, s->cd_azx, s->cd_azy, s->cd_azz};
  double* dv[9] = {s->dvdx_xx, s->dvdx_xy, s->dvdx_xz, s->dvdx_yx, s->dvdx_yy,
                   s->dvdx_yz, s->dvdx_zx, s->dvdx_zy, s->dvdx_zz};
  for (int k = 0; k < 24; k++) a.cd[k] = cd[k];
  for (int k = 0; k < 9; k++) a.dvdx[k] = dv[k];
  TimedScope ts(c, MHD_TIMING_FORCE, st);
  MHD_DISPATCH(force_launch, c, a, n, st);
  c->launches++;
}

}  // namespace mhd
