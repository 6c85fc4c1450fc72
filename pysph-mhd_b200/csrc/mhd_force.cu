// mhd_force.cu -- the fused force pass of the SPMHD right-hand side, in FP64
// or with FP32 pair arithmetic (sm_100a).
//
// k_force_prologue: DensityFromSmoothingLength, IdealGasEOS and
//   MagneticStateReconstruction (src/equations.py:109-118, 97-106, 474-485),
//   then one packed record per particle (ForceRec, sorted order) holding
//   everything a neighbour contributes.  The FP64 form takes pair geometry
//   from the record's FP64 positions and applies the exact FP64 neighbour
//   rule of the oracle (r^2 < (R h_i)^2 or r^2 < (R h_j)^2), so its
//   neighbour sets are bit-identical to the reference's.  The FP32 form
//   takes geometry from fixed-point positions (one wrapped 32-bit
//   difference per axis, the minimum image for free) and tests
//   r^2 < (R max(h_i, h_j))^2 in FP32: a pair within ~1e-7 (relative) of the
//   cut-off may be admitted or rejected differently from the exact rule.
//   Every compact kernel vanishes there, so the sums change by nothing but
//   FP32 rounding; for the Gaussian kernels (truncated at R = 3, W(R) ~ 1e-4
//   W(0)) such a pair changes a sum by at most one truncated-tail term.
// k_force_pass: CullenDehnenAlphaDiagnostics, MHDAccelerations,
//   MagneticStressAccelerations and MagneticStateRates as one loop over the
//   compacted neighbour list (src/equations.py:318-354, 217-275, 149-195,
//   507-559), then their post_loops, SmoothingLengthRateFromForceDivergence,
//   EnergyLimiter, DivBCorrection and AdaptiveTimestep (src/equations.py:
//   357-429, 278-280, 133-140, 562-567, 588-624, 570-585) per particle in
//   FP64.  Gather formulation: one thread per particle, no atomics on forces.
//   The pair terms are the reference's, regrouped around the displacement
//   x_ij (grad_i r-hat = omega_i |grad W_i| r-hat = omega_i t_i x_ij) so that
//   r-hat is never formed and the thermal and isotropic magnetic pressures
//   share one coefficient.  With T = float the momentum, energy, induction
//   and divergence sums are Kahan-compensated; the Cullen-Dehnen moments
//   feed a clipped limiter and use plain FP32 sums.
#include <cuda_runtime.h>

#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

// ------------------------------------------------------------ helpers
template <class T>
struct alignas(4 * sizeof(T)) V4 {
  T x, y, z, w;
};

__device__ __forceinline__ V4<float> ld4(const V4<float>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return V4<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const V4<double>* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return V4<double>{a.x, a.y, b.x, b.y};
}

// Plain FP64 sum, or a Kahan-compensated FP32 sum.
template <class T>
struct Acc {
  T s = 0;
  __device__ __forceinline__ void add(T v) { s += v; }
  __device__ __forceinline__ double get() const { return (double)s; }
};
template <>
struct Acc<float> {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float y = __fsub_rn(v, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  __device__ __forceinline__ double get() const { return (double)s - (double)c; }
};

// A kernel parameter in the pair precision: the FP32 copy or the FP64 value.
template <class T>
__device__ __forceinline__ T prm_t(float f, double d) {
  if constexpr (sizeof(T) == 4) return f;
  else return d;
}

// FP32: the MUFU approximations (about 2 ulp); FP64: IEEE division and sqrt.
__device__ __forceinline__ float fast_rcp(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double fast_rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float fast_sqrt(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }
__device__ __forceinline__ double fast_sqrt(double x) { return sqrt(x); }

// Asynchronous 16-byte copies global -> shared (cached in L1 too), so a
// neighbour's record is in flight without holding registers.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until at most one group of this thread's copies is still in flight.
__device__ __forceinline__ void cp_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// ------------------------------------------------------------ records
// The force-pass records of the particles, in the cell-sorted order: seven
// planes of four-vectors of the pair precision T (structure of arrays, so
// the 32 lanes of a warp, which mostly read consecutive neighbours, load a
// plane's entries from a few whole lines):
//   q0  FP32 {x, y, z fixed point (Grid::fx_lo), h}; FP64 {x, y, z, h}
//   q1  {m, rho, 1/rho, omega}
//   q2  {Ptot, alpha1 v_wave, v_wave, 1/rho^2}
//   q3  {upred, vpred, wpred, epred}
//   q4  {au', av', aw', 1/h}                     (a' = previous RHS)
//   q5  {Bx, By, Bz, p}
//   q6  {Bx, By, Bz / (rho sqrt(mu0)), psi c_h / rho^2}
// with Ptot = p / rho^2 + |B|^2 / (2 mu0 rho^2), the thermal and isotropic
// magnetic pressure terms that MHDAccelerations and
// MagneticStressAccelerations both weight by omega grad W.
constexpr int kForcePlanes = 7;
template <class T>
struct ForceRec {
  V4<T>* q[kForcePlanes];
};

template <class T>
struct ForceOut {
  double *au, *av, *aw, *ae, *ah, *div, *div_for_psi, *dt_cfl, *dt_adapt, *aBx, *aBy, *aBz, *apsi, *divBsymm,
      *divBdiff, *alphaloc;
  const double *cs, *psipred, *p, *rho, *h, *epred, *alpha1, *omega;  // FP64 per-particle values for the epilogue
  double *xilimiter, *divvdt;
  double* cd[24];   // rxx rxy rxz ryy ryz rzz vxx..vzz axx..azz
  double* dvdx[9];  // xx xy xz yx yy yz zx zy zz
};

// Prologue: G2 (rho from h), G3 (EOS), G5 (B = B/rho * rho) and the records.
template <int DIM, class T>
__global__ void __launch_bounds__(256) k_force_prologue(int n, DevParams P, MhdState s, const double* __restrict__ aup,
                                                        const double* __restrict__ avp,
                                                        const double* __restrict__ awp, const Grid* __restrict__ grids,
                                                        const int* __restrict__ inst, ForceRec<T> rec,
                                                        float4* __restrict__ posf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h = s.h[i];
  reinterpret_cast<float*>(posf + i)[3] = (float)h;  // h after the density iteration
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
  const double b2 = bx * bx + by * by + bz * bz;
  const double vw = sqrt(cs * cs + b2 / (P.mu0 * rho));
  const double ir = 1.0 / rho, ir2 = ir * ir;
  const double om = s.omega[i];
  const double bs = ir * sqrt(P.inv_mu0);
  const double x = s.x[i], y = s.y[i], z = DIM == 3 ? s.z[i] : 0.0;
  if constexpr (sizeof(T) == 4) {
    const Grid& G = grid_of(grids, inst, i);
    rec.q[0][i] = V4<T>{__uint_as_float(fixed_coord(G, 0, x)), __uint_as_float(fixed_coord(G, 1, y)),
                        DIM == 3 ? __uint_as_float(fixed_coord(G, 2, z)) : 0.f, (float)h};
  } else {
    rec.q[0][i] = V4<T>{(T)x, (T)y, (T)z, (T)h};
  }
  rec.q[1][i] = V4<T>{(T)s.m[i], (T)rho, (T)ir, (T)om};
  rec.q[2][i] = V4<T>{(T)(p * ir2 + 0.5 * b2 * P.inv_mu0 * ir2), (T)(s.alpha1[i] * vw), (T)vw, (T)ir2};
  rec.q[3][i] = V4<T>{(T)s.upred[i], (T)s.vpred[i], (T)s.wpred[i], (T)s.epred[i]};
  rec.q[4][i] = V4<T>{(T)aup[i], (T)avp[i], (T)awp[i], (T)(1.0 / h)};
  rec.q[5][i] = V4<T>{(T)bx, (T)by, (T)bz, (T)p};
  rec.q[6][i] = V4<T>{(T)(bx * bs), (T)(by * bs), (T)(bz * bs), (T)(s.psipred[i] * (P.clean_speed * vw) * ir2)};
}

// Cullen-Dehnen moments of one particle (src/equations.py:329-354):
// R_ab = -sum x_a m grad_b W, V_ab = sum dv_a m grad_b W, A_ab = sum da_a
// m grad_b W with grad W = t x_ij.  In a 2-D layout the limiter takes the
// determinant-free branch, which needs only V and the trace of A, so only
// those are summed there.
template <int DIM, class T>
struct CdMoments {
  T rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
  T vxx = 0, vxy = 0, vxz = 0, vyx = 0, vyy = 0, vyz = 0, vzx = 0, vzy = 0, vzz = 0;
  T axx = 0, axy = 0, axz = 0, ayx = 0, ayy = 0, ayz = 0, azx = 0, azy = 0, azz = 0;
  __device__ __forceinline__ void add(T c, T dx, T dy, T dz, T dvx, T dvy, T dvz, T dax, T day, T daz) {
    const T cx = c * dx, cy = c * dy, cz = c * dz;
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
};

// CullenDehnenAlphaDiagnostics.post_loop (src/equations.py:357-429) and
// StrainDiagnostics (:432-471) in FP64: alpha_loc, and the diagnostics the
// caller asked for.
template <int DIM, class T>
__device__ __forceinline__ void cd_post(const CdMoments<DIM, T>& M, int i, const DevParams& P, const ForceOut<T>& o) {
  const double termnorm = o.omega[i] / o.rho[i];
  const double Rxx = M.rxx, Rxy = M.rxy, Rxz = M.rxz, Ryy = M.ryy, Ryz = M.ryz, Rzz = M.rzz;
  const double Vxx = M.vxx, Vxy = M.vxy, Vxz = M.vxz, Vyx = M.vyx, Vyy = M.vyy, Vyz = M.vyz, Vzx = M.vzx,
               Vzy = M.vzy, Vzz = M.vzz;
  const double Axx = M.axx, Axy = M.axy, Axz = M.axz, Ayx = M.ayx, Ayy = M.ayy, Ayz = M.ayz, Azx = M.azx,
               Azy = M.azy, Azz = M.azz;
  double div_a, dvxdx, dvxdy, dvxdz, dvydx, dvydy, dvydz, dvzdx, dvzdy, dvzdz;
  const double denom =
      DIM == 3 ? Rxx * Ryy * Rzz + 2.0 * Rxy * Rxz * Ryz - Rxx * Ryz * Ryz - Ryy * Rxz * Rxz - Rzz * Rxy * Rxy : 0.0;
  if (fabs(denom) > kFloatTiny) {
    const double dd = 1.0 / denom;
    const double t0 = (Ryy * Rzz - Ryz * Ryz) * dd, t1 = (Rxz * Ryz - Rzz * Rxy) * dd;
    const double t2 = (Rxy * Ryz - Rxz * Ryy) * dd, t3 = (Rzz * Rxx - Rxz * Rxz) * dd;
    const double t4 = (Rxy * Rxz - Rxx * Ryz) * dd, t5 = (Rxx * Ryy - Rxy * Rxy) * dd;
    div_a = -((Axx * t0 + Axy * t1 + Axz * t2) + (Ayx * t1 + Ayy * t3 + Ayz * t4) + (Azx * t2 + Azy * t4 + Azz * t5));
    dvxdx = -(Vxx * t0 + Vxy * t1 + Vxz * t2);
    dvxdy = -(Vxx * t1 + Vxy * t3 + Vxz * t4);
    dvxdz = -(Vxx * t2 + Vxy * t4 + Vxz * t5);
    dvydx = -(Vyx * t0 + Vyy * t1 + Vyz * t2);
    dvydy = -(Vyx * t1 + Vyy * t3 + Vyz * t4);
    dvydz = -(Vyx * t2 + Vyy * t4 + Vyz * t5);
    dvzdx = -(Vzx * t0 + Vzy * t1 + Vzz * t2);
    dvzdy = -(Vzx * t1 + Vzy * t3 + Vzz * t4);
    dvzdz = -(Vzx * t2 + Vzy * t4 + Vzz * t5);
  } else {
    div_a = -termnorm * (Axx + Ayy + Azz);
    dvxdx = -termnorm * Vxx; dvxdy = -termnorm * Vxy; dvxdz = -termnorm * Vxz;
    dvydx = -termnorm * Vyx; dvydy = -termnorm * Vyy; dvydz = -termnorm * Vyz;
    dvzdx = -termnorm * Vzx; dvzdy = -termnorm * Vzy; dvzdz = -termnorm * Vzz;
  }
  const double divvdt =
      div_a - (dvxdx * dvxdx + dvydy * dvydy + dvzdz * dvzdz + 2.0 * (dvxdy * dvydx + dvxdz * dvzdx + dvydz * dvzdy));
  const double divv = dvxdx + dvydy + dvzdz;
  const double curlx = dvzdy - dvydz, curly = dvxdz - dvzdx, curlz = dvydx - dvxdy;
  const double compression = fmax(-divv, 0.0);
  const double fac = compression * compression;
  const double denominator = fac + (curlx * curlx + curly * curly + curlz * curlz);
  const double xil = denominator > 0.0 ? fac / denominator : 1.0;
  const double hid = o.h[i];
  const double source = 10.0 * hid * hid * xil * fmax(-divvdt, 0.0);
  const double csi = o.cs[i];
  // alpha clip: reference literal [0, 1] (src/equations.py:428); alpha_min/max extend it
  o.alphaloc[i] = fmax(fmin(source / (csi * csi), P.alpha_max), P.alpha_min);
  if (o.xilimiter) o.xilimiter[i] = xil;
  if (o.divvdt) o.divvdt[i] = divvdt;
  if (o.cd[0]) {
    const double v[24] = {Rxx, Rxy, Rxz, Ryy, Ryz, Rzz, Vxx, Vxy, Vxz, Vyx, Vyy, Vyz,
                          Vzx, Vzy, Vzz, Axx, Axy, Axz, Ayx, Ayy, Ayz, Azx, Azy, Azz};
#pragma unroll
    for (int k = 0; k < 24; k++)
      if (o.cd[k]) o.cd[k][i] = v[k];
  }
  if (o.dvdx[0]) {
    const double v[9] = {dvxdx, dvxdy, dvxdz, dvydx, dvydy, dvydz, dvzdx, dvzdy, dvzdz};
#pragma unroll
    for (int k = 0; k < 9; k++)
      if (o.dvdx[k]) o.dvdx[k][i] = v[k];
  }
}

// Launch shapes (threads per block, minimum resident blocks per SM): the
// second number caps the registers and so sets the occupancy.
constexpr int kForceShapes[][2] = {{128, 2}, {128, 3}, {128, 4}, {256, 2}};
constexpr int kForceShapeCount = 4;

// One particle i of the force pass: its record values, the pair sums and
// the pair terms (CullenDehnenAlphaDiagnostics, MHDAccelerations,
// MagneticStressAccelerations, MagneticStateRates loops) with neighbour
// records j, and the FP64 epilogue.  Shared by the list-driven pass and the
// cell-tile pass, which differ only in how they walk the neighbours.
template <int K, int DIM, class T>
struct ForceParticle {
  V4<T> pi;
  T h1i, norm, faci1, rhoi, irhoi, omegai, ptoti, AI, vwi, irho2i, ui, vi, wi, epi, aui, avi, awi, bxi, byi, bzi,
      p_i, bsxi, bsyi, bszi, psii, pr2i, av, ac, ar, inv_mu0;
  float Rf, rhi2f;
  double rhi2;
  CdMoments<DIM, T> M;
  Acc<T> fx, fy, fz, fe, fdiv, bxr, byr, bzr, dbs, dbd;
  T dtc;

  __device__ __forceinline__ void init(int i, const DevParams& P, const ForceRec<T>& rec) {
    pi = rec.q[0][i];
    const V4<T> i1 = rec.q[1][i], i2 = rec.q[2][i], i3 = rec.q[3][i], i4 = rec.q[4][i], i5 = rec.q[5][i],
                i6 = rec.q[6][i];
    h1i = i4.w;
    norm = prm_t<T>(P.normf, P.norm);
    // grad W(h_i) = faci1 dw(q) / r * x_ij
    faci1 = norm * (DIM == 2 ? h1i * h1i * h1i : (h1i * h1i) * (h1i * h1i));
    rhoi = i1.y; irhoi = i1.z; omegai = i1.w;
    ptoti = i2.x; AI = i2.y; vwi = i2.z; irho2i = i2.w;
    ui = i3.x; vi = i3.y; wi = i3.z; epi = i3.w;
    aui = i4.x; avi = i4.y; awi = i4.z;
    bxi = i5.x; byi = i5.y; bzi = i5.z; p_i = i5.w;
    bsxi = i6.x; bsyi = i6.y; bszi = i6.z; psii = i6.w;
    pr2i = p_i * irho2i;
    av = prm_t<T>(P.avf, P.av); ac = prm_t<T>(P.acf, P.ac); ar = prm_t<T>(P.arf, P.ar);
    inv_mu0 = prm_t<T>(P.inv_mu0f, P.inv_mu0);
    // neighbour test r^2 < (R max(h_i, h_j))^2: FP32 on the FP32 form, the
    // exact FP64 rule of the oracle on the FP64 form
    Rf = P.Rf;
    rhi2f = (Rf * (float)pi.w) * (Rf * (float)pi.w);
    rhi2 = rh2_exact(P.R, (double)pi.w);
    dtc = 0;
  }

  // the self pair: every sum term carries a zero kernel gradient or a zero
  // displacement; only the signal speed max(vw_i - 2 dot, 0) = vw_i enters
  // dt_cfl
  __device__ __forceinline__ void self_pair() { dtc = fmax(dtc, vwi); }

  // A candidate j: the neighbour test, then the pair terms.
  __device__ __forceinline__ void pair(const Grid& G, const DevParams& P, const V4<T>& pj, const V4<T>& j1,
                                       const V4<T>& j2, const V4<T>& j3, const V4<T>& j4, const V4<T>& j5,
                                       const V4<T>& j6) {
    const T two = (T)2, half = (T)0.5, zero = (T)0;
    T dx, dy, dz, r, inv_r;
    if constexpr (sizeof(T) == 4) {
      // FP32 geometry: one wrapped fixed-point difference per axis
      dx = fixed_delta(G, 0, __float_as_uint(pi.x), __float_as_uint(pj.x));
      dy = fixed_delta(G, 1, __float_as_uint(pi.y), __float_as_uint(pj.y));
      dz = DIM == 3 ? fixed_delta(G, 2, __float_as_uint(pi.z), __float_as_uint(pj.z)) : 0.f;
      const float r2 = dx * dx + dy * dy + dz * dz;
      const float rhj = Rf * pj.w;
      if (!(r2 < fmaxf(rhi2f, rhj * rhj))) return;
      inv_r = r2 > 0.f ? rsqrtf(r2) : 0.f;
      r = r2 * inv_r;
    } else {
      // FP64 geometry and the exact neighbour test of the oracle
      const double dxd = min_image((double)pi.x - pj.x, G.L[0], G.half[0], G.periodic[0]);
      const double dyd = min_image((double)pi.y - pj.y, G.L[1], G.half[1], G.periodic[1]);
      const double dzd = DIM == 3 ? min_image((double)pi.z - pj.z, G.L[2], G.half[2], G.periodic[2]) : 0.0;
      const double r2d = r2_exact(dxd, dyd, dzd);
      if (!(r2d < rhi2 || r2d < rh2_exact(P.R, pj.w))) return;
      dx = dxd;
      dy = dyd;
      dz = dzd;
      r = sqrt(r2d);
      inv_r = r > 0.0 ? 1.0 / r : 0.0;
    }
    const T mj = j1.x, rhoj = j1.y, irhoj = j1.z, omegaj = j1.w;
    const T h1j = j4.w;
    // DWI = ti XIJ, DWJ = tj XIJ (zero at r <= 1e-12); oti, otj carry omega
    T ti = 0, tj = 0;
    if (r > (T)kPairDistanceEpsilon) {
      T w, dw;
      w_dw<K>(r * h1i, DIM, w, dw);
      ti = faci1 * dw * inv_r;
      w_dw<K>(r * h1j, DIM, w, dw);
      tj = norm * (DIM == 2 ? h1j * h1j * h1j : (h1j * h1j) * (h1j * h1j)) * dw * inv_r;
    }
    const T oti = omegai * ti, otj = omegaj * tj;
    const T dvx = ui - j3.x, dvy = vi - j3.y, dvz = wi - j3.z;
    const T vdotx = dvx * dx + dvy * dy + dvz * dz;

    // ---- CullenDehnenAlphaDiagnostics.loop
    M.add(mj * ti, dx, dy, dz, dvx, dvy, dvz, aui - j4.x, avi - j4.y, awi - j4.z);
    // ---- MHDAccelerations, MagneticStressAccelerations and
    // MagneticStateRates loops, in the displacement x_ij instead of r-hat:
    // grad_i r-hat = omega_i ti x_ij = oti x_ij wherever grad_i != 0.
    // MHDAccelerations drops r-hat (and so dot, the viscosity, conduction
    // and div v terms) below r = 1e-8.
    const bool far = r >= (T)kInteractionDistanceEpsilon;
    const T vdf = far ? vdotx : zero;  // (v_ij . r-hat) r
    const T dot = vdf * inv_r;
    // artificial viscosity (v_ij . r-hat < 0)
    T qi = zero, qj = zero;
    if (dot < zero) {
      qi = -half * irhoi * fmax(AI - two * dot, zero) * dot * av;
      qj = -half * irhoj * fmax(j2.y - two * dot, zero) * dot * av;
    }
    dtc = fmax(dtc, fmax(vwi, j2.z) - two * dot);
    // momentum: -x_ij m_j (oti (Ptot_i + q_i) + otj (Ptot_j + q_j)) + the
    // anisotropic Maxwell stress m_j (b_i (b_i . x_ij) oti + b_j (b_j . x_ij) otj)
    const T S = oti * (ptoti + qi) + otj * (j2.x + qj);
    const T ai = oti * (bsxi * dx + bsyi * dy + bszi * dz);
    const T aj = otj * (j6.x * dx + j6.y * dy + j6.z * dz);
    fx.add(mj * (-dx * S + (bsxi * ai + j6.x * aj)));
    fy.add(mj * (-dy * S + (bsyi * ai + j6.y * aj)));
    fz.add(mj * (-dz * S + (bszi * ai + j6.z * aj)));
    // div v, energy (thermal, viscous, conduction with v_sig = sqrt(|dp| / rho_bar))
    const T mo = mj * oti;
    fdiv.add(mo * vdf);
    const T vsig2 = fast_sqrt(fabs(p_i - j5.w) * fast_rcp(half * (rhoi + rhoj)));
    const T rf = far ? r : zero;
    T fei = mo * (pr2i * vdotx + qi * vdf);
    fei += ac * vsig2 * (epi - j3.w) * (half * mj * rf * (oti * irhoi + otj * irhoj));
    // induction, resistivity (v_sig,B = |v_ij - (v_ij . r-hat) r-hat|), cleaning
    const T xbi = bxi * dx + byi * dy + bzi * dz;
    const T xbj = j5.x * dx + j5.y * dy + j5.z * dz;
    const T wi_ = oti * irho2i, wj_ = otj * j2.w;
    const T pv = vdotx * (inv_r * inv_r);
    const T tx = dvx - pv * dx, ty = dvy - pv * dy, tz = dvz - pv * dz;
    const T vsig_b = fast_sqrt(tx * tx + ty * ty + tz * tz);
    const T diss = half * mj * r * (wi_ + wj_) * vsig_b * ar;
    const T dbx = bxi - j5.x, dby = byi - j5.y, dbz = bzi - j5.z;
    const T d_brho = -mj * wi_ * xbi;
    const T cpsi = mj * (oti * psii + otj * j6.w);
    bxr.add(d_brho * dvx + diss * dbx - cpsi * dx);
    byr.add(d_brho * dvy + diss * dby - cpsi * dy);
    bzr.add(d_brho * dvz + diss * dbz - cpsi * dz);
    fe.add(fei + (-half * (dbx * dbx + dby * dby + dbz * dbz) * diss * inv_mu0));
    dbs.add(mj * (wi_ * xbi + wj_ * xbj));
    dbd.add(-mo * (xbi - xbj));
  }

  // Post-loops in FP64: CullenDehnenAlphaDiagnostics (+ StrainDiagnostics),
  // MHDAccelerations, SmoothingLengthRateFromForceDivergence,
  // MagneticStateRates, EnergyLimiter, DivBCorrection, AdaptiveTimestep.
  __device__ __forceinline__ void finish(int i, const DevParams& P, const ForceOut<T>& o) const {
    const double rhoi_d = o.rho[i], irho_d = 1.0 / rhoi_d;
    const double hid = o.h[i], csi = o.cs[i];
    cd_post<DIM, T>(M, i, P, o);
    // MHDAccelerations.post_loop, SmoothingLengthRateFromForceDivergence
    const double divi = -fdiv.get() * irho_d;
    // MagneticStateRates.post_loop (src/equations.py:562-567)
    const double vwid =
        sqrt(csi * csi + ((double)bxi * bxi + (double)byi * byi + (double)bzi * bzi) * P.inv_mu0 * irho_d);
    const double chi = P.clean_speed * vwid;
    const double psipi = o.psipred[i];
    const double dbdv = dbd.get(), dbsv = dbs.get();
    const double apsi = -chi * dbdv * irho_d - P.clean_damp * psipi * chi / hid - 0.5 * P.clean_active * psipi * divi;
    double dtcd = dtc;
    dtcd = fmax(dtcd, vwid);
    dtcd = fmax(dtcd, chi);
    // EnergyLimiter (src/equations.py:594-598)
    double fed = fe.get();
    const double epid = o.epred[i];
    if (dtcd > 0.0) {
      const double dtcour = P.c_cour * hid / dtcd;
      if (epid + dtcour * fed < 0.0 && epid > 0.0) fed /= 1.0 - dtcour * fed / epid;
    }
    // DivBCorrection (src/equations.py:607-624)
    double ax = fx.get(), ay = fy.get(), az = fz.get();
    {
      const double bxd = bxi, byd = byi, bzd = bzi;
      const double b2 = bxd * bxd + byd * byd + bzd * bzd;
      double frac = 0.0;
      if (b2 > 0.0) {
        const double betap = 2.0 * P.mu0 * o.p[i] / b2;
        frac = fmax(0.0, fmin(1.0, (10.0 - betap) * 0.125));
      }
      const double cf = dbsv * frac * P.inv_mu0;
      ax -= bxd * cf;
      ay -= byd * cf;
      az -= bzd * cf;
    }
    // AdaptiveTimestep (src/equations.py:578-585)
    double dta = kBigNumber;
    if (dtcd > 0.0) dta = P.c_cour * hid / dtcd;
    const double f2 = ax * ax + ay * ay + az * az;
    if (f2 > 0.0) dta = fmin(dta, P.c_force * sqrt(hid / sqrt(f2)));

    o.au[i] = ax;
    o.av[i] = ay;
    o.aw[i] = az;
    o.ae[i] = fed;
    o.ah[i] = hid * divi * (1.0 / (double)DIM);
    o.div[i] = divi;
    o.div_for_psi[i] = divi;
    o.dt_cfl[i] = dtcd;
    o.dt_adapt[i] = dta;
    o.aBx[i] = bxr.get();
    o.aBy[i] = byr.get();
    o.aBz[i] = bzr.get();
    o.apsi[i] = apsi;
    o.divBsymm[i] = rhoi_d * dbsv;
    o.divBdiff[i] = dbdv;
  }
};

// List-driven pass: one thread per particle walks its compacted neighbour
// list.  STAGED: each thread copies its next neighbour's record into its own
// slot of a two-stage shared-memory buffer (cp.async) while it computes the
// current pair, so a pair no longer waits on a gather from L1/L2.
template <int K, int DIM, class T, int SHAPE, bool STAGED>
__global__ void __launch_bounds__(kForceShapes[SHAPE][0], kForceShapes[SHAPE][1])
    k_force_pass(int n, DevParams P, NbrList L, const Grid* __restrict__ grids, const int* __restrict__ inst,
                 const ForceRec<T> rec, ForceOut<T> o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& G = grid_of(grids, inst, i);
  ForceParticle<K, DIM, T> F;
  F.init(i, P, rec);

  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  // Staged: slot [stage][plane][thread] of the dynamic shared buffer; the
  // list entries run two pairs ahead of the computed pair, its record one.
  // Register gather: the list entry is fetched one pair ahead and every
  // record of a pair is requested before its neighbour test, so a pair waits
  // on one memory round trip instead of three (entry, position, records).
  constexpr int NT = kForceShapes[SHAPE][0];
  extern __shared__ __align__(16) unsigned char force_smem[];
  V4<T>* __restrict__ sb = reinterpret_cast<V4<T>*>(force_smem) + threadIdx.x;
  auto fetch = [&](int stage, int jj) {
#pragma unroll
    for (int p = 0; p < kForcePlanes; p++) {
      V4<T>* dst = sb + (stage * kForcePlanes + p) * NT;
      const V4<T>* src = rec.q[p] + jj;
#pragma unroll
      for (int b = 0; b < (int)(sizeof(V4<T>) / 16); b++)
        cp_async16(reinterpret_cast<char*>(dst) + 16 * b, reinterpret_cast<const char*>(src) + 16 * b);
    }
    cp_async_commit();
  };
  int jn = cnt > 0 ? row[0] : i;
  int jn2 = i;
  if constexpr (STAGED) {
    fetch(0, jn);
    jn2 = cnt > 1 ? row[32] : i;
  }
  for (int k = 0; k < cnt; k++) {
    const int j = jn;
    if constexpr (STAGED) {
      jn = jn2;
      if (k + 1 < cnt) fetch((k + 1) & 1, jn);
      else cp_async_commit();  // an empty group keeps the wait below uniform
      if (k + 2 < cnt) jn2 = row[(k + 2) * 32];
      cp_async_wait_all_but_one();
      if (j == i) {
        F.self_pair();
        continue;
      }
      const V4<T>* st = sb + ((k & 1) * kForcePlanes) * NT;
      F.pair(G, P, st[0], st[NT], st[2 * NT], st[3 * NT], st[4 * NT], st[5 * NT], st[6 * NT]);
    } else {
      if (k + 1 < cnt) jn = row[(k + 1) * 32];
      if (j == i) {
        F.self_pair();
        continue;
      }
      F.pair(G, P, ld4(rec.q[0] + j), ld4(rec.q[1] + j), ld4(rec.q[2] + j), ld4(rec.q[3] + j), ld4(rec.q[4] + j),
             ld4(rec.q[5] + j), ld4(rec.q[6] + j));
    }
  }
  F.finish(i, P, o);
}

// Cell-tile pass (FP32 form, an alternative kept for comparison): no
// neighbour list.  Each warp takes 32 consecutive particles of the sorted
// order, walks the union of their search stencils row by row (one
// contiguous index range per row piece, as the list build does), stages 32
// candidate records at a time in shared memory with coalesced 16-byte loads
// (each record read from memory once per warp), and every lane tests every
// staged candidate against its own particle and adds the pair terms of its
// neighbours.  A big particle (h beyond what the grid's stencil covers) can
// reach a particle from beyond that union; its pairs are then missed, so
// this pass is exact only while no particle is big.
constexpr int kTileThreads = 128;
template <int K, int DIM>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_force_tiles(int n, DevParams P, const Grid* __restrict__ grids, const int* __restrict__ inst,
                  const int* __restrict__ cell_start, const int* __restrict__ cellc, const ForceRec<float> rec,
                  ForceOut<float> o) {
  using T = float;
  __shared__ V4<T> tile[kTileThreads / 32][kForcePlanes][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = (blockIdx.x * kTileThreads + threadIdx.x) & ~31;
  if (i0 >= n) return;
  const int i = i0 + lane;
  const bool live = i < n;
  const int ii = live ? i : i0;
  const Grid& G = grid_of(grids, inst, ii);
  ForceParticle<K, DIM, T> F;
  F.init(ii, P, rec);
  // the warp's cell extents (the warp's particles share one instance: a
  // warp that straddles two instances takes the first one's grid, and the
  // second instance's particles are taken whole by their own warps)
  int cx, cy, cz;
  unpack_cell<DIM>(cellc[ii], cx, cy, cz);
  int lo[3] = {cx, cy, cz}, hi[3] = {cx, cy, cz};
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  const int sw = G.sw;
  const int nc[3] = {G.nc[0], G.nc[1], DIM == 3 ? G.nc[2] : 1};
  int a_lo[3], a_hi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const bool whole = a >= DIM || nc[a] < 2 * sw + 1 + (hi[a] - lo[a]);
    a_lo[a] = whole ? 0 : lo[a] - sw;
    a_hi[a] = whole ? nc[a] - 1 : hi[a] + sw;
  }
  V4<T>(*buf)[32] = tile[warp];
  for (int zu = a_lo[2]; zu <= a_hi[2]; zu++) {
    const int zc = zu < 0 ? zu + nc[2] : (zu >= nc[2] ? zu - nc[2] : zu);
    if (!G.periodic[2] && zc != zu) continue;
    for (int yu = a_lo[1]; yu <= a_hi[1]; yu++) {
      const int yc = yu < 0 ? yu + nc[1] : (yu >= nc[1] ? yu - nc[1] : yu);
      if (!G.periodic[1] && yc != yu) continue;
      const int base = G.cell_base + (zc * nc[1] + yc) * nc[0];
      // x pieces: below 0, inside, above nx - 1 (periodic wrap)
      for (int piece = 0; piece < 3; piece++) {
        int xl, xh;
        if (piece == 0) { xl = a_lo[0]; xh = min(a_hi[0], -1); }
        else if (piece == 1) { xl = max(a_lo[0], 0); xh = min(a_hi[0], nc[0] - 1); }
        else { xl = max(a_lo[0], nc[0]); xh = a_hi[0]; }
        if (xl > xh) continue;
        if (piece != 1) {
          if (!G.periodic[0]) continue;
          const int s = piece == 0 ? nc[0] : -nc[0];
          xl += s;
          xh += s;
        }
        const int jb = cell_start[base + xl], je = cell_start[base + xh + 1];
        for (int t0 = jb; t0 < je; t0 += 32) {
          const int m = min(32, je - t0);
          __syncwarp();
          if (lane < m) {
#pragma unroll
            for (int p = 0; p < kForcePlanes; p++) buf[p][lane] = ld4(rec.q[p] + t0 + lane);
          }
          __syncwarp();
          for (int c = 0; c < m; c++) {
            const int j = t0 + c;
            if (j == ii) {
              F.self_pair();
              continue;
            }
            F.pair(G, P, buf[0][c], buf[1][c], buf[2][c], buf[3][c], buf[4][c], buf[5][c], buf[6][c]);
          }
        }
      }
    }
  }
  if (live) F.finish(i, P, o);
}

// 2-D complement of the Cullen-Dehnen moments.  In a 2-D layout the force
// pass takes the fallback branch of the limiter (the 3x3 determinant is
// zero), which needs neither R_ab nor the off-diagonal A_ab, so it does not
// sum R_xx, R_xy, R_yy, A_xy, A_yx, A_zx, A_zy (A_z* is non-zero when a field
// component along z gives a z acceleration).  When the caller asks for the cd_*
// diagnostics this pass sums them as CullenDehnenAlphaDiagnostics.loop does
// (src/equations.py:318-354), in FP64 over the neighbour list, and writes
// them over the force pass's zeros.
template <int K>
__global__ void __launch_bounds__(128) k_cd_complement_2d(int n, DevParams P, NbrList L, const Grid* __restrict__ grids,
                                                          const int* __restrict__ inst, const double* __restrict__ x,
                                                          const double* __restrict__ y, const double* __restrict__ h,
                                                          const double* __restrict__ m, const double* __restrict__ aup,
                                                          const double* __restrict__ avp,
                                                          const double* __restrict__ awp, double* __restrict__ rxx,
                                                          double* __restrict__ rxy, double* __restrict__ ryy,
                                                          double* __restrict__ axy, double* __restrict__ ayx,
                                                          double* __restrict__ azx, double* __restrict__ azy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& G = grid_of(grids, inst, i);
  const double xi = x[i], yi = y[i], hi = h[i];
  const double h1 = 1.0 / hi, fac = P.norm * (h1 * h1), rhi2 = rh2_exact(P.R, hi);
  const double aui = aup[i], avi = avp[i], awi = awp[i];
  double sxx = 0.0, sxy = 0.0, syy = 0.0, sab = 0.0, sba = 0.0, szx = 0.0, szy = 0.0;
  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  for (int k = 0; k < cnt; k++) {
    const int j = row[k * 32];
    const double dx = min_image(xi - x[j], G.L[0], G.half[0], G.periodic[0]);
    const double dy = min_image(yi - y[j], G.L[1], G.half[1], G.periodic[1]);
    const double r2 = r2_exact(dx, dy, 0.0);
    if (!(r2 < rhi2)) continue;  // W(h_i) and its gradient vanish beyond R h_i
    const double r = sqrt(r2);
    if (!(r > kPairDistanceEpsilon)) continue;
    double w, dw;
    w_dw<K>(r * h1, 2, w, dw);
    const double t = fac * dw * h1 / r;
    const double runx = m[j] * (t * dx), runy = m[j] * (t * dy);
    sxx += -dx * runx;
    sxy += -dx * runy;
    syy += -dy * runy;
    sab += (aui - aup[j]) * runy;
    sba += (avi - avp[j]) * runx;
    const double daz = awi - awp[j];
    szx += daz * runx;
    szy += daz * runy;
  }
  if (rxx) rxx[i] = sxx;
  if (rxy) rxy[i] = sxy;
  if (ryy) ryy[i] = syy;
  if (axy) axy[i] = sab;
  if (ayx) ayx[i] = sba;
  if (azx) azx[i] = szx;
  if (azy) azy[i] = szy;
}

// ------------------------------------------------------------- dispatch
template <class T>
static ForceRec<T> records(Ctx* c) {
  ForceRec<T> r;
  V4<T>* base = reinterpret_cast<V4<T>*>(c->frec);
  for (int k = 0; k < kForcePlanes; k++) r.q[k] = base + (size_t)k * c->n_pad;
  return r;
}

template <class T>
static void prologue_launch(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  const ForceRec<T> rec = records<T>(c);
  if (c->P.dim == 3)
    k_force_prologue<3, T><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->au_prev, c->av_prev, c->aw_prev,
                                                            c->d_grids, c->inst, rec, c->posf);
  else
    k_force_prologue<2, T><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->au_prev, c->av_prev, c->aw_prev,
                                                            c->d_grids, c->inst, rec, c->posf);
}

void launch_force_prologue(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  TimedScope ts(c, MHD_TIMING_PROLOGUE, st);
  if (c->P.fp32)
    prologue_launch<float>(c, s, n, st);
  else
    prologue_launch<double>(c, s, n, st);
  c->launches++;
}

// Dynamic shared memory of the staged force pass: two stages of the seven
// record planes per thread.
template <class T>
constexpr size_t force_stage_bytes(int threads) {
  return (size_t)2 * kForcePlanes * sizeof(V4<T>) * threads;
}

template <int K, int DIM, class T, int SHAPE, bool STAGED>
static void force_launch_one(Ctx* c, const ForceOut<T>& o, int n, cudaStream_t st) {
  constexpr int bs = kForceShapes[SHAPE][0];
  const size_t smem = STAGED ? force_stage_bytes<T>(bs) : 0;
  k_force_pass<K, DIM, T, SHAPE, STAGED><<<(n + bs - 1) / bs, bs, smem, st>>>(n, c->P, c->lists(), c->d_grids,
                                                                            c->inst, records<T>(c), o);
}

template <int K, int DIM, class T, bool STAGED>
static void force_launch_shape(Ctx* c, const ForceOut<T>& o, int n, cudaStream_t st) {
  // default shapes measured on the 128^3 blast (FP64 uncapped, FP32 capped
  // for occupancy); the autotuner may pick another
  const int s = c->force_shape >= 0 ? c->force_shape : (sizeof(T) == 4 ? 2 : 0);
  switch (s) {
    case 1: force_launch_one<K, DIM, T, 1, STAGED>(c, o, n, st); break;
    case 2: force_launch_one<K, DIM, T, 2, STAGED>(c, o, n, st); break;
    case 3: force_launch_one<K, DIM, T, 3, STAGED>(c, o, n, st); break;
    default: force_launch_one<K, DIM, T, 0, STAGED>(c, o, n, st);
  }
}

// The FP32 form stages its neighbours' records in shared memory (measured
// on the 128^3 blast: 1.87 ms per pass against 1.99 for the register
// gather); the FP64 form gathers into registers (4.69 ms against 5.71 ms
// staged, whose 57 KB of shared memory per block halves the resident blocks).
template <int K, int DIM, class T>
static void force_launch_t(Ctx* c, const ForceOut<T>& o, int n, cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    if (c->force_tiles) {
      k_force_tiles<K, DIM><<<(n + kTileThreads - 1) / kTileThreads, kTileThreads, 0, st>>>(
          n, c->P, c->d_grids, c->inst, c->cell_start, c->cellc, records<T>(c), o);
      return;
    }
    if (c->force_staged) {
      force_launch_shape<K, DIM, T, true>(c, o, n, st);
      return;
    }
  }
  force_launch_shape<K, DIM, T, false>(c, o, n, st);
}

// The staged passes need more dynamic shared memory than the default
// limit: raise it for every launch shape of the context's kernel,
// dimension and precision (at set-up, never inside a stream capture).
template <int K, int DIM, class T>
static cudaError_t configure_shapes() {
  cudaError_t e = cudaSuccess;
  auto one = [&](auto fn, int threads) {
    const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)force_stage_bytes<T>(threads));
    if (r != cudaSuccess) e = r;
  };
  one(k_force_pass<K, DIM, T, 0, true>, kForceShapes[0][0]);
  one(k_force_pass<K, DIM, T, 1, true>, kForceShapes[1][0]);
  one(k_force_pass<K, DIM, T, 2, true>, kForceShapes[2][0]);
  one(k_force_pass<K, DIM, T, 3, true>, kForceShapes[3][0]);
  return e;
}

template <int K, int DIM>
static cudaError_t configure_kd(Ctx* c) {
  return c->P.fp32 ? configure_shapes<K, DIM, float>() : cudaSuccess;
}

cudaError_t configure_force_pass(Ctx* c) {
  const int d3 = c->P.dim == 3;
  switch (c->P.kernel) {
    case MHD_KERNEL_CUBIC: return d3 ? configure_kd<0, 3>(c) : configure_kd<0, 2>(c);
    case MHD_KERNEL_QUINTIC: return d3 ? configure_kd<1, 3>(c) : configure_kd<1, 2>(c);
    case MHD_KERNEL_WENDLAND_C2: return d3 ? configure_kd<2, 3>(c) : configure_kd<2, 2>(c);
    case MHD_KERNEL_WENDLAND_C4: return d3 ? configure_kd<3, 3>(c) : configure_kd<3, 2>(c);
    case MHD_KERNEL_WENDLAND_C6: return d3 ? configure_kd<4, 3>(c) : configure_kd<4, 2>(c);
    case MHD_KERNEL_GAUSSIAN: return d3 ? configure_kd<5, 3>(c) : configure_kd<5, 2>(c);
    default: return d3 ? configure_kd<6, 3>(c) : configure_kd<6, 2>(c);
  }
}

template <int K, int DIM>
static void force_launch(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  auto fill = [&](auto& o) {
    o.au = s->au; o.av = s->av; o.aw = s->aw; o.ae = s->ae; o.ah = s->ah; o.div = s->div;
    o.div_for_psi = s->div_for_psi; o.dt_cfl = s->dt_cfl; o.dt_adapt = s->dt_adapt;
    o.aBx = s->aBevolx; o.aBy = s->aBevoly; o.aBz = s->aBevolz; o.apsi = s->apsi; o.divBsymm = s->divBsymm;
    o.divBdiff = s->divBdiff; o.alphaloc = s->alphaloc;
    o.cs = s->cs; o.psipred = s->psipred; o.p = s->p; o.rho = s->rho; o.h = s->h; o.epred = s->epred;
    o.alpha1 = s->alpha1; o.omega = s->omega;
    o.xilimiter = s->xilimiter; o.divvdt = s->divvdt;
    double* cd[24] = {s->cd_rxx, s->cd_rxy, s->cd_rxz, s->cd_ryy, s->cd_ryz, s->cd_rzz, s->cd_vxx, s->cd_vxy,
                      s->cd_vxz, s->cd_vyx, s->cd_vyy, s->cd_vyz, s->cd_vzx, s->cd_vzy, s->cd_vzz, s->cd_axx,
                      s->cd_axy, s->cd_axz, s->cd_ayx, s->cd_ayy, s->cd_ayz, s->cd_azx, s->cd_azy, s->cd_azz};
    double* dv[9] = {s->dvdx_xx, s->dvdx_xy, s->dvdx_xz, s->dvdx_yx, s->dvdx_yy,
                     s->dvdx_yz, s->dvdx_zx, s->dvdx_zy, s->dvdx_zz};
    for (int k = 0; k < 24; k++) o.cd[k] = cd[k];
    for (int k = 0; k < 9; k++) o.dvdx[k] = dv[k];
  };
  if (c->P.fp32) {
    ForceOut<float> o;
    fill(o);
    force_launch_t<K, DIM, float>(c, o, n, st);
  } else {
    ForceOut<double> o;
    fill(o);
    force_launch_t<K, DIM, double>(c, o, n, st);
  }
}

template <int K>
static void cd_complement_launch(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  k_cd_complement_2d<K><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->lists(), c->d_grids, c->inst, s->x, s->y, s->h,
                                                         s->m, c->au_prev, c->av_prev, c->aw_prev, s->cd_rxx,
                                                         s->cd_rxy, s->cd_ryy, s->cd_axy, s->cd_ayx, s->cd_azx,
                                                         s->cd_azy);
}

void launch_force_pass(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  if (c->timing) launch_pair_stats(c, s, n, st);  // outside the timed scope
  {
    TimedScope ts(c, MHD_TIMING_FORCE, st);
    const int d3 = c->P.dim == 3;
    switch (c->P.kernel) {
      case MHD_KERNEL_CUBIC: d3 ? force_launch<0, 3>(c, s, n, st) : force_launch<0, 2>(c, s, n, st); break;
      case MHD_KERNEL_QUINTIC: d3 ? force_launch<1, 3>(c, s, n, st) : force_launch<1, 2>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C2: d3 ? force_launch<2, 3>(c, s, n, st) : force_launch<2, 2>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C4: d3 ? force_launch<3, 3>(c, s, n, st) : force_launch<3, 2>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C6: d3 ? force_launch<4, 3>(c, s, n, st) : force_launch<4, 2>(c, s, n, st); break;
      case MHD_KERNEL_GAUSSIAN: d3 ? force_launch<5, 3>(c, s, n, st) : force_launch<5, 2>(c, s, n, st); break;
      default: d3 ? force_launch<6, 3>(c, s, n, st) : force_launch<6, 2>(c, s, n, st); break;
    }
    c->launches++;
  }
  if (c->P.dim == 2 && (s->cd_rxx || s->cd_rxy || s->cd_ryy || s->cd_axy || s->cd_ayx || s->cd_azx || s->cd_azy)) {
    switch (c->P.kernel) {
      case MHD_KERNEL_CUBIC: cd_complement_launch<0>(c, s, n, st); break;
      case MHD_KERNEL_QUINTIC: cd_complement_launch<1>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C2: cd_complement_launch<2>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C4: cd_complement_launch<3>(c, s, n, st); break;
      case MHD_KERNEL_WENDLAND_C6: cd_complement_launch<4>(c, s, n, st); break;
      case MHD_KERNEL_GAUSSIAN: cd_complement_launch<5>(c, s, n, st); break;
      default: cd_complement_launch<6>(c, s, n, st); break;
    }
    c->launches++;
  }
}

}  // namespace mhd
