// mhd_force.cu -- the fused force pass of the SPMHD right-hand side, in FP64
// or with FP32 pair arithmetic (sm_100a).
//
// k_force_prologue: DensityFromSmoothingLength, IdealGasEOS and
//   MagneticStateReconstruction (src/equations.py:109-118, 97-106, 474-485),
//   then the per-particle factors the pair loop reuses, packed into
//   4-vectors of the pair precision T (sorted order):
//     r0 = {m, rho, 1/rho, omega}        r1 = {p omega/rho^2, alpha1 v_wave, v_wave, p}
//     r2 = {upred, vpred, wpred, epred}  r3 = {au', av', aw', 1/h}   (a' = previous RHS)
//     r4 = {Bx, By, Bz, psi c_h}         r5 = {Bx/rho, By/rho, Bz/rho, |B/rho|^2/mu0}
//   and an FP64 {x, y, z, h} record.  The FP64 form takes pair geometry
//   from that record and applies the exact FP64 neighbour rule of the
//   oracle (r^2 < (R h_i)^2 or r^2 < (R h_j)^2), so its neighbour sets are
//   bit-identical to the reference's.  The FP32 form takes geometry from the
//   packed cell-relative FP32 positions and tests r^2 < (R max(h_i, h_j))^2
//   in FP32: a pair within ~1e-7 (relative) of the cut-off may be admitted
//   or rejected differently from the exact rule.  Every compact kernel
//   vanishes there, so the sums change by nothing but FP32 rounding; for the
//   Gaussian kernels (truncated at R = 3, W(R) ~ 1e-4 W(0)) such a pair
//   changes a sum by at most one truncated-tail term.
// k_force_pass: CullenDehnenAlphaDiagnostics, MHDAccelerations,
//   MagneticStressAccelerations and MagneticStateRates as one loop over the
//   compacted neighbour list (src/equations.py:318-354, 217-275, 149-195,
//   507-559), then their post_loops, SmoothingLengthRateFromForceDivergence,
//   EnergyLimiter, DivBCorrection and AdaptiveTimestep (src/equations.py:
//   357-429, 278-280, 133-140, 562-567, 588-624, 570-585) per particle in
//   FP64.  Gather formulation: one thread per particle, no atomics on forces.
//   With T = float the momentum, energy, induction and divergence sums are
//   Kahan-compensated; the Cullen-Dehnen moments feed a clipped limiter and
//   use plain FP32 sums.
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

// ------------------------------------------------------------ records
template <class T>
struct ForceRecords {
  const V4<double>* pos;  // {x, y, z, h}
  const V4<T>* r[6];
  const float4* posf;     // packed FP32 positions (geometry of the FP32 form)
  const int* cellc;
  const Grid* grids;  // per-instance geometry
  const int* inst;    // instance of each particle (null: one instance)
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
                                                        const double* __restrict__ awp, V4<double>* __restrict__ pos,
                                                        V4<T>* __restrict__ r0, V4<T>* __restrict__ r1,
                                                        V4<T>* __restrict__ r2, V4<T>* __restrict__ r3,
                                                        V4<T>* __restrict__ r4, V4<T>* __restrict__ r5,
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
  const double vw = sqrt(cs * cs + (bx * bx + by * by + bz * bz) / (P.mu0 * rho));
  const double ir = 1.0 / rho;
  const double om = s.omega[i];
  const double brx = bx * ir, bry = by * ir, brz = bz * ir;
  pos[i] = V4<double>{s.x[i], s.y[i], s.z[i], h};
  r0[i] = V4<T>{(T)s.m[i], (T)rho, (T)ir, (T)om};
  r1[i] = V4<T>{(T)(p * ir * ir * om), (T)(s.alpha1[i] * vw), (T)vw, (T)p};
  r2[i] = V4<T>{(T)s.upred[i], (T)s.vpred[i], (T)s.wpred[i], (T)s.epred[i]};
  r3[i] = V4<T>{(T)aup[i], (T)avp[i], (T)awp[i], (T)(1.0 / h)};
  r4[i] = V4<T>{(T)bx, (T)by, (T)bz, (T)(s.psipred[i] * (P.clean_speed * vw))};
  r5[i] = V4<T>{(T)brx, (T)bry, (T)brz, (T)((brx * brx + bry * bry + brz * brz) * P.inv_mu0)};
}

// Launch shapes (threads per block, minimum resident blocks per SM): the
// second number caps the registers and so sets the occupancy.
constexpr int kForceShapes[][2] = {{128, 2}, {128, 3}, {128, 4}, {256, 2}};
constexpr int kForceShapeCount = 4;

template <int K, int DIM, class T, int SHAPE>
__global__ void __launch_bounds__(kForceShapes[SHAPE][0], kForceShapes[SHAPE][1])
    k_force_pass(int n, DevParams P, NbrList L, ForceRecords<T> R, ForceOut<T> o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& G = grid_of(R.grids, R.inst, i);
  const V4<double> pi = R.pos[i];
  const V4<T> i0 = R.r[0][i], i1 = R.r[1][i], i2 = R.r[2][i], i3 = R.r[3][i], i4 = R.r[4][i], i5 = R.r[5][i];
  const double xi = pi.x, yi = pi.y, zi = DIM == 3 ? pi.z : 0.0, hi = pi.w;
  const double rhi2 = rh2_exact(P.R, hi);
  const T h1i = i3.w;
  const T norm = prm_t<T>(P.normf, P.norm);
  const T faci = norm * (DIM == 2 ? h1i * h1i : h1i * h1i * h1i);
  const T rhoi = i0.y, irhoi = i0.z, omegai = i0.w;
  const T PI = i1.x, AI = i1.y, vwi = i1.z, p_i = i1.w;
  const T ui = i2.x, vi = i2.y, wi = i2.z, epi = i2.w;
  const T aui = i3.x, avi = i3.y, awi = i3.z;
  const T bxi = i4.x, byi = i4.y, bzi = i4.z, psichi = i4.w;
  const T brxi = i5.x, bryi = i5.y, brzi = i5.z, bro2i = i5.w;
  const T rhoi2inv = irhoi * irhoi;
  const T av = prm_t<T>(P.avf, P.av), ac = prm_t<T>(P.acf, P.ac), ar = prm_t<T>(P.arf, P.ar),
          inv_mu0 = prm_t<T>(P.inv_mu0f, P.inv_mu0);
  const T two = (T)2, half = (T)0.5, zero = (T)0;

  // Cullen-Dehnen moments (src/equations.py:329-354)
  T rxx = 0, rxy = 0, rxz = 0, ryy = 0, ryz = 0, rzz = 0;
  T vxx = 0, vxy = 0, vxz = 0, vyx = 0, vyy = 0, vyz = 0, vzx = 0, vzy = 0, vzz = 0;
  T axx = 0, axy = 0, axz = 0, ayx = 0, ayy = 0, ayz = 0, azx = 0, azy = 0, azz = 0;
  Acc<T> fx, fy, fz, fe, fdiv, bxr, byr, bzr, dbs, dbd;
  T dtc = 0;

  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  float4 pif = make_float4(0.f, 0.f, 0.f, 0.f);
  int cif = 0;
  if constexpr (sizeof(T) == 4) {
    pif = R.posf[i];
    cif = R.cellc[i];
  }
  const float Rf = P.Rf;
  // the list entry is fetched one pair ahead, and every record of a pair is
  // requested before its neighbour test, so a pair waits on one memory
  // round trip instead of three (entry, position, records)
  int jn = cnt > 0 ? row[0] : i;
  for (int k = 0; k < cnt; k++) {
    const int j = jn;
    if (k + 1 < cnt) jn = row[(k + 1) * 32];
    if (j == i) {
      // the self pair: every sum term carries a zero kernel gradient or a
      // zero displacement; only the signal speed max(vw_i - 2 dot, 0) = vw_i
      // enters dt_cfl
      dtc = fmax(dtc, vwi);
      continue;
    }
    const V4<T> j0 = ld4(R.r[0] + j), j1 = ld4(R.r[1] + j), j2 = ld4(R.r[2] + j), j3 = ld4(R.r[3] + j);
    const V4<T> j4 = ld4(R.r[4] + j), j5 = ld4(R.r[5] + j);
    T dx, dy, dz, r, inv_r0;
    if constexpr (sizeof(T) == 4) {
      // FP32 geometry from the packed positions; FP32 neighbour test
      const float4 pj = __ldg(R.posf + j);
      rel_dx<DIM>(G, pif, cif, pj, __ldg(R.cellc + j), dx, dy, dz);
      const float r2 = dx * dx + dy * dy + dz * dz;
      const float rh = Rf * fmaxf(pif.w, pj.w);
      if (!(r2 < rh * rh)) continue;
      inv_r0 = r2 > 0.f ? rsqrtf(r2) : 0.f;
      r = r2 * inv_r0;
    } else {
      // FP64 geometry and the exact neighbour test of the oracle
      const V4<double> pj = ld4(R.pos + j);
      const double dxd = min_image(xi - pj.x, G.L[0], G.half[0], G.periodic[0]);
      const double dyd = min_image(yi - pj.y, G.L[1], G.half[1], G.periodic[1]);
      const double dzd = DIM == 3 ? min_image(zi - pj.z, G.L[2], G.half[2], G.periodic[2]) : 0.0;
      const double r2d = r2_exact(dxd, dyd, dzd);
      if (!(r2d < rhi2 || r2d < rh2_exact(P.R, pj.w))) continue;
      dx = dxd;
      dy = dyd;
      dz = dzd;
      r = sqrt(r2d);
      inv_r0 = 0;
    }
    const T mj = j0.x, rhoj = j0.y, irhoj = j0.z, omegaj = j0.w;
    const T h1j = j3.w;
    // DWI = ti * XIJ, DWJ = tj * XIJ (zero at r <= 1e-12)
    T ti = 0, tj = 0, inv_r = 0;
    if (r > (T)kPairDistanceEpsilon) {
      inv_r = sizeof(T) == 4 ? inv_r0 : fast_rcp(r);
      T w, dw;
      w_dw<K>(r * h1i, DIM, w, dw);
      ti = faci * dw * h1i * inv_r;
      w_dw<K>(r * h1j, DIM, w, dw);
      tj = norm * (DIM == 2 ? h1j * h1j : h1j * h1j * h1j) * dw * h1j * inv_r;
    }
    const T dvx = ui - j2.x, dvy = vi - j2.y, dvz = wi - j2.z;
    const T vdotx = dvx * dx + dvy * dy + dvz * dz;

    // ---- CullenDehnenAlphaDiagnostics.loop
    {
      const T c = mj * ti;
      const T cx = c * dx, cy = c * dy, cz = c * dz;
      const T dax = aui - j3.x, day = avi - j3.y, daz = awi - j3.z;
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
    // ---- MHDAccelerations.loop (r-hat is zero below 1e-8 here); its
    // momentum and energy terms join the magnetic ones below in one
    // compensated add per sum
    T mf, fei;
    {
      const bool far = r >= (T)kInteractionDistanceEpsilon;
      const T dot = far ? vdotx * inv_r : zero;
      const T g6 = far ? r : zero;
      const T grad_i = omegai * ti * g6;
      const T grad_j = omegaj * tj * g6;
      fdiv.add(mj * dot * grad_i);
      const T pj = j1.w, vwj = j1.z;
      const T vsig2 = fast_sqrt(fabs(p_i - pj) * fast_rcp(half * (rhoi + rhoj)));
      T c = vwi - two * dot;
      c = fmax(c, vwj - two * dot);
      c = fmax(c, zero);
      dtc = fmax(dtc, c);
      T fcoef = PI * ti + j1.x * tj;
      fei = mj * PI * ti * vdotx;
      if (dot < zero) {
        const T vsigav_i = fmax(AI - two * dot, zero);
        const T vsigav_j = fmax(j1.y - two * dot, zero);
        const T qi = -half * irhoi * vsigav_i * dot * av;
        const T qj = -half * irhoj * vsigav_j * dot * av;
        fcoef += qi * omegai * ti + qj * omegaj * tj;
        fei += mj * qi * dot * grad_i;
      }
      mf = mj * fcoef;
      const T eij = epi - j2.w;
      fei += ac * vsig2 * eij * (half * mj * (irhoi * grad_i + irhoj * grad_j));
    }
    // ---- MagneticStressAccelerations.loop and MagneticStateRates.loop
    {
      const T rux = dx * inv_r, ruy = dy * inv_r, ruz = dz * inv_r;
      const T g8 = r > (T)kPairDistanceEpsilon ? r : zero;
      const T grad_i = omegai * ti * g8;
      const T grad_j = omegaj * tj * g8;
      const T gradp = mj * half * (bro2i * grad_i + j5.w * grad_j);
      const T si = (brxi * rux + bryi * ruy + brzi * ruz) * grad_i;
      const T sj = (j5.x * rux + j5.y * ruy + j5.z * ruz) * grad_j;
      const T ms = mj * inv_mu0;
      const T bxj = j4.x, byj = j4.y, bzj = j4.z;
      const T proj_bi = bxi * rux + byi * ruy + bzi * ruz;
      const T proj_bj = bxj * rux + byj * ruy + bzj * ruz;
      const T dbx = bxi - bxj, dby = byi - byj, dbz = bzi - bzj;
      const T proj_db = dbx * rux + dby * ruy + dbz * ruz;
      const T delta_b2 = dbx * dbx + dby * dby + dbz * dbz;
      const T pmi = mj * rhoi2inv * grad_i;
      const T pmj = mj * irhoj * irhoj * grad_j;
      const T d_brho = -(pmi * proj_bi);
      const T projv = vdotx * inv_r;
      const T tx = dvx - projv * rux, ty = dvy - projv * ruy, tz = dvz - projv * ruz;
      const T vsig_b = fast_sqrt(tx * tx + ty * ty + tz * tz);
      const T diss = half * (pmi + pmj) * vsig_b * ar;
      const T dpsi = pmi * psichi + pmj * j4.w;
      fx.add(-mf * dx + (-rux * gradp + ms * (brxi * si + j5.x * sj)));
      fy.add(-mf * dy + (-ruy * gradp + ms * (bryi * si + j5.y * sj)));
      fz.add(-mf * dz + (-ruz * gradp + ms * (brzi * si + j5.z * sj)));
      bxr.add(d_brho * dvx + diss * dbx - dpsi * rux);
      byr.add(d_brho * dvy + diss * dby - dpsi * ruy);
      bzr.add(d_brho * dvz + diss * dbz - dpsi * ruz);
      fe.add(fei + (-half * delta_b2 * diss * inv_mu0));
      dbs.add(pmi * proj_bi + pmj * proj_bj);
      dbd.add(-mj * proj_db * grad_i);
    }
  }

  // ---- per-particle epilogue in FP64
  const double rhoi_d = o.rho[i], irho_d = 1.0 / rhoi_d, omega_d = o.omega[i];
  // CullenDehnenAlphaDiagnostics.post_loop (src/equations.py:357-429)
  const double termnorm = omega_d * irho_d;
  const double Rxx = rxx, Rxy = rxy, Rxz = rxz, Ryy = ryy, Ryz = ryz, Rzz = rzz;
  const double Vxx = vxx, Vxy = vxy, Vxz = vxz, Vyx = vyx, Vyy = vyy, Vyz = vyz, Vzx = vzx, Vzy = vzy, Vzz = vzz;
  const double Axx = axx, Axy = axy, Axz = axz, Ayx = ayx, Ayy = ayy, Ayz = ayz, Azx = azx, Azy = azy, Azz = azz;
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
  const double hid = hi;
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
  // MHDAccelerations.post_loop, SmoothingLengthRateFromForceDivergence
  const double divi = -fdiv.get() * irho_d;
  // MagneticStateRates.post_loop (src/equations.py:562-567)
  const double vwid = sqrt(csi * csi + ((double)bxi * bxi + (double)byi * byi + (double)bzi * bzi) * P.inv_mu0 * irho_d);
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
  (void)rhoi;
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
static ForceRecords<T> records(Ctx* c) {
  ForceRecords<T> R;
  R.pos = reinterpret_cast<const V4<double>*>(c->rec_pos);
  for (int k = 0; k < 6; k++) R.r[k] = reinterpret_cast<const V4<T>*>(c->rec[k]);
  R.posf = c->posf;
  R.cellc = c->cellc;
  R.grids = c->d_grids;
  R.inst = c->inst;
  return R;
}

template <class T>
static void prologue_launch(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  V4<T>* r[6];
  for (int k = 0; k < 6; k++) r[k] = reinterpret_cast<V4<T>*>(c->rec[k]);
  V4<double>* pos = reinterpret_cast<V4<double>*>(c->rec_pos);
  if (c->P.dim == 3)
    k_force_prologue<3, T><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->au_prev, c->av_prev, c->aw_prev, pos,
                                                            r[0], r[1], r[2], r[3], r[4], r[5], c->posf);
  else
    k_force_prologue<2, T><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, *s, c->au_prev, c->av_prev, c->aw_prev, pos,
                                                            r[0], r[1], r[2], r[3], r[4], r[5], c->posf);
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

template <int K, int DIM, class T>
static void force_launch_t(Ctx* c, const ForceOut<T>& o, int n, cudaStream_t st) {
  // default shapes measured on the 128^3 blast: FP64 uncapped (208-220
  // registers, no spills), FP32 capped at 128 registers (16 warps per SM)
  const int s = c->force_shape >= 0 ? c->force_shape : (sizeof(T) == 4 ? 2 : 0);
  const int bs = kForceShapes[s][0];
  const int grid = (n + bs - 1) / bs;
  switch (s) {
    case 1: k_force_pass<K, DIM, T, 1><<<grid, bs, 0, st>>>(n, c->P, c->lists(), records<T>(c), o); break;
    case 2: k_force_pass<K, DIM, T, 2><<<grid, bs, 0, st>>>(n, c->P, c->lists(), records<T>(c), o); break;
    case 3: k_force_pass<K, DIM, T, 3><<<grid, bs, 0, st>>>(n, c->P, c->lists(), records<T>(c), o); break;
    default: k_force_pass<K, DIM, T, 0><<<grid, bs, 0, st>>>(n, c->P, c->lists(), records<T>(c), o);
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
