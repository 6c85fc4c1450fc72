/*
 * mhd_oracle.c -- FP64 CPU restatement of the reference SPMHD right-hand side
 * and predictor-evaluate-corrector step.
 *
 * TEST INFRASTRUCTURE AND CPU BASELINE ONLY.  Nothing in the product links or
 * calls this file; the tests, the smoke check and the benchmark's CPU leg use
 * it as the checker.  The CUDA path never falls back to it.
 *
 * Restates, literally and in the same group order (src/scheme.py:66-81):
 *   G1  DensityIteration                      src/equations.py:14-94
 *   G2  SmoothingLengthRateFromDensityRelation src/equations.py:121-130
 *       DensityFromSmoothingLength            src/equations.py:109-118
 *   G3  IdealGasEOS                           src/equations.py:97-106
 *   G4  CullenDehnenAlphaDiagnostics          src/equations.py:283-429
 *   G5  StrainDiagnostics                     src/equations.py:432-471
 *       MagneticStateReconstruction           src/equations.py:474-485
 *   G6  MHDAccelerations                      src/equations.py:198-280
 *   G7  SmoothingLengthRateFromForceDivergence src/equations.py:133-140
 *   G8  MagneticStressAccelerations           src/equations.py:143-195
 *   G9  MagneticStateRates                    src/equations.py:488-567
 *   G10 EnergyLimiter, DivBCorrection, AdaptiveTimestep
 *                                             src/equations.py:588-624, 570-585
 *   MHDStep.initialize / stage1 / stage2      src/integrator.py:12-82
 * Every arithmetic expression keeps the reference's evaluation order, and the
 * file is compiled with -ffp-contract=off, so that with neighbours summed in
 * ascending index order ("exact_order") the results equal, bit for bit, the
 * golden fixtures produced by executing the reference's own Python code.
 *
 * PySPH semantics restated here (PySPH is not available; unpinned):
 * kernel forms and normalisations; the neighbour rule
 * r2 < (R h_i)^2 || r2 < (R h_j)^2 on the minimum-image x_i - x_j, self
 * included; neighbours recomputed from the current h before every density
 * pass; iterated-group stopping rule; PEC stage order; periodic wrap.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- property table (names are the reference's, src/particles.py) ---- */
#define PROPS(X)                                                                                       \
  X(x) X(y) X(z) X(u) X(v) X(w) X(rho) X(rho_sum) X(h) X(m) X(cs) X(p) X(e) X(au) X(av) X(aw)          \
  X(arho) X(ae) X(ah) X(x0) X(y0) X(z0) X(u0) X(v0) X(w0) X(upred) X(vpred) X(wpred) X(epred) X(e0)  \
  X(h0) X(div) X(dt_cfl) X(dt_adapt) X(grhox) X(grhoy) X(grhoz) X(dwdh) X(omega) X(converged)         \
  X(alpha1) X(alpha10) X(Bx) X(By) X(Bz) X(Bevolx) X(Bevoly) X(Bevolz) X(psi) X(Bevolxpred)          \
  X(Bevolypred) X(Bevolzpred) X(psipred) X(Bxpred) X(Bypred) X(Bzpred) X(aBevolx) X(aBevoly)         \
  X(aBevolz) X(apsi) X(Bevolx0) X(Bevoly0) X(Bevolz0) X(psi0) X(divBsymm) X(divBdiff) X(div_for_psi) \
  X(alphaloc) X(xilimiter) X(divvdt) X(cd_rxx) X(cd_rxy) X(cd_rxz) X(cd_ryy) X(cd_ryz) X(cd_rzz)      \
  X(cd_vxx) X(cd_vxy) X(cd_vxz) X(cd_vyx) X(cd_vyy) X(cd_vyz) X(cd_vzx) X(cd_vzy) X(cd_vzz)           \
  X(cd_axx) X(cd_axy) X(cd_axz) X(cd_ayx) X(cd_ayy) X(cd_ayz) X(cd_azx) X(cd_azy) X(cd_azz)           \
  X(dvdx_xx) X(dvdx_xy) X(dvdx_xz) X(dvdx_yx) X(dvdx_yy) X(dvdx_yz) X(dvdx_zx) X(dvdx_zy) X(dvdx_zz)

enum {
#define X(n) P_##n,
  PROPS(X)
#undef X
      P_COUNT
};

static const char* PROP_NAMES[] = {
#define X(n) #n,
    PROPS(X)
#undef X
};

int oracle_nprops(void) { return P_COUNT; }
const char* oracle_prop_name(int i) { return (i >= 0 && i < P_COUNT) ? PROP_NAMES[i] : 0; }

/* Must match oracle/__init__.py (ctypes). */
typedef struct OracleParams {
  int dim;
  int kernel; /* 0 cubic, 1 quintic, 2 wendland_c2, 3 wendland_c4, 4 wendland_c6, 5 gaussian, 6 super_gaussian */
  int iterate;
  int min_iter;
  int max_iter;
  int exact_order;
  int nthreads;
  int periodic[3];
  double hfact, gamma, mu0, av, ac, ar, clean_speed, clean_damp, timestep_factor, alpha_min, alpha_max;
  double lo[3], hi[3];
} OracleParams;

#define DENSITY_TOLERANCE 1.0e-4
#define COURANT_FACTOR 0.3
#define FORCE_FACTOR 0.25
#define PAIR_DISTANCE_EPSILON 1.0e-12
#define INTERACTION_DISTANCE_EPSILON 1.0e-8
#define FLOAT_TINY 2.2250738585072014e-308

#define A(name) (P[P_##name])

static inline double pymax(double a, double b) { return (b > a) ? b : a; }
static inline double pymin(double a, double b) { return (b < a) ? b : a; }

/* ---------------------------------------------------------------- kernels */
static double radius_scale(int kernel) { return (kernel == 1 || kernel == 5 || kernel == 6) ? 3.0 : 2.0; }

static double kernel_norm(int kernel, int dim) {
  switch (kernel) {
    case 0: return dim == 1 ? 2.0 / 3.0 : dim == 2 ? 10.0 / (7.0 * M_PI) : 1.0 / M_PI;
    case 1: return dim == 1 ? 1.0 / 120.0 : dim == 2 ? 7.0 / (478.0 * M_PI) : 1.0 / (120.0 * M_PI);
    case 2: return dim == 1 ? 3.0 / 4.0 : dim == 2 ? 7.0 / (4.0 * M_PI) : 21.0 / (16.0 * M_PI);
    case 3: return dim == 1 ? 5.0 / 8.0 : dim == 2 ? 9.0 / (4.0 * M_PI) : 495.0 / (256.0 * M_PI);
    case 4: return dim == 1 ? 55.0 / 64.0 : dim == 2 ? 78.0 / (28.0 * M_PI) : 1365.0 / (512.0 * M_PI);
    default: return dim == 1 ? 1.0 / sqrt(M_PI) : dim == 2 ? 1.0 / M_PI : 1.0 / (M_PI * sqrt(M_PI));
  }
}

/* w(q) and dw/dq, unnormalised. */
static inline void w_dw(int kernel, int dim, double q, double* w, double* dw) {
  switch (kernel) {
    case 0:
      if (q > 2.0) { *w = 0.0; *dw = 0.0; }
      else if (q > 1.0) { double t = 2.0 - q; *w = 0.25 * t * t * t; *dw = -0.75 * t * t; }
      else { *w = 1.0 - 1.5 * q * q * (1.0 - 0.5 * q); *dw = -3.0 * q * (1.0 - 0.75 * q); }
      return;
    case 1: {
      if (q > 3.0) { *w = 0.0; *dw = 0.0; return; }
      double t3 = 3.0 - q, t2 = 2.0 - q, t1 = 1.0 - q;
      double ww = t3 * t3 * t3 * t3 * t3;
      double dd = -5.0 * t3 * t3 * t3 * t3;
      if (!(q > 2.0)) {
        ww -= 6.0 * t2 * t2 * t2 * t2 * t2;
        dd += 30.0 * t2 * t2 * t2 * t2;
        if (!(q > 1.0)) {
          ww += 15.0 * t1 * t1 * t1 * t1 * t1;
          dd -= 75.0 * t1 * t1 * t1 * t1;
        }
      }
      *w = ww; *dw = dd;
      return;
    }
    case 2: {
      if (q >= 2.0) { *w = 0.0; *dw = 0.0; return; }
      double s = 1.0 - 0.5 * q, s3 = s * s * s;
      *w = s3 * s * (2.0 * q + 1.0); *dw = -5.0 * q * s3;
      return;
    }
    case 3: {
      if (q >= 2.0) { *w = 0.0; *dw = 0.0; return; }
      double s = 1.0 - 0.5 * q, s5 = s * s * s * s * s;
      *w = s5 * s * (35.0 / 12.0 * q * q + 3.0 * q + 1.0);
      *dw = -14.0 / 3.0 * q * (1.0 + 2.5 * q) * s5;
      return;
    }
    case 4: {
      if (q >= 2.0) { *w = 0.0; *dw = 0.0; return; }
      double s = 1.0 - 0.5 * q, s7 = s * s * s * s * s * s * s;
      *w = s7 * s * (4.0 * q * q * q + 6.25 * q * q + 4.0 * q + 1.0);
      *dw = -5.5 * q * (1.0 + 3.5 * q + 4.0 * q * q) * s7;
      return;
    }
    case 5: {
      if (q >= 3.0) { *w = 0.0; *dw = 0.0; return; }
      double e = exp(-q * q);
      *w = e; *dw = -2.0 * q * e;
      return;
    }
    default: {
      if (q >= 3.0) { *w = 0.0; *dw = 0.0; return; }
      double e = exp(-q * q), d2 = 0.5 * dim;
      *w = e * (d2 + 1.0 - q * q); *dw = -2.0 * q * e * (d2 + 2.0 - q * q);
      return;
    }
  }
}

typedef struct {
  int kernel, dim;
  double norm, R;
} Kern;

static inline double hfac(const Kern* k, double h1) {
  if (k->dim == 1) return k->norm * h1;
  if (k->dim == 2) return k->norm * h1 * h1;
  return k->norm * h1 * h1 * h1;
}
static inline double kern_w(const Kern* k, double rij, double h) {
  double h1 = 1.0 / h, q = rij * h1, w, dw;
  w_dw(k->kernel, k->dim, q, &w, &dw);
  return w * hfac(k, h1);
}
static inline void kern_grad(const Kern* k, const double* xij, double rij, double h, double* g) {
  double h1 = 1.0 / h, tmp;
  if (rij > 1.0e-12) {
    double q = rij * h1, w, dw;
    w_dw(k->kernel, k->dim, q, &w, &dw);
    tmp = hfac(k, h1) * dw * h1 / rij;
  } else {
    tmp = 0.0;
  }
  g[0] = tmp * xij[0];
  g[1] = tmp * xij[1];
  g[2] = tmp * xij[2];
}
static inline double kern_gradh(const Kern* k, double rij, double h) {
  double h1 = 1.0 / h, q = rij * h1, w, dw;
  w_dw(k->kernel, k->dim, q, &w, &dw);
  return -hfac(k, h1) * h1 * (dw * q + w * (double)k->dim);
}

/* --------------------------------------------------------- neighbour grid */
typedef struct {
  int nc[3];
  double lo[3], cs[3];
  int64_t ncells;
  int64_t* start; /* ncells + 1 */
  int64_t* idx;   /* particles grouped by cell, ascending index inside a cell */
  int64_t* cell_of;
} Grid;

static inline double min_image(const OracleParams* pr, int a, double d) {
  if (!pr->periodic[a]) return d;
  double L = pr->hi[a] - pr->lo[a], half = 0.5 * L;
  if (d > half) d = d - L;
  if (d < -half) d = d + L;
  return d;
}

static void grid_build(Grid* g, const OracleParams* pr, int64_t n, double* const* P, double cutoff) {
  const double* pos[3] = {A(x), A(y), A(z)};
  for (int a = 0; a < 3; a++) {
    double lo, hi;
    if (a >= pr->dim) { g->nc[a] = 1; g->lo[a] = 0.0; g->cs[a] = 1.0; continue; }
    if (pr->periodic[a]) {
      lo = pr->lo[a];
      hi = pr->hi[a];
    } else {
      lo = INFINITY; hi = -INFINITY;
      for (int64_t i = 0; i < n; i++) { lo = fmin(lo, pos[a][i]); hi = fmax(hi, pos[a][i]); }
      hi += 1e-12 * (fabs(hi) + 1.0);
    }
    int c = (int)floor((hi - lo) / cutoff);
    if (c < 1) c = 1;
    if (c > 4096) c = 4096;
    if (pr->periodic[a] && c < 3) c = 1;
    g->nc[a] = c;
    g->lo[a] = lo;
    g->cs[a] = (hi - lo) / c;
  }
  g->ncells = (int64_t)g->nc[0] * g->nc[1] * g->nc[2];
  g->start = (int64_t*)calloc(g->ncells + 1, sizeof(int64_t));
  g->idx = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  g->cell_of = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) {
    int64_t cc[3];
    for (int a = 0; a < 3; a++) {
      int64_t c = 0;
      if (a < pr->dim) {
        c = (int64_t)floor((pos[a][i] - g->lo[a]) / g->cs[a]);
        if (c < 0) c = 0;
        if (c >= g->nc[a]) c = g->nc[a] - 1;
      }
      cc[a] = c;
    }
    int64_t cid = (cc[2] * g->nc[1] + cc[1]) * g->nc[0] + cc[0];
    g->cell_of[i] = cid;
    g->start[cid + 1]++;
  }
  for (int64_t c = 0; c < g->ncells; c++) g->start[c + 1] += g->start[c];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (g->ncells + 1));
  memcpy(fill, g->start, sizeof(int64_t) * (g->ncells + 1));
  for (int64_t i = 0; i < n; i++) g->idx[fill[g->cell_of[i]]++] = i;
  free(fill);
}

static void grid_free(Grid* g) {
  free(g->start);
  free(g->idx);
  free(g->cell_of);
}

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

/* Neighbours of i under the symmetric rule; ascending when exact_order. */
static int64_t neighbours(const Grid* g, const OracleParams* pr, double* const* P, double R, int64_t i,
                          int64_t* out) {
  const double* X = A(x);
  const double* Y = A(y);
  const double* Z = A(z);
  const double* H = A(h);
  int64_t cid = g->cell_of[i];
  int c0 = (int)(cid % g->nc[0]);
  int c1 = (int)((cid / g->nc[0]) % g->nc[1]);
  int c2 = (int)(cid / ((int64_t)g->nc[0] * g->nc[1]));
  double rhi = R * H[i], rhi2 = rhi * rhi;
  int64_t cnt = 0;
  int lo[3], hi[3];
  int cc[3] = {c0, c1, c2};
  for (int a = 0; a < 3; a++) {
    if (g->nc[a] == 1) { lo[a] = 0; hi[a] = 0; }
    else { lo[a] = -1; hi[a] = 1; }
  }
  for (int oz = lo[2]; oz <= hi[2]; oz++) {
    int z = cc[2] + oz;
    if (z < 0 || z >= g->nc[2]) {
      if (!pr->periodic[2]) continue;
      z = (z + g->nc[2]) % g->nc[2];
    }
    for (int oy = lo[1]; oy <= hi[1]; oy++) {
      int y = cc[1] + oy;
      if (y < 0 || y >= g->nc[1]) {
        if (!pr->periodic[1]) continue;
        y = (y + g->nc[1]) % g->nc[1];
      }
      for (int ox = lo[0]; ox <= hi[0]; ox++) {
        int x = cc[0] + ox;
        if (x < 0 || x >= g->nc[0]) {
          if (!pr->periodic[0]) continue;
          x = (x + g->nc[0]) % g->nc[0];
        }
        int64_t c = ((int64_t)z * g->nc[1] + y) * g->nc[0] + x;
        for (int64_t k = g->start[c]; k < g->start[c + 1]; k++) {
          int64_t j = g->idx[k];
          double dx = min_image(pr, 0, X[i] - X[j]);
          double dy = min_image(pr, 1, Y[i] - Y[j]);
          double dz = pr->dim == 3 ? min_image(pr, 2, Z[i] - Z[j]) : 0.0;
          double r2 = dx * dx + dy * dy + dz * dz;
          double rhj = R * H[j];
          if (r2 < rhi2 || r2 < rhj * rhj) out[cnt++] = j;
        }
      }
    }
  }
  if (pr->exact_order) qsort(out, (size_t)cnt, sizeof(int64_t), cmp_i64);
  return cnt;
}

static double max_h(int64_t n, const double* h) {
  double m = 0.0;
  for (int64_t i = 0; i < n; i++) m = h[i] > m ? h[i] : m;
  return m;
}

typedef struct {
  double xij[3], rij;
} Pair;

static inline Pair make_pair(const OracleParams* pr, double* const* P, int64_t i, int64_t j) {
  Pair q;
  q.xij[0] = min_image(pr, 0, A(x)[i] - A(x)[j]);
  q.xij[1] = min_image(pr, 1, A(y)[i] - A(y)[j]);
  q.xij[2] = pr->dim == 3 ? min_image(pr, 2, A(z)[i] - A(z)[j]) : 0.0;
  q.rij = sqrt(q.xij[0] * q.xij[0] + q.xij[1] * q.xij[1] + q.xij[2] * q.xij[2]);
  return q;
}

#define NBR_MAX 4096

/* ----------------------------------------------------- G1 density pass */
/* One pass of DensityIteration (src/equations.py:24-88). Returns the
   equation_has_converged value (1 or -1). */
static int density_pass(const OracleParams* pr, const Kern* K, int64_t n, double** P) {
  const double k = pr->hfact;
  const double dim = (double)pr->dim;
  const int once = !pr->iterate;
  Grid g;
  grid_build(&g, pr, n, P, K->R * max_h(n, A(h)));
  int conv = 1;
#pragma omp parallel reduction(min : conv)
  {
    int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * NBR_MAX * 8);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
      /* initialize (:25-35) */
      A(rho)[i] = 0.0;
      A(div)[i] = 0.0;
      A(grhox)[i] = 0.0;
      A(grhoy)[i] = 0.0;
      A(grhoz)[i] = 0.0;
      A(arho)[i] = 0.0;
      A(dwdh)[i] = 0.0;
      /* loop (:38-50) */
      int64_t cnt = neighbours(&g, pr, P, K->R, i, nb);
      double hi = A(h)[i];
      for (int64_t t = 0; t < cnt; t++) {
        int64_t j = nb[t];
        Pair q = make_pair(pr, P, i, j);
        double WI = kern_w(K, q.rij, hi), DWI[3], GHI = kern_gradh(K, q.rij, hi);
        kern_grad(K, q.xij, q.rij, hi, DWI);
        double mj = A(m)[j];
        double dvx = A(upred)[i] - A(upred)[j];
        double dvy = A(vpred)[i] - A(vpred)[j];
        double dvz = A(wpred)[i] - A(wpred)[j];
        double vijdotdwij = dvx * DWI[0] + dvy * DWI[1] + dvz * DWI[2];
        A(rho)[i] += mj * WI;
        A(arho)[i] += mj * vijdotdwij;
        A(grhox)[i] += mj * DWI[0];
        A(grhoy)[i] += mj * DWI[1];
        A(grhoz)[i] += mj * DWI[2];
        A(dwdh)[i] += mj * GHI;
      }
    }
    free(nb);
  }
  /* post_loop (:53-88) */
#pragma omp parallel for reduction(min : conv) schedule(static)
  for (int64_t i = 0; i < n; i++) {
    if (A(converged)[i] != 1) {
      double mi = A(m)[i], hi = A(h)[i], hi0 = A(h0)[i];
      double rhoi = mi / pow(hi / k, dim);
      double dhdrhoi = -hi / (dim * rhoi);
      double dwdhi = A(dwdh)[i];
      double omegai = 1.0 - dhdrhoi * dwdhi;
      double gradhi = 1.0 / omegai;
      A(omega)[i] = gradhi;
      double func = rhoi - A(rho)[i];
      double dfdh1 = omegai > 0.0 ? dhdrhoi / omegai : dhdrhoi / fabs(omegai + 2.220446049250313e-16);
      double hnew = hi - func * dfdh1;
      if (hnew > 1.2 * hi) hnew = 1.2 * hi;
      else if (hnew < 0.8 * hi) hnew = 0.8 * hi;
      double diff = fabs(hnew - hi) / hi0;
      int finalize = ((diff < DENSITY_TOLERANCE) && (omegai > 0.0) && (hi > 0.0)) || once;
      if (!finalize) {
        conv = -1;
        A(h)[i] = hnew;
        A(converged)[i] = 0;
      } else {
        A(arho)[i] *= A(omega)[i];
        A(ah)[i] = A(arho)[i] * dhdrhoi;
        A(h)[i] = k * pow(mi / A(rho)[i], 1.0 / dim);
        A(converged)[i] = 1;
      }
    }
    A(div)[i] = -A(arho)[i] / A(rho)[i];
  }
  grid_free(&g);
  return conv;
}

/* ------------------------------------------------- G4-G9 pair loops */
static void cd_loop(const OracleParams* pr, const Kern* K, double** P, int64_t i, const int64_t* nb, int64_t cnt) {
  /* CullenDehnenAlphaDiagnostics.initialize (:288-315) */
  A(alphaloc)[i] = 0.0;
  A(xilimiter)[i] = 1.0;
  A(divvdt)[i] = 0.0;
  for (int c = P_cd_rxx; c <= P_cd_azz; c++) P[c][i] = 0.0;
  double hi = A(h)[i];
  for (int64_t t = 0; t < cnt; t++) {
    int64_t j = nb[t];
    Pair q = make_pair(pr, P, i, j);
    double DWI[3];
    kern_grad(K, q.xij, q.rij, hi, DWI);
    const double* XIJ = q.xij;
    /* loop (:318-354) */
    double runx = A(m)[j] * DWI[0];
    double runy = A(m)[j] * DWI[1];
    double runz = A(m)[j] * DWI[2];
    double dvx = A(upred)[i] - A(upred)[j];
    double dvy = A(vpred)[i] - A(vpred)[j];
    double dvz = A(wpred)[i] - A(wpred)[j];
    double dax = A(au)[i] - A(au)[j];
    double day = A(av)[i] - A(av)[j];
    double daz = A(aw)[i] - A(aw)[j];
    A(cd_rxx)[i] += -XIJ[0] * runx;
    A(cd_rxy)[i] += -XIJ[0] * runy;
    A(cd_rxz)[i] += -XIJ[0] * runz;
    A(cd_ryy)[i] += -XIJ[1] * runy;
    A(cd_ryz)[i] += -XIJ[1] * runz;
    A(cd_rzz)[i] += -XIJ[2] * runz;
    A(cd_vxx)[i] += dvx * runx;
    A(cd_vxy)[i] += dvx * runy;
    A(cd_vxz)[i] += dvx * runz;
    A(cd_vyx)[i] += dvy * runx;
    A(cd_vyy)[i] += dvy * runy;
    A(cd_vyz)[i] += dvy * runz;
    A(cd_vzx)[i] += dvz * runx;
    A(cd_vzy)[i] += dvz * runy;
    A(cd_vzz)[i] += dvz * runz;
    A(cd_axx)[i] += dax * runx;
    A(cd_axy)[i] += dax * runy;
    A(cd_axz)[i] += dax * runz;
    A(cd_ayx)[i] += day * runx;
    A(cd_ayy)[i] += day * runy;
    A(cd_ayz)[i] += day * runz;
    A(cd_azx)[i] += daz * runx;
    A(cd_azy)[i] += daz * runy;
    A(cd_azz)[i] += daz * runz;
  }
}

static void cd_post(const OracleParams* pr, double** P, int64_t i) {
  /* post_loop (:357-429) */
  double rxx = A(cd_rxx)[i], rxy = A(cd_rxy)[i], rxz = A(cd_rxz)[i];
  double ryy = A(cd_ryy)[i], ryz = A(cd_ryz)[i], rzz = A(cd_rzz)[i];
  double denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy;
  double termnorm = A(omega)[i] / A(rho)[i];
  double div_a, dvxdx, dvxdy, dvxdz, dvydx, dvydy, dvydz, dvzdx, dvzdy, dvzdz;
  if (fabs(denom) > FLOAT_TINY) {
    double ddenom = 1.0 / denom;
    double term_xx = ryy * rzz - ryz * ryz;
    double term_xy = rxz * ryz - rzz * rxy;
    double term_xz = rxy * ryz - rxz * ryy;
    double term_yy = rzz * rxx - rxz * rxz;
    double term_yz = rxy * rxz - rxx * ryz;
    double term_zz = rxx * ryy - rxy * rxy;
    double gradaxdx = (A(cd_axx)[i] * term_xx + A(cd_axy)[i] * term_xy + A(cd_axz)[i] * term_xz) * ddenom;
    double gradaydy = (A(cd_ayx)[i] * term_xy + A(cd_ayy)[i] * term_yy + A(cd_ayz)[i] * term_yz) * ddenom;
    double gradazdz = (A(cd_azx)[i] * term_xz + A(cd_azy)[i] * term_yz + A(cd_azz)[i] * term_zz) * ddenom;
    div_a = -(gradaxdx + gradaydy + gradazdz);
    double gradvxdx = (A(cd_vxx)[i] * term_xx + A(cd_vxy)[i] * term_xy + A(cd_vxz)[i] * term_xz) * ddenom;
    double gradvxdy = (A(cd_vxx)[i] * term_xy + A(cd_vxy)[i] * term_yy + A(cd_vxz)[i] * term_yz) * ddenom;
    double gradvxdz = (A(cd_vxx)[i] * term_xz + A(cd_vxy)[i] * term_yz + A(cd_vxz)[i] * term_zz) * ddenom;
    double gradvydx = (A(cd_vyx)[i] * term_xx + A(cd_vyy)[i] * term_xy + A(cd_vyz)[i] * term_xz) * ddenom;
    double gradvydy = (A(cd_vyx)[i] * term_xy + A(cd_vyy)[i] * term_yy + A(cd_vyz)[i] * term_yz) * ddenom;
    double gradvydz = (A(cd_vyx)[i] * term_xz + A(cd_vyy)[i] * term_yz + A(cd_vyz)[i] * term_zz) * ddenom;
    double gradvzdx = (A(cd_vzx)[i] * term_xx + A(cd_vzy)[i] * term_xy + A(cd_vzz)[i] * term_xz) * ddenom;
    double gradvzdy = (A(cd_vzx)[i] * term_xy + A(cd_vzy)[i] * term_yy + A(cd_vzz)[i] * term_yz) * ddenom;
    double gradvzdz = (A(cd_vzx)[i] * term_xz + A(cd_vzy)[i] * term_yz + A(cd_vzz)[i] * term_zz) * ddenom;
    dvxdx = -gradvxdx; dvxdy = -gradvxdy; dvxdz = -gradvxdz;
    dvydx = -gradvydx; dvydy = -gradvydy; dvydz = -gradvydz;
    dvzdx = -gradvzdx; dvzdy = -gradvzdy; dvzdz = -gradvzdz;
  } else {
    div_a = -termnorm * (A(cd_axx)[i] + A(cd_ayy)[i] + A(cd_azz)[i]);
    dvxdx = -termnorm * A(cd_vxx)[i]; dvxdy = -termnorm * A(cd_vxy)[i]; dvxdz = -termnorm * A(cd_vxz)[i];
    dvydx = -termnorm * A(cd_vyx)[i]; dvydy = -termnorm * A(cd_vyy)[i]; dvydz = -termnorm * A(cd_vyz)[i];
    dvzdx = -termnorm * A(cd_vzx)[i]; dvzdy = -termnorm * A(cd_vzy)[i]; dvzdz = -termnorm * A(cd_vzz)[i];
  }
  double divvdt = div_a - (dvxdx * dvxdx + dvydy * dvydy + dvzdz * dvzdz + 2.0 * (dvxdy * dvydx + dvxdz * dvzdx + dvydz * dvzdy));
  double divv = dvxdx + dvydy + dvzdz;
  double curlvx = dvzdy - dvydz;
  double curlvy = dvxdz - dvzdx;
  double curlvz = dvydx - dvxdy;
  double compression = pymax(-divv, 0.0);
  double fac = compression * compression;
  double trace_s = curlvx * curlvx + curlvy * curlvy + curlvz * curlvz;
  double denominator = fac + trace_s;
  double xilimiter = denominator > 0.0 ? fac / denominator : 1.0;
  A(divvdt)[i] = divvdt;
  A(xilimiter)[i] = xilimiter;
  double source = 10.0 * A(h)[i] * A(h)[i] * A(xilimiter)[i] * pymax(-A(divvdt)[i], 0.0);
  double temp = A(cs)[i] * A(cs)[i];
  /* alpha clip: reference literal is [0, 1] (:428); alpha_min/alpha_max extend it */
  A(alphaloc)[i] = pymax(pymin(source / temp, pr->alpha_max), pr->alpha_min);
}

static void strain_and_bfield(double** P, int64_t i) {
  /* StrainDiagnostics.initialize (:434-471) */
  double rxx = A(cd_rxx)[i], rxy = A(cd_rxy)[i], rxz = A(cd_rxz)[i];
  double ryy = A(cd_ryy)[i], ryz = A(cd_ryz)[i], rzz = A(cd_rzz)[i];
  double denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy;
  if (fabs(denom) > FLOAT_TINY) {
    double ddenom = 1.0 / denom;
    double term_xx = ryy * rzz - ryz * ryz;
    double term_xy = rxz * ryz - rzz * rxy;
    double term_xz = rxy * ryz - rxz * ryy;
    double term_yy = rzz * rxx - rxz * rxz;
    double term_yz = rxy * rxz - rxx * ryz;
    double term_zz = rxx * ryy - rxy * rxy;
    A(dvdx_xx)[i] = -(A(cd_vxx)[i] * term_xx + A(cd_vxy)[i] * term_xy + A(cd_vxz)[i] * term_xz) * ddenom;
    A(dvdx_xy)[i] = -(A(cd_vxx)[i] * term_xy + A(cd_vxy)[i] * term_yy + A(cd_vxz)[i] * term_yz) * ddenom;
    A(dvdx_xz)[i] = -(A(cd_vxx)[i] * term_xz + A(cd_vxy)[i] * term_yz + A(cd_vxz)[i] * term_zz) * ddenom;
    A(dvdx_yx)[i] = -(A(cd_vyx)[i] * term_xx + A(cd_vyy)[i] * term_xy + A(cd_vyz)[i] * term_xz) * ddenom;
    A(dvdx_yy)[i] = -(A(cd_vyx)[i] * term_xy + A(cd_vyy)[i] * term_yy + A(cd_vyz)[i] * term_yz) * ddenom;
    A(dvdx_yz)[i] = -(A(cd_vyx)[i] * term_xz + A(cd_vyy)[i] * term_yz + A(cd_vyz)[i] * term_zz) * ddenom;
    A(dvdx_zx)[i] = -(A(cd_vzx)[i] * term_xx + A(cd_vzy)[i] * term_xy + A(cd_vzz)[i] * term_xz) * ddenom;
    A(dvdx_zy)[i] = -(A(cd_vzx)[i] * term_xy + A(cd_vzy)[i] * term_yy + A(cd_vzz)[i] * term_yz) * ddenom;
    A(dvdx_zz)[i] = -(A(cd_vzx)[i] * term_xz + A(cd_vzy)[i] * term_yz + A(cd_vzz)[i] * term_zz) * ddenom;
  } else {
    double termnorm = A(omega)[i] / A(rho)[i];
    A(dvdx_xx)[i] = -termnorm * A(cd_vxx)[i];
    A(dvdx_xy)[i] = -termnorm * A(cd_vxy)[i];
    A(dvdx_xz)[i] = -termnorm * A(cd_vxz)[i];
    A(dvdx_yx)[i] = -termnorm * A(cd_vyx)[i];
    A(dvdx_yy)[i] = -termnorm * A(cd_vyy)[i];
    A(dvdx_yz)[i] = -termnorm * A(cd_vyz)[i];
    A(dvdx_zx)[i] = -termnorm * A(cd_vzx)[i];
    A(dvdx_zy)[i] = -termnorm * A(cd_vzy)[i];
    A(dvdx_zz)[i] = -termnorm * A(cd_vzz)[i];
  }
  /* MagneticStateReconstruction.initialize (:476-485) */
  double bxpred = A(Bevolxpred)[i] * A(rho)[i];
  double bypred = A(Bevolypred)[i] * A(rho)[i];
  double bzpred = A(Bevolzpred)[i] * A(rho)[i];
  A(Bx)[i] = bxpred;
  A(By)[i] = bypred;
  A(Bz)[i] = bzpred;
  A(Bxpred)[i] = bxpred;
  A(Bypred)[i] = bypred;
  A(Bzpred)[i] = bzpred;
}

static void mhd_acc_loop(const OracleParams* pr, const Kern* K, double** P, int64_t i, const int64_t* nb, int64_t cnt) {
  const double beta = 2.0, mu0 = pr->mu0;
  /* initialize (:207-214) */
  A(au)[i] = 0.0; A(av)[i] = 0.0; A(aw)[i] = 0.0; A(ae)[i] = 0.0;
  A(dt_cfl)[i] = 0.0; A(div)[i] = 0.0; A(div_for_psi)[i] = 0.0;
  double hi = A(h)[i];
  for (int64_t t = 0; t < cnt; t++) {
    int64_t j = nb[t];
    Pair q = make_pair(pr, P, i, j);
    double DWI[3], DWJ[3];
    kern_grad(K, q.xij, q.rij, hi, DWI);
    kern_grad(K, q.xij, q.rij, A(h)[j], DWJ);
    const double* XIJ = q.xij;
    double RIJ = q.rij;
    double RHOIJ = 0.5 * (A(rho)[i] + A(rho)[j]);
    /* loop (:217-275) */
    double p_i = A(p)[i], pj = A(p)[j];
    double rhoi = A(rho)[i], rhoj = A(rho)[j];
    double rhoi2 = rhoi * rhoi, rhoj2 = rhoj * rhoj;
    double pibrhoi2 = p_i / rhoi2, pjbrhoj2 = pj / rhoj2;
    double mj = A(m)[j];
    double bi2 = A(Bxpred)[i] * A(Bxpred)[i] + A(Bypred)[i] * A(Bypred)[i] + A(Bzpred)[i] * A(Bzpred)[i];
    double bj2 = A(Bxpred)[j] * A(Bxpred)[j] + A(Bypred)[j] * A(Bypred)[j] + A(Bzpred)[j] * A(Bzpred)[j];
    double vwave_i = sqrt(A(cs)[i] * A(cs)[i] + bi2 / (mu0 * rhoi));
    double vwave_j = sqrt(A(cs)[j] * A(cs)[j] + bj2 / (mu0 * rhoj));
    double runix, runiy, runiz;
    if (RIJ < INTERACTION_DISTANCE_EPSILON) { runix = 0.0; runiy = 0.0; runiz = 0.0; }
    else { runix = XIJ[0] / RIJ; runiy = XIJ[1] / RIJ; runiz = XIJ[2] / RIJ; }
    double dvx = A(upred)[i] - A(upred)[j];
    double dvy = A(vpred)[i] - A(vpred)[j];
    double dvz = A(wpred)[i] - A(wpred)[j];
    double dot = dvx * runix + dvy * runiy + dvz * runiz;
    double omegai = A(omega)[i], omegaj = A(omega)[j];
    double grad_i = omegai * (runix * DWI[0] + runiy * DWI[1] + runiz * DWI[2]);
    double grad_j = omegaj * (runix * DWJ[0] + runiy * DWJ[1] + runiz * DWJ[2]);
    A(div)[i] += A(m)[j] * dot * grad_i;
    double pdiff = fabs(p_i - pj);
    double vsig2 = sqrt(pdiff / RHOIJ);
    double dt_cfl = vwave_i - beta * dot;
    dt_cfl = pymax(dt_cfl, vwave_j - beta * dot);
    dt_cfl = pymax(dt_cfl, 0.0);
    A(dt_cfl)[i] = pymax(A(dt_cfl)[i], dt_cfl);
    if (dot < 0.0) {
      double vsigav_i = pymax(A(alpha1)[i] * vwave_i - beta * dot, 0.0);
      double vsigav_j = pymax(A(alpha1)[j] * vwave_j - beta * dot, 0.0);
      double qrho2_i = -0.5 / rhoi * vsigav_i * dot * pr->av;
      double qrho2_j = -0.5 / rhoj * vsigav_j * dot * pr->av;
      A(au)[i] += -mj * (qrho2_i * omegai * DWI[0] + qrho2_j * omegaj * DWJ[0]);
      A(av)[i] += -mj * (qrho2_i * omegai * DWI[1] + qrho2_j * omegaj * DWJ[1]);
      A(aw)[i] += -mj * (qrho2_i * omegai * DWI[2] + qrho2_j * omegaj * DWJ[2]);
      A(ae)[i] += mj * qrho2_i * dot * grad_i;
    }
    A(au)[i] += -mj * (pibrhoi2 * omegai * DWI[0] + pjbrhoj2 * omegaj * DWJ[0]);
    A(av)[i] += -mj * (pibrhoi2 * omegai * DWI[1] + pjbrhoj2 * omegaj * DWJ[1]);
    A(aw)[i] += -mj * (pibrhoi2 * omegai * DWI[2] + pjbrhoj2 * omegaj * DWJ[2]);
    double vijdotdwi = dvx * DWI[0] + dvy * DWI[1] + dvz * DWI[2];
    A(ae)[i] += mj * pibrhoi2 * omegai * vijdotdwi;
    double eij = A(epred)[i] - A(epred)[j];
    A(ae)[i] += pr->ac * vsig2 * eij * (0.5 * A(m)[j] / rhoi * grad_i + 0.5 * mj / rhoj * grad_j);
  }
  /* post_loop (:278-280) */
  A(div_for_psi)[i] = -A(div)[i] / A(rho)[i];
  A(div)[i] = -A(div)[i] / A(rho)[i];
}

static void maxwell_loop(const OracleParams* pr, const Kern* K, double** P, int64_t i, const int64_t* nb, int64_t cnt) {
  const double mu0 = pr->mu0;
  double hi = A(h)[i];
  for (int64_t t = 0; t < cnt; t++) {
    int64_t j = nb[t];
    Pair q = make_pair(pr, P, i, j);
    double DWI[3], DWJ[3];
    kern_grad(K, q.xij, q.rij, hi, DWI);
    kern_grad(K, q.xij, q.rij, A(h)[j], DWJ);
    const double* XIJ = q.xij;
    double RIJ = q.rij;
    /* loop (:149-195) */
    double runix, runiy, runiz;
    if (RIJ > PAIR_DISTANCE_EPSILON) { runix = XIJ[0] / RIJ; runiy = XIJ[1] / RIJ; runiz = XIJ[2] / RIJ; }
    else { runix = 0.0; runiy = 0.0; runiz = 0.0; }
    double grad_i = A(omega)[i] * (runix * DWI[0] + runiy * DWI[1] + runiz * DWI[2]);
    double grad_j = A(omega)[j] * (runix * DWJ[0] + runiy * DWJ[1] + runiz * DWJ[2]);
    double rho_i = A(rho)[i], rho_j = A(rho)[j];
    double brhox_i = A(Bxpred)[i] / rho_i, brhoy_i = A(Bypred)[i] / rho_i, brhoz_i = A(Bzpred)[i] / rho_i;
    double brhox_j = A(Bxpred)[j] / rho_j, brhoy_j = A(Bypred)[j] / rho_j, brhoz_j = A(Bzpred)[j] / rho_j;
    double bro2_i = (brhox_i * brhox_i + brhoy_i * brhoy_i + brhoz_i * brhoz_i) / mu0;
    double bro2_j = (brhox_j * brhox_j + brhoy_j * brhoy_j + brhoz_j * brhoz_j) / mu0;
    double sm = A(m)[j];
    double gradp = sm * (0.5 * bro2_i * grad_i + 0.5 * bro2_j * grad_j);
    double sxx_i = -sm * brhox_i * brhox_i / mu0;
    double sxy_i = -sm * brhox_i * brhoy_i / mu0;
    double sxz_i = -sm * brhox_i * brhoz_i / mu0;
    double syy_i = -sm * brhoy_i * brhoy_i / mu0;
    double syz_i = -sm * brhoy_i * brhoz_i / mu0;
    double szz_i = -sm * brhoz_i * brhoz_i / mu0;
    double sxx_j = -sm * brhox_j * brhox_j / mu0;
    double sxy_j = -sm * brhox_j * brhoy_j / mu0;
    double sxz_j = -sm * brhox_j * brhoz_j / mu0;
    double syy_j = -sm * brhoy_j * brhoy_j / mu0;
    double syz_j = -sm * brhoy_j * brhoz_j / mu0;
    double szz_j = -sm * brhoz_j * brhoz_j / mu0;
    double projsx = (sxx_i * runix + sxy_i * runiy + sxz_i * runiz) * grad_i + (sxx_j * runix + sxy_j * runiy + sxz_j * runiz) * grad_j;
    double projsy = (sxy_i * runix + syy_i * runiy + syz_i * runiz) * grad_i + (sxy_j * runix + syy_j * runiy + syz_j * runiz) * grad_j;
    double projsz = (sxz_i * runix + syz_i * runiy + szz_i * runiz) * grad_i + (sxz_j * runix + syz_j * runiy + szz_j * runiz) * grad_j;
    double ax = -runix * gradp - projsx;
    double ay = -runiy * gradp - projsy;
    double az = -runiz * gradp - projsz;
    A(au)[i] += ax;
    A(av)[i] += ay;
    A(aw)[i] += az;
  }
}

static void magrates_loop(const OracleParams* pr, const Kern* K, double** P, int64_t i, const int64_t* nb, int64_t cnt) {
  const double mu0 = pr->mu0;
  /* initialize (:498-504) */
  A(aBevolx)[i] = 0.0; A(aBevoly)[i] = 0.0; A(aBevolz)[i] = 0.0;
  A(apsi)[i] = 0.0; A(divBsymm)[i] = 0.0; A(divBdiff)[i] = 0.0;
  double hi = A(h)[i];
  for (int64_t t = 0; t < cnt; t++) {
    int64_t j = nb[t];
    Pair q = make_pair(pr, P, i, j);
    double DWI[3], DWJ[3];
    kern_grad(K, q.xij, q.rij, hi, DWI);
    kern_grad(K, q.xij, q.rij, A(h)[j], DWJ);
    const double* XIJ = q.xij;
    double RIJ = q.rij;
    /* loop (:507-559) */
    double runix, runiy, runiz;
    if (RIJ > PAIR_DISTANCE_EPSILON) { runix = XIJ[0] / RIJ; runiy = XIJ[1] / RIJ; runiz = XIJ[2] / RIJ; }
    else { runix = 0.0; runiy = 0.0; runiz = 0.0; }
    double grad_i = A(omega)[i] * (runix * DWI[0] + runiy * DWI[1] + runiz * DWI[2]);
    double grad_j = A(omega)[j] * (runix * DWJ[0] + runiy * DWJ[1] + runiz * DWJ[2]);
    double rho_i = A(rho)[i], rho_j = A(rho)[j];
    double bx_i = A(Bxpred)[i], by_i = A(Bypred)[i], bz_i = A(Bzpred)[i];
    double bx_j = A(Bxpred)[j], by_j = A(Bypred)[j], bz_j = A(Bzpred)[j];
    double proj_bi = bx_i * runix + by_i * runiy + bz_i * runiz;
    double proj_bj = bx_j * runix + by_j * runiy + bz_j * runiz;
    double dbx = bx_i - bx_j, dby = by_i - by_j, dbz = bz_i - bz_j;
    double proj_db = dbx * runix + dby * runiy + dbz * runiz;
    double delta_b2 = dbx * dbx + dby * dby + dbz * dbz;
    double rho_i2_inv = 1.0 / (rho_i * rho_i);
    double rho_j2_inv = 1.0 / (rho_j * rho_j);
    double sm = A(m)[j];
    double pmj_rho21_grad_i = sm * rho_i2_inv * grad_i;
    double pmj_rho21_grad_j = sm * rho_j2_inv * grad_j;
    double d_brho_term = -(pmj_rho21_grad_i * proj_bi);
    double dvx = A(upred)[i] - A(upred)[j];
    double dvy = A(vpred)[i] - A(vpred)[j];
    double dvz = A(wpred)[i] - A(wpred)[j];
    double projv = dvx * runix + dvy * runiy + dvz * runiz;
    double dvxt = dvx - projv * runix;
    double dvyt = dvy - projv * runiy;
    double dvzt = dvz - projv * runiz;
    double vsig_b = sqrt(dvxt * dvxt + dvyt * dvyt + dvzt * dvzt);
    double d_b_diss_term = 0.5 * (sm * rho_i2_inv * grad_i + sm * rho_j2_inv * grad_j) * vsig_b * pr->ar;
    double vwave_i = sqrt(A(cs)[i] * A(cs)[i] + (bx_i * bx_i + by_i * by_i + bz_i * bz_i) / (mu0 * rho_i));
    double vwave_j = sqrt(A(cs)[j] * A(cs)[j] + (bx_j * bx_j + by_j * by_j + bz_j * bz_j) / (mu0 * rho_j));
    double ch_i = pr->clean_speed * vwave_i;
    double ch_j = pr->clean_speed * vwave_j;
    double dpsi_term = pmj_rho21_grad_i * A(psipred)[i] * ch_i + pmj_rho21_grad_j * A(psipred)[j] * ch_j;
    A(aBevolx)[i] += d_brho_term * dvx + d_b_diss_term * dbx - dpsi_term * runix;
    A(aBevoly)[i] += d_brho_term * dvy + d_b_diss_term * dby - dpsi_term * runiy;
    A(aBevolz)[i] += d_brho_term * dvz + d_b_diss_term * dbz - dpsi_term * runiz;
    A(ae)[i] += -0.5 * delta_b2 * d_b_diss_term / mu0;
    A(divBsymm)[i] += pmj_rho21_grad_i * proj_bi + pmj_rho21_grad_j * proj_bj;
    A(divBdiff)[i] += -sm * proj_db * grad_i;
  }
  /* post_loop (:562-567) */
  double vwave = sqrt(A(cs)[i] * A(cs)[i] + (A(Bxpred)[i] * A(Bxpred)[i] + A(Bypred)[i] * A(Bypred)[i] + A(Bzpred)[i] * A(Bzpred)[i]) / (mu0 * A(rho)[i]));
  double ch = pr->clean_speed * vwave;
  double cleaning_active = pr->clean_speed > 0.0 ? 1.0 : 0.0;
  A(apsi)[i] = -ch * A(divBdiff)[i] / A(rho)[i] - pr->clean_damp * A(psipred)[i] * ch / A(h)[i] - 0.5 * cleaning_active * A(psipred)[i] * A(div_for_psi)[i];
  A(dt_cfl)[i] = pymax(A(dt_cfl)[i], vwave);
  A(dt_cfl)[i] = pymax(A(dt_cfl)[i], ch);
}

static void g10(const OracleParams* pr, double** P, int64_t i) {
  const double c_cour = pr->timestep_factor * COURANT_FACTOR;
  const double c_force = pr->timestep_factor * FORCE_FACTOR;
  const double mu0 = pr->mu0;
  /* EnergyLimiter.initialize (:594-598) */
  if (A(dt_cfl)[i] > 0.0) {
    double dtc = c_cour * A(h)[i] / A(dt_cfl)[i];
    if (A(epred)[i] + dtc * A(ae)[i] < 0.0 && A(epred)[i] > 0.0) A(ae)[i] /= 1.0 - dtc * A(ae)[i] / A(epred)[i];
  }
  /* DivBCorrection.initialize (:607-624) */
  double bx = A(Bxpred)[i], by = A(Bypred)[i], bz = A(Bzpred)[i];
  double b2 = bx * bx + by * by + bz * bz;
  double divb = A(divBsymm)[i];
  double frac_divb = 0.0;
  if (b2 > 0.0) {
    double beta = 2.0 * mu0 * A(p)[i] / b2;
    frac_divb = pymax(0.0, pymin(1.0, (10.0 - beta) * 0.125));
  }
  double ax = -bx * divb * frac_divb / mu0;
  double ay = -by * divb * frac_divb / mu0;
  double az = -bz * divb * frac_divb / mu0;
  A(au)[i] += ax;
  A(av)[i] += ay;
  A(aw)[i] += az;
  A(divBsymm)[i] = A(rho)[i] * divb;
  /* AdaptiveTimestep.initialize (:578-585) */
  double dt_adapt = 1.0e29;
  if (A(dt_cfl)[i] > 0.0) dt_adapt = c_cour * A(h)[i] / A(dt_cfl)[i];
  double f2 = A(au)[i] * A(au)[i] + A(av)[i] * A(av)[i] + A(aw)[i] * A(aw)[i];
  if (f2 > 0.0) dt_adapt = pymin(dt_adapt, c_force * sqrt(A(h)[i] / sqrt(f2)));
  A(dt_adapt)[i] = dt_adapt;
}

typedef void (*pair_fn)(const OracleParams*, const Kern*, double**, int64_t, const int64_t*, int64_t);

static void pair_group(const OracleParams* pr, const Kern* K, int64_t n, double** P, const Grid* g, pair_fn fn) {
#pragma omp parallel
  {
    int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * NBR_MAX * 8);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
      int64_t cnt = neighbours(g, pr, P, K->R, i, nb);
      fn(pr, K, P, i, nb, cnt);
    }
    free(nb);
  }
}

static void set_threads(const OracleParams* pr) {
#ifdef _OPENMP
  if (pr->nthreads > 0) omp_set_num_threads(pr->nthreads);
#else
  (void)pr;
#endif
}

/* One right-hand-side evaluation: the ten groups of src/scheme.py:70-81.
   Returns the number of density passes. */
int oracle_rhs(const OracleParams* pr, int64_t n, double** P, int32_t* itype) {
  (void)itype;
  set_threads(pr);
  Kern K = {pr->kernel, pr->dim, kernel_norm(pr->kernel, pr->dim), radius_scale(pr->kernel)};
  const double k = pr->hfact, dim = (double)pr->dim;
  /* G1: iterated DensityIteration (src/scheme.py:71) */
  int passes = 0;
  int min_it = pr->iterate ? pr->min_iter : 0;
  int max_it = pr->iterate ? pr->max_iter : 1;
  for (;;) {
    int conv = density_pass(pr, &K, n, P);
    passes++;
    if (!pr->iterate) break;
    if ((passes >= min_it && conv > 0) || passes == max_it) break;
  }
  /* G2, G3 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    double rhoh = A(m)[i] / pow(A(h)[i] / k, dim);
    A(ah)[i] *= rhoh / A(rho)[i];
    A(rho_sum)[i] = A(rho)[i];
    A(rho)[i] = A(m)[i] / pow(A(h)[i] / k, dim);
    A(p)[i] = (pr->gamma - 1.0) * A(rho)[i] * A(epred)[i];
    A(cs)[i] = sqrt(pr->gamma * A(p)[i] / A(rho)[i]);
  }
  Grid g;
  grid_build(&g, pr, n, P, K.R * max_h(n, A(h)));
  /* G4 */
  pair_group(pr, &K, n, P, &g, cd_loop);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) cd_post(pr, P, i);
  /* G5 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) strain_and_bfield(P, i);
  /* G6 */
  pair_group(pr, &K, n, P, &g, mhd_acc_loop);
  /* G7 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) A(ah)[i] = A(h)[i] * A(div)[i] * (1.0 / dim);
  /* G8, G9 */
  pair_group(pr, &K, n, P, &g, maxwell_loop);
  pair_group(pr, &K, n, P, &g, magrates_loop);
  /* G10 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) g10(pr, P, i);
  grid_free(&g);
  return passes;
}

/* Neighbour count of every particle under the rule of the pair loops
   (r_ij < R max(h_i, h_j), minimum image, self included) with the current
   h: the oracle's own cell search, for checking the device's lists. */
int oracle_neighbour_counts(const OracleParams* pr, int64_t n, double** P, int32_t* counts) {
  set_threads(pr);
  Kern K = {pr->kernel, pr->dim, kernel_norm(pr->kernel, pr->dim), radius_scale(pr->kernel)};
  Grid g;
  grid_build(&g, pr, n, P, K.R * max_h(n, A(h)));
#pragma omp parallel
  {
    int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * NBR_MAX * 8);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) counts[i] = (int32_t)neighbours(&g, pr, P, K.R, i, nb);
    free(nb);
  }
  grid_free(&g);
  return 0;
}

/* MHDStep.initialize (src/integrator.py:12-35) */
static void stage_initialize(int64_t n, double** P) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    A(x0)[i] = A(x)[i]; A(y0)[i] = A(y)[i]; A(z0)[i] = A(z)[i];
    A(u0)[i] = A(u)[i]; A(v0)[i] = A(v)[i]; A(w0)[i] = A(w)[i];
    A(upred)[i] = A(u)[i]; A(vpred)[i] = A(v)[i]; A(wpred)[i] = A(w)[i];
    A(e0)[i] = A(e)[i]; A(epred)[i] = A(e)[i]; A(h0)[i] = A(h)[i];
    A(converged)[i] = 0; A(omega)[i] = 1.0; A(alpha10)[i] = A(alpha1)[i];
    A(Bevolx0)[i] = A(Bevolx)[i]; A(Bevoly0)[i] = A(Bevoly)[i]; A(Bevolz0)[i] = A(Bevolz)[i]; A(psi0)[i] = A(psi)[i];
    A(Bevolxpred)[i] = A(Bevolx)[i]; A(Bevolypred)[i] = A(Bevoly)[i]; A(Bevolzpred)[i] = A(Bevolz)[i];
    A(psipred)[i] = A(psi)[i];
  }
}

/* MHDStep.stage1 (src/integrator.py:38-65); in dim 2 z is not a coordinate. */
static void stage_1(const OracleParams* pr, int64_t n, double** P, const int32_t* itype, double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    if (itype[i] != 1) continue;
    double dtb2 = 0.5 * dt;
    A(u)[i] = A(u0)[i] + dtb2 * A(au)[i];
    A(v)[i] = A(v0)[i] + dtb2 * A(av)[i];
    A(w)[i] = A(w0)[i] + dtb2 * A(aw)[i];
    A(upred)[i] = A(u0)[i] + dt * A(au)[i];
    A(vpred)[i] = A(v0)[i] + dt * A(av)[i];
    A(wpred)[i] = A(w0)[i] + dt * A(aw)[i];
    A(x)[i] = A(x0)[i] + dt * A(u)[i];
    A(y)[i] = A(y0)[i] + dt * A(v)[i];
    if (pr->dim == 3) A(z)[i] = A(z0)[i] + dt * A(w)[i];
    A(e)[i] = A(e0)[i] + dtb2 * A(ae)[i];
    A(epred)[i] = A(e0)[i] + dt * A(ae)[i];
    A(h)[i] = A(h0)[i] + dt * A(ah)[i];
    double decay_rate = 0.1 * A(cs)[i] / A(h)[i];
    if (A(alpha10)[i] < A(alphaloc)[i]) A(alpha1)[i] = A(alphaloc)[i];
    else A(alpha1)[i] = (A(alpha10)[i] + dt * A(alphaloc)[i] * decay_rate) / (1.0 + dt * decay_rate);
    A(Bevolx)[i] = A(Bevolx0)[i] + dtb2 * A(aBevolx)[i];
    A(Bevoly)[i] = A(Bevoly0)[i] + dtb2 * A(aBevoly)[i];
    A(Bevolz)[i] = A(Bevolz0)[i] + dtb2 * A(aBevolz)[i];
    A(psi)[i] = A(psi0)[i] + dtb2 * A(apsi)[i];
    A(Bevolxpred)[i] = A(Bevolx0)[i] + dt * A(aBevolx)[i];
    A(Bevolypred)[i] = A(Bevoly0)[i] + dt * A(aBevoly)[i];
    A(Bevolzpred)[i] = A(Bevolz0)[i] + dt * A(aBevolz)[i];
    A(psipred)[i] = A(psi0)[i] + dt * A(apsi)[i];
  }
}

/* MHDStep.stage2 (src/integrator.py:68-82) */
static void stage_2(const OracleParams* pr, int64_t n, double** P, const int32_t* itype, double dt) {
  const double gamma1 = pr->gamma - 1.0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    if (itype[i] != 1) continue;
    double dtb2 = 0.5 * dt;
    A(u)[i] += dtb2 * A(au)[i];
    A(v)[i] += dtb2 * A(av)[i];
    A(w)[i] += dtb2 * A(aw)[i];
    A(e)[i] += dtb2 * A(ae)[i];
    A(p)[i] = gamma1 * A(rho)[i] * A(e)[i];
    A(Bevolx)[i] += dtb2 * A(aBevolx)[i];
    A(Bevoly)[i] += dtb2 * A(aBevoly)[i];
    A(Bevolz)[i] += dtb2 * A(aBevolz)[i];
    A(psi)[i] += dtb2 * A(apsi)[i];
    A(Bx)[i] = A(Bevolx)[i] * A(rho)[i];
    A(By)[i] = A(Bevoly)[i] * A(rho)[i];
    A(Bz)[i] = A(Bevolz)[i] * A(rho)[i];
  }
}

/* Periodic wrap of positions into the box (PySPH DomainManager, restated). */
static void wrap(const OracleParams* pr, int64_t n, double** P) {
  double* pos[3] = {A(x), A(y), A(z)};
  for (int a = 0; a < pr->dim; a++) {
    if (!pr->periodic[a]) continue;
    double lo = pr->lo[a], hi = pr->hi[a], L = hi - lo;
    for (int64_t i = 0; i < n; i++) {
      if (pos[a][i] < lo) pos[a][i] = pos[a][i] + L;
      if (pos[a][i] > hi) pos[a][i] = pos[a][i] - L;
    }
  }
}

/* PECIntegrator.one_timestep (restated): returns the density passes. */
int oracle_step(const OracleParams* pr, int64_t n, double** P, int32_t* itype, double dt) {
  set_threads(pr);
  stage_initialize(n, P);
  stage_1(pr, n, P, itype, dt);
  wrap(pr, n, P);
  int passes = oracle_rhs(pr, n, P, itype);
  stage_2(pr, n, P, itype, dt);
  wrap(pr, n, P);
  return passes;
}

/* The two halves of PECIntegrator.one_timestep around its right-hand side,
   for drivers that evaluate the right-hand side themselves (the domain
   decomposition tests): MHDStep.initialize + stage1 + wrap, and
   MHDStep.stage2 + wrap (src/integrator.py:12-82). */
int oracle_predict(const OracleParams* pr, int64_t n, double** P, int32_t* itype, double dt) {
  set_threads(pr);
  stage_initialize(n, P);
  stage_1(pr, n, P, itype, dt);
  wrap(pr, n, P);
  return 0;
}

int oracle_correct(const OracleParams* pr, int64_t n, double** P, int32_t* itype, double dt) {
  set_threads(pr);
  stage_2(pr, n, P, itype, dt);
  wrap(pr, n, P);
  return 0;
}

/* min over particles of dt_adapt (the adaptive-timestep rule). */
double oracle_min_dt(int64_t n, double** P) {
  double m = INFINITY;
  for (int64_t i = 0; i < n; i++) m = A(dt_adapt)[i] < m ? A(dt_adapt)[i] : m;
  return m;
}
