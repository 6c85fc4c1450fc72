// mhd_adjoint.cu -- reverse-mode (adjoint) derivative of the SPMHD step loop.
//
// Differentiates L = sum_i m_i |B_i|^2 / (2 mu0 rho_i) after K literal PEC
// steps (MHDStep + the ten groups of src/scheme.py:66-81, single density
// pass, step sizes given and frozen) with respect to the state at the first
// step and to alpha_max.  The forward sweep keeps the 24-field step state
// every `every` steps (checkpoints); the reverse sweep re-runs each segment
// from its checkpoint with a tape of the intermediates (predicted state,
// density, EOS, Cullen-Dehnen and force sums) and walks it backwards.
//
// Every stage is a pair sum or a pointwise map of mhd_step_fns.cuh.  Its
// vector-Jacobian product is formed from the local Jacobian of that map,
// obtained by evaluating the same function on dual numbers seeded with the
// identity over the stage's per-particle inputs: pointwise maps and posts
// per particle, pair terms per pair in gather form (a particle collects the
// terms in which it is the i side and those in which it is the j side, so
// there are no atomics).  The energy limiter's time scale (from dt_cfl) is
// held at its value, like the step size.  Neighbours: the cell grid of
// mhd_pairgrid.cuh over each pass's positions and smoothing lengths, with
// the exact rule.  Compiled with --fmad=false like the forward-mode file.
#include <cuda_runtime.h>

#include <string>

#include "mhd_common.cuh"
#include "mhd_dual.cuh"
#include "mhd_internal.h"
#include "mhd_pairgrid.cuh"
#include "mhd_step_fns.cuh"

namespace mhd {
namespace adj {

constexpr int kTile = 128;
constexpr int NS = kStateDirs;  // 24 state fields
// state field offsets (field-major arrays of n)
enum { SX = 0, SV = 3, SE = 6, SH = 7, SA1 = 8, SB = 9, SPSI = 12, SA = 13, SAE = 16, SAH = 17, SALOC = 18,
       SCS = 19, SAB = 20, SAPSI = 23 };
// tape offsets (per step): the input state, the predicted state, the density
// pass, the EOS, the Cullen-Dehnen sums and the force sums
enum { T_S = 0, T_X = 24, T_VH = 27, T_VP = 30, T_EH = 33, T_EP = 34, T_HP = 35, T_A1 = 36, T_BH = 37, T_BP = 40,
       T_PSIH = 43, T_PSIP = 44, T_RS = 45, T_DW = 46, T_OM = 47, T_HN = 48, T_RHO = 49, T_P = 50, T_CS = 51,
       T_B = 52, T_CD = 55, T_ALOC = 82, T_FS = 83, T_DTCFL = 97, NT = 98 };
// workspace offsets: lambdas of the intermediates, the sum adjoints and the
// lambdas of the rates
enum { L_X = 0, L_VH = 3, L_VP = 6, L_EH = 9, L_EP = 10, L_HP = 11, L_A1 = 12, L_BH = 13, L_BP = 16, L_PSIH = 19,
       L_PSIP = 20, L_HN = 21, L_OM = 22, L_RHO = 23, L_P = 24, L_CS = 25, L_B = 26, M_D = 29, M_CD = 31, M_F = 58,
       L_RATES = 72, NL = 81 };  // L_RATES: au 3, ae, ah, ab 3, apsi

template <int N>
__device__ inline Dual<N> seeded(double v, int k) {
  Dual<N> r(v);
  if (k >= 0) r.d[k] = 1.0;
  return r;
}

struct Args {
  int n;
  DevParams P;
  double dt;
  double amax;
  const double* m;
  const int* itype;
  const double* s_in;      // forward: S_n (NS x n)
  double* s_out;           // forward: S_{n+1}
  const double* tape;      // this step's tape (NT x n)
  double* tape_w;          // forward: tape written
  const double* lam_next;  // reverse: lambda(S_{n+1})
  double* lam;             // reverse: lambda(S_n)
  double* w;               // reverse: workspace (NL x n)
  double* g_amax;          // reverse: per-particle dL/d alpha_max (accumulating over steps)
  const double* s_final;   // reverse, last step: S_K (loss terms)
  double* dta_out;         // forward: dt_adapt of the step (adaptive step sizes)
  double* slices;          // per-slice partial sums of the pair passes
  int dual_pairs;          // reverse: force and CD pair VJPs from dual Jacobians (check path) instead of by hand
  // the neighbour search of the pair passes (mhd_pairgrid.cuh), rebuilt
  // before each pass over its positions and smoothing lengths
  const PairGrid* pg;
  const int* cell_start;
  const int* perm;
  const double4* pos;
  int nslices;
};

// f(j, dx, dy, dz) for every neighbour j of particle i (i < n) under the
// exact rule, among the particles of this block's slice (grid y).
template <int DIM, class F>
__device__ inline void a_pairs(const Args& a, int i, F&& f) {
  if (i >= a.n) return;
  pair_grid_visit<DIM>(*a.pg, a.cell_start, a.perm, a.pos, a.P, i, (int)blockIdx.y, a.nslices, f);
}

#define TP(k, i) a.tape_w[(size_t)(k) * a.n + (i)]
#define TR(k, i) a.tape[(size_t)(k) * a.n + (i)]
#define SI(k, i) a.s_in[(size_t)(k) * a.n + (i)]
#define SO(k, i) a.s_out[(size_t)(k) * a.n + (i)]
#define LN(k, i) a.lam_next[(size_t)(k) * a.n + (i)]
#define LS(k, i) a.lam[(size_t)(k) * a.n + (i)]
#define W(k, i) a.w[(size_t)(k) * a.n + (i)]

// Pair passes split over a.nslices slices of the particles (grid y,
// a_pairs): each writes `width` partial sums per particle and slice, value
// q of slice s at slices[(s * width + q) * n + i], and a per-particle
// kernel adds the slices in slice order (deterministic).
constexpr int kSliceWidth = 24;  // the widest partial record (the 24 CD moments)
__device__ inline double& slice_part(const Args& a, int width, int q, int i) {
  return a.slices[((size_t)blockIdx.y * width + q) * a.n + i];
}
__device__ inline double slices_sum(const Args& a, int width, int q, int i) {
  double v = 0.0;
  for (int s = 0; s < a.nslices; s++) v += a.slices[((size_t)s * width + q) * a.n + i];
  return v;
}

template <class D>
__device__ inline StepState<D> state_at(const double* s, int n, int i, int seed_base) {
  StepState<D> q;
  auto g = [&](int k) { return seeded<sizeof(D) / sizeof(double) - 1>(s[(size_t)k * n + i], seed_base < 0 ? -1 : k); };
  for (int c = 0; c < 3; c++) {
    q.x[c] = g(SX + c);
    q.v[c] = g(SV + c);
    q.bev[c] = g(SB + c);
    q.a[c] = g(SA + c);
    q.abev[c] = g(SAB + c);
  }
  q.e = g(SE);
  q.h = g(SH);
  q.alpha1 = g(SA1);
  q.psi = g(SPSI);
  q.ae = g(SAE);
  q.ah = g(SAH);
  q.aloc = g(SALOC);
  q.cs = g(SCS);
  q.apsi = g(SAPSI);
  return q;
}

__device__ inline StepState<double> state_values(const double* s, int n, int i) {
  StepState<double> q;
  auto g = [&](int k) { return s[(size_t)k * n + i]; };
  for (int c = 0; c < 3; c++) {
    q.x[c] = g(SX + c);
    q.v[c] = g(SV + c);
    q.bev[c] = g(SB + c);
    q.a[c] = g(SA + c);
    q.abev[c] = g(SAB + c);
  }
  q.e = g(SE);
  q.h = g(SH);
  q.alpha1 = g(SA1);
  q.psi = g(SPSI);
  q.ae = g(SAE);
  q.ah = g(SAH);
  q.aloc = g(SALOC);
  q.cs = g(SCS);
  q.apsi = g(SAPSI);
  return q;
}

// Side of particle i from a tape, as dual numbers seeded at `base` (or not).
template <class D>
__device__ inline Side<D> side_at(const double* t, int n, int i, int base) {
  auto g = [&](int k, int s) {
    D r(t[(size_t)k * n + i]);
    if (base >= 0) r.d[base + s] = 1.0;
    return r;
  };
  Side<D> s;
  s.h = g(T_HN, 0);
  s.rho = g(T_RHO, 1);
  s.p = g(T_P, 2);
  s.omega = g(T_OM, 3);
  s.cs = g(T_CS, 4);
  for (int c = 0; c < 3; c++) {
    s.b[c] = g(T_B + c, 5 + c);
    s.v[c] = g(T_VP + c, 8 + c);
  }
  s.e = g(T_EP, 11);
  s.alpha = g(T_A1, 12);
  s.psi = g(T_PSIP, 13);
  return s;
}

// Side of particle i with only the directions lo .. lo + N - 1 of the
// kSideDirs side inputs seeded (local direction s - lo).
template <int N>
__device__ inline Side<Dual<N>> side_window(const double* t, int n, int i, int lo) {
  using D = Dual<N>;
  auto g = [&](int k, int s) {
    D r(t[(size_t)k * n + i]);
    if (s >= lo && s < lo + N) r.d[s - lo] = 1.0;
    return r;
  };
  Side<D> s;
  s.h = g(T_HN, 0);
  s.rho = g(T_RHO, 1);
  s.p = g(T_P, 2);
  s.omega = g(T_OM, 3);
  s.cs = g(T_CS, 4);
  for (int c = 0; c < 3; c++) {
    s.b[c] = g(T_B + c, 5 + c);
    s.v[c] = g(T_VP + c, 8 + c);
  }
  s.e = g(T_EP, 11);
  s.alpha = g(T_A1, 12);
  s.psi = g(T_PSIP, 13);
  return s;
}

__device__ inline Side<double> side_values(const double* t, int n, int i) {
  auto g = [&](int k) { return t[(size_t)k * n + i]; };
  Side<double> s;
  s.h = g(T_HN);
  s.rho = g(T_RHO);
  s.p = g(T_P);
  s.omega = g(T_OM);
  s.cs = g(T_CS);
  for (int c = 0; c < 3; c++) {
    s.b[c] = g(T_B + c);
    s.v[c] = g(T_VP + c);
  }
  s.e = g(T_EP);
  s.alpha = g(T_A1);
  s.psi = g(T_PSIP);
  return s;
}

// ====================================================== taped forward step
__global__ void __launch_bounds__(256) k_f_predict(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int k = 0; k < NS; k++) TP(T_S + k, i) = SI(k, i);
  const StepState<double> s = state_values(a.s_in, a.n, i);
  Predicted<double> o;
  f_predict(a.P, s, a.itype[i] == 1, a.dt, o);
  for (int c = 0; c < 3; c++) {
    TP(T_X + c, i) = o.x[c];
    TP(T_VH + c, i) = o.vhalf[c];
    TP(T_VP + c, i) = o.vpred[c];
    TP(T_BH + c, i) = o.bhalf[c];
    TP(T_BP + c, i) = o.bpred[c];
  }
  TP(T_EH, i) = o.ehalf;
  TP(T_EP, i) = o.epred;
  TP(T_HP, i) = o.h;
  TP(T_A1, i) = o.alpha1;
  TP(T_PSIH, i) = o.psihalf;
  TP(T_PSIP, i) = o.psipred;
}

template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_f_density_pair(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const double* HP = a.tape_w + (size_t)T_HP * n;
  double rho = 0.0, dwdh = 0.0;
  const double hi = i < n ? HP[i] : 1.0;
  a_pairs<DIM>(a, i, [&](int j, double dx, double dy, double dz) {
    const double xij[3] = {dx, dy, dz};
    f_density_pair<K, DIM>(a.P.norm, xij, hi, a.m[j], rho, dwdh);
  });
  if (i >= n) return;
  slice_part(a, 2, 0, i) = rho;
  slice_part(a, 2, 1, i) = dwdh;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_f_density(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (i >= n) return;
  const double hi = TP(T_HP, i);
  const double rho = slices_sum(a, 2, 0, i), dwdh = slices_sum(a, 2, 1, i);
  double om, hn;
  f_density_post<DIM>(a.P.hfact, hi, a.m[i], rho, dwdh, om, hn);
  TP(T_RS, i) = rho;
  TP(T_DW, i) = dwdh;
  TP(T_OM, i) = om;
  TP(T_HN, i) = hn;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_f_prologue(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double bp[3] = {TP(T_BP, i), TP(T_BP + 1, i), TP(T_BP + 2, i)};
  double rho, p, cs, b[3];
  f_prologue<DIM>(a.P, TP(T_HN, i), a.m[i], TP(T_EP, i), bp, rho, p, cs, b);
  TP(T_RHO, i) = rho;
  TP(T_P, i) = p;
  TP(T_CS, i) = cs;
  for (int c = 0; c < 3; c++) TP(T_B + c, i) = b[c];
}

template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_f_cd_pair(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const double* HN = a.tape_w + (size_t)T_HN * n;
  double r[6] = {}, vv[9] = {}, aa[9] = {};
  const int ii = i < n ? i : 0;
  const double hi = HN[ii];
  a_pairs<DIM>(a, i, [&](int j, double dx, double dy, double dz) {
    const double xij[3] = {dx, dy, dz};
    double dv[3], da[3];
    for (int c = 0; c < 3; c++) {
      dv[c] = TP(T_VP + c, i) - TP(T_VP + c, j);
      da[c] = SI(SA + c, i) - SI(SA + c, j);
    }
    f_cd_pair<K, DIM>(a.P.norm, xij, hi, a.m[j], dv, da, r, vv, aa);
  });
  if (i >= n) return;
  for (int k = 0; k < 6; k++) slice_part(a, 24, k, i) = r[k];
  for (int k = 0; k < 9; k++) {
    slice_part(a, 24, 6 + k, i) = vv[k];
    slice_part(a, 24, 15 + k, i) = aa[k];
  }
}

__global__ void __launch_bounds__(256) k_f_cd(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (i >= n) return;
  const double hi = TP(T_HN, i);
  double r[6], vv[9], aa[9];
  for (int k = 0; k < 6; k++) r[k] = slices_sum(a, 24, k, i);
  for (int k = 0; k < 9; k++) {
    vv[k] = slices_sum(a, 24, 6 + k, i);
    aa[k] = slices_sum(a, 24, 15 + k, i);
  }
  for (int k = 0; k < 6; k++) TP(T_CD + k, i) = r[k];
  for (int k = 0; k < 9; k++) {
    TP(T_CD + 6 + k, i) = vv[k];
    TP(T_CD + 15 + k, i) = aa[k];
  }
  TP(T_ALOC, i) = f_cd_post(r, vv, aa, TP(T_OM, i), TP(T_RHO, i), hi, TP(T_CS, i), a.amax, a.P.alpha_min);
}

// Force pair sums over one slice of the candidate tiles (grid y, as the
// reverse force pairs): partial sums of the 14 sums and the dt_cfl max.
constexpr int kFwdSums = kFSumDirs + 1;

template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_f_force_pair(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const Side<double> I = side_values(a.tape_w, n, i < n ? i : 0);
  FSums<double> S;
  S.zero();
  a_pairs<DIM>(a, i, [&](int j, double dx, double dy, double dz) {
    const double xij[3] = {dx, dy, dz};
    f_force_pair<K, DIM>(a.P, I, side_values(a.tape_w, n, j), a.m[j], xij, S);
  });
  if (i >= n) return;
  double* sp[kFSumDirs];
  fsum_ptrs(S, sp);
  double* part = a.slices + (size_t)blockIdx.y * kFwdSums * n;
  for (int k = 0; k < kFSumDirs; k++) part[(size_t)k * n + i] = *sp[k];
  part[(size_t)kFSumDirs * n + i] = S.dtcfl;
}

// The slices' sums added in slice order, then the force post-loop, stage2
// and the next state.
template <int DIM>
__global__ void __launch_bounds__(kTile) k_f_force(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (i >= n) return;
  const Side<double> I = side_values(a.tape_w, n, i);
  FSums<double> S;
  S.zero();
  double* sp[kFSumDirs];
  fsum_ptrs(S, sp);
  for (int sl = 0; sl < a.nslices; sl++) {
    const double* part = a.slices + (size_t)sl * kFwdSums * n;
    for (int k = 0; k < kFSumDirs; k++) *sp[k] += part[(size_t)k * n + i];
    S.dtcfl = fmax(S.dtcfl, part[(size_t)kFSumDirs * n + i]);
  }
  for (int k = 0; k < kFSumDirs; k++) TP(T_FS + k, i) = *sp[k];
  TP(T_DTCFL, i) = S.dtcfl;
  FOut<double> o;
  f_force_post<DIM>(a.P, I, S, o);
  // S_{n+1}: the rates, stage2 (src/integrator.py:68-82) and the carried fields
  const double dtb2 = a.itype[i] == 1 ? 0.5 * a.dt : 0.0;
  for (int c = 0; c < 3; c++) {
    SO(SX + c, i) = TP(T_X + c, i);
    SO(SA + c, i) = o.au[c];
    SO(SAB + c, i) = o.ab[c];
    SO(SV + c, i) = TP(T_VH + c, i) + dtb2 * o.au[c];
    SO(SB + c, i) = TP(T_BH + c, i) + dtb2 * o.ab[c];
  }
  SO(SE, i) = TP(T_EH, i) + dtb2 * o.ae;
  SO(SPSI, i) = TP(T_PSIH, i) + dtb2 * o.apsi;
  SO(SH, i) = TP(T_HN, i);
  SO(SA1, i) = TP(T_A1, i);
  SO(SAE, i) = o.ae;
  SO(SAH, i) = o.ah;
  SO(SALOC, i) = TP(T_ALOC, i);
  SO(SCS, i) = TP(T_CS, i);
  SO(SAPSI, i) = o.apsi;
  if (a.dta_out) a.dta_out[i] = o.dta;
}

// min over particles (one block): the adaptive step size.
__global__ void __launch_bounds__(256) k_min(int n, const double* v, double* out) {
  __shared__ double sh[256];
  double m = INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, v[i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// L = sum m |Bevol rho|^2 / (2 mu0 rho) with rho of the last right-hand side.
__global__ void __launch_bounds__(256) k_f_energy(int n, double mu0, const double* m, const double* s,
                                                  const double* tape, double* part) {
  __shared__ double sh[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < n) {
    const double rho = tape[(size_t)T_RHO * n + i];
    double b2 = 0.0;
    for (int c = 0; c < 3; c++) {
      const double b = s[(size_t)(SB + c) * n + i] * rho;
      b2 += b * b;
    }
    e = m[i] * b2 / (2.0 * mu0 * rho);
  }
  sh[threadIdx.x] = e;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_blocks(int nb, const double* part, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += part[b];
  *out = s;
}

// ============================================================ reverse step
// Loss seed: lambda(Bevol_K) = m Bevol rho / mu0 (the rho term goes to the
// last step's EOS, see k_r_correct).
__global__ void __launch_bounds__(256) k_r_seed(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  double* lam = const_cast<double*>(a.lam_next);
  for (int k = 0; k < NS; k++) lam[(size_t)k * a.n + i] = 0.0;
  const double rho = TR(T_RHO, i);
  for (int c = 0; c < 3; c++)
    lam[(size_t)(SB + c) * a.n + i] = a.m[i] * a.s_final[(size_t)(SB + c) * a.n + i] * rho / a.P.mu0;
}

// Stage2 and the carried fields (the forward k_f_force tail) reversed.
__global__ void __launch_bounds__(256) k_r_correct(Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int k = 0; k < NL; k++) W(k, i) = 0.0;
  for (int k = 0; k < NS; k++) LS(k, i) = 0.0;
  const double dtb2 = a.itype[i] == 1 ? 0.5 * a.dt : 0.0;
  for (int c = 0; c < 3; c++) {
    W(L_X + c, i) = LN(SX + c, i);
    W(L_VH + c, i) = LN(SV + c, i);
    W(L_RATES + c, i) = LN(SA + c, i) + dtb2 * LN(SV + c, i);
    W(L_BH + c, i) = LN(SB + c, i);
    W(L_RATES + 5 + c, i) = LN(SAB + c, i) + dtb2 * LN(SB + c, i);
  }
  W(L_EH, i) = LN(SE, i);
  W(L_RATES + 3, i) = LN(SAE, i) + dtb2 * LN(SE, i);
  W(L_RATES + 4, i) = LN(SAH, i);
  W(L_PSIH, i) = LN(SPSI, i);
  W(L_RATES + 8, i) = LN(SAPSI, i) + dtb2 * LN(SPSI, i);
  W(L_HN, i) = LN(SH, i);
  W(L_A1, i) = LN(SA1, i);
  W(L_CS, i) = LN(SCS, i);
  if (a.s_final) {
    double b2 = 0.0;
    for (int c = 0; c < 3; c++) {
      const double b = a.s_final[(size_t)(SB + c) * a.n + i];
      b2 += b * b;
    }
    W(L_RHO, i) += a.m[i] * b2 / (2.0 * a.P.mu0);
  }
}

// Force posts (G6 post, G7, G9 post, G10) reversed: lambda of the side of i
// and the sum adjoints mu_F.
template <int DIM>
__global__ void __launch_bounds__(64) k_r_force_post(Args a) {
  using D = Dual<kSideDirs + kFSumDirs>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const Side<D> I = side_at<D>(a.tape, a.n, i, 0);
  FSums<D> S;
  S.zero();
  D* sp[kFSumDirs];
  fsum_ptrs(S, sp);
  for (int k = 0; k < kFSumDirs; k++) *sp[k] = seeded<kSideDirs + kFSumDirs>(TR(T_FS + k, i), kSideDirs + k);
  S.dtcfl = D(TR(T_DTCFL, i));
  FOut<D> o;
  f_force_post<DIM>(a.P, I, S, o);
  const D* out[kFOutDirs] = {&o.au[0], &o.au[1], &o.au[2], &o.ae, &o.ah, &o.ab[0], &o.ab[1], &o.ab[2], &o.apsi};
  double g[kSideDirs + kFSumDirs];
  for (int d = 0; d < kSideDirs + kFSumDirs; d++) {
    double s = 0.0;
    for (int q = 0; q < kFOutDirs; q++) s += W(L_RATES + q, i) * out[q]->d[d];
    g[d] = s;
  }
  W(L_HN, i) += g[0];
  W(L_RHO, i) += g[1];
  W(L_P, i) += g[2];
  W(L_OM, i) += g[3];
  W(L_CS, i) += g[4];
  for (int c = 0; c < 3; c++) {
    W(L_B + c, i) += g[5 + c];
    W(L_VP + c, i) += g[8 + c];
  }
  W(L_EP, i) += g[11];
  W(L_A1, i) += g[12];
  W(L_PSIP, i) += g[13];
  for (int k = 0; k < kFSumDirs; k++) W(M_F + k, i) = g[kSideDirs + k];
}

__device__ inline void add_side(const Args& a, int i, const double* g, double sign_x, const double* gx) {
  W(L_HN, i) += g[0];
  W(L_RHO, i) += g[1];
  W(L_P, i) += g[2];
  W(L_OM, i) += g[3];
  W(L_CS, i) += g[4];
  for (int c = 0; c < 3; c++) {
    W(L_B + c, i) += g[5 + c];
    W(L_VP + c, i) += g[8 + c];
    W(L_X + c, i) += sign_x * gx[c];
  }
  W(L_EP, i) += g[11];
  W(L_A1, i) += g[12];
  W(L_PSIP, i) += g[13];
}

// Force pair terms reversed, gather form: particle k collects the terms of
// the pairs (k, j) through its i side and x_k, and of the pairs (j, k)
// through its j side and x_k.  The kSideDirs + 3 input directions are
// evaluated a window of kForceWindow at a time, so the dual sums a thread
// holds stay small (the same derivatives as one pass over all directions).
// The particles are dealt to a.nslices slices (grid y, a_pairs), so that a
// small particle count still fills the GPU; each slice writes its partial
// sums and k_r_force_pair_sum adds them in slice order (deterministic).
constexpr int kForceWindow = 6;
constexpr int kForceDirs = kSideDirs + 3;

template <int K, int DIM, bool DUAL>
__global__ void __launch_bounds__(kTile) k_r_force_pair(Args a) {
  constexpr int NW = kForceWindow, ND = kForceDirs;
  using D = Dual<NW>;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const int kk = k < n ? k : 0;
  double gs[kSideDirs] = {}, gx[3] = {};
  if constexpr (!DUAL) {
    // hand-written VJP (vjp_force_pair)
    const Side<double> Kv = side_values(a.tape, n, kk);
    a_pairs<DIM>(a, k, [&](int j, double dx, double dy, double dz) {
      const Side<double> Jv = side_values(a.tape, n, j);
      double w[kFSumDirs], gI[kSideDirs], gJ[kSideDirs], gxx[3];
      // (k, j): k is the i side
      for (int q = 0; q < kFSumDirs; q++) w[q] = W(M_F + q, k);
      const double xkj[3] = {dx, dy, dz};
      vjp_force_pair<K, DIM>(a.P, Kv, Jv, a.m[j], xkj, w, gI, gJ, gxx);
      for (int d = 0; d < kSideDirs; d++) gs[d] += gI[d];
      for (int c = 0; c < 3; c++) gx[c] += gxx[c];
      // (j, k): k is the j side, x_j - x_k = -(dx, dy, dz)
      for (int q = 0; q < kFSumDirs; q++) w[q] = W(M_F + q, j);
      const double xjk[3] = {-dx, -dy, -dz};
      vjp_force_pair<K, DIM>(a.P, Jv, Kv, a.m[k], xjk, w, gI, gJ, gxx);
      for (int d = 0; d < kSideDirs; d++) gs[d] += gJ[d];
      for (int c = 0; c < 3; c++) gx[c] -= gxx[c];
    });
  } else {
  a_pairs<DIM>(a, k, [&](int j, double dx, double dy, double dz) {
    const Side<D> Jval = side_at<D>(a.tape, n, j, -1);
    for (int lo = 0; lo < ND; lo += NW) {
      const Side<D> Kseed = side_window<NW>(a.tape, n, kk, lo);
      // the displacement directions kSideDirs .. kSideDirs + 2 in this window
      auto xs = [&](double v, int c) {
        const int l = kSideDirs + c - lo;
        return seeded<NW>(v, l >= 0 && l < NW ? l : -1);
      };
      // (k, j): k is the i side
      {
        const D xij[3] = {xs(dx, 0), xs(dy, 1), xs(dz, 2)};
        FSums<D> S;
        S.zero();
        f_force_pair<K, DIM>(a.P, Kseed, Jval, D(a.m[j]), xij, S);
        D* sp[kFSumDirs];
        fsum_ptrs(S, sp);
        for (int d = 0; d < NW && lo + d < ND; d++) {
          double v = 0.0;
          for (int q = 0; q < kFSumDirs; q++) v += W(M_F + q, k) * sp[q]->d[d];
          if (lo + d < kSideDirs) gs[lo + d] += v;
          else gx[lo + d - kSideDirs] += v;
        }
      }
      // (j, k): k is the j side, x_j - x_k = -(dx, dy, dz)
      {
        const D xji[3] = {xs(-dx, 0), xs(-dy, 1), xs(-dz, 2)};
        FSums<D> S;
        S.zero();
        f_force_pair<K, DIM>(a.P, Jval, Kseed, D(a.m[k]), xji, S);
        D* sp[kFSumDirs];
        fsum_ptrs(S, sp);
        for (int d = 0; d < NW && lo + d < ND; d++) {
          double v = 0.0;
          for (int q = 0; q < kFSumDirs; q++) v += W(M_F + q, j) * sp[q]->d[d];
          if (lo + d < kSideDirs) gs[lo + d] += v;
          else gx[lo + d - kSideDirs] -= v;
        }
      }
    }
  });
  }
  if (k >= n) return;
  double* part = a.slices + (size_t)blockIdx.y * ND * n;
  for (int d = 0; d < kSideDirs; d++) part[(size_t)d * n + k] = gs[d];
  for (int c = 0; c < 3; c++) part[(size_t)(kSideDirs + c) * n + k] = gx[c];
}

__global__ void __launch_bounds__(256) k_r_force_pair_sum(Args a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (k >= n) return;
  double g[kForceDirs];
  for (int d = 0; d < kForceDirs; d++) {
    double v = 0.0;
    for (int s = 0; s < a.nslices; s++) v += a.slices[((size_t)s * kForceDirs + d) * n + k];
    g[d] = v;
  }
  add_side(a, k, g, 1.0, g + kSideDirs);
}

// Cullen-Dehnen post reversed: the sum adjoints mu_CD and the lambdas of
// Omega, rho, h, cs; alpha_max's derivative accumulates per particle.
__global__ void __launch_bounds__(64) k_r_cd_post(Args a) {
  using D = Dual<32>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  D r[6], vv[9], aa[9];
  for (int k = 0; k < 6; k++) r[k] = seeded<32>(TR(T_CD + k, i), k);
  for (int k = 0; k < 9; k++) {
    vv[k] = seeded<32>(TR(T_CD + 6 + k, i), 6 + k);
    aa[k] = seeded<32>(TR(T_CD + 15 + k, i), 15 + k);
  }
  const D om = seeded<32>(TR(T_OM, i), 27), rho = seeded<32>(TR(T_RHO, i), 28);
  const D h = seeded<32>(TR(T_HN, i), 29), cs = seeded<32>(TR(T_CS, i), 30);
  const D amax = seeded<32>(a.amax, 31);
  const D al = f_cd_post(r, vv, aa, om, rho, h, cs, amax, a.P.alpha_min);
  const double lam = LN(SALOC, i);
  for (int k = 0; k < 27; k++) W(M_CD + k, i) = lam * al.d[k];
  W(L_OM, i) += lam * al.d[27];
  W(L_RHO, i) += lam * al.d[28];
  W(L_HN, i) += lam * al.d[29];
  W(L_CS, i) += lam * al.d[30];
  a.g_amax[i] += lam * al.d[31];
}

// Cullen-Dehnen pair terms reversed (gather form, as the force pairs).
template <int K, int DIM, bool DUAL>
__global__ void __launch_bounds__(kTile) k_r_cd_pair(Args a) {
  using D = Dual<10>;  // x_ij 3, h_i, dv 3, da 3
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const double* HN = a.tape + (size_t)T_HN * n;
  const int kk = k < n ? k : 0;
  double gx[3] = {}, gh = 0.0, gv[3] = {}, ga[3] = {};
  a_pairs<DIM>(a, k, [&](int j, double dx, double dy, double dz) {
    for (int side = 0; side < 2; side++) {
      // side 0: pair (k, j); side 1: pair (j, k)
      const int ii = side ? j : kk, jj = side ? kk : j;
      const double sgn = side ? -1.0 : 1.0;
      const double xv[3] = {sgn * dx, sgn * dy, sgn * dz};
      double dvv[3], dav[3];
      for (int c = 0; c < 3; c++) {
        dvv[c] = TR(T_VP + c, ii) - TR(T_VP + c, jj);
        dav[c] = TR(T_S + SA + c, ii) - TR(T_S + SA + c, jj);
      }
      double g[10] = {};
      if constexpr (DUAL) {
        const D xij[3] = {seeded<10>(xv[0], 0), seeded<10>(xv[1], 1), seeded<10>(xv[2], 2)};
        const D hi = seeded<10>(HN[ii], side ? -1 : 3);
        D dv[3], da[3];
        for (int c = 0; c < 3; c++) {
          dv[c] = seeded<10>(dvv[c], 4 + c);
          da[c] = seeded<10>(dav[c], 7 + c);
        }
        D r[6], vv[9], aa[9];
        for (int q = 0; q < 6; q++) r[q] = D(0.0);
        for (int q = 0; q < 9; q++) vv[q] = aa[q] = D(0.0);
        f_cd_pair<K, DIM>(a.P.norm, xij, hi, D(a.m[jj]), dv, da, r, vv, aa);
        for (int d = 0; d < 10; d++) {
          double s = 0.0;
          for (int q = 0; q < 6; q++) s += W(M_CD + q, ii) * r[q].d[d];
          for (int q = 0; q < 9; q++) s += W(M_CD + 6 + q, ii) * vv[q].d[d] + W(M_CD + 15 + q, ii) * aa[q].d[d];
          g[d] = s;
        }
      } else {
        double w[24];
        for (int q = 0; q < 24; q++) w[q] = W(M_CD + q, ii);
        vjp_cd_pair<K, DIM>(a.P.norm, xv, HN[ii], a.m[jj], dvv, dav, w, g);
      }
      for (int c = 0; c < 3; c++) {
        gx[c] += sgn * g[c];
        gv[c] += sgn * g[4 + c];
        ga[c] += sgn * g[7 + c];
      }
      if (!side) gh += g[3];
    }
  });
  if (k >= n) return;
  for (int c = 0; c < 3; c++) {
    slice_part(a, 10, c, k) = gx[c];
    slice_part(a, 10, 3 + c, k) = gv[c];
    slice_part(a, 10, 6 + c, k) = ga[c];
  }
  slice_part(a, 10, 9, k) = gh;
}

__global__ void __launch_bounds__(256) k_r_cd_sum(Args a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  for (int c = 0; c < 3; c++) {
    W(L_X + c, k) += slices_sum(a, 10, c, k);
    W(L_VP + c, k) += slices_sum(a, 10, 3 + c, k);
    LS(SA + c, k) += slices_sum(a, 10, 6 + c, k);
  }
  W(L_HN, k) += slices_sum(a, 10, 9, k);
}

// EOS and magnetic-state reconstruction reversed.
template <int DIM>
__global__ void __launch_bounds__(256) k_r_prologue(Args a) {
  using D = Dual<5>;  // h, epred, bpred 3
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const D h = seeded<5>(TR(T_HN, i), 0), ep = seeded<5>(TR(T_EP, i), 1);
  const D bp[3] = {seeded<5>(TR(T_BP, i), 2), seeded<5>(TR(T_BP + 1, i), 3), seeded<5>(TR(T_BP + 2, i), 4)};
  D rho, p, cs, b[3];
  f_prologue<DIM>(a.P, h, D(a.m[i]), ep, bp, rho, p, cs, b);
  double g[5];
  for (int d = 0; d < 5; d++)
    g[d] = W(L_RHO, i) * rho.d[d] + W(L_P, i) * p.d[d] + W(L_CS, i) * cs.d[d] + W(L_B, i) * b[0].d[d] +
           W(L_B + 1, i) * b[1].d[d] + W(L_B + 2, i) * b[2].d[d];
  W(L_HN, i) += g[0];
  W(L_EP, i) += g[1];
  for (int c = 0; c < 3; c++) W(L_BP + c, i) += g[2 + c];
}

// Density post reversed: lambda(h before the pass) and mu_D.
template <int DIM>
__global__ void __launch_bounds__(256) k_r_density_post(Args a) {
  using D = Dual<3>;  // h, rho_sum, dwdh
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const D h = seeded<3>(TR(T_HP, i), 0), rho = seeded<3>(TR(T_RS, i), 1), dw = seeded<3>(TR(T_DW, i), 2);
  D om, hn;
  f_density_post<DIM>(a.P.hfact, h, D(a.m[i]), rho, dw, om, hn);
  double g[3];
  for (int d = 0; d < 3; d++) g[d] = W(L_OM, i) * om.d[d] + W(L_HN, i) * hn.d[d];
  W(L_HP, i) += g[0];
  W(M_D, i) = g[1];
  W(M_D + 1, i) = g[2];
}

// Density pair terms reversed (gather form).
template <int K, int DIM>
__global__ void __launch_bounds__(kTile) k_r_density_pair(Args a) {
  using D = Dual<4>;  // x_ij 3, h_i
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  const double* HP = a.tape + (size_t)T_HP * n;
  const int kk = k < n ? k : 0;
  double gx[3] = {}, gh = 0.0;
  a_pairs<DIM>(a, k, [&](int j, double dx, double dy, double dz) {
    for (int side = 0; side < 2; side++) {
      const int ii = side ? j : kk, jj = side ? kk : j;
      const double sgn = side ? -1.0 : 1.0;
      const D xij[3] = {seeded<4>(sgn * dx, 0), seeded<4>(sgn * dy, 1), seeded<4>(sgn * dz, 2)};
      const D hi = seeded<4>(HP[ii], side ? -1 : 3);
      D rho(0.0), dw(0.0);
      f_density_pair<K, DIM>(a.P.norm, xij, hi, D(a.m[jj]), rho, dw);
      for (int c = 0; c < 3; c++) gx[c] += sgn * (W(M_D, ii) * rho.d[c] + W(M_D + 1, ii) * dw.d[c]);
      if (!side) gh += W(M_D, ii) * rho.d[3] + W(M_D + 1, ii) * dw.d[3];
    }
  });
  if (k >= n) return;
  for (int c = 0; c < 3; c++) slice_part(a, 4, c, k) = gx[c];
  slice_part(a, 4, 3, k) = gh;
}

__global__ void __launch_bounds__(256) k_r_density_sum(Args a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  for (int c = 0; c < 3; c++) W(L_X + c, k) += slices_sum(a, 4, c, k);
  W(L_HP, k) += slices_sum(a, 4, 3, k);
}

// initialize + stage1 + wrap reversed: lambda(S_n).
__global__ void __launch_bounds__(64) k_r_predict(Args a) {
  using D = Dual<NS>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const StepState<D> s = state_at<D>(a.tape + (size_t)T_S * a.n, a.n, i, 0);
  Predicted<D> o;
  f_predict(a.P, s, a.itype[i] == 1, a.dt, o);
  for (int d = 0; d < NS; d++) {
    double g = 0.0;
    for (int c = 0; c < 3; c++)
      g += W(L_X + c, i) * o.x[c].d[d] + W(L_VH + c, i) * o.vhalf[c].d[d] + W(L_VP + c, i) * o.vpred[c].d[d] +
           W(L_BH + c, i) * o.bhalf[c].d[d] + W(L_BP + c, i) * o.bpred[c].d[d];
    g += W(L_EH, i) * o.ehalf.d[d] + W(L_EP, i) * o.epred.d[d] + W(L_HP, i) * o.h.d[d] + W(L_A1, i) * o.alpha1.d[d] +
         W(L_PSIH, i) * o.psihalf.d[d] + W(L_PSIP, i) * o.psipred.d[d];
    LS(d, i) += g;
  }
}

// Gather S_0 from a state's fields into the checkpoint layout.
__global__ void __launch_bounds__(256) k_pack_state(int n, MhdState s, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* f[NS] = {s.x,      s.y,      s.z,      s.u,    s.v,  s.w,  s.e,  s.h,
                         s.alpha1, s.Bevolx, s.Bevoly, s.Bevolz, s.psi, s.au, s.av, s.aw,
                         s.ae,     s.ah,     s.alphaloc, s.cs, s.aBevolx, s.aBevoly, s.aBevolz, s.apsi};
  for (int k = 0; k < NS; k++) out[(size_t)k * n + i] = f[k][i];
}

#undef TP
#undef TR
#undef SI
#undef SO
#undef LN
#undef LS
#undef W

// {x, y, z, h} of a tape's positions and one of its smoothing lengths, for
// the grid build.
template <int DIM>
__global__ void __launch_bounds__(256) k_pack_pos(int n, const double* __restrict__ X,
                                                  const double* __restrict__ H, double4* __restrict__ pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] = make_double4(X[i], X[n + i], DIM == 3 ? X[2 * n + i] : 0.0, H[i]);
}

// The grid of a tape's positions and the smoothing lengths at offset `h`.
template <int DIM>
static void grid_for(Ctx* c, Args& a, const double* tape, int h, cudaStream_t st) {
  k_pack_pos<DIM><<<(a.n + 255) / 256, 256, 0, st>>>(a.n, tape + (size_t)T_X * a.n, tape + (size_t)h * a.n,
                                                     c->pgrid.pos);
  c->launches++;
  build_pair_grid(c, c->pgrid, a.n, st);
  a.pg = c->pgrid.grid;
  a.cell_start = c->pgrid.cell_start;
  a.perm = c->pgrid.perm;
  a.pos = c->pgrid.pos;
}

template <int K, int DIM>
static void forward_step(Ctx* c, Args a, cudaStream_t st) {
  const int nb = (a.n + kTile - 1) / kTile, np = (a.n + 255) / 256;
  const dim3 sliced(nb, a.nslices);
  k_f_predict<<<np, 256, 0, st>>>(a);
  grid_for<DIM>(c, a, a.tape_w, T_HP, st);  // the density pass: predicted h
  k_f_density_pair<K, DIM><<<sliced, kTile, 0, st>>>(a);
  k_f_density<DIM><<<np, 256, 0, st>>>(a);
  k_f_prologue<DIM><<<np, 256, 0, st>>>(a);
  grid_for<DIM>(c, a, a.tape_w, T_HN, st);  // the later groups: the new h
  k_f_cd_pair<K, DIM><<<sliced, kTile, 0, st>>>(a);
  k_f_cd<<<np, 256, 0, st>>>(a);
  k_f_force_pair<K, DIM><<<sliced, kTile, 0, st>>>(a);
  k_f_force<DIM><<<nb, kTile, 0, st>>>(a);
}

template <int K, int DIM>
static void reverse_step(Ctx* c, Args a, cudaStream_t st) {
  const int nb = (a.n + kTile - 1) / kTile, np = (a.n + 255) / 256, n64 = (a.n + 63) / 64;
  const dim3 sliced(nb, a.nslices);
  k_r_correct<<<np, 256, 0, st>>>(a);
  k_r_force_post<DIM><<<n64, 64, 0, st>>>(a);
  grid_for<DIM>(c, a, a.tape, T_HN, st);
  if (a.dual_pairs)
    k_r_force_pair<K, DIM, true><<<sliced, kTile, 0, st>>>(a);
  else
    k_r_force_pair<K, DIM, false><<<sliced, kTile, 0, st>>>(a);
  k_r_force_pair_sum<<<np, 256, 0, st>>>(a);
  k_r_cd_post<<<n64, 64, 0, st>>>(a);
  if (a.dual_pairs)
    k_r_cd_pair<K, DIM, true><<<sliced, kTile, 0, st>>>(a);
  else
    k_r_cd_pair<K, DIM, false><<<sliced, kTile, 0, st>>>(a);
  k_r_cd_sum<<<np, 256, 0, st>>>(a);
  k_r_prologue<DIM><<<np, 256, 0, st>>>(a);
  k_r_density_post<DIM><<<np, 256, 0, st>>>(a);
  grid_for<DIM>(c, a, a.tape, T_HP, st);
  k_r_density_pair<K, DIM><<<sliced, kTile, 0, st>>>(a);
  k_r_density_sum<<<np, 256, 0, st>>>(a);
  k_r_predict<<<n64, 64, 0, st>>>(a);
}

#define MHD_A_DISPATCH(FN, ...)                                                                   \
  do {                                                                                            \
    const int d3 = c->P.dim == 3;                                                                 \
    switch (c->P.kernel) {                                                                        \
      case MHD_KERNEL_CUBIC: d3 ? FN<0, 3>(__VA_ARGS__) : FN<0, 2>(__VA_ARGS__); break;           \
      case MHD_KERNEL_QUINTIC: d3 ? FN<1, 3>(__VA_ARGS__) : FN<1, 2>(__VA_ARGS__); break;         \
      case MHD_KERNEL_WENDLAND_C2: d3 ? FN<2, 3>(__VA_ARGS__) : FN<2, 2>(__VA_ARGS__); break;     \
      case MHD_KERNEL_WENDLAND_C4: d3 ? FN<3, 3>(__VA_ARGS__) : FN<3, 2>(__VA_ARGS__); break;     \
      case MHD_KERNEL_WENDLAND_C6: d3 ? FN<4, 3>(__VA_ARGS__) : FN<4, 2>(__VA_ARGS__); break;     \
      case MHD_KERNEL_GAUSSIAN: d3 ? FN<5, 3>(__VA_ARGS__) : FN<5, 2>(__VA_ARGS__); break;        \
      default: d3 ? FN<6, 3>(__VA_ARGS__) : FN<6, 2>(__VA_ARGS__); break;                         \
    }                                                                                             \
  } while (0)

}  // namespace adj
}  // namespace mhd

using namespace mhd;
using namespace mhd::adj;

namespace {

#define A_FAIL(code, msg) \
  do {                    \
    c->err = (msg);       \
    return (code);        \
  } while (0)
#define A_CK(call)                                                 \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) {                                       \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return MHD_ERR_CUDA;                                         \
    }                                                              \
  } while (0)

const char* const kAdjointFields[NS] = {"x",  "y",  "z",  "u",  "v",  "w",        "e",   "h",
                                        "alpha1", "Bevolx", "Bevoly", "Bevolz", "psi", "au", "av", "aw",
                                        "ae", "ah", "alphaloc", "cs", "aBevolx", "aBevoly", "aBevolz", "apsi"};

// Workspace of the adjoint: two states, `every` tapes, the reverse
// workspace, two lambdas, the per-particle alpha_max derivative, partials.
struct AdjLayout {
  size_t state[2], tape, w, lam[2], g_amax, dta, part, slices, total;
};

AdjLayout layout(int64_t n, int every) {
  AdjLayout L;
  size_t off = 0;
  auto take = [&](size_t cnt) {
    const size_t o = off;
    off += (cnt + 31) & ~(size_t)31;
    return o;
  };
  L.state[0] = take(NS * n);
  L.state[1] = take(NS * n);
  L.tape = take((size_t)every * NT * n);
  L.w = take(NL * n);
  L.lam[0] = take(NS * n);
  L.lam[1] = take(NS * n);
  L.g_amax = take(n);
  L.dta = take(n);
  L.part = take(n / 256 + 64);
  static_assert(kFwdSums <= kSliceWidth && kForceDirs <= kSliceWidth, "slice records fit the buffer");
  L.slices = take((size_t)derivative_slices(n) * kSliceWidth * n);
  L.total = off;
  return L;
}

int check_adjoint(Ctx* c, const MhdState* s, int64_t n, int steps, const double* dts, int every, bool adaptive) {
  if (!s || !s->m || !s->itype) A_FAIL(MHD_ERR_INVALID, "state, m or itype is null");
  if (n < 1 || n > c->n_max) A_FAIL(MHD_ERR_INVALID, "n must be in [1, n_max]");
  if (c->P.iterate) A_FAIL(MHD_ERR_INVALID, "the adjoint needs the single density pass (iterate = 0)");
  if (steps < 1 || !dts) A_FAIL(MHD_ERR_INVALID, "steps must be >= 1 and dts non-null");
  if (every < 1 || every > 256) A_FAIL(MHD_ERR_INVALID, "every must be in [1, 256]");
  for (int k = 0; k < steps; k++) {
    if (adaptive && k > 0 && dts[k] < 0.0) continue;
    if (!(dts[k] >= 0.0) || !isfinite(dts[k])) A_FAIL(MHD_ERR_INVALID, "step sizes must be finite and >= 0");
  }
  const AdjLayout L = layout(n, every);
  if (c->adj_size < L.total) {
    cudaFree(c->adj_buf);
    c->adj_buf = nullptr;
    c->adj_size = 0;
    A_CK(cudaMalloc(&c->adj_buf, sizeof(double) * L.total));
    c->adj_size = L.total;
  }
  if (alloc_pair_grid(c->pgrid, c->n_max) != MHD_OK) A_FAIL(MHD_ERR_CUDA, "pair grid allocation failed");
  return MHD_OK;
}

Args base_args(Ctx* c, const MhdState* s, int64_t n, double amax) {
  Args a;
  memset(&a, 0, sizeof a);
  a.n = (int)n;
  a.P = c->P;
  a.amax = amax;
  a.m = s->m;
  a.itype = s->itype;
  a.nslices = derivative_slices(n);
  return a;
}

// Run steps [k0, k1) from `s0` with tapes (tape slot t - k0); returns the
// state buffer holding S_{k1}.  A negative dts[t + 1] is replaced by the
// adaptive rule (min dt_adapt, clipped so that time + dt <= tf).
double* run_segment(Ctx* c, Args a, const AdjLayout& L, const double* s0, int k0, int k1, double* dts, int steps,
                    double& time, cudaStream_t st) {
  double* buf = (double*)c->adj_buf;
  const double* cur = s0;
  int which = 0;
  for (int t = k0; t < k1; t++) {
    a.s_in = cur;
    a.s_out = buf + L.state[which];
    a.tape_w = buf + L.tape + (size_t)(t - k0) * NT * a.n;
    a.dt = dts[t];
    a.dta_out = buf + L.dta;
    a.slices = buf + L.slices;
    MHD_A_DISPATCH(forward_step, c, a, st);
    c->launches += 8;
    time += dts[t];
    if (t + 1 < steps && dts[t + 1] < 0.0) {
      k_min<<<1, 256, 0, st>>>(a.n, buf + L.dta, buf + L.part);
      c->launches++;
      double dmin = 0.0;
      if (cudaMemcpyAsync(&dmin, buf + L.part, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return nullptr;
      dts[t + 1] = time + dmin > c->P.tf ? c->P.tf - time : dmin;
    }
    cur = a.s_out;
    which ^= 1;
  }
  return const_cast<double*>(cur);
}

}  // namespace

extern "C" {

int mhd_adjoint_field_count(void) { return NS; }
const char* mhd_adjoint_field_name(int32_t k) { return (k >= 0 && k < NS) ? kAdjointFields[k] : nullptr; }

int mhd_adjoint_forward(void* ctx, const MhdState* s, int64_t n, int32_t steps, double* dts, int32_t every,
                        double* checkpoints, double* loss, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  int rc = check_adjoint(c, s, n, steps, dts, every, true);
  if (rc != MHD_OK) return rc;
  if (!checkpoints || !loss) A_FAIL(MHD_ERR_INVALID, "checkpoints and loss must be non-null");
  const cudaStream_t st = (cudaStream_t)stream;
  const AdjLayout L = layout(n, every);
  double* buf = (double*)c->adj_buf;
  const int np = (int)((n + 255) / 256);
  k_pack_state<<<np, 256, 0, st>>>((int)n, *s, checkpoints);
  c->launches++;
  Args a = base_args(c, s, n, c->P.alpha_max);
  const double* cur = checkpoints;
  const int nseg = (steps + every - 1) / every;
  double time = 0.0;
  for (int g = 0; g < nseg; g++) {
    const int k0 = g * every, k1 = k0 + every < steps ? k0 + every : steps;
    double* end = run_segment(c, a, L, cur, k0, k1, dts, steps, time, st);
    if (!end) A_FAIL(MHD_ERR_CUDA, "adaptive step size read-back failed");
    double* next_cp = checkpoints + (size_t)(g + 1) * NS * n;
    A_CK(cudaMemcpyAsync(next_cp, end, sizeof(double) * NS * n, cudaMemcpyDeviceToDevice, st));
    cur = next_cp;
    if (g == nseg - 1) {
      const double* last_tape = buf + L.tape + (size_t)(k1 - 1 - k0) * NT * n;
      k_f_energy<<<np, 256, 0, st>>>((int)n, c->P.mu0, s->m, cur, last_tape, buf + L.part);
      k_sum_blocks<<<1, 32, 0, st>>>(np, buf + L.part, buf + L.part + np);
      c->launches += 2;
    }
  }
  A_CK(cudaGetLastError());
  A_CK(cudaMemcpyAsync(loss, buf + L.part + np, sizeof(double), cudaMemcpyDeviceToHost, st));
  A_CK(cudaStreamSynchronize(st));
  return MHD_OK;
}

int mhd_adjoint_backward(void* ctx, const MhdState* s, int64_t n, int32_t steps, const double* dts, int32_t every,
                         const double* checkpoints, double* lambda0, double* dloss_dalpha_max, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  int rc = check_adjoint(c, s, n, steps, dts, every, false);
  if (rc != MHD_OK) return rc;
  if (!checkpoints || !lambda0 || !dloss_dalpha_max) A_FAIL(MHD_ERR_INVALID, "output pointers must be non-null");
  double* dts_w = const_cast<double*>(dts);  // all >= 0: run_segment only reads them
  const cudaStream_t st = (cudaStream_t)stream;
  const AdjLayout L = layout(n, every);
  double* buf = (double*)c->adj_buf;
  const int np = (int)((n + 255) / 256);
  A_CK(cudaMemsetAsync(buf + L.g_amax, 0, sizeof(double) * n, st));
  Args a = base_args(c, s, n, c->P.alpha_max);
  a.w = buf + L.w;
  a.g_amax = buf + L.g_amax;
  a.slices = buf + L.slices;
  {
    const char* e = getenv("MHD_ADJOINT_DUAL");
    a.dual_pairs = e && atoi(e) != 0;
  }
  double* lam_next = buf + L.lam[0];
  double* lam = buf + L.lam[1];
  const int nseg = (steps + every - 1) / every;
  for (int g = nseg - 1; g >= 0; g--) {
    const int k0 = g * every, k1 = k0 + every < steps ? k0 + every : steps;
    double time = 0.0;
    const double* s_end = run_segment(c, a, L, checkpoints + (size_t)g * NS * n, k0, k1, dts_w, steps, time, st);
    for (int t = k1 - 1; t >= k0; t--) {
      Args r = a;
      r.tape = buf + L.tape + (size_t)(t - k0) * NT * n;
      r.dt = dts[t];
      r.lam_next = lam_next;
      r.lam = lam;
      r.s_final = t == steps - 1 ? s_end : nullptr;
      if (t == steps - 1) {
        k_r_seed<<<np, 256, 0, st>>>(r);
        c->launches++;
      }
      MHD_A_DISPATCH(reverse_step, c, r, st);
      c->launches += 12;
      double* tmp = lam_next;
      lam_next = lam;
      lam = tmp;
    }
  }
  A_CK(cudaGetLastError());
  A_CK(cudaMemcpyAsync(lambda0, lam_next, sizeof(double) * NS * n, cudaMemcpyDeviceToDevice, st));
  k_sum_blocks<<<1, 32, 0, st>>>((int)n, buf + L.g_amax, buf + L.part);
  c->launches++;
  A_CK(cudaMemcpyAsync(dloss_dalpha_max, buf + L.part, sizeof(double), cudaMemcpyDeviceToHost, st));
  A_CK(cudaStreamSynchronize(st));
  return MHD_OK;
}

}  // extern "C"
