// mhd_pairs.cu -- density pass and neighbour lists of the SPMHD right-hand
// side (sm_100a).
//
// k_density_pass: one pass of DensityIteration (src/equations.py:14-94) --
//   pair sums rho = sum m W(h_i), dwdh = sum m dW/dh(h_i), then the Newton
//   update of h with the [0.8h, 1.2h] clip and the convergence test, one
//   thread per particle of the cell-sorted order, h read from one buffer and
//   written to another (Jacobi semantics of PySPH's post_loop).
// k_build_lists & co.: the compacted neighbour lists every pair pass reads
//   (PySPH's NNPS, src/application.py:63-78), carried across sorts where
//   they stay valid.
// The fused force pass (groups G2-G10) is in mhd_force.cu.
#include <cuda_runtime.h>

#include <climits>

#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

// FP64 sum, or a Kahan-compensated FP32 sum.
template <class T>
struct SumT {
  T s = 0;
  __device__ __forceinline__ void add(T v) { s += v; }
  __device__ __forceinline__ double get() const { return (double)s; }
};
template <>
struct SumT<float> {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float y = __fsub_rn(v, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  __device__ __forceinline__ double get() const { return (double)s - (double)c; }
};

// ------------------------------------------------------------ density pass
// One particle of a density pass; returns whether it is still unconverged.
template <int K, int DIM, class T>
__device__ __forceinline__ bool density_particle(int i, const DevParams& P, const NbrList& L,
                                                 const double* __restrict__ x, const double* __restrict__ y,
                                                 const double* __restrict__ z, const double* __restrict__ m,
                                                 const double* __restrict__ h_in, double* __restrict__ h_out,
                                                 const double* __restrict__ h0, double* __restrict__ rho_sum,
                                                 double* __restrict__ omega, double* __restrict__ converged,
                                                 const Grid* __restrict__ grids, const int* __restrict__ inst,
                                                 const uint4* __restrict__ posq, DevScalars* sc) {
  const double hi = h_in[i];
  if (converged[i] == 1.0) {
    // Already finalised: its h is frozen; a re-summation would only refresh
    // the unconsumed rho_sum diagnostic (src/equations.py:117).
    h_out[i] = hi;
    return false;
  }
  const Grid& G = grid_of(grids, inst, i);
  const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
  const T h1 = (T)(1.0 / hi);
  const T fac = (T)P.norm * (DIM == 2 ? h1 * h1 : h1 * h1 * h1);
  const T fgh = -fac * h1;
  const double rhi2 = rh2_exact(P.R, hi);
  constexpr bool compact = K <= MHD_KERNEL_WENDLAND_C6;
  SumT<T> rs, ds;
  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  // FP32 form: geometry and mass from the packed {x, y, z fixed point, m}
  // records; FP64: exact geometry.
  uint4 piq = make_uint4(0u, 0u, 0u, 0u);
  float rhi2f = 0.f;
  if constexpr (sizeof(T) == 4) {
    piq = posq[i];
    const float rh = (float)P.R * (float)hi;
    rhi2f = rh * rh;
  }
  // the list entry is fetched one pair ahead, so a pair waits on one memory
  // round trip (its record) instead of two
  int jn = cnt > 0 ? row[0] : i;
  for (int k = 0; k < cnt; k++) {
    const int j = jn;
    if (k + 1 < cnt) jn = row[(k + 1) * 32];
    T r, mj;
    bool nb;
    if constexpr (sizeof(T) == 4) {
      const uint4 pj = __ldg(posq + j);
      mj = __uint_as_float(pj.w);
      const float dx = fixed_delta(G, 0, piq.x, pj.x);
      const float dy = fixed_delta(G, 1, piq.y, pj.y);
      const float dz = DIM == 3 ? fixed_delta(G, 2, piq.z, pj.z) : 0.f;
      const float r2 = dx * dx + dy * dy + dz * dz;
      nb = r2 < rhi2f;
      if (!compact && !nb) {
        const float rh = (float)P.R * (float)h_in[j];
        nb = r2 < rh * rh;
      }
      r = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
    } else {
      mj = m[j];  // requested with the position, before the neighbour test
      const double dx = min_image(xi - x[j], G.L[0], G.half[0], G.periodic[0]);
      const double dy = min_image(yi - y[j], G.L[1], G.half[1], G.periodic[1]);
      const double dz = DIM == 3 ? min_image(zi - z[j], G.L[2], G.half[2], G.periodic[2]) : 0.0;
      const double r2 = r2_exact(dx, dy, dz);
      // For compact kernels a pair admitted only by R*h_j has W(h_i) = 0 and
      // dW/dh(h_i) = 0, so the h_i test alone gives the same sums.
      nb = r2 < rhi2;
      if (!compact && !nb) nb = r2 < rh2_exact(P.R, h_in[j]);
      r = nb ? sqrt(r2) : 0.0;
    }
    if (nb) {
      const T q = r * h1;
      T w, dw;
      w_dw<K>(q, DIM, w, dw);
      rs.add(mj * (w * fac));
      ds.add(mj * (fgh * (dw * q + w * (T)DIM)));
    }
  }
  // post_loop (src/equations.py:53-86), FP64
  const double rsum = rs.get(), dsum = ds.get();
  const double mi = m[i];
  const double rhoi = mi / pow_dim<DIM>(hi / P.hfact);
  const double dhdrhoi = -hi / ((double)DIM * rhoi);
  const double omegai = 1.0 - dhdrhoi * dsum;
  omega[i] = 1.0 / omegai;
  const double func = rhoi - rsum;
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
  } else {
    hout = P.hfact * pow(mi / rsum, 1.0 / (double)DIM);
    converged[i] = 1.0;
  }
  h_out[i] = hout;
  rho_sum[i] = rsum;
  // The lists hold every j within R * max(h_i, h_j) of the h they were built
  // with, enlarged by the list margin; a larger h needs new lists.
  if (!(hout <= L.hlim[i])) atomicExch(&sc->relist, 1);
  return !finalize;
}

// A density pass over all particles, grid-stride (a pass after the group
// stopped returns at once).
template <int K, int DIM, class T>
__global__ void __launch_bounds__(128) k_density_pass(int n, int pass, DevParams P, NbrList L,
                                                      const double* __restrict__ x, const double* __restrict__ y,
                                                      const double* __restrict__ z, const double* __restrict__ m,
                                                      const double* __restrict__ h_in, double* __restrict__ h_out,
                                                      const double* __restrict__ h0, double* __restrict__ rho_sum,
                                                      double* __restrict__ omega, double* __restrict__ converged,
                                                      const Grid* __restrict__ grids, const int* __restrict__ inst,
                                                      const uint4* __restrict__ posq, DevScalars* sc) {
  // pass < 0: the body of the captured density loop -- the pass index comes
  // from the device, and the h buffers alternate with its parity
  if (pass < 0) {
    pass = sc->loop_pass;
    if (pass & 1) {
      double* a = const_cast<double*>(h_in);
      h_in = h_out;
      h_out = a;
    }
  }
  // Stop when the iterated group already stopped after pass `pass` (1-based
  // count), or when the neighbour lists no longer cover the current h.
  if (sc->relist) return;
  if (pass > 0) {
    const bool stop = !P.iterate || pass >= P.max_iter || (pass >= P.min_iter && sc->n_unconverged[pass - 1] == 0);
    if (stop) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&sc->passes_done, pass + 1);
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const bool unconv = density_particle<K, DIM, T>(i, P, L, x, y, z, m, h_in, h_out, h0, rho_sum, omega,
                                                    converged, grids, inst, posq, sc);
    const unsigned act = __activemask();
    const unsigned b = __ballot_sync(act, unconv);
    if (b && (int)(threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(&sc->n_unconverged[pass], __popc(b));
  }
}

// ----------------------------------------- density pass with diagnostics
// The density-pass outputs that no later equation reads (src/equations.py:
// 24-50, 80-86): rho_sum, arho (scaled by the new omega when a particle is
// finalised), grhox/y/z and dwdh.  Written when the caller passes any of the
// arrays.  As in the reference every particle is summed in every pass --
// converged ones too, with their frozen h -- so after the group these hold
// the last pass's sums; the post-loop (Newton update, convergence test) runs
// for unconverged particles only and is the fast pass's, op for op, so h,
// omega and converged do not depend on whether diagnostics are written.
// Pair arithmetic is FP64 in both precision forms.
struct DensityDiag {
  double *arho, *grhox, *grhoy, *grhoz, *dwdh;
  const double *upred, *vpred, *wpred;
};

template <int K, int DIM>
__global__ void __launch_bounds__(128) k_density_pass_diag(int n, int pass, DevParams P, NbrList L,
                                                           const double* __restrict__ x, const double* __restrict__ y,
                                                           const double* __restrict__ z, const double* __restrict__ m,
                                                           const double* __restrict__ h_in, double* __restrict__ h_out,
                                                           const double* __restrict__ h0,
                                                           double* __restrict__ rho_sum, double* __restrict__ omega,
                                                           double* __restrict__ converged,
                                                           const Grid* __restrict__ grids, const int* __restrict__ inst,
                                                           DensityDiag D, DevScalars* sc) {
  if (sc->relist) return;
  if (pass > 0) {
    const bool stop = !P.iterate || pass >= P.max_iter || (pass >= P.min_iter && sc->n_unconverged[pass - 1] == 0);
    if (stop) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&sc->passes_done, pass + 1);
  const int stride = gridDim.x * blockDim.x;
  constexpr bool compact = K <= MHD_KERNEL_WENDLAND_C6;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double hi = h_in[i];
    const Grid& G = grid_of(grids, inst, i);
    const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
    const double h1 = 1.0 / hi;
    const double fac = P.norm * (DIM == 2 ? h1 * h1 : h1 * h1 * h1);
    const double fgh = -fac * h1;
    const double rhi2 = rh2_exact(P.R, hi);
    const double ui = D.upred[i], vi = D.vpred[i], wi = D.wpred[i];
    double rsum = 0.0, dsum = 0.0, ar = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    const int cnt = L.cnt[i];
    const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
    for (int k = 0; k < cnt; k++) {
      const int j = row[k * 32];
      const double dx = min_image(xi - x[j], G.L[0], G.half[0], G.periodic[0]);
      const double dy = min_image(yi - y[j], G.L[1], G.half[1], G.periodic[1]);
      const double dz = DIM == 3 ? min_image(zi - z[j], G.L[2], G.half[2], G.periodic[2]) : 0.0;
      const double r2 = r2_exact(dx, dy, dz);
      bool nb = r2 < rhi2;
      if (!compact && !nb) nb = r2 < rh2_exact(P.R, h_in[j]);
      if (!nb) continue;
      const double r = sqrt(r2);
      const double mj = m[j];
      const double q = r * h1;
      double w, dw;
      w_dw<K>(q, DIM, w, dw);
      // DWI = fac dw h1 / r * XIJ (zero at r <= 1e-12), GHI = -fac h1 (dw q + d w)
      const double t = r > kPairDistanceEpsilon ? fac * dw * h1 / r : 0.0;
      const double dwx = t * dx, dwy = t * dy, dwz = t * dz;
      const double vdw = (ui - D.upred[j]) * dwx + (vi - D.vpred[j]) * dwy + (wi - D.wpred[j]) * dwz;
      rsum += mj * (w * fac);
      ar += mj * vdw;
      gx += mj * dwx;
      gy += mj * dwy;
      gz += mj * dwz;
      dsum += mj * (fgh * (dw * q + w * (double)DIM));
    }
    bool unconv = false;
    if (converged[i] != 1.0) {
      // post_loop (src/equations.py:53-86), as in density_particle
      const double mi = m[i];
      const double rhoi = mi / pow_dim<DIM>(hi / P.hfact);
      const double dhdrhoi = -hi / ((double)DIM * rhoi);
      const double omegai = 1.0 - dhdrhoi * dsum;
      const double om = 1.0 / omegai;
      omega[i] = om;
      const double func = rhoi - rsum;
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
        unconv = true;
      } else {
        ar *= om;
        hout = P.hfact * pow(mi / rsum, 1.0 / (double)DIM);
        converged[i] = 1.0;
      }
      h_out[i] = hout;
      if (!(hout <= L.hlim[i])) atomicExch(&sc->relist, 1);
    } else {
      h_out[i] = hi;
    }
    rho_sum[i] = rsum;
    if (D.arho) D.arho[i] = ar;
    if (D.grhox) D.grhox[i] = gx;
    if (D.grhoy) D.grhoy[i] = gy;
    if (D.grhoz) D.grhoz[i] = gz;
    if (D.dwdh) D.dwdh[i] = dsum;
    const unsigned act = __activemask();
    const unsigned b = __ballot_sync(act, unconv);
    if (b && (int)(threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(&sc->n_unconverged[pass], __popc(b));
  }
}

// ------------------------------------------------------- neighbour lists
// A list holds every j within the margin-enlarged symmetric radius
// R * max(h_i, h_j) * (1 + margin) of the h it was built with.  The tests run
// in FP32 on the packed positions with a relative slack of 4e-6 on r^2 (FP32
// geometry errors are ~1e-7), and a list is declared valid only up to
// h_i * (1 + margin) * (1 - 1e-4): every pair the exact FP64 criterion admits
// while each h stays within its limit is in the list.  Three passes: gather
// (each particle's own search), scatter (big particles add themselves where
// a smaller search cannot reach them), ordering of the scattered entries.

// Grid of the big-particle passes (a grid-stride loop over the big
// particles, one warp each): up to 16 blocks of 4 warps per multiprocessor,
// enough for every big particle of a step to start at once (a big
// particle's search is a chain of dependent row lookups, so these passes
// are bound by latency, not by issue).
static int big_blocks(const Ctx* c, int n) {
  const int want = (n + 3) / 4;
  const int cap = c->num_sms * 16;
  return want < 1 ? 1 : (want < cap ? want : cap);
}

// FP32 squared distance from the packed positions, rounded op by op so that
// it is the same whichever particle of the pair computes it.
template <int DIM>
__device__ __forceinline__ float sym_r2(const Grid& G, const float4& pa, int ca, const float4& pb, int cb) {
  float dx, dy, dz;
  rel_dx<DIM>(G, pa, ca, pb, cb, dx, dy, dz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// (Rg * h)^2 * slack, rounded op by op.
__device__ __forceinline__ float reach2(float Rg, float h, float slack) {
  const float rh = __fmul_rn(Rg, h);
  return __fmul_rn(__fmul_rn(rh, rh), slack);
}

// Search half-width and cut-off of a particle: the grid's for a normal
// particle, its own R * h * (1 + margin) for a big one.
__device__ __forceinline__ void search_extent(const Grid& G, int dim, float Rg, float h, bool big, int& sw,
                                              double& cut) {
  sw = G.sw;
  cut = G.cut * (1.0 + 1e-6);
  if (!big) return;
  cut = (double)Rg * (double)h * (1.0 + 1e-5);
  for (int a = 0; a < dim; a++) {
    const int s = (int)ceil(cut * G.inv_cs[a]);
    sw = s > sw ? s : sw;
  }
}

// Gather pass: every particle lists the j it finds in its own search.  A
// normal particle searches the grid's +-sw stencil and keeps every normal j
// with r < R * max(h_i, h_j) * (1 + margin); big j are left to the scatter
// pass.  A big particle searches its own extended stencil and keeps normal j
// under the same rule and big j within its own R * h_i * (1 + margin).
// Positions are the packed FP32 cell-relative ones: per cell the particle's
// position is shifted by the cell offset, so a candidate costs one float4
// load.  Counts beyond `cap` are recorded, not stored, and flag a rebuild
// with a larger capacity.
constexpr int kGatherUnroll = 4;
// (a carried build runs this over a few percent of the particles: few blocks
// have work, so the registers the unrolled loads take cost no occupancy that
// matters)
template <int DIM>
__global__ void __launch_bounds__(128, 2) k_build_lists(int n, DevParams P, const Grid* __restrict__ grids,
                                                     const int* __restrict__ inst, const int* __restrict__ cell_start,
                                                     const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ z, const double* __restrict__ h,
                                                     const float4* __restrict__ posf, const int* __restrict__ cellc,
                                                     float grow, int cap, int* __restrict__ idx,
                                                     int* __restrict__ cnt_out, int* __restrict__ gcnt_out,
                                                     double* __restrict__ hlim, int* __restrict__ big_idx,
                                                     const int* __restrict__ reb_idx, DevScalars* sc) {
  // a carried build lists the rebuilt particles only (reb_idx, in sorted
  // order within each warp's share), a full one every particle
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (reb_idx ? sc->n_reb : n)) return;
  const int i = reb_idx ? reb_idx[t] : t;
  const Grid& G = grid_of(grids, inst, i);
  const float4 pi = posf[i];
  const int ci = cellc[i];
  const float Rg = __fmul_rn((float)P.R, grow);
  const float slack = 1.0f + 4e-6f;
  const float rhi2 = reach2(Rg, pi.w, 1.0f);
  const float hbig = G.h_bigf;
  const bool big_i = pi.w > hbig;
  int sw;
  double cut;
  search_extent(G, DIM, Rg, pi.w, big_i, sw, cut);
  if (big_i) {
    // its extended search runs in k_build_lists_big, one warp per particle
    big_idx[atomicAdd(&sc->n_big, 1)] = i;
    return;
  }
  const float own2 = reach2(Rg, pi.w, slack);
  int* __restrict__ row = idx + (size_t)(i >> 5) * cap * 32 + (i & 31);
  int cnt = 0;
  int cxi, cyi, czi;
  unpack_cell<DIM>(ci, cxi, cyi, czi);
  const int whole = 2 * sw + 1;
  const bool mx = G.periodic[0] && G.nc[0] < whole, my = G.periodic[1] && G.nc[1] < whole,
             mz = DIM == 3 && G.periodic[2] && G.nc[2] < whole;
  const float Lx = (float)G.L[0], Ly = (float)G.L[1], Lz = (float)G.L[2];
  const float csx = G.csf[0], csy = G.csf[1], csz = G.csf[2];
  // One contiguous index range per stencil row piece: the x shift of a
  // candidate follows from its packed cell x and the piece's image offset.
  constexpr int xmask = DIM == 3 ? 2047 : 65535;
  for_each_row_trimmed<DIM>(G, sw, cell_start, x[i], y[i], DIM == 3 ? z[i] : 0.0, cut,
                            [&](int cyu, int czu, int jb, int je, int xoff) {
    const float sy = pi.y + (float)(cyi - cyu) * csy;
    const float sz = DIM == 3 ? pi.z + (float)(czi - czu) * csz : 0.f;
    const int cxo = cxi - xoff;
    auto test = [&](int j, const float4& pj, int cj) {
      const float sx = pi.x + (float)(cxo - (cj & xmask)) * csx;
      bool keep;
      if (pj.w > hbig) {
        // big j: kept here only by a big i, within i's own reach (the
        // scatter pass adds it everywhere else)
        keep = big_i && sym_r2<DIM>(G, pi, ci, pj, cj) < own2;
      } else {
        float dx = sx - pj.x, dy = sy - pj.y, dz = DIM == 3 ? sz - pj.z : 0.f;
        if (mx) dx = dx > 0.5f * Lx ? dx - Lx : (dx < -0.5f * Lx ? dx + Lx : dx);
        if (my) dy = dy > 0.5f * Ly ? dy - Ly : (dy < -0.5f * Ly ? dy + Ly : dy);
        if (mz) dz = dz > 0.5f * Lz ? dz - Lz : (dz < -0.5f * Lz ? dz + Lz : dz);
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rhj = Rg * pj.w;
        keep = r2 < fmaxf(rhi2, rhj * rhj) * slack;
      }
      if (keep) {
        if (cnt < cap) row[cnt * 32] = j;
        cnt++;
      }
    };
    // kGatherUnroll candidates at a time, every record of a group requested
    // before the first test (a thread's candidates are a chain of L1/L2 round
    // trips otherwise)
    int j = jb;
    for (; j + kGatherUnroll <= je; j += kGatherUnroll) {
      float4 pq[kGatherUnroll];
      int cq[kGatherUnroll];
#pragma unroll
      for (int u = 0; u < kGatherUnroll; u++) {
        pq[u] = __ldg(posf + j + u);
        cq[u] = __ldg(cellc + j + u);
      }
#pragma unroll
      for (int u = 0; u < kGatherUnroll; u++) test(j + u, pq[u], cq[u]);
    }
    for (; j < je; j++) test(j, __ldg(posf + j), __ldg(cellc + j));
  });
  const int stored = cnt < cap ? cnt : cap;
  cnt_out[i] = stored;
  gcnt_out[i] = stored;
  hlim[i] = h[i] * (double)grow * (1.0 - 1e-4);
  if (cnt > cap) {
    atomicMax(&sc->list_max, cnt);
    atomicExch(&sc->relist, 1);
  }
}

// Scatter pass: every big particle j searches its extended stencil and
// appends itself to the list of each i with r < R * h_j * (1 + margin) that
// did not keep j in its own gather pass (every normal i; a big i only beyond
// its own reach).  The test is the gather pass's, from the other side, with
// the same op-by-op rounding, so each pair is listed exactly once.
template <int DIM>
__global__ void __launch_bounds__(128) k_scatter_big(DevParams P, const Grid* __restrict__ grids,
                                                     const int* __restrict__ inst, const int* __restrict__ cell_start,
                                                     const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ z, const float4* __restrict__ posf,
                                                     const int* __restrict__ cellc, float grow, int cap,
                                                     int* __restrict__ idx, int* __restrict__ cnt,
                                                     const int* __restrict__ big_idx, const int* __restrict__ mark,
                                                     const int* __restrict__ gcnt, int* __restrict__ app_idx,
                                                     DevScalars* sc) {
  // one warp per big particle: the lanes take consecutive candidates
  const int nb = sc->n_big, lane = threadIdx.x & 31;
  const float Rg = __fmul_rn((float)P.R, grow);
  const float slack = 1.0f + 4e-6f;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nb; t += nwarps) {
    const int j = big_idx[t];
    const Grid& G = grid_of(grids, inst, j);
    const float4 pj = posf[j];
    const int cj = cellc[j];
    const float hbig = G.h_bigf;
    const float reach_j = reach2(Rg, pj.w, slack);
    int sw;
    double cut;
    search_extent(G, DIM, Rg, pj.w, true, sw, cut);
    // the extended stencil's rows looked up 32 at a time, candidates 32 at
    // a time (the appends land in atomic order; the ordering pass sorts them)
    warp_rows<DIM>(G, sw, cell_start, x[j], y[j], DIM == 3 ? z[j] : 0.0, cut, [&](int i, int, int, int) {
      if (i < 0 || i == j) return;
      const float4 pi = __ldg(posf + i);
      const float r2 = sym_r2<DIM>(G, pi, __ldg(cellc + i), pj, cj);
      if (!(r2 < reach_j)) return;
      if (pi.w > hbig && r2 < reach2(Rg, pi.w, slack)) return;  // i kept j itself
      int* __restrict__ irow = idx + (size_t)(i >> 5) * cap * 32 + (i & 31);
      if (mark && !mark[i]) {
        // a carried-over list may hold j already (its appended entries of
        // this build start after gcnt)
        const int g = gcnt[i];
        bool held = false;
        for (int e = 0; e < g && !held; e++) held = irow[(size_t)e * 32] == j;
        if (held) return;
      }
      const int slot = atomicAdd(cnt + i, 1);
      // the first entry appended to i's list enrols i for the ordering pass
      if (slot == __ldg(gcnt + i)) app_idx[atomicAdd(&sc->n_app, 1)] = i;
      if (slot < cap) {
        irow[(size_t)slot * 32] = j;
      } else {
        atomicMax(&sc->list_max, slot + 1);
        atomicExch(&sc->relist, 1);
      }
    });
  }
}

// Gather pass of the big particles, one warp per particle: the lanes test
// consecutive candidates of each row piece and append the kept ones in
// candidate order (ballot prefix), so the list is what a single thread
// scanning the extended stencil would write.
template <int DIM>
__global__ void __launch_bounds__(128) k_build_lists_big(DevParams P, const Grid* __restrict__ grids,
                                                         const int* __restrict__ inst,
                                                         const int* __restrict__ cell_start,
                                                         const double* __restrict__ x, const double* __restrict__ y,
                                                         const double* __restrict__ z, const double* __restrict__ h,
                                                         const float4* __restrict__ posf,
                                                         const int* __restrict__ cellc, float grow, int cap,
                                                         int* __restrict__ idx, int* __restrict__ cnt_out,
                                                         int* __restrict__ gcnt_out, double* __restrict__ hlim,
                                                         const int* __restrict__ big_idx, DevScalars* sc) {
  const int nb = sc->n_big, lane = threadIdx.x & 31;
  const float Rg = __fmul_rn((float)P.R, grow);
  const float slack = 1.0f + 4e-6f;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  constexpr int xmask = DIM == 3 ? 2047 : 65535;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nb; t += nwarps) {
    const int i = big_idx[t];
    const Grid& G = grid_of(grids, inst, i);
    const float4 pi = posf[i];
    const int ci = cellc[i];
    const float rhi2 = reach2(Rg, pi.w, 1.0f), own2 = reach2(Rg, pi.w, slack);
    const float hbig = G.h_bigf;
    int sw;
    double cut;
    search_extent(G, DIM, Rg, pi.w, true, sw, cut);
    int cxi, cyi, czi;
    unpack_cell<DIM>(ci, cxi, cyi, czi);
    const int whole = 2 * sw + 1;
    const bool mx = G.periodic[0] && G.nc[0] < whole, my = G.periodic[1] && G.nc[1] < whole,
               mz = DIM == 3 && G.periodic[2] && G.nc[2] < whole;
    const float Lx = (float)G.L[0], Ly = (float)G.L[1], Lz = (float)G.L[2];
    const float csx = G.csf[0], csy = G.csf[1], csz = G.csf[2];
    int* __restrict__ row = idx + (size_t)(i >> 5) * cap * 32 + (i & 31);
    int cnt = 0;
    // the extended stencil's rows looked up 32 at a time (a big particle's
    // search has up to (2 sw + 1)^2 rows), candidates 32 at a time
    warp_rows<DIM>(G, sw, cell_start, x[i], y[i], DIM == 3 ? z[i] : 0.0, cut, [&](int j, int cyu, int czu, int xoff) {
      bool keep = false;
      if (j >= 0) {
        const float4 pj = __ldg(posf + j);
        const int cjj = __ldg(cellc + j);
        if (pj.w > hbig) {
          keep = sym_r2<DIM>(G, pi, ci, pj, cjj) < own2;
        } else {
          const float sy = pi.y + (float)(cyi - cyu) * csy;
          const float sz = DIM == 3 ? pi.z + (float)(czi - czu) * csz : 0.f;
          const int cxo = cxi - xoff;
          const float sx = pi.x + (float)(cxo - (cjj & xmask)) * csx;
          float dx = sx - pj.x, dy = sy - pj.y, dz = DIM == 3 ? sz - pj.z : 0.f;
          if (mx) dx = dx > 0.5f * Lx ? dx - Lx : (dx < -0.5f * Lx ? dx + Lx : dx);
          if (my) dy = dy > 0.5f * Ly ? dy - Ly : (dy < -0.5f * Ly ? dy + Ly : dy);
          if (mz) dz = dz > 0.5f * Lz ? dz - Lz : (dz < -0.5f * Lz ? dz + Lz : dz);
          const float r2 = dx * dx + dy * dy + dz * dz;
          const float rhj = Rg * pj.w;
          keep = r2 < fmaxf(rhi2, rhj * rhj) * slack;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (pos < cap) row[pos * 32] = j;
      }
      cnt += __popc(bal);
    });
    if (lane == 0) {
      const int stored = cnt < cap ? cnt : cap;
      cnt_out[i] = stored;
      gcnt_out[i] = stored;
      hlim[i] = h[i] * (double)grow * (1.0 - 1e-4);
      if (cnt > cap) {
        atomicMax(&sc->list_max, cnt);
        atomicExch(&sc->relist, 1);
      }
    }
  }
}

// Order the scattered entries of every list by index (the scatter pass
// appends them in whatever order its atomics resolve) and cap the counts.
// One warp per particle the scatter pass enrolled: up to 32 appended entries
// are sorted across the lanes by a bitonic network (one entry per lane,
// padded with INT_MAX), up to 32 kRankRegs by rank (each entry's position is
// the count of smaller entries), longer runs, rare, by one lane's insertion
// sort.
constexpr int kRankRegs = 8;
__global__ void __launch_bounds__(128) k_sort_appended(int cap, int* __restrict__ idx, int* __restrict__ cnt,
                                                       const int* __restrict__ gcnt,
                                                       const int* __restrict__ app_idx,
                                                       const DevScalars* __restrict__ sc) {
  const int na = sc->n_app, lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < na; t += nwarps) {
    const int i = app_idx[t];
    int c = cnt[i];
    if (c > cap) c = cap;
    __syncwarp();
    if (lane == 0) cnt[i] = c;
    const int g = gcnt[i];
    const int m = c - g;
    if (m < 2) continue;
    int* __restrict__ row = idx + (size_t)(i >> 5) * cap * 32 + (i & 31);
    if (m <= 32) {
      int v = lane < m ? row[(size_t)(g + lane) * 32] : INT_MAX;
#pragma unroll
      for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
          const int o = __shfl_xor_sync(0xffffffffu, v, j);
          const bool ascending = (lane & k) == 0, lower = (lane & j) == 0;
          v = (lower == ascending) ? min(v, o) : max(v, o);
        }
      }
      if (lane < m) row[(size_t)(g + lane) * 32] = v;
    } else if (m <= 32 * kRankRegs) {
      // up to 32 kRankRegs entries: each lane holds kRankRegs of them, every
      // entry's rank is the count of entries before it in (value, position)
      // order, counted against all entries passed round the warp
      int v[kRankRegs], rank[kRankRegs];
#pragma unroll
      for (int r = 0; r < kRankRegs; r++) {
        const int e = r * 32 + lane;
        v[r] = e < m ? row[(size_t)(g + e) * 32] : INT_MAX;
        rank[r] = 0;
      }
      for (int r2 = 0; r2 < kRankRegs && r2 * 32 < m; r2++)
        for (int src = 0; src < 32; src++) {
          const int o = __shfl_sync(0xffffffffu, v[r2], src);
          const int op = r2 * 32 + src;
#pragma unroll
          for (int r = 0; r < kRankRegs; r++) rank[r] += (o < v[r] || (o == v[r] && op < r * 32 + lane)) ? 1 : 0;
        }
      __syncwarp();
#pragma unroll
      for (int r = 0; r < kRankRegs; r++)
        if (r * 32 + lane < m) row[(size_t)(g + rank[r]) * 32] = v[r];
    } else if (lane == 0) {
      for (int a = g + 1; a < c; a++) {
        const int v = row[(size_t)a * 32];
        int b = a - 1;
        while (b >= g && row[(size_t)b * 32] > v) {
          row[(size_t)(b + 1) * 32] = row[(size_t)b * 32];
          b--;
        }
        row[(size_t)(b + 1) * 32] = v;
      }
    }
  }
}

// ------------------------------------------------- lists across sorts
// A list built at time t_b holds every j with r(t_b) < R (1 + margin)
// (1 - 1e-4) max(h_i(t_b), h_j(t_b)).  Every particle k keeps an epoch: a
// reference position xr_k, md_k = the largest |x_k - xr_k| seen since, and
// hm_k = the smallest h_k seen since (h at the start of each right-hand
// side).  Any particle moved by at most 2 md since any time of its epoch, so
// a pair absent from a list has r(now) >= R (1 + margin)(1 - 1e-4) hm - 4 D,
// D the largest md of the two, and the list stays valid while
//   h_k <= hlim_k = (1 + margin)(1 - 1e-4) hm_k - 4 D_k / R
// for every k, D_k the largest md in the cells within sw + 1 of k's cell
// (every partner within reach, one cell of slack).  A particle failing the
// test (with a quarter of the margin as headroom for the coming density
// iteration), and every big particle, is dirty: it starts a new epoch, and
// every list within sw + 1 cells of it is rebuilt, so no list built before
// that epoch can lack it while it is in reach.  Big particles (rebuilt every
// time) append themselves to carried-over lists that lack them.  md is also
// recorded in the cell of xr: if the state was changed behind the lists'
// back, the particle now at an index is not the one the lists name, and the
// distance between the two marks both places.

__device__ __forceinline__ int cell_key(const Grid& G, double x, double y, double z) {
  const int cx = cell_coord(G, 0, x), cy = cell_coord(G, 1, y), cz = cell_coord(G, 2, z);
  return G.cell_base + (cz * G.nc[1] + cy) * G.nc[0] + cx;
}

// Epoch bookkeeping of sorted particle k (source index o = perm[k]): xr, hm
// and md carried from the old slot and updated; md marked in the cells of x
// and xr.  With `full` every epoch starts now.
template <int DIM>
__global__ void __launch_bounds__(256) k_track(int n, int full, const Grid* __restrict__ grids,
                                               const int* __restrict__ inst, const int* __restrict__ perm,
                                               const double* __restrict__ x, const double* __restrict__ y,
                                               const double* __restrict__ z, const double* __restrict__ h,
                                               const double* __restrict__ xr_old, const double* __restrict__ hm_old,
                                               const float* __restrict__ md_old, double* __restrict__ xr_new,
                                               double* __restrict__ hm_new, float* __restrict__ md_new, int64_t pad,
                                               int* __restrict__ new_of_old, unsigned* __restrict__ cell_md,
                                               DevScalars* sc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (k == 0) {
    atomicAdd(&sc->n_listed, (unsigned long long)n);
    if (full) atomicAdd(&sc->n_rebuilt, (unsigned long long)n);
  }
  const double xk = x[k], yk = y[k], zk = DIM == 3 ? z[k] : 0.0, hk = h[k];
  if (full) {
    xr_new[k] = xk;
    xr_new[pad + k] = yk;
    xr_new[2 * pad + k] = zk;
    hm_new[k] = hk;
    md_new[k] = 0.f;
    return;
  }
  const Grid& G = grid_of(grids, inst, k);
  const int o = perm[k];
  new_of_old[o] = k;
  const double rx = xr_old[o], ry = xr_old[pad + o], rz = DIM == 3 ? xr_old[2 * pad + o] : 0.0;
  const double dx = min_image(xk - rx, G.L[0], G.half[0], G.periodic[0]);
  const double dy = min_image(yk - ry, G.L[1], G.half[1], G.periodic[1]);
  const double dz = DIM == 3 ? min_image(zk - rz, G.L[2], G.half[2], G.periodic[2]) : 0.0;
  float m = __double2float_ru(sqrt(dx * dx + dy * dy + dz * dz));
  const float mo = md_old[o];
  m = mo > m ? mo : m;
  if (!(m <= 3.0e38f)) m = INFINITY;  // non-finite: moved arbitrarily far
  const double hmo = hm_old[o];
  xr_new[k] = rx;
  xr_new[pad + k] = ry;
  xr_new[2 * pad + k] = rz;
  hm_new[k] = hmo < hk ? hmo : hk;
  md_new[k] = m;
  const unsigned bits = __float_as_uint(m);
  if (bits) {
    atomicMax(cell_md + cell_key(G, xk, yk, zk), bits);
    atomicMax(cell_md + cell_key(G, rx, ry, rz), bits);
  }
}

// out = the max of `in` over the cells within sw + 1 along one axis of each
// instance's grid (periodic wrap; an axis of at most 2 (sw + 1) + 1 cells is
// taken whole).  Values are non-negative FP32 bit patterns or flags.
__global__ void __launch_bounds__(256) k_dilate(int ncells, int n_inst, const Grid* __restrict__ grids, int axis,
                                                const unsigned* __restrict__ in, unsigned* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int lo = 0, hi = n_inst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (grids[mid].cell_base <= c) lo = mid;
    else hi = mid - 1;
  }
  const Grid& G = grids[lo];
  const int local = c - G.cell_base;
  if (local >= G.ncells) {
    out[c] = 0u;
    return;
  }
  const int nx = G.nc[0], ny = G.nc[1];
  const int coord = axis == 0 ? local % nx : (axis == 1 ? (local / nx) % ny : local / (nx * ny));
  const int stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
  const int nc = G.nc[axis], base = c - coord * stride, w = G.sw + 1;
  unsigned m = 0u;
  if (nc <= 2 * w + 1) {
    for (int t = 0; t < nc; t++) m = max(m, in[base + t * stride]);
  } else {
    for (int d = -w; d <= w; d++) {
      int t = coord + d;
      if (t < 0 || t >= nc) {
        if (!G.periodic[axis]) continue;
        t = t < 0 ? t + nc : t - nc;
      }
      m = max(m, in[base + t * stride]);
    }
  }
  out[c] = m;
}

// Dirty particles: big ones, and those whose limit leaves no headroom.
// Writes the limit (the density iteration's check) and flags the cells.
__global__ void __launch_bounds__(256) k_mark(int n, DevParams P, const Grid* __restrict__ grids,
                                              const int* __restrict__ inst, const uint32_t* __restrict__ keys,
                                              const double* __restrict__ h, const float4* __restrict__ posf,
                                              const double* __restrict__ hm, const unsigned* __restrict__ cell_md,
                                              double grow1, double headroom, double* __restrict__ hlim,
                                              int* __restrict__ mark, unsigned* __restrict__ cell_dirty) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const Grid& G = grid_of(grids, inst, k);
  const uint32_t key = keys[k];
  const double D = (double)__uint_as_float(cell_md[key]);
  const double lim = grow1 * hm[k] - 4.0 * D / P.R;
  const bool dirty = posf[k].w > G.h_bigf || !(h[k] * headroom <= lim);
  hlim[k] = lim;
  mark[k] = dirty ? 1 : 0;
  if (dirty) cell_dirty[key] = 1u;
}

// Carry the clean lists over (entry j of the source order becomes
// new_of_old[j]); a dirty particle starts a new epoch; mark becomes "rebuild"
// for dirty particles and every particle within sw + 1 cells of one.
__global__ void __launch_bounds__(256) k_remap(int n, int cap, const int* __restrict__ perm,
                                               const uint32_t* __restrict__ keys, const int* __restrict__ new_of_old,
                                               const unsigned* __restrict__ cell_dirty, int* __restrict__ mark,
                                               const double* __restrict__ x, const double* __restrict__ y,
                                               const double* __restrict__ z, const double* __restrict__ h,
                                               double* __restrict__ xr_new, double* __restrict__ hm_new,
                                               float* __restrict__ md_new, int64_t pad,
                                               const int* __restrict__ idx_old, const int* __restrict__ cnt_old,
                                               int* __restrict__ idx_new, int* __restrict__ cnt_new,
                                               int* __restrict__ gcnt_new, int* __restrict__ reb_idx,
                                               DevScalars* sc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool rebuild = false;
  if (k < n) {
    const int dirty = mark[k];
    if (dirty) {
      xr_new[k] = x[k];
      xr_new[pad + k] = y[k];
      xr_new[2 * pad + k] = z[k];
      hm_new[k] = h[k];
      md_new[k] = 0.f;
    }
    rebuild = dirty || cell_dirty[keys[k]] != 0u;
    mark[k] = rebuild ? 1 : 0;
  }
  {
    // the gather pass runs over the rebuilt particles only: each warp enrols
    // its rebuilt lanes in lane order with one atomic
    const unsigned b = __ballot_sync(0xffffffffu, rebuild);
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0 && b) base = atomicAdd(&sc->n_reb, __popc(b));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (rebuild) reb_idx[base + __popc(b & ((1u << lane) - 1u))] = k;
  }
  const int nr = __syncthreads_count(rebuild);
  if (threadIdx.x == 0 && nr) atomicAdd(&sc->n_rebuilt, (unsigned long long)nr);
  if (k >= n || rebuild) return;
  const int o = perm[k];
  int c = cnt_old[o];
  c = c < cap ? c : cap;
  const int* __restrict__ src = idx_old + (size_t)(o >> 5) * cap * 32 + (o & 31);
  int* __restrict__ dst = idx_new + (size_t)(k >> 5) * cap * 32 + (k & 31);
  for (int e = 0; e < c; e++) dst[(size_t)e * 32] = new_of_old[src[(size_t)e * 32]];
  cnt_new[k] = c;
  gcnt_new[k] = c;
}

// Neighbours of each particle under the exact FP64 rule of the oracle
// (r2 < (R h_i)^2 or r2 < (R h_j)^2, self included), counted over its list.
template <int DIM>
__global__ void __launch_bounds__(128) k_neighbour_counts(int n, DevParams P, const Grid* __restrict__ grids,
                                                          const int* __restrict__ inst, NbrList L,
                                                          const double* __restrict__ x, const double* __restrict__ y,
                                                          const double* __restrict__ z, const double* __restrict__ h,
                                                          int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& G = grid_of(grids, inst, i);
  const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
  const double rhi2 = rh2_exact(P.R, h[i]);
  const int cnt = L.cnt[i];
  const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
  int nb = 0;
  for (int k = 0; k < cnt; k++) {
    const int j = row[k * 32];
    const double dx = min_image(xi - x[j], G.L[0], G.half[0], G.periodic[0]);
    const double dy = min_image(yi - y[j], G.L[1], G.half[1], G.periodic[1]);
    const double dz = DIM == 3 ? min_image(zi - z[j], G.L[2], G.half[2], G.periodic[2]) : 0.0;
    const double r2 = r2_exact(dx, dy, dz);
    nb += (r2 < rhi2 || r2 < rh2_exact(P.R, h[j])) ? 1 : 0;
  }
  out[i] = nb;
}

// Pairs under the exact rule and list entries, summed over the particles
// (one atomic pair per block).
template <int DIM>
__global__ void __launch_bounds__(256) k_pair_stats(int n, DevParams P, const Grid* __restrict__ grids,
                                                    const int* __restrict__ inst, NbrList L,
                                                    const double* __restrict__ x, const double* __restrict__ y,
                                                    const double* __restrict__ z, const double* __restrict__ h,
                                                    DevScalars* sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned nb = 0, cnt = 0;
  if (i < n) {
    const Grid& G = grid_of(grids, inst, i);
    const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
    const double rhi2 = rh2_exact(P.R, h[i]);
    cnt = (unsigned)L.cnt[i];
    const int* __restrict__ row = L.idx + (size_t)(i >> 5) * L.cap * 32 + (i & 31);
    for (unsigned k = 0; k < cnt; k++) {
      const int j = row[(size_t)k * 32];
      const double dx = min_image(xi - x[j], G.L[0], G.half[0], G.periodic[0]);
      const double dy = min_image(yi - y[j], G.L[1], G.half[1], G.periodic[1]);
      const double dz = DIM == 3 ? min_image(zi - z[j], G.L[2], G.half[2], G.periodic[2]) : 0.0;
      const double r2 = r2_exact(dx, dy, dz);
      nb += (r2 < rhi2 || r2 < rh2_exact(P.R, h[j])) ? 1u : 0u;
    }
  }
  __shared__ unsigned long long acc[2];
  if (threadIdx.x == 0) acc[0] = acc[1] = 0ULL;
  __syncthreads();
  atomicAdd(&acc[0], (unsigned long long)nb);
  atomicAdd(&acc[1], (unsigned long long)cnt);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&sc->n_pairs, acc[0]);
    atomicAdd(&sc->n_candidates, acc[1]);
  }
}

void launch_pair_stats(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  if (c->P.dim == 3)
    k_pair_stats<3><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, c->d_grids, c->inst, c->lists(), s->x, s->y, s->z,
                                                     s->h, c->d_sc);
  else
    k_pair_stats<2><<<(n + 255) / 256, 256, 0, st>>>(n, c->P, c->d_grids, c->inst, c->lists(), s->x, s->y, s->z,
                                                     s->h, c->d_sc);
  c->launches++;
}

void launch_neighbour_counts(Ctx* c, const MhdState* s, int n, int* out, cudaStream_t st) {
  if (n <= 0) return;
  if (c->P.dim == 3)
    k_neighbour_counts<3><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->d_grids, c->inst, c->lists(), s->x, s->y,
                                                           s->z, s->h, out);
  else
    k_neighbour_counts<2><<<(n + 127) / 128, 128, 0, st>>>(n, c->P, c->d_grids, c->inst, c->lists(), s->x, s->y,
                                                           s->z, s->h, out);
  c->launches++;
}

// Max of a per-cell array over the cells within sw + 1 of each cell, one
// axis at a time between `in` and `tmp`; returns the buffer holding it.
static unsigned* dilate_cells(Ctx* c, unsigned* in, unsigned* tmp, cudaStream_t st) {
  const int nb = (c->key_cells + 255) / 256;
  for (int a = 0; a < c->P.dim; a++) {
    k_dilate<<<nb, 256, 0, st>>>(c->key_cells, c->n_inst, c->d_grids, a, in, tmp);
    unsigned* t = in;
    in = tmp;
    tmp = t;
  }
  c->launches += c->P.dim;
  return in;
}

template <int DIM>
static void build_lists_dim(Ctx* c, const MhdState* s, int n, cudaStream_t st, const Ctx::ListSlot* O,
                            Ctx::ListSlot& S) {
  const float grow = (float)(1.0 + c->list_margin);
  const int nb = (n + 127) / 128, nb256 = (n + 255) / 256;
  const int64_t pad = c->n_pad;
  const bool full = O == nullptr;
  int* mark = nullptr;
  if (!full) cudaMemsetAsync(c->cell_scr[0], 0, sizeof(unsigned) * c->key_cells, st);
  k_track<DIM><<<nb256, 256, 0, st>>>(n, full ? 1 : 0, c->d_grids, c->inst, c->perm, s->x, s->y, s->z, s->h,
                                      full ? nullptr : O->xr, full ? nullptr : O->hm, full ? nullptr : O->md, S.xr,
                                      S.hm, S.md, pad, c->new_of_old, c->cell_scr[0], c->d_sc);
  c->launches++;
  if (!full) {
    unsigned* md_dil = dilate_cells(c, c->cell_scr[0], c->cell_scr[1], st);
    unsigned* flags = md_dil == c->cell_scr[0] ? c->cell_scr[1] : c->cell_scr[0];
    cudaMemsetAsync(flags, 0, sizeof(unsigned) * c->key_cells, st);
    k_mark<<<nb256, 256, 0, st>>>(n, c->P, c->d_grids, c->inst, c->sorted_keys, s->h, c->posf, S.hm, md_dil,
                                  (double)grow * (1.0 - 1e-4), 1.0 + 0.25 * c->list_margin, c->nbr_hlim,
                                  c->nbr_mark, flags);
    unsigned* dirty_dil = dilate_cells(c, flags, md_dil, st);
    k_remap<<<nb256, 256, 0, st>>>(n, c->list_cap, c->perm, c->sorted_keys, c->new_of_old, dirty_dil, c->nbr_mark,
                                   s->x, s->y, s->z, s->h, S.xr, S.hm, S.md, pad, O->idx, O->cnt, S.idx, S.cnt,
                                   S.gcnt, c->reb_idx, c->d_sc);
    c->launches += 2;
    mark = c->nbr_mark;
  }
  k_build_lists<DIM><<<nb, 128, 0, st>>>(n, c->P, c->d_grids, c->inst, c->cell_start, s->x, s->y, s->z, s->h,
                                         c->posf, c->cellc, grow, c->list_cap, S.idx, S.cnt, S.gcnt, c->nbr_hlim,
                                         c->big_idx, mark ? c->reb_idx : nullptr, c->d_sc);
  k_build_lists_big<DIM><<<big_blocks(c, n), 128, 0, st>>>(c->P, c->d_grids, c->inst, c->cell_start, s->x, s->y,
                                                         s->z, s->h, c->posf, c->cellc, grow, c->list_cap, S.idx,
                                                         S.cnt, S.gcnt, c->nbr_hlim, c->big_idx, c->d_sc);
  k_scatter_big<DIM><<<big_blocks(c, n), 128, 0, st>>>(c->P, c->d_grids, c->inst, c->cell_start, s->x, s->y, s->z,
                                                     c->posf, c->cellc, grow, c->list_cap, S.idx, S.cnt,
                                                     c->big_idx, mark, S.gcnt, c->app_idx, c->d_sc);
  k_sort_appended<<<big_blocks(c, n), 128, 0, st>>>(c->list_cap, S.idx, S.cnt, S.gcnt, c->app_idx, c->d_sc);
  c->launches += 4;
}

void launch_build_lists(Ctx* c, const MhdState* s, int n, cudaStream_t st, const MhdState* src) {
  if (n <= 0) return;
  TimedScope ts(c, MHD_TIMING_LISTS, st);
  // the slot of s (or the least recently used one not holding src's lists)
  int nw = -1, od = -1;
  for (int k = 0; k < 2; k++) {
    if (c->slots[k].key == s->x) nw = k;
    if (src && c->slots[k].key == src->x) od = k;
  }
  if (nw < 0 || nw == od) nw = od >= 0 ? 1 - od : (c->slots[0].use <= c->slots[1].use ? 0 : 1);
  const bool carry = c->list_reuse && od >= 0 && c->slots[od].n == n && c->slots[od].layout == c->layout_gen;
  Ctx::ListSlot& S = c->slots[nw];
  S.key = nullptr;
  c->nbr_idx = S.idx;
  c->nbr_cnt = S.cnt;
  c->nbr_gcnt = S.gcnt;
  cudaMemsetAsync(&c->d_sc->n_big, 0, 3 * sizeof(int), st);  // n_big, n_app and n_reb
  if (c->P.dim == 3)
    build_lists_dim<3>(c, s, n, st, carry ? &c->slots[od] : nullptr, S);
  else
    build_lists_dim<2>(c, s, n, st, carry ? &c->slots[od] : nullptr, S);
  S.key = s->x;
  S.n = n;
  S.layout = c->layout_gen;
  S.use = ++c->slot_clock;
}

// ------------------------------------------------------------- dispatch
template <int K, int DIM>
static void density_launch(Ctx* c, MhdState* s, int n, int pass, const double* h_in, double* h_out, cudaStream_t st) {
  // Passes 0 and 1 cover the particles with one thread each; later passes,
  // which most groups skip (and which then return at once), use about one
  // wave of blocks, so a skipped pass costs little in a captured run.
  const int full = (n + 127) / 128;
  const int grid = pass < 2 ? full : std::min(full, c->num_sms * 8);
  if (s->arho || s->grhox || s->grhoy || s->grhoz || s->dwdh) {
    const DensityDiag D{s->arho, s->grhox, s->grhoy, s->grhoz, s->dwdh, s->upred, s->vpred, s->wpred};
    k_density_pass_diag<K, DIM><<<grid, 128, 0, st>>>(n, pass, c->P, c->lists(), s->x, s->y, s->z, s->m, h_in, h_out,
                                                      s->h0, s->rho_sum, s->omega, s->converged, c->d_grids, c->inst,
                                                      D, c->d_sc);
    return;
  }
  if (c->P.fp32) {
    k_density_pass<K, DIM, float><<<grid, 128, 0, st>>>(n, pass, c->P, c->lists(), s->x, s->y, s->z, s->m, h_in, h_out,
                                                        s->h0, s->rho_sum, s->omega, s->converged, c->d_grids, c->inst,
                                                        c->posq, c->d_sc);
    return;
  }
  k_density_pass<K, DIM, double><<<grid, 128, 0, st>>>(n, pass, c->P, c->lists(), s->x, s->y, s->z, s->m, h_in, h_out,
                                                       s->h0, s->rho_sum, s->omega, s->converged, c->d_grids, c->inst,
                                                       c->posq, c->d_sc);
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

// End of a captured density iteration (a fixed number of passes, each with
// the on-device stop test): the latest h is in h_alt after an odd number of
// passes; a group that had not stopped when the passes ran out raises an
// event (the run is replayed uncaptured).
__global__ void __launch_bounds__(256) k_finish_density(int n, DevParams P, int passes, double* __restrict__ h,
                                                        const double* __restrict__ h_alt, DevScalars* sc) {
  const int done = sc->passes_done;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    const bool stopped = done >= P.max_iter || (!P.iterate && done > 0) ||
                         (done >= P.min_iter && done > 0 && sc->n_unconverged[done - 1] == 0);
    if (!stopped && done >= passes) atomicOr(&sc->events, 1);
  }
  if (i < n && (done & 1)) h[i] = h_alt[i];
}

__global__ void __launch_bounds__(32) k_density_loop_control(DevParams P, DevScalars* sc,
                                                              cudaGraphConditionalHandle h, int first) {
  if (threadIdx.x != 0) return;
  const int next = first >= 0 ? first : sc->loop_pass + 1;
  sc->loop_pass = next;
  if (first < 0) sc->loop_iters++;
  const int done = sc->passes_done;
  const bool stopped = done >= P.max_iter || !P.iterate ||
                       (done >= P.min_iter && done > 0 && sc->n_unconverged[done - 1] == 0);
  const int cap = P.max_iter < kDensityLoopCap ? P.max_iter : kDensityLoopCap;
  cudaGraphSetConditional(h, (!stopped && !sc->relist && next < cap) ? 1u : 0u);
}

void launch_density_loop_control(Ctx* c, cudaGraphConditionalHandle h, int first, cudaStream_t st) {
  k_density_loop_control<<<1, 32, 0, st>>>(c->P, c->d_sc, h, first);
  c->launches++;
}

void launch_finish_density(Ctx* c, MhdState* s, int n, int passes, cudaStream_t st) {
  if (n <= 0) return;
  k_finish_density<<<(n + 255) / 256, 256, 0, st>>>(n, c->P, passes, s->h, c->h_alt, c->d_sc);
  c->launches++;
}

}  // namespace mhd
