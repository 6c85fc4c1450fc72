// mhd_abi.cu -- the extern "C" entry points declared in include/mhd_b200.h.
//
// Host-side orchestration of the sm_100a kernels: context workspace, grid
// planning, the iterated density group with device-side early exit, and the
// PEC step order.  No C++ exception crosses the ABI; every entry point
// returns MHD_OK or a negative MHD_ERR_* code.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "mhd_b200.h"
#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

double kernel_norm(int kernel, int dim) {
  const double pi = M_PI;
  switch (kernel) {
    case MHD_KERNEL_CUBIC: return dim == 2 ? 10.0 / (7.0 * pi) : 1.0 / pi;
    case MHD_KERNEL_QUINTIC: return dim == 2 ? 7.0 / (478.0 * pi) : 1.0 / (120.0 * pi);
    case MHD_KERNEL_WENDLAND_C2: return dim == 2 ? 7.0 / (4.0 * pi) : 21.0 / (16.0 * pi);
    case MHD_KERNEL_WENDLAND_C4: return dim == 2 ? 9.0 / (4.0 * pi) : 495.0 / (256.0 * pi);
    case MHD_KERNEL_WENDLAND_C6: return dim == 2 ? 78.0 / (28.0 * pi) : 1365.0 / (512.0 * pi);
    default: return dim == 2 ? 1.0 / pi : 1.0 / (pi * sqrt(pi));
  }
}

}  // namespace mhd

using namespace mhd;

namespace {
thread_local std::string g_err;
}  // namespace

void mhd::set_library_error(const std::string& msg) { g_err = msg; }

namespace {

const char* const kFieldNames[] = {
#define MHD_NAME_(n) #n,
    MHD_STATE_REQUIRED(MHD_NAME_) MHD_STATE_OPTIONAL(MHD_NAME_)
#undef MHD_NAME_
    "itype"};
constexpr int kFieldCount = sizeof(kFieldNames) / sizeof(kFieldNames[0]);

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return MHD_ERR_CUDA;                                                         \
    }                                                                              \
  } while (0)

#define FAIL(code, msg)  \
  do {                   \
    c->err = (msg);      \
    return (code);       \
  } while (0)

int fill_params(Ctx* c, const MhdParams* p) {
  if (!p) FAIL(MHD_ERR_INVALID, "params is null");
  if (p->dim != 2 && p->dim != 3) FAIL(MHD_ERR_INVALID, "dim must be 2 or 3");
  if (p->kernel < 0 || p->kernel > 6) FAIL(MHD_ERR_INVALID, "unknown kernel id");
  if (!(p->hfact > 0.0)) FAIL(MHD_ERR_INVALID, "hfact must be > 0");
  if (!(p->gamma > 1.0)) FAIL(MHD_ERR_INVALID, "gamma must be > 1 (src/integrator.py:8)");
  if (!(p->mu0 > 0.0)) FAIL(MHD_ERR_INVALID, "mu0 must be > 0");
  if (p->max_iter < 1 || p->max_iter > 256) FAIL(MHD_ERR_INVALID, "max_iter must be in [1, 256]");
  if (p->min_iter < 0) FAIL(MHD_ERR_INVALID, "min_iter must be >= 0");
  if (p->precision != MHD_PRECISION_FP64 && p->precision != MHD_PRECISION_FP32)
    FAIL(MHD_ERR_INVALID, "unknown precision");
  for (int a = 0; a < 3; a++)
    if (p->periodic[a] && a < p->dim && !(p->hi[a] > p->lo[a])) FAIL(MHD_ERR_INVALID, "periodic box has hi <= lo");
  c->params = *p;
  DevParams& P = c->P;
  memset(&P, 0, sizeof P);
  P.dim = p->dim;
  P.kernel = p->kernel;
  P.iterate = p->iterate ? 1 : 0;
  P.min_iter = p->iterate ? p->min_iter : 0;
  P.max_iter = p->iterate ? p->max_iter : 1;
  for (int a = 0; a < 3; a++) {
    P.periodic[a] = (a < p->dim && p->periodic[a]) ? 1 : 0;
    P.lo[a] = p->lo[a];
    P.hi[a] = p->hi[a];
    P.L[a] = p->hi[a] - p->lo[a];
    P.half[a] = 0.5 * P.L[a];
  }
  P.R = radius_scale_of(p->kernel);
  P.hfact = p->hfact;
  P.gamma = p->gamma;
  P.gamma1 = p->gamma - 1.0;
  P.mu0 = p->mu0;
  P.inv_mu0 = 1.0 / p->mu0;
  P.av = p->av;
  P.ac = p->ac;
  P.ar = p->ar;
  P.clean_speed = p->clean_speed;
  P.clean_damp = p->clean_damp;
  P.clean_active = p->clean_speed > 0.0 ? 1.0 : 0.0;
  P.c_cour = p->timestep_factor * kCourantFactor;
  P.c_force = p->timestep_factor * kForceFactor;
  P.alpha_min = p->alpha_min;
  P.alpha_max = p->alpha_max;
  P.tf = p->tf;
  P.norm = kernel_norm(p->kernel, p->dim);
  P.fp32 = p->precision == MHD_PRECISION_FP32 ? 1 : 0;
  return MHD_OK;
}

bool check_state(Ctx* c, const MhdState* s, bool integrator_copies) {
  if (!s) {
    c->err = "state is null";
    return false;
  }
#define MHD_REQ_(n)                                    \
  if (!s->n) {                                         \
    c->err = "required state field '" #n "' is null"; \
    return false;                                      \
  }
  MHD_STATE_REQUIRED(MHD_REQ_)
#undef MHD_REQ_
  if (!s->itype) {
    c->err = "required state field 'itype' is null";
    return false;
  }
  if (integrator_copies) {
#define MHD_REQ_(n)                                                                   \
  if (!s->n) {                                                                        \
    c->err = "MHDStep.initialize/stage1 need state field '" #n "' (non-null)";        \
    return false;                                                                     \
  }
    MHD_REQ_(x0) MHD_REQ_(y0) MHD_REQ_(z0) MHD_REQ_(u0) MHD_REQ_(v0) MHD_REQ_(w0) MHD_REQ_(e0) MHD_REQ_(alpha10)
    MHD_REQ_(Bevolx0) MHD_REQ_(Bevoly0) MHD_REQ_(Bevolz0) MHD_REQ_(psi0)
#undef MHD_REQ_
  }
  return true;
}

template <class T>
int dev_alloc(Ctx* c, T** p, int64_t count) {
  CK(cudaMalloc((void**)p, sizeof(T) * (size_t)(count > 0 ? count : 1)));
  return MHD_OK;
}

// Persistent fields carried through the neighbour sort.
int build_gather(const MhdState* src, MhdState* dst, GatherSet& g) {
  int k = 0;
#define MHD_G_(n)          \
  g.src[k] = src->n;       \
  g.dst[k] = dst->n;       \
  k++;
  MHD_SORTED_FIELDS(MHD_G_)
#undef MHD_G_
  g.nf = k;
  g.isrc = src->itype;
  g.idst = dst->itype;
  return k;
}

// h_max and bounding box -> uniform grid with cells >= R * h_max * margin.
int plan_grid(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  DevScalars init;
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  init = *c->h_sc;
  init.h_max_bits = 0ULL;
  for (int a = 0; a < 3; a++) {
    init.lo_bits[a] = ~0ULL;
    init.hi_bits[a] = 0ULL;
  }
  *c->h_sc = init;
  CK(cudaMemcpyAsync(c->d_sc, c->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice, st));
  launch_reduce_hbox(c, s, n, st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const DevScalars& h = *c->h_sc;
  if (h.status != MHD_OK) FAIL(h.status, "non-finite or non-positive smoothing length");
  const double hmax = n > 0 ? dbl_unorder(h.h_max_bits) : 1.0;
  const DevParams& P = c->P;
  const double cutoff = P.R * hmax * c->grid_margin * (1.0 + c->list_margin);
  Grid g;
  memset(&g, 0, sizeof g);
  double extent[3];
  for (int a = 0; a < 3; a++) {
    if (a >= P.dim) {
      g.nc[a] = 1;
      g.lo[a] = 0.0;
      extent[a] = 1.0;
      continue;
    }
    double lo, ext;
    if (P.periodic[a]) {
      lo = P.lo[a];
      ext = P.L[a];
    } else {
      lo = n > 0 ? dbl_unorder(h.lo_bits[a]) : 0.0;
      const double hi = n > 0 ? dbl_unorder(h.hi_bits[a]) : 1.0;
      ext = (hi - lo) * (1.0 + 1e-12) + 1e-300;
    }
    if (!isfinite(lo) || !isfinite(ext)) FAIL(MHD_ERR_NONFINITE, "non-finite particle position");
    // packed cell coordinates hold 11/11/10 bits in 3-D, 16/16 in 2-D
    const double axis_max = P.dim == 3 ? (a == 2 ? 1023.0 : 2047.0) : 65535.0;
    double ncd = floor(ext * c->stencil / cutoff);
    int nc = ncd < 1.0 ? 1 : (ncd > axis_max ? (int)axis_max : (int)ncd);
    g.nc[a] = nc;
    g.lo[a] = lo;
    extent[a] = ext;
  }
  // Keep the table within 2^24 cells; coarser cells stay valid.
  const int64_t cap = (int64_t)1 << 24;
  while ((int64_t)g.nc[0] * g.nc[1] * g.nc[2] > cap) {
    int a = 0;
    for (int b = 1; b < 3; b++)
      if (g.nc[b] > g.nc[a]) a = b;
    g.nc[a] = std::max(1, (int)(g.nc[a] * 0.8));
  }
  // The stencil of +-stencil cells covers the cut-off on every axis with at
  // least 2*stencil+1 cells; smaller axes are scanned whole.
  double hplan = INFINITY;
  g.sw = c->stencil;
  for (int a = 0; a < 3; a++) {
    g.cs[a] = extent[a] / g.nc[a];
    g.csf[a] = (float)g.cs[a];
    g.inv_cs[a] = a < P.dim ? 1.0 / g.cs[a] : 0.0;
    const bool limits = a < P.dim && g.nc[a] >= 2 * g.sw + 1;
    if (limits) hplan = std::min(hplan, g.sw * g.cs[a] / (P.R * (1.0 + c->list_margin)) * (1.0 - 1e-9));
  }
  g.h_plan = hplan;
  c->list_cut = cutoff;
  g.ncells = g.nc[0] * g.nc[1] * g.nc[2];
  if ((int64_t)g.ncells + 1 > c->cell_cap) {
    if (c->cell_start) cudaFree(c->cell_start);
    c->cell_start = nullptr;
    c->cell_cap = 0;
    const int64_t want = (int64_t)g.ncells + 1 + (g.ncells >> 2);
    if (dev_alloc(c, &c->cell_start, want) != MHD_OK) return MHD_ERR_CUDA;
    c->cell_cap = want;
  }
  g.cell_base = 0;
  g.cut = cutoff;
  for (int a = 0; a < 3; a++) {
    g.periodic[a] = P.periodic[a];
    g.L[a] = P.L[a];
    g.half[a] = P.half[a];
  }
  c->grid = g;
  c->key_cells = g.ncells;
  // The stream was synchronised above, so the previous upload of the staging
  // copy has completed.
  c->h_grids[0] = g;
  CK(cudaMemcpyAsync(c->d_grids, c->h_grids, sizeof(Grid), cudaMemcpyHostToDevice, st));
  c->have_grid = true;
  return MHD_OK;
}

// Allocate (or grow) the neighbour-list storage for `cap` entries per particle.
int ensure_list_storage(Ctx* c, int cap) {
  if (cap <= c->list_cap && c->nbr_idx) return MHD_OK;
  cudaFree(c->nbr_idx);
  c->nbr_idx = nullptr;
  c->list_cap = 0;
  if (dev_alloc(c, &c->nbr_idx, c->n_pad * (int64_t)cap) != MHD_OK) return MHD_ERR_CUDA;
  c->list_cap = cap;
  return MHD_OK;
}

// Sort src into dst, carry the previous accelerations into au_prev and build
// the neighbour lists of the sorted particles.
int sort_into(Ctx* c, const MhdState* src, MhdState* dst, int n, cudaStream_t st) {
  {
    TimedScope ts(c, MHD_TIMING_CELLS, st);
    launch_sort_cells(c, src, n, st);
    GatherSet g;
    memset(&g, 0, sizeof g);
    build_gather(src, dst, g);
    launch_gather(c, g, n, st);
    GatherSet a;
    memset(&a, 0, sizeof a);
    a.src[0] = src->au;
    a.src[1] = src->av;
    a.src[2] = src->aw;
    a.dst[0] = c->au_prev;
    a.dst[1] = c->av_prev;
    a.dst[2] = c->aw_prev;
    a.nf = 3;
    launch_gather(c, a, n, st);
  }
  launch_pack_positions(c, dst, n, st);
  launch_build_lists(c, dst, n, st);
  c->lists_checked = false;
  CK(cudaGetLastError());
  return MHD_OK;
}

// Re-sort `s` in place for a grid planned from its current h and rebuild
// the lists (an h outgrew its list during the density iteration).  Uses the
// context's spare buffers.
int resort_in_place(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  int rc = plan_grid(c, s, n, st);
  if (rc != MHD_OK) return rc;
  {
    TimedScope ts(c, MHD_TIMING_CELLS, st);
    launch_sort_cells(c, s, n, st);
    GatherSet g;
    memset(&g, 0, sizeof g);
    build_gather(s, s, g);
    const int nf = g.nf;
    // au_prev & co. ride along.
    g.src[nf] = c->au_prev;
    g.src[nf + 1] = c->av_prev;
    g.src[nf + 2] = c->aw_prev;
    double* home[kGatherMax];
    for (int f = 0; f < nf; f++) home[f] = g.dst[f];
    home[nf] = c->au_prev;
    home[nf + 1] = c->av_prev;
    home[nf + 2] = c->aw_prev;
    g.nf = nf + 3;
    for (int f = 0; f < g.nf; f++) {
      if (!c->spare[f] && dev_alloc(c, &c->spare[f], c->n_max) != MHD_OK) return MHD_ERR_CUDA;
      g.dst[f] = c->spare[f];
    }
    int32_t* itmp = (int32_t*)c->keys[c->sorted_keys == c->keys[0] ? 1 : 0];
    g.idst = itmp;
    launch_gather(c, g, n, st);
    for (int f = 0; f < g.nf; f++)
      CK(cudaMemcpyAsync(home[f], c->spare[f], sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->itype, itmp, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
  }
  launch_pack_positions(c, s, n, st);
  launch_build_lists(c, s, n, st);
  c->lists_checked = false;
  CK(cudaGetLastError());
  return MHD_OK;
}

// React to a raised `relist` (h_sc must hold a fresh copy of the device
// scalars): grow the list capacity after an overflow, then re-plan, re-sort
// and rebuild.
int relist(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  const int need = c->h_sc->list_max;
  if (need > c->list_cap) {
    int rc = ensure_list_storage(c, ((need + need / 4) + 7) & ~7);
    if (rc != MHD_OK) return rc;
  }
  CK(cudaMemsetAsync(&c->d_sc->relist, 0, 2 * sizeof(int), st));  // relist, list_max
  return resort_in_place(c, s, n, st);
}

// Synchronise and make sure the lists cover the current h of `s`.
int ensure_lists(Ctx* c, MhdState* s, int n, cudaStream_t st, int* rebuilds) {
  for (int tries = 0; tries < 16; tries++) {
    CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!c->h_sc->relist) {
      c->lists_checked = true;
      return MHD_OK;
    }
    int rc = relist(c, s, n, st);
    if (rc != MHD_OK) return rc;
    if (rebuilds) (*rebuilds)++;
  }
  FAIL(MHD_ERR_CAPACITY, "neighbour lists rebuilt too often");
}

int density_iterate(Ctx* c, MhdState* s, int n, MhdRhsStats* stats, cudaStream_t st) {
  if (!c->have_grid) FAIL(MHD_ERR_INVALID, "mhd_cells_build must precede the density iteration");
  const DevParams& P = c->P;
  if (n == 0) {
    if (stats) stats->density_passes = 0;
    return MHD_OK;
  }
  // reset pass counters (a relist raised by the list build stays raised)
  {
    DevScalars* d = c->d_sc;
    CK(cudaMemsetAsync(&d->n_unconverged[0], 0, sizeof(d->n_unconverged), st));
    CK(cudaMemsetAsync(&d->passes_done, 0, sizeof(int), st));
  }
  double* buf[2] = {s->h, c->h_alt};
  int pass = 0, rebuilds = 0, chunk = std::min(4, P.max_iter);
  int64_t unconv = 0;
  for (;;) {
    for (int k = pass; k < pass + chunk && k < P.max_iter; k++)
      launch_density_pass(c, s, n, k, buf[k & 1], buf[(k + 1) & 1], st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const DevScalars& h = *c->h_sc;
    const int done = h.passes_done;
    const bool stopped =
        done >= P.max_iter || (!P.iterate && done > 0) || (done >= P.min_iter && done > 0 && h.n_unconverged[done - 1] == 0);
    unconv = done > 0 ? h.n_unconverged[done - 1] : 0;
    if (h.relist) {
      // bring the latest h home, re-sort and rebuild the lists for it, go on
      if (done & 1) CK(cudaMemcpyAsync(s->h, c->h_alt, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      int rc = relist(c, s, n, st);
      if (rc != MHD_OK) return rc;
      CK(cudaMemcpyAsync(c->h_alt, s->h, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      rebuilds++;
      if (rebuilds > 64) FAIL(MHD_ERR_CAPACITY, "neighbour lists rebuilt too often");
      if (stopped) {
        rc = ensure_lists(c, s, n, st, &rebuilds);
        if (rc != MHD_OK) return rc;
        break;
      }
      pass = done;
      continue;
    }
    if (stopped) {
      if (done & 1) CK(cudaMemcpyAsync(s->h, c->h_alt, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      c->lists_checked = true;
      break;
    }
    if (done <= pass) FAIL(MHD_ERR_CUDA, "density pass made no progress");
    pass = done;
    chunk = std::min(chunk * 2, 32);
  }
  if (stats) {
    stats->density_passes = c->h_sc->passes_done;
    stats->grid_rebuilds += rebuilds;
    stats->n_unconverged = unconv;
    stats->n_cells = c->grid.ncells;
  }
  return MHD_OK;
}

int force_pass(Ctx* c, MhdState* s, int n, cudaStream_t st) {
  if (!c->have_grid) FAIL(MHD_ERR_INVALID, "mhd_cells_build must precede the force pass");
  if (!c->lists_checked) {
    int rc = ensure_lists(c, s, n, st, nullptr);
    if (rc != MHD_OK) return rc;
  }
  launch_force_prologue(c, s, n, st);
  launch_force_pass(c, s, n, st);
  CK(cudaGetLastError());
  return MHD_OK;
}

int read_status(Ctx* c, cudaStream_t st) {
  CK(cudaMemcpyAsync(&c->h_sc->status, &c->d_sc->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (c->h_sc->status != MHD_OK) {
    const int code = c->h_sc->status;
    CK(cudaMemsetAsync(&c->d_sc->status, 0, sizeof(int), st));
    FAIL(code, "device reported a non-finite value (timestep or smoothing length)");
  }
  return MHD_OK;
}

inline cudaStream_t S(void* stream) { return (cudaStream_t)stream; }

}  // namespace

// =========================================================================
extern "C" {

int mhd_abi_version(void) { return MHD_ABI_VERSION; }
int mhd_state_field_count(void) { return kFieldCount; }
const char* mhd_state_field_name(int32_t i) { return (i >= 0 && i < kFieldCount) ? kFieldNames[i] : nullptr; }

static const char* const kSortedNames[] = {
#define MHD_NAME_(n) #n,
    MHD_SORTED_FIELDS(MHD_NAME_)
#undef MHD_NAME_
    "itype"};
int mhd_sorted_field_count(void) { return (int)(sizeof(kSortedNames) / sizeof(kSortedNames[0])); }
const char* mhd_sorted_field_name(int32_t i) {
  return (i >= 0 && i < mhd_sorted_field_count()) ? kSortedNames[i] : nullptr;
}

int mhd_ctx_create(const MhdParams* params, int64_t n_max, void** out) {
  if (!out) return MHD_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    g_err = "no CUDA device";
    return MHD_ERR_NO_DEVICE;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  if (prop.major != 10) {
    g_err = std::string("this library is built for sm_100a; device is ") + prop.name;
    return MHD_ERR_NO_DEVICE;
  }
  if (n_max < 0 || n_max > ((int64_t)1 << 31) - 4096) {
    g_err = "n_max out of range";
    return MHD_ERR_INVALID;
  }
  Ctx* c = new Ctx();
  c->device = dev;
  c->n_max = n_max;
  int rc = fill_params(c, params);
  if (rc != MHD_OK) {
    g_err = c->err;
    delete c;
    return rc;
  }
  const int64_t N = n_max > 0 ? n_max : 1;
  const int sb = max_sort_blocks(N);
  bool ok = dev_alloc(c, &c->keys[0], N) == MHD_OK && dev_alloc(c, &c->keys[1], N) == MHD_OK &&
            dev_alloc(c, &c->vals[0], N) == MHD_OK && dev_alloc(c, &c->vals[1], N) == MHD_OK &&
            dev_alloc(c, &c->hist, (int64_t)256 * sb) == MHD_OK &&
            dev_alloc(c, &c->scan_sums, scan_sums_needed(N)) == MHD_OK && dev_alloc(c, &c->h_alt, N) == MHD_OK &&
            dev_alloc(c, &c->au_prev, N) == MHD_OK && dev_alloc(c, &c->av_prev, N) == MHD_OK &&
            dev_alloc(c, &c->aw_prev, N) == MHD_OK && dev_alloc(c, &c->d_sc, 1) == MHD_OK;
  for (int k = 0; k < 7 && ok; k++) {
    double* p = nullptr;
    ok = dev_alloc(c, &p, 4 * ((N + 31) / 32 * 32)) == MHD_OK;
    if (k == 0) c->rec_pos = p;
    else c->rec[k - 1] = p;
  }
  c->n_pad = (N + 31) / 32 * 32;
  {
    const double rr = radius_scale_of(params->kernel) * params->hfact * (1.0 + c->list_margin);
    const double vol = params->dim == 3 ? 4.0 / 3.0 * M_PI * rr * rr * rr : M_PI * rr * rr;
    const int cap = ((int)(1.5 * vol) + 16 + 7) & ~7;
    ok = ok && dev_alloc(c, &c->posf, c->n_pad) == MHD_OK && dev_alloc(c, &c->cellc, c->n_pad) == MHD_OK;
    ok = ok && dev_alloc(c, &c->nbr_cnt, c->n_pad) == MHD_OK && dev_alloc(c, &c->nbr_hlim, c->n_pad) == MHD_OK &&
         ensure_list_storage(c, cap) == MHD_OK;
  }
  if (ok && cudaMallocHost((void**)&c->h_sc, sizeof(DevScalars)) != cudaSuccess) ok = false;
  ok = ok && dev_alloc(c, &c->d_grids, 1) == MHD_OK;
  if (ok && cudaMallocHost((void**)&c->h_grids, sizeof(Grid)) != cudaSuccess) ok = false;
  if (ok) c->grid_slots = 1;
  if (!ok) {
    g_err = c->err.empty() ? "workspace allocation failed" : c->err;
    mhd_ctx_destroy(c);
    return MHD_ERR_CUDA;
  }
  memset(c->h_sc, 0, sizeof(DevScalars));
  c->h_sc->dt_min_bits = ~0ULL;
  if (cudaMemcpy(c->d_sc, c->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice) != cudaSuccess) {
    g_err = "workspace initialisation failed";
    mhd_ctx_destroy(c);
    return MHD_ERR_CUDA;
  }
  if (const char* m = getenv("MHD_GRID_MARGIN")) c->grid_margin = std::max(1.0, atof(m));
  if (const char* m = getenv("MHD_FORCE_SHAPE")) c->force_shape = std::max(0, std::min(3, atoi(m)));
  if (const char* m = getenv("MHD_STENCIL")) c->stencil = std::max(1, std::min(3, atoi(m)));
  *out = c;
  return MHD_OK;
}

int mhd_ctx_destroy(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_OK;
  cudaFree(c->keys[0]);
  cudaFree(c->keys[1]);
  cudaFree(c->vals[0]);
  cudaFree(c->vals[1]);
  cudaFree(c->hist);
  cudaFree(c->scan_sums);
  cudaFree(c->cell_start);
  cudaFree(c->h_alt);
  cudaFree(c->au_prev);
  cudaFree(c->av_prev);
  cudaFree(c->aw_prev);
  cudaFree(c->rec_pos);
  for (void* p : c->rec) cudaFree(p);
  cudaFree(c->posf);
  cudaFree(c->cellc);
  cudaFree(c->nbr_idx);
  cudaFree(c->nbr_cnt);
  cudaFree(c->nbr_hlim);
  for (double* p : c->spare) cudaFree(p);
  for (auto& e : c->events) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  cudaFree(c->d_sc);
  if (c->h_sc) cudaFreeHost(c->h_sc);
  cudaFree(c->d_grids);
  if (c->h_grids) cudaFreeHost(c->h_grids);
  cudaFree(c->inst);
  delete c;
  return MHD_OK;
}

int mhd_ctx_set_params(void* ctx, const MhdParams* params) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  return fill_params(c, params);
}

const char* mhd_last_error(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  return c ? c->err.c_str() : g_err.c_str();
}

int64_t mhd_launch_count(void* ctx) { return ctx ? ((Ctx*)ctx)->launches : 0; }

int mhd_timing_enable(void* ctx, int32_t enable) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  c->timing = enable != 0;
  return MHD_OK;
}

int mhd_timing_read(void* ctx, double* ms, int64_t* launches) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !ms || !launches) return MHD_ERR_INVALID;
  for (int k = 0; k < MHD_TIMING_KINDS; k++) {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  for (size_t e = 0; e < c->events_used; e++) {
    CK(cudaEventSynchronize(c->events[e].b));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->events[e].a, c->events[e].b));
    ms[c->events[e].kind] += t;
    launches[c->events[e].kind] += 1;
  }
  c->events_used = 0;
  return MHD_OK;
}

int mhd_probe_fma_peak(int32_t precision, double* flops_per_second, void* stream) {
  if (!flops_per_second) return MHD_ERR_INVALID;
  return probe_fma_peak(precision, flops_per_second, S(stream));
}

int mhd_pair_counts(void* ctx, int64_t* pairs, int64_t* candidates, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  const cudaStream_t st = S(stream);
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (pairs) *pairs = (int64_t)c->h_sc->n_pairs;
  if (candidates) *candidates = (int64_t)c->h_sc->n_candidates;
  CK(cudaMemsetAsync(&c->d_sc->n_pairs, 0, 2 * sizeof(unsigned long long), st));
  return MHD_OK;
}

int mhd_neighbour_counts(void* ctx, MhdState* s, int64_t n, int32_t* counts, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!counts || !check_state(c, s, false)) FAIL(MHD_ERR_INVALID, "counts or state is null");
  if (!c->have_grid) FAIL(MHD_ERR_INVALID, "mhd_cells_build must precede mhd_neighbour_counts");
  const cudaStream_t st = S(stream);
  int rc = ensure_lists(c, s, (int)n, st, nullptr);
  if (rc != MHD_OK) return rc;
  launch_neighbour_counts(c, s, (int)n, counts, st);
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_cells_build(void* ctx, const MhdState* src, MhdState* dst, int64_t n, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, src, false) || !check_state(c, dst, false)) return MHD_ERR_INVALID;
  if (src->x == dst->x) FAIL(MHD_ERR_INVALID, "src and dst must not alias");
  const cudaStream_t st = S(stream);
  int rc = plan_grid(c, src, (int)n, st);
  if (rc != MHD_OK) return rc;
  return sort_into(c, src, dst, (int)n, st);
}

int mhd_density_iterate(void* ctx, MhdState* s, int64_t n, MhdRhsStats* stats, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, s, false)) return MHD_ERR_INVALID;
  return density_iterate(c, s, (int)n, stats, S(stream));
}

int mhd_force_pass(void* ctx, MhdState* s, int64_t n, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, s, false)) return MHD_ERR_INVALID;
  return force_pass(c, s, (int)n, S(stream));
}

int mhd_rhs(void* ctx, const MhdState* src, MhdState* dst, int64_t n, MhdRhsStats* stats, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (stats) memset(stats, 0, sizeof *stats);
  int rc = mhd_cells_build(ctx, src, dst, n, stream);
  if (rc != MHD_OK) return rc;
  if (stats) stats->grid_rebuilds = 1;
  rc = density_iterate(c, dst, (int)n, stats, S(stream));
  if (rc != MHD_OK) return rc;
  return force_pass(c, dst, (int)n, S(stream));
}

int mhd_timestep(void* ctx, const MhdState* s, int64_t n, double t, double* dt_host, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 1 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n must be in [1, n_max]");
  if (!s || !s->dt_adapt) FAIL(MHD_ERR_INVALID, "dt_adapt is null");
  const cudaStream_t st = S(stream);
  launch_dt_reduce(c, s, (int)n, t, st);
  CK(cudaGetLastError());
  if (dt_host) {
    CK(cudaMemcpyAsync(&c->h_sc->dt_next, &c->d_sc->dt_next, sizeof(double), cudaMemcpyDeviceToHost, st));
    int rc = read_status(c, st);
    if (rc != MHD_OK) return rc;
    *dt_host = c->h_sc->dt_next;
  }
  return MHD_OK;
}

int mhd_clock_set(void* ctx, double t, double dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  launch_clock_set(c, t, dt, S(stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_clock_get(void* ctx, double* t, double* dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  const cudaStream_t st = S(stream);
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (t) *t = c->h_sc->t;
  if (dt) *dt = c->h_sc->dt;
  if (c->h_sc->status != MHD_OK) return read_status(c, st);
  return MHD_OK;
}

int mhd_step_initialize(void* ctx, MhdState* s, int64_t n, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, s, true)) return MHD_ERR_INVALID;
  launch_stage(c, s, (int)n, 0, 0.0, S(stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_step_stage1(void* ctx, MhdState* s, int64_t n, double dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, s, true)) return MHD_ERR_INVALID;
  launch_stage(c, s, (int)n, 1, dt, S(stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_step_stage2(void* ctx, MhdState* s, int64_t n, double dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (!check_state(c, s, false)) return MHD_ERR_INVALID;
  launch_stage(c, s, (int)n, 2, dt, S(stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_corrector_predictor(void* ctx, MhdState* s, int64_t n, int32_t mode, double dt_cur, double dt_next,
                            void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 0 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n exceeds the context's n_max");
  if (mode < 1 || mode > 3) FAIL(MHD_ERR_INVALID, "mode must be 1, 2 or 3");
  if (!check_state(c, s, false)) return MHD_ERR_INVALID;
  launch_corrector_predictor(c, s, (int)n, mode, dt_cur, dt_next, S(stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_step(void* ctx, MhdState* src, MhdState* dst, int64_t n, double dt, MhdRhsStats* stats, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  const cudaStream_t st = S(stream);
  if (dt < 0.0) {
    double t = 0.0;
    int rc = mhd_clock_get(ctx, &t, &dt, stream);
    if (rc != MHD_OK) return rc;
  }
  int rc = mhd_step_initialize(ctx, src, n, stream);
  if (rc != MHD_OK) return rc;
  rc = mhd_step_stage1(ctx, src, n, dt, stream);
  if (rc != MHD_OK) return rc;
  rc = mhd_rhs(ctx, src, dst, n, stats, stream);
  if (rc != MHD_OK) return rc;
  rc = mhd_step_stage2(ctx, dst, n, dt, stream);
  if (rc != MHD_OK) return rc;
  (void)st;
  return MHD_OK;
}

}  // extern "C"
