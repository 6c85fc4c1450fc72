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
  P.Rf = (float)P.R;
  P.normf = (float)P.norm;
  P.avf = (float)P.av;
  P.acf = (float)P.ac;
  P.arf = (float)P.ar;
  P.inv_mu0f = (float)P.inv_mu0;
  P.fp32 = p->precision == MHD_PRECISION_FP32 ? 1 : 0;
  const cudaError_t e = configure_force_pass(c);
  if (e != cudaSuccess) FAIL(MHD_ERR_CUDA, std::string("force pass set-up: ") + cudaGetErrorString(e));
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

// Persistent fields carried through the neighbour sort.  With rhs_follows
// (the sort of a right-hand side, whose prologue rewrites them before
// anything reads them: DensityFromSmoothingLength, IdealGasEOS and
// MagneticStateReconstruction) rho, p, cs and B are not carried.
int build_gather(const MhdState* src, MhdState* dst, GatherSet& g, bool rhs_follows = false) {
  int k = 0;
#define MHD_G_(n)                                                                          \
  if (!(rhs_follows && (&src->n == &src->rho || &src->n == &src->p || &src->n == &src->cs || \
                        &src->n == &src->Bx || &src->n == &src->By || &src->n == &src->Bz))) { \
    g.src[k] = src->n;                                                                     \
    g.dst[k] = dst->n;                                                                     \
    k++;                                                                                   \
  }
  MHD_SORTED_FIELDS(MHD_G_)
#undef MHD_G_
  g.nf = k;
  g.isrc = src->itype;
  g.idst = dst->itype;
  return k;
}

void refresh_spec(Ctx* c) {
  PlanSpec& S = c->spec;
  const DevParams& P = c->P;
  S.dim = P.dim;
  S.stencil = c->stencil;
  for (int a = 0; a < 3; a++) {
    S.periodic[a] = P.periodic[a];
    S.lo[a] = P.lo[a];
    S.L[a] = P.L[a];
    S.half[a] = P.half[a];
  }
  S.R = P.R;
  S.grid_margin = c->grid_margin;
  S.list_margin = c->list_margin;
  S.cell_kappa = c->cell_kappa;
}

int grow_cell_table(Ctx* c, int64_t cells) {
  if (cells + 1 <= c->cell_cap) return MHD_OK;
  if (c->cell_start) cudaFree(c->cell_start);
  for (unsigned*& p : c->cell_scr) {
    cudaFree(p);
    p = nullptr;
  }
  c->cell_start = nullptr;
  c->cell_cap = 0;
  const int64_t want = cells + 1 + (cells >> 2);
  if (dev_alloc(c, &c->cell_start, want) != MHD_OK || dev_alloc(c, &c->cell_scr[0], want) != MHD_OK ||
      dev_alloc(c, &c->cell_scr[1], want) != MHD_OK)
    return MHD_ERR_CUDA;
  c->cell_cap = want;
  c->generation++;
  return MHD_OK;
}

// h_max and bounding box -> uniform grid with cells >= R * h_max * margin.
// A single simulation plans on the host (the cell table grows as needed);
// a batched context plans every instance on the device, within the cell
// capacities fixed when its instances were set, with no synchronisation.
int plan_grid(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  refresh_spec(c);
  if (c->batched) {
    launch_reduce_hbox(c, s, n, st);
    launch_plan_grids(c, st);
    CK(cudaGetLastError());
    c->have_grid = true;
    return MHD_OK;
  }
  launch_reduce_hbox(c, s, n, st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_inst, c->d_inst, sizeof(InstScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&c->h_sc->status, &c->d_sc->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  launch_reset_hbox(c, st);
  if (c->h_sc->status != MHD_OK) FAIL(c->h_sc->status, "non-finite or non-positive smoothing length");
  const InstScalars& q = *c->h_inst;
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = dbl_unorder(q.lo_bits[a]);
    hi[a] = dbl_unorder(q.hi_bits[a]);
  }
  Grid g;
  const double hmax = dbl_unorder(q.h_max_bits);
  if (plan_instance(c->spec, n, hmax, mean_h(hmax, q.h_sum, n), lo, hi, nullptr, g) != MHD_OK)
    FAIL(MHD_ERR_NONFINITE, "non-finite particle position");
  g.cell_base = 0;
  c->list_cut = g.cut;
  if (grow_cell_table(c, g.ncells) != MHD_OK) return MHD_ERR_CUDA;
  c->grid = g;
  c->key_cells = g.ncells;
  // The stream was synchronised above, so the previous upload of the staging
  // copy has completed.
  c->h_grids[0] = g;
  CK(cudaMemcpyAsync(c->d_grids, c->h_grids, sizeof(Grid), cudaMemcpyHostToDevice, st));
  c->have_grid = true;
  return MHD_OK;
}

// (Re)allocate the per-instance tables for n_inst instances whose particles
// start at start[0..n_inst] and reset their clocks and reductions.  The
// instance index array is left to the caller.
int alloc_instances(Ctx* c, int n_inst, const int64_t* start) {
  if (n_inst > c->grid_slots) {
    cudaFree(c->d_grids);
    cudaFree(c->d_inst);
    cudaFree(c->d_stage);
    if (c->h_grids) cudaFreeHost(c->h_grids);
    if (c->h_inst) cudaFreeHost(c->h_inst);
    c->d_grids = nullptr;
    c->d_inst = nullptr;
    c->d_stage = nullptr;
    c->h_grids = nullptr;
    c->h_inst = nullptr;
    c->grid_slots = 0;
    if (dev_alloc(c, &c->d_grids, n_inst) != MHD_OK || dev_alloc(c, &c->d_inst, n_inst) != MHD_OK ||
        dev_alloc(c, &c->d_stage, 2 * n_inst) != MHD_OK)
      return MHD_ERR_CUDA;
    if (cudaMallocHost((void**)&c->h_grids, sizeof(Grid) * n_inst) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_inst, sizeof(InstScalars) * n_inst) != cudaSuccess)
      FAIL(MHD_ERR_CUDA, "pinned allocation failed");
    c->grid_slots = n_inst;
    c->generation++;
  }
  for (int k = 0; k < n_inst; k++) {
    InstScalars& q = c->h_inst[k];
    memset(&q, 0, sizeof q);
    q.dt_min_bits = ~0ULL;
    q.h_max_bits = 0ULL;
    for (int a = 0; a < 3; a++) {
      q.lo_bits[a] = ~0ULL;
      q.hi_bits[a] = 0ULL;
      q.nc_cap[a] = 1;
    }
    q.n = (int)(start[k + 1] - start[k]);
  }
  CK(cudaMemcpy(c->d_inst, c->h_inst, sizeof(InstScalars) * n_inst, cudaMemcpyHostToDevice));
  c->n_inst = n_inst;
  c->inst_start.assign(start, start + n_inst + 1);
  return MHD_OK;
}

// Allocate (or grow) the neighbour-list storage for `cap` entries per particle.
int ensure_list_storage(Ctx* c, int cap) {
  if (cap <= c->list_cap && c->slots[0].idx && c->slots[1].idx) return MHD_OK;
  for (Ctx::ListSlot& S : c->slots) {
    cudaFree(S.idx);
    S.idx = nullptr;
    S.key = nullptr;  // no lists to carry over
  }
  c->nbr_idx = nullptr;
  c->list_cap = 0;
  for (Ctx::ListSlot& S : c->slots)
    if (dev_alloc(c, &S.idx, c->n_pad * (int64_t)cap) != MHD_OK) return MHD_ERR_CUDA;
  c->nbr_idx = c->slots[0].idx;
  c->list_cap = cap;
  c->generation++;
  return MHD_OK;
}

// Sort src into dst, carry the previous accelerations into au_prev and build
// the neighbour lists of the sorted particles.
int sort_into(Ctx* c, const MhdState* src, MhdState* dst, int n, cudaStream_t st, bool rhs_follows) {
  {
    TimedScope ts(c, MHD_TIMING_CELLS, st);
    launch_sort_cells(c, src, n, st);
    GatherSet g;
    memset(&g, 0, sizeof g);
    build_gather(src, dst, g, rhs_follows);
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
  launch_build_lists(c, dst, n, st, src);
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
  launch_build_lists(c, s, n, st, nullptr);
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
    stats->n_cells = c->batched ? c->key_cells : c->grid.ncells;
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

// The rest of a captured density iteration as a conditional while node:
// an arming kernel sets the loop's condition after passes [0, first), and
// the body -- one density pass whose index and h buffers come from the
// device, then the control kernel that advances the index and sets the
// condition again -- repeats until the group stops, a list needs
// rebuilding, or the passes reach min(max_iter, kDensityLoopCap).  The
// index rises by one per iteration, so the loop ends after at most
// kDensityLoopCap - first iterations whatever the particles do.
int capture_density_loop(Ctx* c, MhdState* dst, int n, int first, cudaStream_t st) {
  cudaStreamCaptureStatus status;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &nd));
  if (status != cudaStreamCaptureStatusActive) FAIL(MHD_ERR_INVALID, "the density loop needs an active capture");
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  launch_density_loop_control(c, h, first, st);
  CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, deps, nd, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if (!c->cap_stream2) CK(cudaStreamCreateWithFlags(&c->cap_stream2, cudaStreamNonBlocking));
  CK(cudaStreamBeginCaptureToGraph(c->cap_stream2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_density_pass(c, dst, n, -1, dst->h, c->h_alt, c->cap_stream2);
  launch_density_loop_control(c, h, -1, c->cap_stream2);
  // the body's launches are counted when they run (DevScalars::loop_iters)
  c->launches -= 2;
  cudaGraph_t captured = nullptr;
  const cudaError_t le = cudaGetLastError();
  const cudaError_t ee = cudaStreamEndCapture(c->cap_stream2, &captured);
  if (le != cudaSuccess || ee != cudaSuccess)
    FAIL(MHD_ERR_CUDA, std::string("density loop body capture failed: ") +
                           cudaGetErrorString(le != cudaSuccess ? le : ee));
  CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  return MHD_OK;
}

// Right-hand side with nothing that synchronises (batched contexts): device
// planning, sort and lists, the density iteration with its on-device stop
// test (its first min_iter passes as plain launches, the rest as a
// conditional while node; with MHD_GRAPH_LOOP=0 or diagnostic outputs, a
// fixed number of passes), the force pass.  Lists that stop covering an h,
// or a group that has not stopped after the captured passes, raise relist
// or an event that the caller reads after the run.
int rhs_captured(Ctx* c, const MhdState* src, MhdState* dst, int n, cudaStream_t st) {
  int rc = plan_grid(c, src, n, st);
  if (rc != MHD_OK) return rc;
  rc = sort_into(c, src, dst, n, st, true);
  if (rc != MHD_OK) return rc;
  CK(cudaMemsetAsync(&c->d_sc->n_unconverged[0], 0, sizeof(c->d_sc->n_unconverged), st));
  CK(cudaMemsetAsync(&c->d_sc->passes_done, 0, sizeof(int), st));
  double* buf[2] = {dst->h, c->h_alt};
  const bool diag = dst->arho || dst->grhox || dst->grhoy || dst->grhoz || dst->dwdh;
  const int cap = std::min(c->P.max_iter, kDensityLoopCap);
  const int first = std::min(cap, std::max(c->P.min_iter, 1));
  if (c->graph_loop && !diag && c->P.iterate && cap > first) {
    for (int k = 0; k < first; k++) launch_density_pass(c, dst, n, k, buf[k & 1], buf[(k + 1) & 1], st);
    rc = capture_density_loop(c, dst, n, first, st);
    if (rc != MHD_OK) return rc;
    launch_finish_density(c, dst, n, cap, st);
  } else {
    const int passes = std::min(c->P.max_iter, c->graph_passes);
    for (int k = 0; k < passes; k++) launch_density_pass(c, dst, n, k, buf[k & 1], buf[(k + 1) & 1], st);
    launch_finish_density(c, dst, n, passes, st);
  }
  launch_force_prologue(c, dst, n, st);
  launch_force_pass(c, dst, n, st);
  CK(cudaGetLastError());
  return MHD_OK;
}

// One fused step on the device clocks: the right-hand side from cur into
// nxt, the per-instance timestep, the corrector-predictor on nxt.
int step_fused(Ctx* c, const MhdState* cur, MhdState* nxt, int n, int mode, bool captured, cudaStream_t st) {
  int rc;
  if (captured) {
    rc = rhs_captured(c, cur, nxt, n, st);
  } else {
    rc = plan_grid(c, cur, n, st);
    if (rc == MHD_OK) rc = sort_into(c, cur, nxt, n, st, true);
    if (rc == MHD_OK) rc = density_iterate(c, nxt, n, nullptr, st);
    if (rc == MHD_OK) rc = force_pass(c, nxt, n, st);
  }
  if (rc != MHD_OK) return rc;
  launch_dt_reduce(c, nxt, n, -1.0, st);
  launch_corrector_predictor(c, nxt, n, mode, -1.0, -1.0, st);
  CK(cudaGetLastError());
  return MHD_OK;
}

// Capture `steps` fused steps (a -> b -> a ...) into an executable graph.
int capture_run(Ctx* c, MhdState* a, MhdState* b, int n, int steps, int finish, Ctx::GraphEntry& e) {
  if (!c->cap_stream) CK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  const cudaStream_t cs = c->cap_stream;
  const bool timing = c->timing;
  const int64_t l0 = c->launches;
  c->timing = false;
  CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = MHD_OK;
  for (int k = 0; k < steps && rc == MHD_OK; k++) {
    const MhdState* cur = (k & 1) ? b : a;
    MhdState* nxt = (k & 1) ? a : b;
    const int mode = (finish && k == steps - 1) ? 1 : 3;
    rc = step_fused(c, cur, nxt, n, mode, true, cs);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(cs, &g);
  c->timing = timing;
  e.launches = c->launches - l0;
  c->launches = l0;
  if (rc != MHD_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) FAIL(MHD_ERR_CUDA, std::string("stream capture failed: ") + cudaGetErrorString(ce));
  const cudaError_t ie = cudaGraphInstantiate(&e.exec, g, 0ULL);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) FAIL(MHD_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(ie));
  e.a = *a;
  e.b = *b;
  e.n = n;
  e.steps = steps;
  e.finish = finish;
  e.generation = c->generation;
  return MHD_OK;
}

void drop_graphs(Ctx* c) {
  for (auto& e : c->graphs) cudaGraphExecDestroy(e.exec);
  c->graphs.clear();
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
  {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0) c->num_sms = sms;
  }
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
  c->n_pad = (N + 31) / 32 * 32;
  {
    double* p = nullptr;
    ok = ok && dev_alloc(c, &p, 32 * c->n_pad) == MHD_OK;  // 256 B per particle
    c->frec = p;
  }
  {
    const double rr = radius_scale_of(params->kernel) * params->hfact * (1.0 + c->list_margin);
    const double vol = params->dim == 3 ? 4.0 / 3.0 * M_PI * rr * rr * rr : M_PI * rr * rr;
    const int cap = ((int)(1.5 * vol) + 16 + 7) & ~7;
    ok = ok && dev_alloc(c, &c->posf, c->n_pad) == MHD_OK && dev_alloc(c, &c->posq, c->n_pad) == MHD_OK &&
         dev_alloc(c, &c->cellc, c->n_pad) == MHD_OK;
    ok = ok && dev_alloc(c, &c->nbr_hlim, c->n_pad) == MHD_OK && dev_alloc(c, &c->big_idx, c->n_pad) == MHD_OK &&
         dev_alloc(c, &c->app_idx, c->n_pad) == MHD_OK &&
         dev_alloc(c, &c->reb_idx, c->n_pad) == MHD_OK &&
         dev_alloc(c, &c->new_of_old, c->n_pad) == MHD_OK && dev_alloc(c, &c->nbr_mark, c->n_pad) == MHD_OK;
    for (Ctx::ListSlot& S : c->slots)
      ok = ok && dev_alloc(c, &S.cnt, c->n_pad) == MHD_OK && dev_alloc(c, &S.gcnt, c->n_pad) == MHD_OK &&
           dev_alloc(c, &S.xr, 3 * c->n_pad) == MHD_OK && dev_alloc(c, &S.hm, c->n_pad) == MHD_OK &&
           dev_alloc(c, &S.md, c->n_pad) == MHD_OK;
    ok = ok && ensure_list_storage(c, cap) == MHD_OK;
    c->nbr_cnt = c->slots[0].cnt;
    c->nbr_gcnt = c->slots[0].gcnt;
  }
  if (ok && cudaMallocHost((void**)&c->h_sc, sizeof(DevScalars)) != cudaSuccess) ok = false;
  const int64_t one[2] = {0, N};
  ok = ok && alloc_instances(c, 1, one) == MHD_OK;
  if (!ok) {
    g_err = c->err.empty() ? "workspace allocation failed" : c->err;
    mhd_ctx_destroy(c);
    return MHD_ERR_CUDA;
  }
  memset(c->h_sc, 0, sizeof(DevScalars));
  if (cudaMemcpy(c->d_sc, c->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice) != cudaSuccess) {
    g_err = "workspace initialisation failed";
    mhd_ctx_destroy(c);
    return MHD_ERR_CUDA;
  }
  if (const char* m = getenv("MHD_GRID_MARGIN")) c->grid_margin = std::max(1.0, atof(m));
  if (const char* m = getenv("MHD_FORCE_SHAPE")) c->force_shape = std::max(0, std::min(3, atoi(m)));
  if (const char* m = getenv("MHD_STENCIL")) c->stencil = std::max(1, std::min(3, atoi(m)));
  if (const char* m = getenv("MHD_GRAPH_PASSES")) c->graph_passes = std::max(1, std::min(256, atoi(m)));
  if (const char* m = getenv("MHD_GRAPH_LOOP")) c->graph_loop = atoi(m) != 0;
  if (const char* m = getenv("MHD_CELL_KAPPA")) c->cell_kappa = std::max(1.0, atof(m));
  if (const char* m = getenv("MHD_LIST_MARGIN")) c->list_margin = std::max(0.005, std::min(0.5, atof(m)));
  if (const char* m = getenv("MHD_LIST_REUSE")) c->list_reuse = atoi(m) != 0;
  if (const char* m = getenv("MHD_FORCE_STAGED")) c->force_staged = atoi(m) != 0;
  if (const char* m = getenv("MHD_FORCE_TILES")) c->force_tiles = atoi(m) != 0;
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
  cudaFree(c->frec);
  cudaFree(c->posf);
  cudaFree(c->posq);
  cudaFree(c->cellc);
  for (Ctx::ListSlot& S : c->slots) {
    cudaFree(S.idx);
    cudaFree(S.cnt);
    cudaFree(S.gcnt);
    cudaFree(S.xr);
    cudaFree(S.hm);
    cudaFree(S.md);
  }
  cudaFree(c->new_of_old);
  cudaFree(c->nbr_mark);
  for (unsigned* p : c->cell_scr) cudaFree(p);
  cudaFree(c->big_idx);
  cudaFree(c->app_idx);
  cudaFree(c->reb_idx);
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
  cudaFree(c->d_inst);
  if (c->h_inst) cudaFreeHost(c->h_inst);
  cudaFree(c->d_stage);
  drop_graphs(c);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  if (c->cap_stream2) cudaStreamDestroy(c->cap_stream2);
  cudaFree(c->tan_work);
  cudaFree(c->adj_buf);
  free_pair_grid(c->pgrid);
  delete c;
  return MHD_OK;
}

int mhd_ctx_set_params(void* ctx, const MhdParams* params) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  c->generation++;
  c->layout_gen++;  // the kernel radius may change: no list is carried over
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

int mhd_list_counts(void* ctx, int64_t* listed, int64_t* rebuilt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  const cudaStream_t st = S(stream);
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (listed) *listed = (int64_t)c->h_sc->n_listed;
  if (rebuilt) *rebuilt = (int64_t)c->h_sc->n_rebuilt;
  CK(cudaMemsetAsync(&c->d_sc->n_listed, 0, 2 * sizeof(unsigned long long), st));
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
  return sort_into(c, src, dst, (int)n, st, false);
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
    CK(cudaMemcpyAsync(&c->h_inst->dt_next, &c->d_inst->dt_next, sizeof(double), cudaMemcpyDeviceToHost, st));
    int rc = read_status(c, st);
    if (rc != MHD_OK) return rc;
    *dt_host = c->h_inst->dt_next;
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
  CK(cudaMemcpyAsync(c->h_inst, c->d_inst, sizeof(InstScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (t) *t = c->h_inst->t;
  if (dt) *dt = c->h_inst->dt;
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

// ------------------------------------------------------------ batched form
int mhd_ctx_set_instances(void* ctx, const MhdState* s, int32_t n_inst, const int64_t* start, double cell_headroom,
                          void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n_inst < 1 || !start) FAIL(MHD_ERR_INVALID, "n_inst must be >= 1 and start non-null");
  if (start[0] != 0) FAIL(MHD_ERR_INVALID, "start[0] must be 0");
  for (int k = 0; k < n_inst; k++)
    if (start[k + 1] <= start[k]) FAIL(MHD_ERR_INVALID, "every instance needs at least one particle");
  const int64_t n = start[n_inst];
  if (n > c->n_max) FAIL(MHD_ERR_INVALID, "instances exceed the context's n_max");
  if (!(cell_headroom >= 1.0 && cell_headroom <= 16.0)) FAIL(MHD_ERR_INVALID, "cell_headroom must be in [1, 16]");
  if (!check_state(c, s, false)) return MHD_ERR_INVALID;
  const cudaStream_t st = S(stream);
  CK(cudaStreamSynchronize(st));
  drop_graphs(c);
  c->batched = false;
  int rc = alloc_instances(c, n_inst, start);
  if (rc != MHD_OK) return rc;
  cudaFree(c->inst);
  c->inst = nullptr;
  if (n_inst > 1) {
    if (dev_alloc(c, &c->inst, c->n_max) != MHD_OK) return MHD_ERR_CUDA;
    std::vector<int> idx((size_t)n);
    for (int k = 0; k < n_inst; k++)
      for (int64_t i = start[k]; i < start[k + 1]; i++) idx[(size_t)i] = k;
    CK(cudaMemcpy(c->inst, idx.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
  }
  // Plan every instance on the host once to fix its cell capacity.
  refresh_spec(c);
  launch_reduce_hbox(c, s, (int)n, st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_inst, c->d_inst, sizeof(InstScalars) * n_inst, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&c->h_sc->status, &c->d_sc->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (c->h_sc->status != MHD_OK) {
    CK(cudaMemsetAsync(&c->d_sc->status, 0, sizeof(int), st));
    FAIL(MHD_ERR_NONFINITE, "non-finite or non-positive smoothing length");
  }
  const double axis_max[3] = {c->P.dim == 3 ? 2047.0 : 65535.0, c->P.dim == 3 ? 2047.0 : 65535.0,
                              c->P.dim == 3 ? 1023.0 : 1.0};
  int64_t base = 0;
  for (int k = 0; k < n_inst; k++) {
    InstScalars& q = c->h_inst[k];
    double lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = dbl_unorder(q.lo_bits[a]);
      hi[a] = dbl_unorder(q.hi_bits[a]);
    }
    Grid g;
    const double hmax = dbl_unorder(q.h_max_bits);
    if (plan_instance(c->spec, q.n, hmax, mean_h(hmax, q.h_sum, q.n), lo, hi, nullptr, g) != MHD_OK)
      FAIL(MHD_ERR_NONFINITE, "non-finite particle position");
    int64_t cells = 1;
    for (int a = 0; a < 3; a++) {
      const double want = a < c->P.dim ? ceil(g.nc[a] * cell_headroom) : 1.0;
      q.nc_cap[a] = (int)std::min(axis_max[a], std::max(1.0, want));
      cells *= q.nc_cap[a];
    }
    if (cells > ((int64_t)1 << 24)) {
      cells = 1;
      for (int a = 0; a < 3; a++) {
        q.nc_cap[a] = g.nc[a];
        cells *= g.nc[a];
      }
    }
    q.cell_base = (int)base;
    base += cells;
    if (base > ((int64_t)1 << 30)) FAIL(MHD_ERR_CAPACITY, "instances need more than 2^30 cells");
    q.h_max_bits = 0ULL;
    q.h_sum = 0ULL;
    for (int a = 0; a < 3; a++) {
      q.lo_bits[a] = ~0ULL;
      q.hi_bits[a] = 0ULL;
    }
    q.dt_min_bits = ~0ULL;
    if (k == 0) {
      g.cell_base = 0;
      c->grid = g;
    }
  }
  CK(cudaMemcpy(c->d_inst, c->h_inst, sizeof(InstScalars) * n_inst, cudaMemcpyHostToDevice));
  if (grow_cell_table(c, base) != MHD_OK) return MHD_ERR_CUDA;
  c->key_cells = (int)base;
  c->batched = true;
  c->generation++;
  c->layout_gen++;
  return MHD_OK;
}

int mhd_clock_set_all(void* ctx, const double* t, const double* dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (!t || !dt) FAIL(MHD_ERR_INVALID, "t and dt must be non-null");
  const cudaStream_t st = S(stream);
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpy(c->d_stage, t, sizeof(double) * c->n_inst, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_stage + c->n_inst, dt, sizeof(double) * c->n_inst, cudaMemcpyHostToDevice));
  launch_clock_load(c, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return MHD_OK;
}

int mhd_clock_get_all(void* ctx, double* t, double* dt, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (!t || !dt) FAIL(MHD_ERR_INVALID, "t and dt must be non-null");
  const cudaStream_t st = S(stream);
  launch_clock_store(c, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpy(t, c->d_stage, sizeof(double) * c->n_inst, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(dt, c->d_stage + c->n_inst, sizeof(double) * c->n_inst, cudaMemcpyDeviceToHost));
  return read_status(c, st);
}

int32_t mhd_instance_count(void* ctx) { return ctx ? ((Ctx*)ctx)->n_inst : 0; }

int mhd_ctx_tune(void* ctx, int32_t stencil, int32_t force_shape) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (stencil < 1 || stencil > 3) FAIL(MHD_ERR_INVALID, "stencil must be 1, 2 or 3");
  if (force_shape < -1 || force_shape > 3) FAIL(MHD_ERR_INVALID, "force_shape must be in -1..3");
  c->stencil = stencil;
  c->force_shape = force_shape;
  drop_graphs(c);
  c->generation++;
  return MHD_OK;
}

int mhd_advance(void* ctx, MhdState* a, MhdState* b, int64_t n, int32_t steps, int32_t finish, int32_t capture,
                void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return MHD_ERR_INVALID;
  if (n < 1 || n > c->n_max) FAIL(MHD_ERR_INVALID, "n must be in [1, n_max]");
  if (steps < 0) FAIL(MHD_ERR_INVALID, "steps must be >= 0");
  if (!check_state(c, a, false) || !check_state(c, b, false)) return MHD_ERR_INVALID;
  if (a->x == b->x) FAIL(MHD_ERR_INVALID, "a and b must not alias");
  if (c->batched && n != c->inst_start.back()) FAIL(MHD_ERR_INVALID, "n differs from the instances' total");
  if (capture && !c->batched) FAIL(MHD_ERR_INVALID, "captured runs need mhd_ctx_set_instances first");
  if (steps == 0) return MHD_OK;
  const cudaStream_t st = S(stream);
  if (!capture) {
    for (int k = 0; k < steps; k++) {
      const MhdState* cur = (k & 1) ? b : a;
      MhdState* nxt = (k & 1) ? a : b;
      const int mode = (finish && k == steps - 1) ? 1 : 3;
      int rc = step_fused(c, cur, nxt, (int)n, mode, false, st);
      if (rc != MHD_OK) return rc;
    }
    return read_status(c, st);
  }
  Ctx::GraphEntry* hit = nullptr;
  for (auto& e : c->graphs)
    if (e.generation == c->generation && e.n == n && e.steps == steps && e.finish == finish &&
        !memcmp(&e.a, a, sizeof(MhdState)) && !memcmp(&e.b, b, sizeof(MhdState)))
      hit = &e;
  if (!hit) {
    if (c->graphs.size() >= 8) drop_graphs(c);
    Ctx::GraphEntry e;
    memset(&e, 0, sizeof e);
    int rc = capture_run(c, a, b, (int)n, steps, finish, e);
    if (rc != MHD_OK) return rc;
    c->graphs.push_back(e);
    hit = &c->graphs.back();
  }
  const unsigned long long iters0 = c->h_sc->loop_iters;
  CK(cudaGraphLaunch(hit->exec, st));
  c->launches += hit->launches;
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  c->launches += 2 * (int64_t)(c->h_sc->loop_iters - iters0);
  const int rc = read_status(c, st);
  if (rc != MHD_OK) return rc;
  if (c->h_sc->relist || c->h_sc->events) {
    CK(cudaMemsetAsync(&c->d_sc->events, 0, sizeof(int), st));
    FAIL(MHD_ERR_RELIST, "the captured run met a neighbour-list rebuild or an unfinished density iteration; "
                         "restore its input state and replay it uncaptured");
  }
  return MHD_OK;
}

}  // extern "C"
