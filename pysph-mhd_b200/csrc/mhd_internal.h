// mhd_internal.h -- context and launch helpers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "mhd_common.cuh"
#include "mhd_pairgrid.cuh"

namespace mhd {

constexpr int kGatherMax = 48;

// Fields permuted by the neighbour sort (besides itype): everything that
// persists from one right-hand side to the next, plus the output properties
// (src/particles.py:53-71) so the caller's view stays consistent.
#define MHD_SORTED_FIELDS(X)                                                                                 \
  X(x) X(y) X(z) X(gid) X(m) X(h) X(h0) X(u) X(v) X(w) X(e) X(upred) X(vpred) X(wpred) X(epred) X(Bevolx)      \
  X(Bevoly) X(Bevolz) X(Bevolxpred) X(Bevolypred) X(Bevolzpred) X(psi) X(psipred) X(alpha1) X(converged)        \
  X(omega) X(rho) X(rho_sum) X(p) X(cs) X(Bx) X(By) X(Bz)

// Arrays gathered by the neighbour sort: dst[f][s] = src[f][perm[s]].
struct GatherSet {
  const double* src[kGatherMax];
  double* dst[kGatherMax];
  int nf;
  const int32_t* isrc;
  int32_t* idst;
};

struct Ctx {
  MhdParams params;
  DevParams P;
  Grid grid;                // host copy of instance 0's grid
  Grid* d_grids = nullptr;  // device grid table, one entry per instance
  Grid* h_grids = nullptr;  // pinned staging copy of d_grids
  int grid_slots = 0;       // entries allocated in d_grids / h_grids
  int* inst = nullptr;      // instance of each particle; null = one instance
  int n_inst = 1;
  bool batched = false;     // instances set: grids planned on the device within fixed capacities
  int key_cells = 0;        // cells over all instances (the sort key range)
  InstScalars* d_inst = nullptr;  // per-instance clock and reductions (n_inst entries)
  InstScalars* h_inst = nullptr;  // pinned staging copy of d_inst
  double* d_stage = nullptr;      // 2 * n_inst doubles for clock uploads / downloads
  std::vector<int64_t> inst_start;  // first particle of each instance (n_inst + 1 entries)
  PlanSpec spec;                  // what every instance's grid plan shares
  int64_t generation = 0;         // bumped when a buffer captured by a graph is reallocated
  int graph_passes = 8;           // density passes captured per right-hand side
  cudaStream_t cap_stream = nullptr;
  cudaStream_t cap_stream2 = nullptr;  // captures the density loop's body graph
  bool graph_loop = true;  // captured density iteration as a conditional while node (MHD_GRAPH_LOOP=0: fixed passes)
  void* tan_work = nullptr;  // derivative form: new h / energy partials (dual records)
  PairGridBufs pgrid;        // derivative forms: the cell grid of their pair passes
  void* adj_buf = nullptr;   // adjoint: states, tapes, reverse workspace (doubles)
  size_t adj_size = 0;
  struct GraphEntry {
    MhdState a, b;
    int64_t n;
    int steps, finish;
    int64_t generation;
    cudaGraphExec_t exec;
    int64_t launches;  // kernels per replay
  };
  std::vector<GraphEntry> graphs;
  bool have_grid = false;
  int64_t n_max = 0;
  int device = 0;
  int64_t launches = 0;
  std::string err;

  // sort workspace
  uint32_t* keys[2] = {nullptr, nullptr};
  int32_t* vals[2] = {nullptr, nullptr};
  uint32_t* sorted_keys = nullptr;
  int32_t* perm = nullptr;
  uint32_t* hist = nullptr;
  uint32_t* scan_sums = nullptr;
  int* cell_start = nullptr;
  int64_t cell_cap = 0;

  // density / force workspace
  double* h_alt = nullptr;
  double* au_prev = nullptr;
  double* av_prev = nullptr;
  double* aw_prev = nullptr;
  // packed per-particle records of the force pass (sorted order): 8
  // four-vectors of the pair precision, 128 B (FP32) or 256 B (FP64) per
  // particle; sized for FP64
  void* frec = nullptr;

  double* spare[kGatherMax] = {};  // replan buffers, allocated on first use
  double grid_margin = 1.0;        // cells are R * h_cell * grid_margin * (1 + list_margin) wide
  double cell_kappa = 1.1;         // h_cell = min(h_max, cell_kappa * h_mean)

  // packed FP32 positions relative to the cell origin, and packed cell
  // coordinates, of the sorted particles (written after every sort)
  float4* posf = nullptr;
  uint4* posq = nullptr;  // {x, y, z fixed-point (Grid::fx_lo), m as float bits}: the FP32 density pass
  int* cellc = nullptr;
  int num_sms = 148;       // multiprocessors of the context's device
  int stencil = 2;       // cells are >= list cut-off / stencil wide
  int force_shape = -1;  // launch-shape variant of the force pass (kForceShapes); -1 = per-precision default
  bool force_staged = true;  // force-pass records staged in shared memory (MHD_FORCE_STAGED=0: register gather)
  bool force_tiles = false;  // FP32 force pass by cell tiles instead of lists (MHD_FORCE_TILES=1; no big particles)
  double list_cut = 0;   // R * h_max * (1 + list_margin) of the current grid

  // compacted neighbour lists (NbrList layout), built with every grid.  The
  // margin covers h growth during the density iteration (far below 2 % per
  // step in practice; more triggers a rebuild); larger margins pull in whole
  // lattice shells (at 5 %, the sqrt(6) shell of a cubic lattice with
  // R h = 2.4 dx: 42 % more entries).
  double list_margin = 0.02;
  int list_cap = 0;
  // current lists: the arrays of the slot built last
  int* nbr_idx = nullptr;
  int* nbr_cnt = nullptr;
  int* nbr_gcnt = nullptr;  // entries of the gather pass (the rest were scattered)
  int* big_idx = nullptr;   // big particles of the last build (DevScalars::n_big of them)
  int* app_idx = nullptr;   // particles given scattered entries by the last build (DevScalars::n_app)
  int* reb_idx = nullptr;   // particles whose lists a carried build rebuilds (DevScalars::n_reb)
  double* nbr_hlim = nullptr;

  // Lists persist across sorts in two slots, one per state buffer the caller
  // alternates between (keyed by the buffer's x array): the sort into a
  // buffer carries each list of the other buffer's slot to its particle's
  // new place, renumbered through the sort, where no pair it lacks can have
  // come within range, and rebuilds the rest.  Per particle a slot keeps an
  // epoch reference position xr, the largest distance md from it seen
  // since, and the smallest h hm seen since (see k_track).
  struct ListSlot {
    const double* key = nullptr;  // x array of the state whose order the lists follow
    int64_t n = -1;
    int64_t layout = -1;          // layout_gen when built
    uint64_t use = 0;
    int* idx = nullptr;
    int* cnt = nullptr;
    int* gcnt = nullptr;
    double* xr = nullptr;  // 3 x n_pad
    double* hm = nullptr;
    float* md = nullptr;
  };
  ListSlot slots[2];
  uint64_t slot_clock = 0;
  int64_t layout_gen = 0;     // bumped when the particle layout (instances) changes
  bool list_reuse = true;     // MHD_LIST_REUSE=0: rebuild every list on every sort
  int* new_of_old = nullptr;  // inverse of the last sort's permutation
  int* nbr_mark = nullptr;    // per particle: dirty, then "rebuild"
  unsigned* cell_scr[2] = {nullptr, nullptr};  // per-cell scratch (cell_cap entries each)
  int64_t last_rebuilt = -1;  // lists rebuilt by the last build (-1: not counted)
  int64_t n_pad = 0;  // n_max rounded up to a multiple of 32
  bool lists_checked = false;  // the host knows the current lists are valid
  NbrList lists() const { return NbrList{nbr_idx, nbr_cnt, nbr_hlim, list_cap}; }

  DevScalars* d_sc = nullptr;
  DevScalars* h_sc = nullptr;  // pinned mirror

  // CUDA-event timing of kernel families (MHD_TIMING_*)
  bool timing = false;
  struct EventPair {
    cudaEvent_t a, b;
    int kind;
  };
  std::vector<EventPair> events;
  size_t events_used = 0;
};

// Records a CUDA event pair around the launches in its scope when timing.
struct TimedScope {
  Ctx* c;
  int kind;
  cudaStream_t st;
  size_t slot = (size_t)-1;
  TimedScope(Ctx* c_, int kind_, cudaStream_t st_) : c(c_), kind(kind_), st(st_) {
    if (!c->timing) return;
    if (c->events_used == c->events.size()) {
      Ctx::EventPair e;
      cudaEventCreate(&e.a);
      cudaEventCreate(&e.b);
      c->events.push_back(e);
    }
    slot = c->events_used++;
    c->events[slot].kind = kind;
    cudaEventRecord(c->events[slot].a, st);
  }
  ~TimedScope() {
    if (slot != (size_t)-1) cudaEventRecord(c->events[slot].b, st);
  }
};

// Message returned by mhd_last_error(NULL) (entry points without a context).
void set_library_error(const std::string& msg);

int max_sort_blocks(int64_t n_max);
int64_t scan_sums_needed(int64_t n_max);
void launch_reduce_hbox(Ctx* c, const MhdState* s, int n, cudaStream_t st);
void launch_sort_cells(Ctx* c, const MhdState* s, int n, cudaStream_t st);
void launch_gather(Ctx* c, const GatherSet& gs, int n, cudaStream_t st);
// Stable sort of (c->keys[0][i], c->vals[0][i]) by key for keys below
// ncells, leaving the sorted keys in c->sorted_keys and the values (the
// permutation) in c->perm, then cell_start[k] = first sorted slot with key
// >= k for k in [0, ncells].
void sort_keys_to_cells(Ctx* c, int n, int64_t ncells, int* cell_start, cudaStream_t st);

void launch_reset_hbox(Ctx* c, cudaStream_t st);
void launch_plan_grids(Ctx* c, cudaStream_t st);
// Lists of the sorted particles of s; src is the state s was sorted from
// (its slot's lists are carried over where they stay valid), or null for a
// full rebuild.
void launch_build_lists(Ctx* c, const MhdState* s, int n, cudaStream_t st, const MhdState* src);
void launch_pack_positions(Ctx* c, const MhdState* s, int n, cudaStream_t st);
void launch_neighbour_counts(Ctx* c, const MhdState* s, int n, int* out, cudaStream_t st);
// adds the exact-rule neighbour pairs and the list entries of the current
// lists to DevScalars::n_pairs / n_candidates (the force pass's pair counts)
void launch_pair_stats(Ctx* c, const MhdState* s, int n, cudaStream_t st);
// density pass `pass` (0-based) reading h_in, writing h_out
void launch_density_pass(Ctx* c, MhdState* s, int n, int pass, const double* h_in, double* h_out, cudaStream_t st);
void launch_finish_density(Ctx* c, MhdState* s, int n, int passes, cudaStream_t st);
// The captured density loop's control (one thread): with first >= 0 it arms
// the loop (the next pass is `first`), otherwise it advances it; then it
// sets the loop condition: the group has not stopped, no list needs
// rebuilding, and the next pass is below min(max_iter, kDensityLoopCap).
constexpr int kDensityLoopCap = 256;
void launch_density_loop_control(Ctx* c, cudaGraphConditionalHandle h, int first, cudaStream_t st);
// Raises the dynamic shared-memory limit of the staged force passes for the
// context's kernel, dimension and precision (set-up only).
cudaError_t configure_force_pass(Ctx* c);
void launch_force_prologue(Ctx* c, MhdState* s, int n, cudaStream_t st);
void launch_force_pass(Ctx* c, MhdState* s, int n, cudaStream_t st);

void launch_dt_reduce(Ctx* c, const MhdState* s, int n, double t, cudaStream_t st);
void launch_stage(Ctx* c, MhdState* s, int n, int which, double dt, cudaStream_t st);
void launch_clock_set(Ctx* c, double t, double dt, cudaStream_t st);
void launch_clock_load(Ctx* c, cudaStream_t st);
void launch_clock_store(Ctx* c, cudaStream_t st);
int probe_fma_peak(int precision, double* flops, cudaStream_t st);
void launch_corrector_predictor(Ctx* c, MhdState* s, int n, int mode, double dt_cur, double dt_next,
                                cudaStream_t st);

}  // namespace mhd
