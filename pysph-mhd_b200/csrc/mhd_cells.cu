// mhd_cells.cu -- neighbour grid for the SPMHD particle update (sm_100a).
//
// Replaces PySPH's NNPS update (src/application.py:63-78) and its
// Solver.reorder_particles (src/solver.py:30-32,69-70): particles are
// binned into a uniform grid whose cells are at least R*h_max wide, sorted
// by linear cell index (x fastest) with a stable LSD radix sort, and the
// persistent particle fields are gathered into the sorted order.  A prefix
// table cell_start[ncells+1] then makes every x-row of three neighbouring
// cells one contiguous index range.
#include <cuda_runtime.h>
#include <string.h>

#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

// ---------------------------------------------------------------- reductions
// Per-instance h_max and bounding box (order-mapped integer atomics into the
// instance's InstScalars, which the consumer resets).  The particles of an
// instance are contiguous, so each block takes one contiguous chunk and a
// thread flushes a partial result only where the instance changes; a warp
// whose lanes all hold the same instance combines them first.
struct HBox {
  double hm, lo[3], hi[3];
  __device__ void reset() {
    hm = 0.0;
    for (int a = 0; a < 3; a++) {
      lo[a] = INFINITY;
      hi[a] = -INFINITY;
    }
  }
  __device__ void flush(InstScalars* is, int k) const {
    atomicMax(&is[k].h_max_bits, dbl_order(hm));
#pragma unroll
    for (int a = 0; a < 3; a++) {
      atomicMin(&is[k].lo_bits[a], dbl_order(lo[a]));
      atomicMax(&is[k].hi_bits[a], dbl_order(hi[a]));
    }
  }
};

__global__ void __launch_bounds__(256) k_reduce_hbox(int n, int chunk, const int* __restrict__ inst,
                                                     const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ z, const double* __restrict__ h,
                                                     InstScalars* is, DevScalars* sc) {
  const double* pos[3] = {x, y, z};
  const int b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  int key = -1;
  HBox acc;
  acc.reset();
  bool bad = false;
  for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    const int k = inst ? inst[i] : 0;
    if (k != key) {
      if (key >= 0) acc.flush(is, key);
      acc.reset();
      key = k;
    }
    const double hv = h[i];
    acc.hm = hv > acc.hm ? hv : acc.hm;
    bad |= !(hv > 0.0) || !isfinite(hv);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double v = pos[a][i];
      acc.lo[a] = fmin(acc.lo[a], v);
      acc.hi[a] = fmax(acc.hi[a], v);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) set_status(sc, MHD_ERR_NONFINITE);
  // warps whose lanes share one instance combine in registers, then the
  // block's warps combine in shared memory: one flush per instance and block
  __shared__ int skey[8];
  __shared__ HBox sacc[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wkey = __reduce_max_sync(0xffffffffu, key);
  if (__all_sync(0xffffffffu, key < 0 || key == wkey)) {
    for (int o = 16; o > 0; o >>= 1) {
      acc.hm = fmax(acc.hm, __shfl_xor_sync(0xffffffffu, acc.hm, o));
#pragma unroll
      for (int a = 0; a < 3; a++) {
        acc.lo[a] = fmin(acc.lo[a], __shfl_xor_sync(0xffffffffu, acc.lo[a], o));
        acc.hi[a] = fmax(acc.hi[a], __shfl_xor_sync(0xffffffffu, acc.hi[a], o));
      }
    }
    if (lane == 0) {
      skey[warp] = wkey;
      sacc[warp] = acc;
    }
  } else {
    if (key >= 0) acc.flush(is, key);
    if (lane == 0) skey[warp] = -1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int cur = -1;
    HBox run;
    run.reset();
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      const int k = skey[w];
      if (k < 0) continue;
      if (k != cur) {
        if (cur >= 0) run.flush(is, cur);
        run.reset();
        cur = k;
      }
      const HBox& b = sacc[w];
      run.hm = fmax(run.hm, b.hm);
      for (int a = 0; a < 3; a++) {
        run.lo[a] = fmin(run.lo[a], b.lo[a]);
        run.hi[a] = fmax(run.hi[a], b.hi[a]);
      }
    }
    if (cur >= 0) run.flush(is, cur);
  }
}

// Per-instance sum of h / h_max in 2^-32 units (integer atomics, so the
// sum and the mean h planned from it do not depend on the order of
// accumulation).  Runs after k_reduce_hbox.
__global__ void __launch_bounds__(256) k_reduce_hsum(int n, int chunk, const int* __restrict__ inst,
                                                     const double* __restrict__ h, InstScalars* is) {
  const int b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  int key = -1;
  double scale = 0.0;
  unsigned long long acc = 0ULL;
  for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    const int k = inst ? inst[i] : 0;
    if (k != key) {
      if (key >= 0 && acc) atomicAdd(&is[key].h_sum, acc);
      acc = 0ULL;
      key = k;
      scale = 4294967296.0 / dbl_unorder(is[k].h_max_bits);
    }
    const double v = h[i] * scale;
    acc += v > 0.0 ? (unsigned long long)fmin(v, 4294967296.0) : 0ULL;
  }
  const int wkey = __reduce_max_sync(0xffffffffu, key);
  if (__all_sync(0xffffffffu, key < 0 || key == wkey)) {
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && wkey >= 0 && acc) atomicAdd(&is[wkey].h_sum, acc);
  } else if (key >= 0 && acc) {
    atomicAdd(&is[key].h_sum, acc);
  }
}

__device__ __forceinline__ void reset_hbox(InstScalars& q) {
  q.h_max_bits = 0ULL;
  q.h_sum = 0ULL;
  for (int a = 0; a < 3; a++) {
    q.lo_bits[a] = ~0ULL;
    q.hi_bits[a] = 0ULL;
  }
}

__global__ void k_reset_hbox(int n_inst, InstScalars* is) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n_inst) reset_hbox(is[k]);
}

// Device planner of a batched context: one thread per instance plans its
// grid from the reductions above (same arithmetic as the host planner),
// within the instance's cell capacity, and resets the reductions.
__global__ void k_plan_grids(int n_inst, PlanSpec S, InstScalars* is, Grid* grids, DevScalars* sc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_inst) return;
  InstScalars& q = is[k];
  const double hmax = dbl_unorder(q.h_max_bits);
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = dbl_unorder(q.lo_bits[a]);
    hi[a] = dbl_unorder(q.hi_bits[a]);
  }
  Grid g;
  const int rc = plan_instance(S, q.n, hmax, mean_h(hmax, q.h_sum, q.n), lo, hi, q.nc_cap, g);
  if (rc != MHD_OK) {
    set_status(sc, rc);
  } else {
    g.cell_base = q.cell_base;
    grids[k] = g;
  }
  reset_hbox(q);
}

// --------------------------------------------------------------- cell keys
template <int DIM>
__global__ void __launch_bounds__(256) k_cell_keys(int n, const Grid* __restrict__ grids,
                                                   const int* __restrict__ inst, const double* __restrict__ x,
                                                   const double* __restrict__ y, const double* __restrict__ z,
                                                   uint32_t* __restrict__ keys, int32_t* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& g = grid_of(grids, inst, i);
  const int cx = cell_coord(g, 0, x[i]);
  const int cy = cell_coord(g, 1, y[i]);
  const int cz = DIM == 3 ? cell_coord(g, 2, z[i]) : 0;
  keys[i] = (uint32_t)(g.cell_base + (cz * g.nc[1] + cy) * g.nc[0] + cx);
  vals[i] = i;
}

// -------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITERS = 16;                    // per warp
constexpr int RS_TILE = RS_THREADS * RS_ITERS;  // keys per block

__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                           uint32_t* __restrict__ hist, int nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int it = 0; it < RS_ITERS; it++) {
    const int idx = base + it * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: warp w owns the contiguous sub-tile [w*512, (w+1)*512) of
// the block tile and walks it in order; equal digits inside one 32-key step
// are ranked by lane (match_any), steps and warps in order, so the pass is
// stable.
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const uint32_t* __restrict__ kin,
                                                              const int32_t* __restrict__ vin,
                                                              uint32_t* __restrict__ kout, int32_t* __restrict__ vout,
                                                              int n, int shift, const uint32_t* __restrict__ offs,
                                                              int nblocks) {
  __shared__ uint32_t wh[RS_WARPS][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = threadIdx.x; k < RS_WARPS * 256; k += RS_THREADS) (&wh[0][0])[k] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE + warp * (RS_ITERS * 32);
  const unsigned lt = (1u << lane) - 1u;
  for (int it = 0; it < RS_ITERS; it++) {
    const int idx = base + it * 32 + lane;
    const bool valid = idx < n;
    const uint32_t d = valid ? ((kin[idx] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) wh[warp][d] += __popc(peers);
  }
  __syncthreads();
  {
    const int d = threadIdx.x;  // RS_THREADS == 256 digits
    uint32_t run = offs[d * nblocks + blockIdx.x];
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) {
      const uint32_t c = wh[w][d];
      wh[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
  for (int it = 0; it < RS_ITERS; it++) {
    const int idx = base + it * 32 + lane;
    const bool valid = idx < n;
    uint32_t key = 0;
    int32_t val = 0;
    if (valid) {
      key = kin[idx];
      val = vin[idx];
    }
    const uint32_t d = valid ? ((key >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (valid) {
      const uint32_t pos = wh[warp][d] + __popc(peers & lt);
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wh[warp][d] += __popc(peers);
    __syncwarp();
  }
}

// ------------------------------------------------------------ prefix scan
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nwarps ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    warp_sums[lane] = s;
  }
  __syncthreads();
  const uint32_t warp_off = warp > 0 ? warp_sums[warp - 1] : 0;
  *total = warp_sums[nwarps - 1];
  __syncthreads();
  return warp_off + incl - v;
}

// Exclusive scan of tiles of SCAN_TILE elements; tile totals to `sums`.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const uint32_t* in, uint32_t* out, int m,
                                                             uint32_t* sums) {
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < m ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < m) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0 && sums) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(uint32_t* __restrict__ out, int m,
                                                           const uint32_t* __restrict__ sums) {
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  const uint32_t add = sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++)
    if (base + k < m) out[base + k] += add;
}

// --------------------------------------------------------------- cell table
// cell_start[c] = first sorted slot whose key >= c, for c in [0, ncells]:
// one thread per cell, a lower-bound search in the sorted keys.  Two threads
// of each block first bound the block's 256 cells, so the per-cell searches
// cover only the slots of those cells.  Long runs of empty cells (capacity
// tails of a batched context) cost no more than occupied ones.
__device__ __forceinline__ int lower_bound_key(const uint32_t* __restrict__ k, int lo, int hi, uint32_t key) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (k[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_cell_starts(int n, int ncells, const uint32_t* __restrict__ skeys,
                                                     int* __restrict__ cell_start) {
  __shared__ int range[2];
  const int c0 = blockIdx.x * 256;
  if (threadIdx.x < 2) {
    const long long c = (long long)c0 + (threadIdx.x ? 256 : 0);
    range[threadIdx.x] = c > ncells ? n : lower_bound_key(skeys, 0, n, (uint32_t)c);
  }
  __syncthreads();
  const int c = c0 + threadIdx.x;
  if (c > ncells) return;
  cell_start[c] = lower_bound_key(skeys, range[0], range[1], (uint32_t)c);
}

// ------------------------------------------------------- packed positions
// posf: FP32 position relative to the particle's cell origin (|error| <=
// 2^-24 cell widths) plus h, with the cell coordinates packed into one int
// (cellc): the geometry of the list build, (pos_i - pos_j) + (cell_i -
// cell_j) * cell width.  posq: the fixed-point position of the FP32 pair
// passes (Grid::fx_lo; the pair displacement is one wrapped integer
// difference per axis) plus m.
template <int DIM>
__global__ void __launch_bounds__(256) k_pack_positions(int n, const Grid* __restrict__ grids,
                                                        const int* __restrict__ inst, const double* __restrict__ x,
                                                        const double* __restrict__ y, const double* __restrict__ z,
                                                        const double* __restrict__ h,
                                                        const double* __restrict__ m, float4* __restrict__ posf,
                                                        uint4* __restrict__ posq, int* __restrict__ cellc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Grid& g = grid_of(grids, inst, i);
  const double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
  const int cx = cell_coord(g, 0, xi);
  const int cy = cell_coord(g, 1, yi);
  const int cz = DIM == 3 ? cell_coord(g, 2, zi) : 0;
  const float rx = (float)(xi - (g.lo[0] + cx * g.cs[0]));
  const float ry = (float)(yi - (g.lo[1] + cy * g.cs[1]));
  const float rz = DIM == 3 ? (float)(zi - (g.lo[2] + cz * g.cs[2])) : 0.f;
  posf[i] = make_float4(rx, ry, rz, (float)h[i]);
  posq[i] = make_uint4(fixed_coord(g, 0, xi), fixed_coord(g, 1, yi), DIM == 3 ? fixed_coord(g, 2, zi) : 0u,
                       __float_as_uint((float)m[i]));
  cellc[i] = pack_cell<DIM>(cx, cy, cz);
}

void launch_pack_positions(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  if (n <= 0) return;
  if (c->P.dim == 3)
    k_pack_positions<3><<<(n + 255) / 256, 256, 0, st>>>(n, c->d_grids, c->inst, s->x, s->y, s->z, s->h, s->m,
                                                         c->posf, c->posq, c->cellc);
  else
    k_pack_positions<2><<<(n + 255) / 256, 256, 0, st>>>(n, c->d_grids, c->inst, s->x, s->y, s->z, s->h, s->m,
                                                         c->posf, c->posq, c->cellc);
  c->launches++;
}

// ------------------------------------------------------------------ gather
__global__ void __launch_bounds__(256) k_gather(int n, const int32_t* __restrict__ perm, GatherSet gs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
  for (int f = 0; f < gs.nf; f++) gs.dst[f][s] = __ldg(gs.src[f] + o);
  if (gs.isrc) gs.idst[s] = __ldg(gs.isrc + o);
}

// ------------------------------------------------------------- host driver
static int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Exclusive scan of m elements, in place allowed; `scratch` holds the tile
// sums of every level (sized by scan_sums_needed).
static void exclusive_scan(Ctx* c, const uint32_t* in, uint32_t* out, int m, uint32_t* scratch, cudaStream_t st) {
  const int tiles = ceil_div(m, SCAN_TILE);
  if (tiles <= 1) {
    k_scan_tiles<<<1, SCAN_THREADS, 0, st>>>(in, out, m, nullptr);
    c->launches++;
    return;
  }
  k_scan_tiles<<<tiles, SCAN_THREADS, 0, st>>>(in, out, m, scratch);
  exclusive_scan(c, scratch, scratch, tiles, scratch + tiles, st);
  k_scan_add<<<tiles, SCAN_THREADS, 0, st>>>(out, m, scratch);
  c->launches += 2;
}

int max_sort_blocks(int64_t n_max) { return ceil_div(n_max > 0 ? n_max : 1, RS_TILE); }
int64_t scan_sums_needed(int64_t n_max) {
  int64_t m = (int64_t)256 * max_sort_blocks(n_max), total = 0;
  while (m > 1) {
    m = ceil_div(m, SCAN_TILE);
    total += m;
  }
  return total + 16;
}

void launch_reduce_hbox(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  const int blocks = n > 0 ? (ceil_div(n, 256) < 1184 ? ceil_div(n, 256) : 1184) : 1;
  const int chunk = n > 0 ? ceil_div(n, blocks) : 1;
  k_reduce_hbox<<<blocks, 256, 0, st>>>(n, chunk, c->inst, s->x, s->y, s->z, s->h, c->d_inst, c->d_sc);
  k_reduce_hsum<<<blocks, 256, 0, st>>>(n, chunk, c->inst, s->h, c->d_inst);
  c->launches += 2;
}

void launch_reset_hbox(Ctx* c, cudaStream_t st) {
  k_reset_hbox<<<ceil_div(c->n_inst, 128), 128, 0, st>>>(c->n_inst, c->d_inst);
  c->launches++;
}

void launch_plan_grids(Ctx* c, cudaStream_t st) {
  k_plan_grids<<<ceil_div(c->n_inst, 128), 128, 0, st>>>(c->n_inst, c->spec, c->d_inst, c->d_grids, c->d_sc);
  c->launches++;
}

// Sort the particles by cell of their instance's grid (keys are
// cell_base + linear cell); leaves perm (sorted slot -> source index) in
// c->perm and the cell table (c->key_cells + 1 entries) in c->cell_start.
void launch_sort_cells(Ctx* c, const MhdState* s, int n, cudaStream_t st) {
  const int nb = ceil_div(n, 256);
  if (n > 0) {
    if (c->P.dim == 3)
      k_cell_keys<3><<<nb, 256, 0, st>>>(n, c->d_grids, c->inst, s->x, s->y, s->z, c->keys[0], c->vals[0]);
    else
      k_cell_keys<2><<<nb, 256, 0, st>>>(n, c->d_grids, c->inst, s->x, s->y, s->z, c->keys[0], c->vals[0]);
    c->launches++;
  }
  sort_keys_to_cells(c, n, c->key_cells, c->cell_start, st);
}

void sort_keys_to_cells(Ctx* c, int n, int64_t ncells, int* cell_start, cudaStream_t st) {
  int bits = 1;
  while ((1LL << bits) < ncells) bits++;
  const int passes = (bits + 7) / 8;
  const int sb = max_sort_blocks(n);
  int cur = 0;
  for (int p = 0; p < passes && n > 0; p++) {
    const int shift = 8 * p;
    k_radix_hist<<<sb, RS_THREADS, 0, st>>>(c->keys[cur], n, shift, c->hist, sb);
    exclusive_scan(c, c->hist, c->hist, 256 * sb, c->scan_sums, st);
    k_radix_scatter<<<sb, RS_THREADS, 0, st>>>(c->keys[cur], c->vals[cur], c->keys[cur ^ 1], c->vals[cur ^ 1], n,
                                               shift, c->hist, sb);
    c->launches += 2;
    cur ^= 1;
  }
  c->sorted_keys = c->keys[cur];
  c->perm = c->vals[cur];
  k_cell_starts<<<ceil_div(ncells + 1, 256), 256, 0, st>>>(n, (int)ncells, c->sorted_keys, cell_start);
  c->launches++;
}

void launch_gather(Ctx* c, const GatherSet& gs, int n, cudaStream_t st) {
  if (n <= 0) return;
  k_gather<<<ceil_div(n, 256), 256, 0, st>>>(n, c->perm, gs);
  c->launches++;
}

}  // namespace mhd
