// mhd_pairgrid.cu -- building the derivative forms' cell grid (see
// mhd_pairgrid.cuh): bounds and largest h, the plan, the cell keys, then
// the stable key sort and cell table of the neighbour search.
#include <cuda_runtime.h>

#include "mhd_internal.h"
#include "mhd_pairgrid.cuh"

namespace mhd {

__global__ void __launch_bounds__(32) k_pg_reset(PairGridRed* r) {
  if (threadIdx.x != 0) return;
  r->h_max = 0ULL;
  for (int a = 0; a < 3; a++) {
    r->lo[a] = ~0ULL;
    r->hi[a] = 0ULL;
  }
}

__global__ void __launch_bounds__(256) k_pg_reduce(const double4* __restrict__ pos, int n, PairGridRed* r) {
  double h = 0.0, lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double4 p = pos[i];
    h = fmax(h, p.w);
    const double v[3] = {p.x, p.y, p.z};
    for (int a = 0; a < 3; a++) {
      lo[a] = fmin(lo[a], v[a]);
      hi[a] = fmax(hi[a], v[a]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    h = fmax(h, __shfl_xor_sync(0xffffffffu, h, o));
    for (int a = 0; a < 3; a++) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&r->h_max, dbl_order(h));
    for (int a = 0; a < 3; a++) {
      atomicMin(&r->lo[a], dbl_order(lo[a]));
      atomicMax(&r->hi[a], dbl_order(hi[a]));
    }
  }
}

// The plan (one thread).
__global__ void __launch_bounds__(32) k_pg_plan(DevParams P, const PairGridRed* r, int cap, PairGrid* g) {
  if (threadIdx.x != 0) return;
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = dbl_unorder(r->lo[a]);
    hi[a] = dbl_unorder(r->hi[a]);
  }
  *g = pair_grid_plan(P, dbl_unorder(r->h_max), lo, hi, cap);
}

__global__ void __launch_bounds__(256) k_pg_keys(const double4* __restrict__ pos, int n,
                                                 const PairGrid* __restrict__ gp, uint32_t* __restrict__ keys,
                                                 int32_t* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pos[i];
  keys[i] = (uint32_t)pair_grid_key(*gp, p.x, p.y, p.z);
  vals[i] = i;
}

void build_pair_grid(Ctx* c, PairGridBufs& b, int n, cudaStream_t st) {
  if (n <= 0) return;
  k_pg_reset<<<1, 32, 0, st>>>(b.red);
  const int blocks = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
  k_pg_reduce<<<blocks, 256, 0, st>>>(b.pos, n, b.red);
  k_pg_plan<<<1, 32, 0, st>>>(c->P, b.red, b.cap, b.grid);
  k_pg_keys<<<(n + 255) / 256, 256, 0, st>>>(b.pos, n, b.grid, c->keys[0], c->vals[0]);
  c->launches += 4;
  sort_keys_to_cells(c, n, b.cap, b.cell_start, st);
  b.perm = c->perm;
}

int alloc_pair_grid(PairGridBufs& b, int64_t n_max) {
  if (b.pos) return MHD_OK;
  // at most one cell per particle (at least 64); a sparse case whose
  // reach-wide cells would be more gets coarser cells (pair_grid_plan)
  b.cap = (int)(n_max > 64 ? n_max : 64);
  bool ok = cudaMalloc(&b.pos, sizeof(double4) * (size_t)n_max) == cudaSuccess &&
            cudaMalloc(&b.grid, sizeof(PairGrid)) == cudaSuccess &&
            cudaMalloc(&b.red, sizeof(PairGridRed)) == cudaSuccess &&
            cudaMalloc(&b.cell_start, sizeof(int) * ((size_t)b.cap + 1)) == cudaSuccess;
  if (!ok) {
    free_pair_grid(b);
    return MHD_ERR_CUDA;
  }
  return MHD_OK;
}

void free_pair_grid(PairGridBufs& b) {
  cudaFree(b.pos);
  cudaFree(b.grid);
  cudaFree(b.red);
  cudaFree(b.cell_start);
  b = PairGridBufs{};
}

}  // namespace mhd
