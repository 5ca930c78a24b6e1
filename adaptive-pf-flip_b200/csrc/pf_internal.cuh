// pf_internal.cuh -- device-side layout shared by the libpfgpu kernels.
//
// Grid storage (a B200-first restatement of SparseMacGrid3D<4>,
// src/grid/sparse_mac_grid3d.h:6-47 and SparseBlockGrid3D<4>,
// src/grid/sparse_block_grid3d.h:10-68):
//   * one tile lattice of 8^3-node tiles shared by all eight fields, with
//     TX = ceil((nx+1)/8) etc. so the extra face layer of u/v/w fits;
//   * a dense block-pointer array tile_slot[tile] -> pool slot or -1;
//   * a slot pool: field f of slot s lives at fld[f][s*512 + local], local =
//     (i&7) | (j&7)<<3 | (k&7)<<6, so a tile is 2 KB contiguous per field;
//   * reference-granular activity: act4[f] holds one byte per 4^3 block of
//     field f's own lattice (bid = bx + nbx*(by + nby*bz)), set wherever the
//     reference's ref()/activateBlock() would activate a block.
// Invariant: nodes of field f whose 4^3 block is inactive hold 0, and every
// slot at or beyond the pool size holds 0 in every field.  That makes the
// reference's get() (0 when inactive) a plain load.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pfgpu.h"

#define PF_TV 512
#define PF_NSAVED 3

namespace pf {

struct Geom {
  int nx, ny, nz;
  int TX, TY, TZ;  // tile lattice
  int ntiles;
  double dx, ox, oy, oz;
  double inv_dx;            // 1/dx, for coordinates that need not round as the reference's
  int dx_pow2;              // dx is a power of two: (p - o) / dx == (p - o) * inv_dx exactly
  int fdim[PF_NFIELDS][3];  // node lattice per field
  int bdim[PF_NFIELDS][3];  // 4^3 block lattice per field
};

// Device view of one grid, passed by value to kernels.
struct DevGrid {
  Geom g;
  const int* tile_slot;
  const int* slot_tile;
  float* fld[PF_NFIELDS];
  float* saved[PF_NSAVED];
  uint8_t* act4[PF_NFIELDS];
};

__host__ __device__ inline int tile_id(const Geom& g, int tx, int ty, int tz) {
  return tx + g.TX * (ty + g.TY * tz);
}

__host__ __device__ inline int local_id(int i, int j, int k) {
  return (i & 7) | ((j & 7) << 3) | ((k & 7) << 6);
}

__host__ __device__ inline bool in_field(const Geom& g, int f, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < g.fdim[f][0] && j < g.fdim[f][1] && k < g.fdim[f][2];
}

__host__ __device__ inline bool in_cells(const Geom& g, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < g.nx && j < g.ny && k < g.nz;
}

// Slot of the tile holding node (i,j,k); -1 when unpooled or off the lattice.
__device__ __forceinline__ int slot_of(const DevGrid& G, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0) return -1;
  const int tx = i >> 3, ty = j >> 3, tz = k >> 3;
  if (tx >= G.g.TX || ty >= G.g.TY || tz >= G.g.TZ) return -1;
  return __ldg(&G.tile_slot[tile_id(G.g, tx, ty, tz)]);
}

// SparseBlockGrid3D::get: 0 outside the field lattice or in unpooled tiles.
__device__ __forceinline__ float fget(const DevGrid& G, int f, int i, int j, int k) {
  if (!in_field(G.g, f, i, j, k)) return 0.0f;
  const int s = slot_of(G, i, j, k);
  if (s < 0) return 0.0f;
  return G.fld[f][(size_t)s * PF_TV + local_id(i, j, k)];
}

__device__ __forceinline__ float sget(const DevGrid& G, int a, int i, int j, int k) {
  if (!in_field(G.g, PF_U + a, i, j, k)) return 0.0f;
  const int s = slot_of(G, i, j, k);
  if (s < 0) return 0.0f;
  return G.saved[a][(size_t)s * PF_TV + local_id(i, j, k)];
}

// Marker of a cell: (int)(mk + 0.5f) as SparseMacGrid3D::cell (sparse_mac_grid3d.h:39).
__device__ __forceinline__ int cell_marker(const DevGrid& G, int i, int j, int k) {
  return (int)(fget(G, PF_MK, i, j, k) + 0.5f);
}

__host__ __device__ inline int act4_index(const Geom& g, int f, int i, int j, int k) {
  return (i >> 2) + g.bdim[f][0] * ((j >> 2) + g.bdim[f][1] * (k >> 2));
}

// Mark the 4^3 block of node (i,j,k) of field f active (idempotent).
__device__ __forceinline__ void activate4(const DevGrid& G, int f, int i, int j, int k) {
  uint8_t* a = &G.act4[f][act4_index(G.g, f, i, j, k)];
  if (*a == 0) *a = 1;
}

// Warp-aggregated atomic increment: lanes sharing `key` get consecutive ranks.
__device__ __forceinline__ int warp_agg_inc(int* counters, int key, unsigned active) {
  const unsigned peers = __match_any_sync(active, key);
  const int leader = __ffs(peers) - 1;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == leader) base = atomicAdd(&counters[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

// Control block of an iterative solve, resident in device memory.
struct SolveCtl {
  double rz;         // r.z of the current direction
  double alpha, beta;
  double res;        // max|r| after the last update
  double res0;
  double tol;        // effective tolerance
  double tol_abs, tol_rel;
  double pAp;
  double aux[4];     // per-solver scratch scalars
  int it;            // completed iterations
  int max_iter;
  int done;          // 0 running, 1 converged, 2 breakdown, 3 iteration cap, 4 non-finite
  int pin;           // pinned linear cell index or -1
  unsigned counter;  // last-CTA-done counter
  int n_cells;
  int touches_air;
  int min_fluid;
  int accepted, rejected;  // learned preconditioner outcomes
  double flex[2];          // flexible PCG: r.D^-1 r and r.z_prev of the current residual
};

// Programmatic dependent launch.  A kernel started by launch_pdl may begin
// while its predecessor on the stream is still running: it calls pdl_wait()
// before it touches memory the predecessor writes (the wait returns once the
// predecessor grid has completed and its writes are visible), and
// pdl_launch_dependents() to let its own successor be scheduled.  Work before
// the wait may only read memory no earlier kernel of the chain writes.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace pf

#define PF_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::pf::set_cuda_error(ctx, _e, #expr, __FILE__, __LINE__); \
  } while (0)
