// pf_transfer.cu -- particle<->grid transfer kernels for sm_100a.
//
//   markCells        src/driver/sparse_sim3d_tp.cpp:22-50
//   spP2G3D_tp       src/driver/sparse_ops3d_tp.cpp:23-75, 95-153
//   applyGravity     src/driver/sparse_sim3d_tp.cpp:52-70
//   applyWallBoundary src/driver/sparse_sim3d_tp.cpp:72-97
//   spG2P3D_tp       src/driver/sparse_ops3d_tp.cpp:155-172 (+ sampleField,
//                    src/driver/sparse_ops3d_common.h:30-63)
//   spAdvect3D_tp    src/driver/sparse_ops3d_tp.cpp:176-232
//   calibrateRhoTilde0 src/transfer/transfer3d_tp.cpp:29-36
//
// P2G design (replaces the reference's 8 colour threads that each rescan every
// particle): particles are binned by cell (tile-major) with warp-aggregated
// atomics; one CTA per tile splats its particles, one thread per cell holding
// a register window per face field, into warp-private shared boxes, combines
// them into a staging box per tile, and the normalisation pass sums the
// staging boxes that reach each node.  Every sum runs in a fixed order, so
// P2G is reproducible bit for bit.  Block activation is decided with the
// reference's FP64 operation order wherever FP32 could differ, so the active
// 4^3 set is bit-identical; weights and accumulation are FP32.
#include <cmath>

#include "pf_ctx.h"

namespace pf {
namespace {

constexpr double kR2 = 2.25;  // KR*KR with KR = 1.5 (sparse_ops3d_tp.cpp:21)
// grid coordinate (pos - o)/dx in the reference's double arithmetic
__device__ __forceinline__ double grid_coord(float p, double o, double dx) {
  return __ddiv_rn(__dsub_rn((double)p, o), dx);
}

// The same double; for a power-of-two dx the product with 1/dx is exact.
__device__ __forceinline__ double grid_coord_g(const Geom& g, float p, double o) {
  const double d = __dsub_rn((double)p, o);
  return g.dx_pow2 ? __dmul_rn(d, g.inv_dx) : __ddiv_rn(d, g.dx);
}

// ---------------------------------------------------------------------------
// Binning.  One pass over the particles: the particle's cell (the reference's
// FP64 (pos - o) / dx, floored and clamped) as a bin key tile * 512 + local
// cell with a rank within the cell, and a request for the tile of the cell.
// The 4^3 activation is decided later, in the splat (reach bits below); the
// pool takes the one-tile dilation of the requested tiles, which holds every
// node a particle's window can reach (within two nodes of its cell).
// ---------------------------------------------------------------------------

// floor((p - o) / dx) clamped to [0, n): with a power-of-two dx and a zero
// origin the FP32 product with 1/dx is exact, so its floor is the FP64 one
__device__ __forceinline__ int bin_cell(const Geom& g, float p, double o, bool fast, float inv_dx_f, int n) {
  const int c = fast ? (int)floorf(p * inv_dx_f) : (int)floor(grid_coord_g(g, p, o));
  return min(max(c, 0), n - 1);
}

// Ranks are aggregated over runs of equal keys in consecutive lanes (the
// caller's particle order is largely spatial, so a warp's particles fall into
// a few cells): the run's first lane takes one counter increment for the run.
// A warp bins kBinPer consecutive 32-particle groups and issues all their
// loads, then all their counter increments, before it waits: the kernel is
// bound by the latency of those round trips, not by bandwidth.  With DO_BIN
// the tiles to pool are read off the counts afterwards (k_need_from_counts);
// without it (cell marking) the run leaders request their cells' tiles.
constexpr int kBinPer = 4;

template <bool DO_BIN>
__global__ void __launch_bounds__(256) k_bin(DevGrid G, const float* __restrict__ px, const float* __restrict__ py,
                                             const float* __restrict__ pz, int n, int* tile_count, int* pkey,
                                             int* prank, uint8_t* need) {
  const int lane = threadIdx.x & 31;
  const long long first = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kBinPer;
  const bool fast = G.g.dx_pow2 && G.g.ox == 0.0 && G.g.oy == 0.0 && G.g.oz == 0.0;
  const float inv_dx_f = (float)G.g.inv_dx;
  float x[kBinPer], y[kBinPer], z[kBinPer];
#pragma unroll
  for (int u = 0; u < kBinPer; ++u) {
    const long long p = first + 32 * u + lane;
    x[u] = y[u] = z[u] = 0.0f;
    if (p < n) {
      x[u] = px[p];
      y[u] = py[p];
      z[u] = pz[p];
    }
  }
  int key[kBinPer], start[kBinPer], base[kBinPer], tile[kBinPer];
  bool lead[kBinPer];
#pragma unroll
  for (int u = 0; u < kBinPer; ++u) {
    const long long p = first + 32 * u + lane;
    const int ci = bin_cell(G.g, x[u], G.g.ox, fast, inv_dx_f, G.g.nx);
    const int cj = bin_cell(G.g, y[u], G.g.oy, fast, inv_dx_f, G.g.ny);
    const int ck = bin_cell(G.g, z[u], G.g.oz, fast, inv_dx_f, G.g.nz);
    tile[u] = tile_id(G.g, ci >> 3, cj >> 3, ck >> 3);
    key[u] = tile[u] * PF_TV + local_id(ci, cj, ck);
    // the particles of this group are a prefix of the warp; a run starts where the key changes
    const unsigned valid = __ballot_sync(0xffffffffu, p < n);
    const int prev = __shfl_up_sync(0xffffffffu, key[u], 1);
    const unsigned heads = __ballot_sync(0xffffffffu, p < n && (lane == 0 || prev != key[u]));
    const unsigned upto = 0xffffffffu >> (31 - lane);  // lanes 0..lane
    start[u] = 31 - __clz(heads & upto | 1u);
    const unsigned after = heads & ~upto;              // heads past this lane
    const int stop = after ? __ffs(after) - 1 : 32 - __clz(valid);
    base[u] = 0;
    lead[u] = p < n && lane == start[u];
    if (DO_BIN && lead[u]) base[u] = atomicAdd(&tile_count[key[u]], stop - start[u]);
  }
  if constexpr (DO_BIN) {
#pragma unroll
    for (int u = 0; u < kBinPer; ++u) {
      const long long p = first + 32 * u + lane;
      const int b = __shfl_sync(0xffffffffu, base[u], start[u]);
      if (p < n) {
        pkey[p] = key[u];
        prank[p] = b + (lane - start[u]);
      }
    }
  } else {
    // a byte is stored only when it reads 0 (stores to hot bytes queue in L2)
    uint8_t seen[kBinPer];
#pragma unroll
    for (int u = 0; u < kBinPer; ++u) seen[u] = lead[u] ? need[tile[u]] : 1;
#pragma unroll
    for (int u = 0; u < kBinPer; ++u)
      if (!seen[u]) need[tile[u]] = 1;
  }
}

// need <- the one-tile dilation of the tiles holding particles: tmp[t] =
// need[t] or any particle binned into tile t (one warp per tile over its 512
// cell counts), then k_need_dilate
__global__ void k_need_from_counts(const int* __restrict__ tile_count, const uint8_t* need, int* tmp, int ntiles) {
  const int t = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (t >= ntiles) return;
  const int4* c = reinterpret_cast<const int4*>(tile_count + (size_t)t * PF_TV);
  int any = 0;
#pragma unroll
  for (int q = 0; q < PF_TV / 128; ++q) {
    const int4 v = c[q * 32 + lane];
    any |= v.x | v.y | v.z | v.w;
  }
  any = __any_sync(0xffffffffu, any != 0);
  if (lane == 0) tmp[t] = any || need[t];
}

__global__ void k_need_dilate(Geom g, const int* tmp, uint8_t* need) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ntiles) return;
  const int tx = t % g.TX, q = t / g.TX, ty = q % g.TY, tz = q / g.TY;
  int any = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = tx + dx, y = ty + dy, z = tz + dz;
        if (x >= 0 && y >= 0 && z >= 0 && x < g.TX && y < g.TY && z < g.TZ) any |= tmp[tile_id(g, x, y, z)];
      }
  if (any) need[t] = 1;
}

// perm[start of the particle's cell + its rank] = particle, kBinPer per thread
// with all gathers issued before the scatters
__global__ void k_bin_scatter(const int* __restrict__ pkey, const int* __restrict__ prank,
                              const int* __restrict__ tile_start, int* perm, int n) {
  const long long first = (long long)blockIdx.x * blockDim.x * kBinPer + threadIdx.x;
  int key[kBinPer], rank[kBinPer], at[kBinPer];
#pragma unroll
  for (int u = 0; u < kBinPer; ++u) {
    const long long p = first + (long long)u * blockDim.x;
    key[u] = p < n ? pkey[p] : 0;
    rank[u] = p < n ? prank[p] : 0;
  }
#pragma unroll
  for (int u = 0; u < kBinPer; ++u) at[u] = first + (long long)u * blockDim.x < n ? tile_start[key[u]] : 0;
#pragma unroll
  for (int u = 0; u < kBinPer; ++u) {
    const long long p = first + (long long)u * blockDim.x;
    if (p < n) perm[at[u] + rank[u]] = (int)p;
  }
}

// ---------------------------------------------------------------------------
// markCells (sparse_sim3d_tp.cpp:22-50)
// ---------------------------------------------------------------------------
// Every marker write also lowers the first-touch key of its 4^3 block to the
// write's position in the reference's markCells sequence: the three wall
// loops (x, y, z walls; position q as enumerated here), then the particles
// (position walls + particle index).  Sorting the active blocks by the key
// gives the reference's activeBlockIds() order of the marker field.
__global__ void k_mark_walls(DevGrid G, uint32_t* first) {
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  const long long nxf = 2LL * ny * nz, nyf = 2LL * nx * nz, nzf = 2LL * nx * ny;
  const long long total = nxf + nyf + nzf;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    if (q < nxf) {
      const long long r = q >> 1;
      j = (int)(r % ny); k = (int)(r / ny); i = (q & 1) ? nx - 1 : 0;
    } else if (q < nxf + nyf) {
      const long long s = q - nxf, r = s >> 1;
      i = (int)(r % nx); k = (int)(r / nx); j = (s & 1) ? ny - 1 : 0;
    } else {
      const long long s = q - nxf - nyf, r = s >> 1;
      i = (int)(r % nx); j = (int)(r / nx); k = (s & 1) ? nz - 1 : 0;
    }
    const int sl = slot_of(G, i, j, k);
    if (sl < 0) continue;  // unreachable: wall tiles are pooled first
    G.fld[PF_MK][(size_t)sl * PF_TV + local_id(i, j, k)] = 2.0f;
    activate4(G, PF_MK, i, j, k);
    atomicMin(&first[act4_index(G.g, PF_MK, i, j, k)], (uint32_t)q);
  }
}

__global__ void k_mark_particles(DevGrid G, const float* __restrict__ px, const float* __restrict__ py,
                                 const float* __restrict__ pz, int n, uint32_t* first, uint32_t walls) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  // (int) truncation, as the reference's cast
  const int i = __double2int_rz(grid_coord_g(G.g, px[p], G.g.ox));
  const int j = __double2int_rz(grid_coord_g(G.g, py[p], G.g.oy));
  const int k = __double2int_rz(grid_coord_g(G.g, pz[p], G.g.oz));
  if (!in_cells(G.g, i, j, k)) return;
  const int sl = slot_of(G, i, j, k);
  if (sl < 0) return;  // unreachable: particle cell tiles are pooled first
  float* m = &G.fld[PF_MK][(size_t)sl * PF_TV + local_id(i, j, k)];
  if ((int)(*m + 0.5f) != 2) {
    *m = 1.0f;
    activate4(G, PF_MK, i, j, k);
    // the block's first-touch key is its smallest particle index: the lanes
    // marking one block send one atomicMin, from the lowest lane (the
    // smallest index of the group)
    const int bid = act4_index(G.g, PF_MK, i, j, k);
    const unsigned peers = __match_any_sync(__activemask(), bid);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicMin(&first[bid], walls + (uint32_t)p);
  }
}

// ---------------------------------------------------------------------------
// P2G splat: one CTA per tile holding particles
// ---------------------------------------------------------------------------
// One thread per cell, passes over the tile's 512 cells.  For face field A
// every particle of cell c touches window nodes c-1..c+2 along the field's
// normal axis L = A and c-1..c+1 along the two transverse axes S1 < S2 (the
// -1/2 shift puts the transverse window base at c-1 whatever the particle's
// position).  A thread accumulates all particles of its cell into a 4x3x3
// register window; the nodes a particle does not reach have |d| >= 1.5 and
// receive weight 0.
//
// Determinism.  Every node's sum is formed in one fixed order, so two runs on
// the same particles give bit-identical fields:
//   * a cell's particles are taken in ascending index (sorted at the start of
//     the kernel; binning ranks particles in arrival order);
//   * each warp adds its 32 cells' windows into a shared box of its own, one
//     window offset at a time (the lanes address distinct nodes);
//   * the 16 warp boxes of the tile are combined node by node in warp order
//     into the tile's staging box in global memory;
//   * k_normalize adds the staging boxes of the (up to 8) tiles covering a
//     node in ascending tile offset.
// No floating-point atomics are used.
//
// Activation (preactivateKernel, sparse_ops3d_tp.cpp:23-40: the 4^3 block of
// every node with w > 0, i.e. fl(fl(dx^2 + dy^2) + dz^2) < 2.25 in FP64).  A
// window spans at most two blocks per axis; a block is reached iff the sum of
// the per-axis minima of d^2/r^2 over its window nodes is below 1.  The
// thread keeps, per window block, the minimum of that FP32 sum over its
// cell's particles: a minimum clear of 1 by kReachEps decides the block for
// the whole cell (the FP32 sums are within 1e-5 of the FP64 ones); a minimum
// inside the band sends every particle of the cell through the reference's
// FP64 arithmetic (exact_reach).  Reached blocks are OR-ed per tile and each
// tile CTA writes its blocks' bytes.
constexpr float kReachEps = 2e-5f;
constexpr int kSplatThreads = 128;                 // threads per tile CTA
constexpr int kSplatPasses = PF_TV / kSplatThreads;
constexpr int kSplatGroups = PF_TV / 32;           // warp boxes per tile (one per warp and pass)
// Warp box of one field: the window nodes of a warp's 8 x 4 x 1 cells.  The x
// pitch is 12 float2 (mom, mass) and a warp's lanes cover the rows y = 0, 2
// (lanes 0-15) and 1, 3 (lanes 16-31), so each half-warp's 64-bit accesses
// fall on 16 distinct bank pairs.
constexpr int kWarpPitch = 12;
constexpr int kWarpBox = kWarpPitch * 6 * 4;       // x pitch * max(GY * GZ) over the fields
// Staging box of one tile and field: nodes -1..9 along the normal axis and
// -1..8 along the transverse axes relative to the tile's first cell.
constexpr int kStageField = 11 * 10 * 10;
constexpr int kStageTile = 3 * kStageField;
constexpr int kBigSortStage = kSplatGroups * kWarpBox * 2;  // ints of the warp boxes reused by the big-cell sort

static_assert(kStageTile == kSplatStageTile, "staging size mismatch");

// Two FP32 values in one 64-bit register, for the packed .f32x2 arithmetic
// of sm_100 (one instruction for both lanes of add, sub, mul and fma).
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// t = min(max(a - b, 0), 1): one saturating subtract
__device__ __forceinline__ float sub_sat(float a, float b) {
  float d;
  asm("sub.rn.sat.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}

// The FP64 decision for one particle and field: bit x + 2y + 4z for window
// block (x, y, z), where window block 0 along an axis holds the window nodes
// before the split s of that axis.  n[] are the global first window nodes.
template <int A>
__device__ unsigned exact_reach(const DevGrid& G, float ppx, float ppy, float ppz, const int* n, const int* sp) {
  constexpr int NX = A == 0 ? 4 : 3, NY = A == 1 ? 4 : 3, NZ = A == 2 ? 4 : 3;
  const int cnt[3] = {NX, NY, NZ};
  const int fv = PF_U + A;
  const double g[3] = {grid_coord(ppx, G.g.ox, G.g.dx), grid_coord(ppy, G.g.oy, G.g.dx),
                       grid_coord(ppz, G.g.oz, G.g.dx)};
  double m[3][2];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const double c = ax == A ? g[ax] : __dsub_rn(g[ax], 0.5);
    m[ax][0] = m[ax][1] = 1e300;
    for (int i = 0; i < cnt[ax]; ++i) {
      const int node = n[ax] + i;
      if (node < 0 || node >= G.g.fdim[fv][ax]) continue;
      const double d = __dsub_rn(c, (double)node);
      const double dd = __dmul_rn(d, d);
      if (i < sp[ax]) m[ax][0] = fmin(m[ax][0], dd);
      else m[ax][1] = fmin(m[ax][1], dd);
    }
  }
  unsigned r = 0u;
#pragma unroll
  for (int z = 0; z < 2; ++z)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int x = 0; x < 2; ++x)
        if (__dadd_rn(__dadd_rn(m[0][x], m[1][y]), m[2][z]) < kR2) r |= 1u << (x + 2 * y + 4 * z);
  return r;
}

// Batcher's odd-even merge sort of N register values (all indices resolve at
// compile time).
template <int N>
__device__ __forceinline__ void sort_net(int (&a)[N]) {
#pragma unroll
  for (int p = 1; p < N; p <<= 1)
#pragma unroll
    for (int k = p; k >= 1; k >>= 1)
#pragma unroll
      for (int j = k % p; j + k < N; j += 2 * k)
#pragma unroll
        for (int i = 0; i < k; ++i)
          if (i + j + k < N && (i + j) / (2 * p) == (i + j + k) / (2 * p)) {
            const int x = a[i + j], y = a[i + j + k];
            a[i + j] = min(x, y);
            a[i + j + k] = max(x, y);
          }
}

template <int N>
__device__ __forceinline__ void sort_segment(int* __restrict__ perm, int beg, int n) {
  int a[N];
#pragma unroll
  for (int i = 0; i < N; ++i) a[i] = i < n ? perm[beg + i] : 0x7fffffff;
  sort_net<N>(a);
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (i < n) perm[beg + i] = a[i];
}

// Cell of thread `tid` in pass `pass`: lane bits 0-2 give x, lane bits 3-4 the
// row (0, 2, 1, 3 in that order, for the warp box's bank pattern), the warp's
// flat index g = warps * pass + warp gives the y half (g & 1) and z (g >> 1).
__device__ __forceinline__ int splat_cell_of(int tid, int pass) {
  const int lane = tid & 31, g = (kSplatThreads / 32) * pass + (tid >> 5);
  const int q = lane >> 3;
  const int y = 4 * (g & 1) + (((q & 1) << 1) | (q >> 1));
  return (lane & 7) + 8 * y + 64 * (g >> 1);
}

// Window geometry of one cell for face field A: 4 nodes along the normal axis
// L = A, 3 along the transverse axes S1 < S2.
template <int A>
struct SplatWindow {
  static constexpr int S1 = A == 0 ? 1 : 0, S2 = A == 2 ? 1 : 2;
  int n[3];      // global first window node per axis (the cell minus one)
  int sp[3];     // window nodes before the 4^3 block boundary per axis
  unsigned off;  // bit 4*axis + i: node i off the field's lattice

  __device__ __forceinline__ SplatWindow(const DevGrid& G, const int (&c)[3], bool edge) {
    off = 0u;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      n[ax] = c[ax] - 1;
      sp[ax] = min(4 - (n[ax] & 3), ax == A ? 4 : 3);
      if (edge)
#pragma unroll
        for (int i = 0; i < (ax == A ? 4 : 3); ++i)
          if (n[ax] + i < 0 || n[ax] + i >= G.g.fdim[PF_U + A][ax]) off |= 1u << (4 * ax + i);
    }
  }

  // a[ax][i] = d^2/r^2 for window node i along axis ax, d = g - i with g the
  // particle's coordinate relative to the first window node (transverse axes
  // shifted by -1/2 onto the node lattice).  With a power-of-two dx and a
  // zero origin the product with 1/dx is exact and the FMA rounds X/dx - n
  // once: the FP64 value rounded to float.  Nodes off the lattice get a = 2
  // (weight 0, never reached).  Pairs (a0, a1), (a2, a3) per axis.
  __device__ __forceinline__ void coords(const DevGrid& G, float X, float Y, float Z, bool fast, float inv_dx_f,
                                         double inv_dx, bool edge, f32x2 (&a)[3][2]) const {
    float g[3];
    if (fast) {
      g[0] = fmaf(X, inv_dx_f, (float)-n[0]);
      g[1] = fmaf(Y, inv_dx_f, (float)-n[1]);
      g[2] = fmaf(Z, inv_dx_f, (float)-n[2]);
    } else {
      g[0] = (float)(((double)X - G.g.ox) * inv_dx - n[0]);
      g[1] = (float)(((double)Y - G.g.oy) * inv_dx - n[1]);
      g[2] = (float)(((double)Z - G.g.oz) * inv_dx - n[2]);
    }
    const f32x2 k2 = f2_pack(1.0f / 2.25f, 1.0f / 2.25f);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      if (ax != A) g[ax] -= 0.5f;
      const f32x2 gg = f2_pack(g[ax], g[ax]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const f32x2 d = f2_sub(gg, f2_pack((float)(2 * h), (float)(2 * h + 1)));
        a[ax][h] = f2_mul(f2_mul(d, d), k2);
      }
    }
    if (edge) {
#pragma unroll
      for (int ax = 0; ax < 3; ++ax)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float lo, hi;
          f2_unpack(a[ax][h], lo, hi);
          if ((off >> (4 * ax + 2 * h)) & 1u) lo = 2.0f;
          if ((off >> (4 * ax + 2 * h + 1)) & 1u) hi = 2.0f;
          a[ax][h] = f2_pack(lo, hi);
        }
    }
  }

  // Per-axis minima of a over the window nodes on each side of the block
  // split.  kNearest: the particle lies in its cell (coordinate in [1, 2) from
  // the first window node along L, [0.5, 1.5) along the transverse axes after
  // the shift), so the nearest node on each side is known without a search.
  template <bool kNearest>
  __device__ __forceinline__ void side_minima(const f32x2 (&a)[3][2], float (&m)[3][2]) const {
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      float v[4];
      f2_unpack(a[ax][0], v[0], v[1]);
      f2_unpack(a[ax][1], v[2], v[3]);
      const int s = sp[ax];
      if (kNearest) {
        if (ax == A) {
          const float m12 = fminf(v[1], v[2]);
          m[ax][0] = s == 1 ? v[0] : s == 2 ? v[1] : m12;
          m[ax][1] = s == 1 ? m12 : s == 2 ? v[2] : s == 3 ? v[3] : 4.0f;
        } else {
          m[ax][0] = s == 1 ? v[0] : v[1];
          m[ax][1] = s == 1 ? v[1] : s == 2 ? v[2] : 4.0f;
        }
      } else {
        m[ax][0] = m[ax][1] = 4.0f;
#pragma unroll
        for (int i = 0; i < (ax == A ? 4 : 3); ++i) {
          if (i < s) m[ax][0] = fminf(m[ax][0], v[i]);
          else m[ax][1] = fminf(m[ax][1], v[i]);
        }
      }
    }
  }
};

// Splat of one cell's particles (perm[beg, end), ascending index) into the
// window accumulators of face field A, and the cell's per-block minima of the
// FP32 reach sums (bmin, block x + 2y + 4z).
//
// Node pair h of transverse row r = s1 + 3*s2 holds L nodes 2h and 2h + 1, so
// one packed f32x2 instruction serves two nodes.  Per node and particle the
// weight is w = t^3 with t = sat((1 - a_L) - (a_S1 + a_S2)), i.e.
// 1 - d^2/r^2 clamped at 0 (t <= 1 holds by itself).  The 36 weights are kept
// in registers between the weight sum and the accumulation.
template <int A, bool kNearest>
__device__ __forceinline__ void splat_particles(const DevGrid& G, const SplatWindow<A>& win, int beg, int end,
                                                const int* __restrict__ perm, const float* __restrict__ px,
                                                const float* __restrict__ py, const float* __restrict__ pz,
                                                const float* __restrict__ vA, const uint8_t* __restrict__ type,
                                                const float* __restrict__ vol, float m_l, float m_g, double inv_dx,
                                                float inv_dx_f, bool fast, bool edge, f32x2 (&am)[9][2],
                                                f32x2 (&ap)[9][2], float (&bmin)[8]) {
  using W = SplatWindow<A>;
  const f32x2 one2 = f2_pack(1.0f, 1.0f);
  // the next particle's attributes are loaded while this one is splatted (the
  // last particle reloads itself, so the loads need no branch)
  int pn = perm[beg];
  float xn = px[pn], yn = py[pn], zn = pz[pn], vn = vA[pn], voln = vol[pn];
  uint8_t tn = type[pn];
  for (int q = beg; q < end; ++q) {
    const float X = xn, Y = yn, Z = zn, VA = vn, VOL = voln;
    const uint8_t TY = tn;
    pn = perm[min(q + 1, end - 1)];
    xn = px[pn];
    yn = py[pn];
    zn = pz[pn];
    vn = vA[pn];
    voln = vol[pn];
    tn = type[pn];
    f32x2 a[3][2];
    win.coords(G, X, Y, Z, fast, inv_dx_f, inv_dx, edge, a);
    {
      float m[3][2];
      win.template side_minima<kNearest>(a, m);
#pragma unroll
      for (int y = 0; y < 2; ++y)
#pragma unroll
        for (int x = 0; x < 2; ++x) {
          const float sxy = m[0][x] + m[1][y];
#pragma unroll
          for (int z = 0; z < 2; ++z) bmin[x + 2 * y + 4 * z] = fminf(bmin[x + 2 * y + 4 * z], sxy + m[2][z]);
        }
    }
    // 1 - a along L, and a_S1 + a_S2 per transverse row
    const f32x2 om2[2] = {f2_sub(one2, a[A][0]), f2_sub(one2, a[A][1])};
    float om[4];
    f2_unpack(om2[0], om[0], om[1]);
    f2_unpack(om2[1], om[2], om[3]);
    float aS1[4], aS2[4];
    f2_unpack(a[W::S1][0], aS1[0], aS1[1]);
    f2_unpack(a[W::S1][1], aS1[2], aS1[3]);
    f2_unpack(a[W::S2][0], aS2[0], aS2[1]);
    f2_unpack(a[W::S2][1], aS2[2], aS2[3]);
    f32x2 w[9][2];
#pragma unroll
    for (int s2 = 0; s2 < 3; ++s2)
#pragma unroll
      for (int s1 = 0; s1 < 3; ++s1) {
        const int r = s1 + 3 * s2;
        const float at = aS1[s1] + aS2[s2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const f32x2 t = f2_pack(sub_sat(om[2 * h], at), sub_sat(om[2 * h + 1], at));
          w[r][h] = f2_mul(f2_mul(t, t), t);
        }
      }
    // the weight sum as a fixed tree (short dependency chains)
    f32x2 q9[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) q9[r] = f2_add(w[r][0], w[r][1]);
    const f32x2 ws = f2_add(f2_add(f2_add(q9[0], q9[1]), f2_add(q9[2], q9[3])),
                            f2_add(f2_add(q9[4], q9[5]), f2_add(f2_add(q9[6], q9[7]), q9[8])));
    float wlo, whi;
    f2_unpack(ws, wlo, whi);
    const float wsum = wlo + whi;
    if (!(wsum > 0.0f)) continue;
    const float mp = (TY == 0 ? m_l : m_g) * VOL;
    const float s_m = __fdividef(mp, wsum);
    const float s_p = s_m * VA;
    const f32x2 sm2 = f2_pack(s_m, s_m), sp2 = f2_pack(s_p, s_p);
#pragma unroll
    for (int r = 0; r < 9; ++r)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        am[r][h] = f2_fma(w[r][h], sm2, am[r][h]);
        ap[r][h] = f2_fma(w[r][h], sp2, ap[r][h]);
      }
  }
}

// Add a warp's window accumulators into its warp box, one (x, y) column of
// window offsets at a time.  The lanes of a warp hold cells of one z layer, so
// within a column the lanes and the z offsets address distinct nodes; between
// columns a lane's node may be another lane's, hence the __syncwarp, which
// also keeps the compiler from reordering the shared accesses across columns.
template <int A>
__device__ __forceinline__ void flush_window(float2* wb, int x, int yl, const f32x2 (&am)[9][2],
                                             const f32x2 (&ap)[9][2]) {
  constexpr int S1 = A == 0 ? 1 : 0, S2 = A == 2 ? 1 : 2;
  constexpr int GY = A == 1 ? 7 : 6;
  constexpr int NX = A == 0 ? 4 : 3, NY = A == 1 ? 4 : 3, NZ = A == 2 ? 4 : 3;
  float2* base = wb + x + kWarpPitch * yl;
#pragma unroll
  for (int ix = 0; ix < NX; ++ix)
#pragma unroll
    for (int iy = 0; iy < NY; ++iy) {
#pragma unroll
      for (int iz = 0; iz < NZ; ++iz) {
        const int idx[3] = {ix, iy, iz};
        const int l = idx[A], r = idx[S1] + 3 * idx[S2];
        float2* p = base + ix + kWarpPitch * (iy + GY * iz);
        float mlo, mhi, plo, phi;
        f2_unpack(am[r][l >> 1], mlo, mhi);
        f2_unpack(ap[r][l >> 1], plo, phi);
        float2 v = *p;
        v.x += (l & 1) ? phi : plo;
        v.y += (l & 1) ? mhi : mlo;
        *p = v;
      }
      __syncwarp();
    }
}

// One field of the splat: every pass's cells into the warp boxes, then the
// warp boxes into the tile's staging box.  Returns this thread's reached
// blocks (bits of the tile's 4x4x4 block box).
template <int A>
__device__ __forceinline__ unsigned long long splat_field(const DevGrid& G, float2* wbox, float2* __restrict__ stage,
                                                          const int* __restrict__ cs, const int* __restrict__ perm,
                                                          const float* __restrict__ px, const float* __restrict__ py,
                                                          const float* __restrict__ pz, const float* __restrict__ vA,
                                                          const uint8_t* __restrict__ type,
                                                          const float* __restrict__ vol, float m_l, float m_g,
                                                          const int (&t0)[3], double inv_dx, float inv_dx_f, bool fast,
                                                          bool edge) {
  constexpr int GY = A == 1 ? 7 : 6, GZ = A == 2 ? 4 : 3;
  constexpr int FX = A == 0 ? 11 : 10, FY = A == 1 ? 11 : 10, FZ = A == 2 ? 11 : 10;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < kSplatGroups * kWarpBox; e += kSplatThreads) wbox[e] = make_float2(0.0f, 0.0f);
  __syncthreads();
  unsigned long long box = 0ull;
#pragma unroll 1
  for (int pass = 0; pass < kSplatPasses; ++pass) {
    const int cl = splat_cell_of(tid, pass);
    const int beg = cs[cl], end = cs[cl + 1];
    const int c[3] = {t0[0] + (cl & 7), t0[1] + ((cl >> 3) & 7), t0[2] + (cl >> 6)};
    const SplatWindow<A> win(G, c, edge);
    f32x2 am[9][2], ap[9][2];
#pragma unroll
    for (int r = 0; r < 9; ++r)
#pragma unroll
      for (int h = 0; h < 2; ++h) am[r][h] = ap[r][h] = 0ull;
    float bmin[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) bmin[b] = 4.0f;
    if (beg < end) {
      if (fast && !edge)
        splat_particles<A, true>(G, win, beg, end, perm, px, py, pz, vA, type, vol, m_l, m_g, inv_dx, inv_dx_f, fast,
                                 edge, am, ap, bmin);
      else
        splat_particles<A, false>(G, win, beg, end, perm, px, py, pz, vA, type, vol, m_l, m_g, inv_dx, inv_dx_f,
                                  fast, edge, am, ap, bmin);
    }
    // this warp's cells into its box (a warp whose cells are all empty adds nothing)
    if (__any_sync(0xffffffffu, beg < end)) {
      const int g = (kSplatThreads / 32) * pass + (tid >> 5);
      const int q = lane >> 3;
      flush_window<A>(wbox + g * kWarpBox, lane & 7, ((q & 1) << 1) | (q >> 1), am, ap);
    }
    // the cell's reached blocks; the FP64 test for a cell with a block in the band
    unsigned reach = 0u;
    bool band = false;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (bmin[b] < 1.0f - kReachEps) reach |= 1u << b;
      band = band || fabsf(bmin[b] - 1.0f) <= kReachEps;
    }
    if (band)
      for (int q2 = beg; q2 < end; ++q2) {
        const int p = perm[q2];
        reach |= exact_reach<A>(G, px[p], py[p], pz[p], win.n, win.sp);
      }
    // window blocks -> the tile's 4x4x4 block box (block of node o -> (o >> 2) - 2*tile - ... )
    const int w0 = (win.n[0] >> 2) - (t0[0] >> 2) + 1, w1 = (win.n[1] >> 2) - (t0[1] >> 2) + 1,
              w2 = (win.n[2] >> 2) - (t0[2] >> 2) + 1;
#pragma unroll
    for (int bb = 0; bb < 8; ++bb)
      if ((reach >> bb) & 1u) box |= 1ull << ((w0 + (bb & 1)) + 4 * ((w1 + ((bb >> 1) & 1)) + 4 * (w2 + (bb >> 2))));
  }
  __syncthreads();
  // warp boxes -> staging box, node by node in warp order (z ascending, then y half)
  float2* st = stage + A * kStageField;
  for (int e = tid; e < FX * FY * FZ; e += kSplatThreads) {
    const int X = e % FX, Y = (e / FX) % FY, Z = e / (FX * FY);
    float2 s = make_float2(0.0f, 0.0f);
    const int zlo = max(0, Z - GZ + 1), zhi = min(7, Z);
    for (int z = zlo; z <= zhi; ++z)
#pragma unroll
      for (int yh = 0; yh < 2; ++yh) {
        const int Yl = Y - 4 * yh;
        if (Yl < 0 || Yl >= GY) continue;
        const float2 v = wbox[(2 * z + yh) * kWarpBox + X + kWarpPitch * (Yl + GY * (Z - z))];
        s.x += v.x;
        s.y += v.y;
      }
    st[e] = s;
  }
  __syncthreads();
  return box;
}

// The tile's 4x4x4 block box: node-block (o >> 2) relative to the tile's first
// 4^3 block minus one, i.e. box index 0 is the block below the tile.
__global__ void __launch_bounds__(kSplatThreads, 3) k_splat(DevGrid G, const int* __restrict__ cell_start,
                                                           int* __restrict__ perm, int* __restrict__ sort_tmp,
                                                           float2* __restrict__ stage,
                                                           const float* __restrict__ px,
                                                           const float* __restrict__ py,
                                                           const float* __restrict__ pz,
                                                           const float* __restrict__ vx,
                                                           const float* __restrict__ vy,
                                                           const float* __restrict__ vz,
                                                           const uint8_t* __restrict__ type,
                                                           const float* __restrict__ vol, float m_l, float m_g) {
  extern __shared__ float2 wbox[];  // [kSplatGroups][kWarpBox]
  __shared__ unsigned sblk[6];      // [3 axes][64 reached blocks of the box]
  __shared__ int nbig;
  __shared__ int big[PF_TV];
  const int t = blockIdx.x;
  const int* cs = cell_start + (size_t)t * PF_TV;
  if (cs[0] >= cs[PF_TV]) return;
  const int tid = threadIdx.x;
  if (tid < 6) sblk[tid] = 0u;
  if (tid == 0) nbig = 0;
  __syncthreads();
  // cells in ascending particle index: small cells in registers, larger ones
  // by ranks counted by the whole CTA
  for (int pass = 0; pass < kSplatPasses; ++pass) {
    const int cl = splat_cell_of(tid, pass);
    const int beg = cs[cl], n = cs[cl + 1] - beg;
    if (n <= 1) continue;
    if (n <= 8) sort_segment<8>(perm, beg, n);
    else if (n <= 16) sort_segment<16>(perm, beg, n);
    else big[atomicAdd(&nbig, 1)] = cl;
  }
  __syncthreads();
  for (int b = 0; b < nbig; ++b) {
    const int cl = big[b];
    const int beg = cs[cl], n = cs[cl + 1] - beg;
    int* sv = reinterpret_cast<int*>(wbox);
    const bool staged = n <= kBigSortStage;
    if (staged)
      for (int i = tid; i < n; i += kSplatThreads) sv[i] = perm[beg + i];
    __syncthreads();
    for (int i = tid; i < n; i += kSplatThreads) {
      const int v = staged ? sv[i] : perm[beg + i];
      int r = 0;
      if (staged)
        for (int j = 0; j < n; ++j) r += sv[j] < v;
      else
        for (int j = 0; j < n; ++j) r += perm[beg + j] < v;
      sort_tmp[beg + r] = v;
    }
    __syncthreads();
    for (int i = tid; i < n; i += kSplatThreads) perm[beg + i] = sort_tmp[beg + i];
    __syncthreads();
  }
  const int tx = t % G.g.TX, tq = t / G.g.TX, ty = tq % G.g.TY, tz = tq / G.g.TY;
  const int t0[3] = {tx * 8, ty * 8, tz * 8};
  const double inv_dx = G.g.inv_dx;
  const float inv_dx_f = (float)inv_dx;
  const bool fast = G.g.dx_pow2 && G.g.ox == 0.0 && G.g.oy == 0.0 && G.g.oz == 0.0;
  // window nodes of this tile's cells span global nodes 8t - 1 .. 8t + 9 per axis
  const bool edge = tx == 0 || ty == 0 || tz == 0 || tx * 8 + 10 > G.g.nx || ty * 8 + 10 > G.g.ny ||
                    tz * 8 + 10 > G.g.nz;
  float2* st = stage + (size_t)t * kStageTile;
  unsigned long long box[3];
  box[0] = splat_field<0>(G, wbox, st, cs, perm, px, py, pz, vx, type, vol, m_l, m_g, t0, inv_dx, inv_dx_f, fast,
                          edge);
  box[1] = splat_field<1>(G, wbox, st, cs, perm, px, py, pz, vy, type, vol, m_l, m_g, t0, inv_dx, inv_dx_f, fast,
                          edge);
  box[2] = splat_field<2>(G, wbox, st, cs, perm, px, py, pz, vz, type, vol, m_l, m_g, t0, inv_dx, inv_dx_f, fast,
                          edge);
  // one shared OR per warp and word
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)box[a]);
    const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(box[a] >> 32));
    if ((tid & 31) == 0) {
      if (lo) atomicOr(&sblk[2 * a], lo);
      if (hi) atomicOr(&sblk[2 * a + 1], hi);
    }
  }
  __syncthreads();
  // activity bytes of the reached blocks (a byte is stored only when it reads 0)
  for (int e = tid; e < 3 * 64; e += kSplatThreads) {
    const int a = e >> 6, idx = e & 63;
    if ((sblk[2 * a + (idx >> 5)] >> (idx & 31)) & 1u) {
      const int fv = PF_U + a;
      const int gbx = 2 * tx - 1 + (idx & 3), gby = 2 * ty - 1 + ((idx >> 2) & 3), gbz = 2 * tz - 1 + (idx >> 4);
      const int bi = gbx + G.g.bdim[fv][0] * (gby + G.g.bdim[fv][1] * gbz);
      if (!G.act4[fv][bi]) G.act4[fv][bi] = 1;
      if (!G.act4[fv + 3][bi]) G.act4[fv + 3][bi] = 1;
    }
  }
}

// The tiles whose cells reach local node l (0..7) of a tile along one axis,
// in ascending offset, with the node's index in each one's staging box: along
// the normal axis a node takes cells l-2..l+1, along a transverse axis
// l-1..l+1, so it has one or two such tiles.  Returns their number.
__device__ __forceinline__ int stage_axis(int l, bool normal, int (&off)[2], int (&idx)[2]) {
  const bool lo = normal ? l <= 1 : l == 0;  // the tile below reaches it
  const bool hi = l == 7;                     // the tile above reaches it
  off[0] = lo ? -1 : 0;
  idx[0] = lo ? l + 9 : l + 1;
  off[1] = lo ? 0 : 1;
  idx[1] = lo ? l + 1 : 0;
  return lo || hi ? 2 : 1;
}

// normalisation u = P/m where m > 0 (sparse_ops3d_tp.cpp:126-152), with the
// optional saved copy (step(): `saved = grid`) and gravity on v where mv > 0
// (applyGravity) fused in.  With `gather` the momentum and raw mass of every
// node are first summed from the staging boxes of the splatted tiles that
// reach it, in ascending tile offset (z, then y, then x).
// Nodes of blocks the exact activation left inactive are cleared: the splat's
// FP32 weights may put a negligible contribution where the reference's FP64
// weight is zero, and inactive blocks stay zero.
__global__ void __launch_bounds__(PF_TV, 4) k_normalize(DevGrid G, const float2* __restrict__ stage, const int* __restrict__ cell_start,
                            int gather, const int* __restrict__ d_nslots, int save, int gravity, float dv) {
  __shared__ int splatted[27];
  const int nslots = *d_nslots;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const int t = G.slot_tile[s];
    const int tx = t % G.g.TX, tq = t / G.g.TX, ty = tq % G.g.TY, tz = tq / G.g.TY;
    if (gather) {
      __syncthreads();
      if (threadIdx.x < 27) {
        const int x = tx + (int)threadIdx.x % 3 - 1, y = ty + ((int)threadIdx.x / 3) % 3 - 1,
                  z = tz + (int)threadIdx.x / 9 - 1;
        int ok = 0;
        if (x >= 0 && y >= 0 && z >= 0 && x < G.g.TX && y < G.g.TY && z < G.g.TZ) {
          const size_t nt = (size_t)tile_id(G.g, x, y, z) * PF_TV;
          ok = cell_start[nt] < cell_start[nt + PF_TV];
        }
        splatted[threadIdx.x] = ok;
      }
      __syncthreads();
    }
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    const int i = tx * 8 + li, j = ty * 8 + lj, k = tz * 8 + lk;
    // every load of the three fields first, then the stores (the stores may
    // alias the field arrays, so interleaving them would serialise the loads)
    float m[3], u[3];
    bool act[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int f = PF_MU + a;
      act[a] = in_field(G.g, f, i, j, k) && G.act4[f][act4_index(G.g, f, i, j, k)];
      m[a] = u[a] = 0.0f;
      if (gather) {
        const int FX = a == 0 ? 11 : 10, FY = a == 1 ? 11 : 10;
        int ox[2], oy[2], oz[2], ix[2], iy[2], iz[2];
        const int nx = stage_axis(li, a == 0, ox, ix), ny = stage_axis(lj, a == 1, oy, iy),
                  nz = stage_axis(lk, a == 2, oz, iz);
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int d = 0; d < 2; ++d) {
              if (c >= nz || b >= ny || d >= nx) continue;
              if (!splatted[(ox[d] + 1) + 3 * ((oy[b] + 1) + 3 * (oz[c] + 1))]) continue;
              const int tn = tile_id(G.g, tx + ox[d], ty + oy[b], tz + oz[c]);
              const float2 v = stage[(size_t)tn * kStageTile + a * kStageField + ix[d] + FX * (iy[b] + FY * iz[c])];
              u[a] += v.x;
              m[a] += v.y;
            }
      } else {
        m[a] = G.fld[f][o];
        u[a] = G.fld[PF_U + a][o];
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float mm = act[a] ? m[a] : 0.0f, uu = act[a] ? u[a] : 0.0f;
      G.fld[PF_MU + a][o] = mm;
      if (mm > 0.0f) uu = uu / mm;
      if (save) G.saved[a][o] = uu;
      if (a == 1 && gravity && mm > 0.0f) uu = uu + dv;
      G.fld[PF_U + a][o] = uu;
    }
  }
}

__global__ void k_save(DevGrid G, const int* __restrict__ d_nslots) {
  const int nslots = *d_nslots;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
#pragma unroll
    for (int a = 0; a < 3; ++a) G.saved[a][o] = G.fld[PF_U + a][o];
  }
}

__global__ void k_gravity(DevGrid G, const int* __restrict__ d_nslots, float dv) {
  const int nslots = *d_nslots;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (G.fld[PF_MV][o] > 0.0f) {
      G.fld[PF_V][o] = G.fld[PF_V][o] + dv;
      const int t = G.slot_tile[s];
      const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
      const int l = threadIdx.x;
      activate4(G, PF_V, tx * 8 + (l & 7), ty * 8 + ((l >> 3) & 7), tz * 8 + (l >> 6));
    }
  }
}

// applyWallBoundary: zero two face layers at every wall
__global__ void k_walls(DevGrid G) {
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  const long long nu = 4LL * ny * nz, nv = 4LL * nx * nz, nw = 4LL * nx * ny;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nu + nv + nw;
       q += (long long)gridDim.x * blockDim.x) {
    int f, i, j, k;
    if (q < nu) {
      const int s = (int)(q & 3); const long long r = q >> 2;
      j = (int)(r % ny); k = (int)(r / ny);
      i = s == 0 ? 0 : s == 1 ? 1 : s == 2 ? nx - 1 : nx;
      f = PF_U;
    } else if (q < nu + nv) {
      const long long qq = q - nu; const int s = (int)(qq & 3); const long long r = qq >> 2;
      i = (int)(r % nx); k = (int)(r / nx);
      j = s == 0 ? 0 : s == 1 ? 1 : s == 2 ? ny - 1 : ny;
      f = PF_V;
    } else {
      const long long qq = q - nu - nv; const int s = (int)(qq & 3); const long long r = qq >> 2;
      i = (int)(r % nx); j = (int)(r / nx);
      k = s == 0 ? 0 : s == 1 ? 1 : s == 2 ? nz - 1 : nz;
      f = PF_W;
    }
    if (!in_field(G.g, f, i, j, k)) continue;
    const int sl = slot_of(G, i, j, k);
    if (sl < 0) continue;  // unreachable: wall tiles are pooled first
    G.fld[f][(size_t)sl * PF_TV + local_id(i, j, k)] = 0.0f;
    activate4(G, f, i, j, k);
  }
}

// ---------------------------------------------------------------------------
// G2P / advection
// ---------------------------------------------------------------------------

// Clamped trilinear sample of face field `a` at grid coordinate (cx,cy,cz),
// current and (optionally) saved values from the same nodes.
template <bool kSaved>
__device__ __forceinline__ void sample2(const DevGrid& G, int a, double cx, double cy, double cz,
                                        float& cur, float& old) {
  const int fv = PF_U + a;
  const int X = G.g.fdim[fv][0], Y = G.g.fdim[fv][1], Z = G.g.fdim[fv][2];
  const int i0 = (int)floor(cx), j0 = (int)floor(cy), k0 = (int)floor(cz);
  const float fx = (float)(cx - i0), fy = (float)(cy - j0), fz = (float)(cz - k0);
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  float s = 0.0f, so = 0.0f;
  // common case: all eight nodes inside the lattice and inside one tile
  if (i0 >= 0 && j0 >= 0 && k0 >= 0 && i0 + 1 < X && j0 + 1 < Y && k0 + 1 < Z && (i0 & 7) != 7 &&
      (j0 & 7) != 7 && (k0 & 7) != 7) {
    const int sl = slot_of(G, i0, j0, k0);
    if (sl < 0) {
      cur = 0.0f;
      old = 0.0f;
      return;
    }
    const float* f = G.fld[fv] + (size_t)sl * PF_TV + local_id(i0, j0, k0);
    const float* h = G.saved[a] + (size_t)sl * PF_TV + local_id(i0, j0, k0);
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const int off = di + 8 * dj + 64 * dk;
          const float w = wx[di] * wy[dj] * wz[dk];
          s += w * __ldg(f + off);
          if (kSaved) so += w * __ldg(h + off);
        }
    cur = s;
    old = so;
    return;
  }
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        const int i = min(max(i0 + di, 0), X - 1);
        const int j = min(max(j0 + dj, 0), Y - 1);
        const int k = min(max(k0 + dk, 0), Z - 1);
        const int sl = slot_of(G, i, j, k);
        const float w = wx[di] * wy[dj] * wz[dk];
        if (sl >= 0) {
          const size_t o = (size_t)sl * PF_TV + local_id(i, j, k);
          s += w * G.fld[fv][o];
          if (kSaved) so += w * G.saved[a][o];
        }
      }
  cur = s;
  old = so;
}

__device__ __forceinline__ float sample1(const DevGrid& G, int a, double cx, double cy, double cz) {
  float c, o;
  sample2<false>(G, a, cx, cy, cz, c, o);
  return c;
}

// (pos - o) / dx as a product with the reciprocal: G2P and advection only need
// it to within rounding, unlike the activation test.
__device__ __forceinline__ double to_grid(double p, double o, double inv_dx) { return (p - o) * inv_dx; }

__device__ __forceinline__ void velocity_at(const DevGrid& G, double x, double y, double z, double out[3]) {
  const double inv_dx = G.g.inv_dx;
  const double gx = to_grid(x, G.g.ox, inv_dx);
  const double gy = to_grid(y, G.g.oy, inv_dx);
  const double gz = to_grid(z, G.g.oz, inv_dx);
  out[0] = sample1(G, 0, gx, gy - 0.5, gz - 0.5);
  out[1] = sample1(G, 1, gx - 0.5, gy, gz - 0.5);
  out[2] = sample1(G, 2, gx - 0.5, gy - 0.5, gz);
}

struct ParticlePtrs {
  float *px, *py, *pz, *vx, *vy, *vz, *vol;
  const uint8_t* type;
};

// FLIP/PIC blend; saved grid either this pool's saved copy (S == nullptr
// semantics via kExternal=false) or another context's u/v/w.
template <bool kExternal>
__global__ void __launch_bounds__(256) k_g2p(DevGrid G, DevGrid S, ParticlePtrs P, int n, double aL, double aG) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double gx = to_grid((double)P.px[p], G.g.ox, G.g.inv_dx);
  const double gy = to_grid((double)P.py[p], G.g.oy, G.g.inv_dx);
  const double gz = to_grid((double)P.pz[p], G.g.oz, G.g.inv_dx);
  const double c[3][3] = {{gx, gy - 0.5, gz - 0.5}, {gx - 0.5, gy, gz - 0.5}, {gx - 0.5, gy - 0.5, gz}};
  const float a = P.type[p] == 0 ? (float)aL : (float)aG;
  float* vp[3] = {P.vx, P.vy, P.vz};
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    float cur, old;
    if (kExternal) {
      cur = sample1(G, ax, c[ax][0], c[ax][1], c[ax][2]);
      old = sample1(S, ax, c[ax][0], c[ax][1], c[ax][2]);
    } else {
      sample2<true>(G, ax, c[ax][0], c[ax][1], c[ax][2], cur, old);
    }
    const float v = vp[ax][p];
    vp[ax][p] = (v + (cur - old)) * a + cur * (1.0f - a);
  }
}

// G2P over the P2G bins (particles have not moved since the binning): one
// CTA per tile with particles stages the current and saved u, v, w of the
// tile's nodes and a one-node halo -- 10^3 nodes per field, node indices
// clamped to the field lattice exactly as sample2 clamps them -- in shared
// memory, then samples its particles from there.  A particle whose stencil
// leaves the box (a position outside the domain) takes sample2.
constexpr int kG2PBox = 10;
constexpr int kG2PBox3 = kG2PBox * kG2PBox * kG2PBox;

__global__ void __launch_bounds__(256) k_g2p_tiles(DevGrid G, const int* __restrict__ cell_start,
                                                   const int* __restrict__ perm, ParticlePtrs P, double aL,
                                                   double aG) {
  __shared__ float2 box[3][kG2PBox3];  // (current, saved)
  const int t = blockIdx.x;
  const int beg = cell_start[(size_t)t * PF_TV], end = cell_start[(size_t)(t + 1) * PF_TV];
  if (beg >= end) return;
  const int tx = t % G.g.TX, tq = t / G.g.TX, ty = tq % G.g.TY, tz = tq / G.g.TY;
  const int b0 = tx * 8 - 1, b1 = ty * 8 - 1, b2 = tz * 8 - 1;
  // the pool slots of the 27 tiles around this one: the box's nodes (clamped
  // to the lattice) lie in them, so each node needs no tile-map load of its own
  __shared__ int nslot[27];
  if (threadIdx.x < 27) {
    const int x = tx + (int)threadIdx.x % 3 - 1, y = ty + ((int)threadIdx.x / 3) % 3 - 1, z = tz + (int)threadIdx.x / 9 - 1;
    nslot[threadIdx.x] = (x >= 0 && y >= 0 && z >= 0 && x < G.g.TX && y < G.g.TY && z < G.g.TZ)
                             ? G.tile_slot[tile_id(G.g, x, y, z)]
                             : -1;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * kG2PBox3; e += blockDim.x) {
    const int a = e / kG2PBox3, s = e - a * kG2PBox3;
    const int fv = PF_U + a;
    const int i = min(max(b0 + s % kG2PBox, 0), G.g.fdim[fv][0] - 1);
    const int j = min(max(b1 + (s / kG2PBox) % kG2PBox, 0), G.g.fdim[fv][1] - 1);
    const int k = min(max(b2 + s / (kG2PBox * kG2PBox), 0), G.g.fdim[fv][2] - 1);
    const int sl = nslot[((i >> 3) - tx + 1) + 3 * (((j >> 3) - ty + 1) + 3 * ((k >> 3) - tz + 1))];
    float2 v = make_float2(0.0f, 0.0f);
    if (sl >= 0) {
      const size_t o = (size_t)sl * PF_TV + local_id(i, j, k);
      v = make_float2(G.fld[fv][o], G.saved[a][o]);
    }
    box[a][s] = v;
  }
  __syncthreads();
  float* vp[3] = {P.vx, P.vy, P.vz};
  const bool fast = G.g.dx_pow2 && G.g.ox == 0.0 && G.g.oy == 0.0 && G.g.oz == 0.0;
  const float inv_dx_f = (float)G.g.inv_dx;
  // the next particle's attributes are loaded while this one is sampled
  int q = beg + threadIdx.x;
  int pn = 0;
  float xn = 0.0f, yn = 0.0f, zn = 0.0f, vn[3] = {0.0f, 0.0f, 0.0f};
  uint8_t tn = 0;
  if (q < end) {
    pn = perm[q];
    xn = P.px[pn]; yn = P.py[pn]; zn = P.pz[pn]; tn = P.type[pn];
    vn[0] = P.vx[pn]; vn[1] = P.vy[pn]; vn[2] = P.vz[pn];
  }
  for (; q < end; q += blockDim.x) {
    const int p = pn;
    const float X = xn, Y = yn, Z = zn, v0[3] = {vn[0], vn[1], vn[2]};
    const uint8_t ty = tn;
    if (q + (int)blockDim.x < end) {
      pn = perm[q + blockDim.x];
      xn = P.px[pn]; yn = P.py[pn]; zn = P.pz[pn]; tn = P.type[pn];
      vn[0] = P.vx[pn]; vn[1] = P.vy[pn]; vn[2] = P.vz[pn];
    }
    // grid coordinates; with a power-of-two dx and a zero origin the FP32
    // product with 1/dx, its half-shifts, floors and fractions are exact and
    // equal the FP64 ones
    float gf[3];
    double gd[3];
    if (fast) {
      gf[0] = X * inv_dx_f;
      gf[1] = Y * inv_dx_f;
      gf[2] = Z * inv_dx_f;
    } else {
      gd[0] = to_grid((double)X, G.g.ox, G.g.inv_dx);
      gd[1] = to_grid((double)Y, G.g.oy, G.g.inv_dx);
      gd[2] = to_grid((double)Z, G.g.oz, G.g.inv_dx);
    }
    const float al = ty == 0 ? (float)aL : (float)aG;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      int n0[3];
      float fr[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (fast) {
          const float c = d == ax ? gf[d] : gf[d] - 0.5f;
          n0[d] = (int)floorf(c);
          fr[d] = c - (float)n0[d];
        } else {
          const double c = d == ax ? gd[d] : gd[d] - 0.5;
          n0[d] = (int)floor(c);
          fr[d] = (float)(c - n0[d]);
        }
      }
      const int li = n0[0] - b0, lj = n0[1] - b1, lk = n0[2] - b2;
      float cur, old;
      if (li >= 0 && lj >= 0 && lk >= 0 && li < kG2PBox - 1 && lj < kG2PBox - 1 && lk < kG2PBox - 1) {
        const float fx = fr[0], fy = fr[1], fz = fr[2];
        const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
        const float2* bp = &box[ax][li + kG2PBox * (lj + kG2PBox * lk)];
        float s = 0.0f, so = 0.0f;
#pragma unroll
        for (int dk = 0; dk < 2; ++dk)
#pragma unroll
          for (int dj = 0; dj < 2; ++dj)
#pragma unroll
            for (int di = 0; di < 2; ++di) {
              const float w = wx[di] * wy[dj] * wz[dk];
              const float2 v = bp[di + kG2PBox * (dj + kG2PBox * dk)];
              s += w * v.x;
              so += w * v.y;
            }
        cur = s;
        old = so;
      } else {
        double c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double g = fast ? (double)gf[d] : gd[d];
          c[d] = d == ax ? g : g - 0.5;
        }
        sample2<true>(G, ax, c[0], c[1], c[2], cur, old);
      }
      vp[ax][p] = (v0[ax] + (cur - old)) * al + cur * (1.0f - al);
    }
  }
}

__device__ __forceinline__ void warp_count(int* counters, int idx, bool flag) {
  const unsigned m = __ballot_sync(__activemask(), flag);
  if (m && (threadIdx.x & 31) == (__ffs(__activemask()) - 1)) atomicAdd(&counters[idx], __popc(m));
}

// RK2 (midpoint) or RK3 advection, boundary clamp, clamp statistics; with
// fuse_g2p the FLIP/PIC update uses the first stage's samples.
__global__ void __launch_bounds__(256) k_advect(DevGrid G, ParticlePtrs P, int n, double dt, int order,
                                                int* counters, int* esc_flags, int fuse_g2p, double aL,
                                                double aG) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  bool low[3] = {false, false, false}, high[3] = {false, false, false};
  int ty = -1;
  if (live) {
    const double x0[3] = {(double)P.px[p], (double)P.py[p], (double)P.pz[p]};
    double k1[3], k2[3], nx[3];
    if (fuse_g2p) {
      const double gx = to_grid(x0[0], G.g.ox, G.g.inv_dx);
      const double gy = to_grid(x0[1], G.g.oy, G.g.inv_dx);
      const double gz = to_grid(x0[2], G.g.oz, G.g.inv_dx);
      const double c[3][3] = {{gx, gy - 0.5, gz - 0.5}, {gx - 0.5, gy, gz - 0.5}, {gx - 0.5, gy - 0.5, gz}};
      const float a = P.type[p] == 0 ? (float)aL : (float)aG;
      float* vp[3] = {P.vx, P.vy, P.vz};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        float cur, old;
        sample2<true>(G, ax, c[ax][0], c[ax][1], c[ax][2], cur, old);
        k1[ax] = cur;
        const float v = vp[ax][p];
        vp[ax][p] = (v + (cur - old)) * a + cur * (1.0f - a);
      }
    } else {
      velocity_at(G, x0[0], x0[1], x0[2], k1);
    }
    if (order == 3) {
      double m1[3], m2[3], k3[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) m1[c] = x0[c] + k1[c] * (0.5 * dt);
      velocity_at(G, m1[0], m1[1], m1[2], k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) m2[c] = (x0[c] - k1[c] * dt) + k2[c] * (2.0 * dt);
      velocity_at(G, m2[0], m2[1], m2[2], k3);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + ((k1[c] + k2[c] * 4.0) + k3[c]) * (dt / 6.0);
    } else {
      double mid[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) mid[c] = x0[c] + k1[c] * (0.5 * dt);
      velocity_at(G, mid[0], mid[1], mid[2], k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + k2[c] * dt;
    }
    const double lo[3] = {G.g.ox + 0.5 * G.g.dx, G.g.oy + 0.5 * G.g.dx, G.g.oz + 0.5 * G.g.dx};
    const double hi[3] = {G.g.ox + (G.g.nx - 0.5) * G.g.dx, G.g.oy + (G.g.ny - 0.5) * G.g.dx,
                          G.g.oz + (G.g.nz - 0.5) * G.g.dx};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      low[c] = nx[c] < lo[c];
      high[c] = nx[c] > hi[c];
      nx[c] = fmax(lo[c], fmin(hi[c], nx[c]));
    }
    P.px[p] = (float)nx[0];
    P.py[p] = (float)nx[1];
    P.pz[p] = (float)nx[2];
    ty = P.type[p];
  }
  const bool clamped = low[0] || high[0] || low[1] || high[1] || low[2] || high[2];
  if (esc_flags && live) esc_flags[p] = clamped ? 1 : 0;
  warp_count(counters, 0, clamped && ty == 0);
  warp_count(counters, 1, clamped && ty == 1);
  warp_count(counters, 2, low[0]);
  warp_count(counters, 3, high[0]);
  warp_count(counters, 4, low[1]);
  warp_count(counters, 5, high[1]);
  warp_count(counters, 6, low[2]);
  warp_count(counters, 7, high[2]);
}

// The last pass of the step over the P2G bins (the particles have not moved
// since the binning): one CTA per tile with particles stages the current and
// saved u, v, w on the tile's nodes with a two-node halo -- 12^3 nodes per
// field, node indices clamped to the field lattice exactly as sample2 clamps
// them -- then, per particle, blends the FLIP/PIC velocity from the first
// stage's samples and takes the RK2 (or RK3) stages from the same box.  A
// sample whose stencil leaves the box (a midpoint more than a cell outside the
// tile, or a position outside the domain) takes the global path.  Every value
// equals k_advect's: the same clamped nodes, weights and summation order.
constexpr int kAdvBox = 12;
constexpr int kAdvBox3 = kAdvBox * kAdvBox * kAdvBox;

// trilinear sample of box field `a` whose stencil origin is (li, lj, lk) in
// box coordinates, with FP32 fractions
template <bool kOld>
__device__ __forceinline__ void box_tri(const float2 (*box)[kAdvBox3], int a, int li, int lj, int lk, float fx,
                                        float fy, float fz, float& cur, float& old) {
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  const float2* bp = &box[a][li + kAdvBox * (lj + kAdvBox * lk)];
  float s = 0.0f, so = 0.0f;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        const float w = wx[di] * wy[dj] * wz[dk];
        const float2 v = bp[di + kAdvBox * (dj + kAdvBox * dk)];
        s += w * v.x;
        if (kOld) so += w * v.y;
      }
  cur = s;
  old = so;
}

// velocity_at from the box where the stencils fit
__device__ __forceinline__ void box_velocity(const DevGrid& G, const float2 (*box)[kAdvBox3], int b0, int b1, int b2,
                                             double x, double y, double z, double out[3]) {
  const double g[3] = {to_grid(x, G.g.ox, G.g.inv_dx), to_grid(y, G.g.oy, G.g.inv_dx),
                       to_grid(z, G.g.oz, G.g.inv_dx)};
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    double c[3];
    int n0[3];
    float fr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      c[d] = d == ax ? g[d] : g[d] - 0.5;
      n0[d] = (int)floor(c[d]);
      fr[d] = (float)(c[d] - n0[d]);
    }
    const int li = n0[0] - b0, lj = n0[1] - b1, lk = n0[2] - b2;
    float cur, old;
    if ((unsigned)li < kAdvBox - 1 && (unsigned)lj < kAdvBox - 1 && (unsigned)lk < kAdvBox - 1)
      box_tri<false>(box, ax, li, lj, lk, fr[0], fr[1], fr[2], cur, old);
    else
      sample2<false>(G, ax, c[0], c[1], c[2], cur, old);
    out[ax] = cur;
  }
}

__global__ void __launch_bounds__(256, 3) k_g2p_advect_tiles(DevGrid G, const int* __restrict__ cell_start,
                                                          const int* __restrict__ perm, ParticlePtrs P, double dt,
                                                          int order, double aL, double aG, int* counters) {
  __shared__ float2 box[3][kAdvBox3];  // (current, saved)
  __shared__ int nslot[27];
  __shared__ int tally[8];
  const int t = blockIdx.x;
  const int beg = cell_start[(size_t)t * PF_TV], end = cell_start[(size_t)(t + 1) * PF_TV];
  if (beg >= end) return;
  const int tx = t % G.g.TX, tq = t / G.g.TX, ty = tq % G.g.TY, tz = tq / G.g.TY;
  const int b0 = tx * 8 - 2, b1 = ty * 8 - 2, b2 = tz * 8 - 2;
  if (threadIdx.x < 27) {
    const int x = tx + (int)threadIdx.x % 3 - 1, y = ty + ((int)threadIdx.x / 3) % 3 - 1, z = tz + (int)threadIdx.x / 9 - 1;
    nslot[threadIdx.x] = (x >= 0 && y >= 0 && z >= 0 && x < G.g.TX && y < G.g.TY && z < G.g.TZ)
                             ? G.tile_slot[tile_id(G.g, x, y, z)]
                             : -1;
  }
  if (threadIdx.x < 8) tally[threadIdx.x] = 0;
  __syncthreads();
  // the box spans nodes [8t - 2, 8t + 10) per axis; clamped into the lattice
  // they lie in tiles t-1 .. t+1
  for (int e = threadIdx.x; e < 3 * kAdvBox3; e += blockDim.x) {
    const int a = e / kAdvBox3, s = e - a * kAdvBox3;
    const int fv = PF_U + a;
    const int i = min(max(b0 + s % kAdvBox, 0), G.g.fdim[fv][0] - 1);
    const int j = min(max(b1 + (s / kAdvBox) % kAdvBox, 0), G.g.fdim[fv][1] - 1);
    const int k = min(max(b2 + s / (kAdvBox * kAdvBox), 0), G.g.fdim[fv][2] - 1);
    const int sl = nslot[((i >> 3) - tx + 1) + 3 * (((j >> 3) - ty + 1) + 3 * ((k >> 3) - tz + 1))];
    float2 v = make_float2(0.0f, 0.0f);
    if (sl >= 0) {
      const size_t o = (size_t)sl * PF_TV + local_id(i, j, k);
      v = make_float2(G.fld[fv][o], G.saved[a][o]);
    }
    box[a][s] = v;
  }
  __syncthreads();
  float* vp[3] = {P.vx, P.vy, P.vz};
  float* pp[3] = {P.px, P.py, P.pz};
  const bool fast = G.g.dx_pow2 && G.g.ox == 0.0 && G.g.oy == 0.0 && G.g.oz == 0.0;
  const float inv_dx_f = (float)G.g.inv_dx;
  const double lo[3] = {G.g.ox + 0.5 * G.g.dx, G.g.oy + 0.5 * G.g.dx, G.g.oz + 0.5 * G.g.dx};
  const double hi[3] = {G.g.ox + (G.g.nx - 0.5) * G.g.dx, G.g.oy + (G.g.ny - 0.5) * G.g.dx,
                        G.g.oz + (G.g.nz - 0.5) * G.g.dx};
  unsigned cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int q = beg + threadIdx.x;
  int pn = 0;
  float xn = 0.0f, yn = 0.0f, zn = 0.0f, vn[3] = {0.0f, 0.0f, 0.0f};
  uint8_t tn = 0;
  if (q < end) {
    pn = perm[q];
    xn = P.px[pn]; yn = P.py[pn]; zn = P.pz[pn]; tn = P.type[pn];
    vn[0] = P.vx[pn]; vn[1] = P.vy[pn]; vn[2] = P.vz[pn];
  }
  for (; q < end; q += blockDim.x) {
    const int p = pn;
    const float X = xn, Y = yn, Z = zn, v0[3] = {vn[0], vn[1], vn[2]};
    const uint8_t ptype = tn;
    if (q + (int)blockDim.x < end) {
      pn = perm[q + blockDim.x];
      xn = P.px[pn]; yn = P.py[pn]; zn = P.pz[pn]; tn = P.type[pn];
      vn[0] = P.vx[pn]; vn[1] = P.vy[pn]; vn[2] = P.vz[pn];
    }
    // stage 1: current and saved samples at the particle (see k_g2p_tiles for
    // the exact FP32 coordinates)
    float gf[3];
    double gd[3];
    if (fast) {
      gf[0] = X * inv_dx_f;
      gf[1] = Y * inv_dx_f;
      gf[2] = Z * inv_dx_f;
    } else {
      gd[0] = to_grid((double)X, G.g.ox, G.g.inv_dx);
      gd[1] = to_grid((double)Y, G.g.oy, G.g.inv_dx);
      gd[2] = to_grid((double)Z, G.g.oz, G.g.inv_dx);
    }
    const float al = ptype == 0 ? (float)aL : (float)aG;
    double k1[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      int n0[3];
      float fr[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (fast) {
          const float c = d == ax ? gf[d] : gf[d] - 0.5f;
          n0[d] = (int)floorf(c);
          fr[d] = c - (float)n0[d];
        } else {
          const double c = d == ax ? gd[d] : gd[d] - 0.5;
          n0[d] = (int)floor(c);
          fr[d] = (float)(c - n0[d]);
        }
      }
      const int li = n0[0] - b0, lj = n0[1] - b1, lk = n0[2] - b2;
      float cur, old;
      if ((unsigned)li < kAdvBox - 1 && (unsigned)lj < kAdvBox - 1 && (unsigned)lk < kAdvBox - 1) {
        box_tri<true>(box, ax, li, lj, lk, fr[0], fr[1], fr[2], cur, old);
      } else {
        double c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double g = fast ? (double)gf[d] : gd[d];
          c[d] = d == ax ? g : g - 0.5;
        }
        sample2<true>(G, ax, c[0], c[1], c[2], cur, old);
      }
      k1[ax] = cur;
      vp[ax][p] = (v0[ax] + (cur - old)) * al + cur * (1.0f - al);
    }
    // the remaining stages, in k_advect's arithmetic
    const double x0[3] = {(double)X, (double)Y, (double)Z};
    double k2[3], nx[3];
    if (order == 3) {
      double m1[3], m2[3], k3[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) m1[c] = x0[c] + k1[c] * (0.5 * dt);
      box_velocity(G, box, b0, b1, b2, m1[0], m1[1], m1[2], k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) m2[c] = (x0[c] - k1[c] * dt) + k2[c] * (2.0 * dt);
      box_velocity(G, box, b0, b1, b2, m2[0], m2[1], m2[2], k3);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + ((k1[c] + k2[c] * 4.0) + k3[c]) * (dt / 6.0);
    } else {
      double mid[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) mid[c] = x0[c] + k1[c] * (0.5 * dt);
      box_velocity(G, box, b0, b1, b2, mid[0], mid[1], mid[2], k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + k2[c] * dt;
    }
    bool any = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool l = nx[c] < lo[c], h = nx[c] > hi[c];
      cnt[2 + 2 * c] += l;
      cnt[3 + 2 * c] += h;
      any = any || l || h;
      pp[c][p] = (float)fmax(lo[c], fmin(hi[c], nx[c]));
    }
    cnt[0] += any && ptype == 0;
    cnt[1] += any && ptype == 1;
  }
  // clamp statistics: one atomic per counter and CTA
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const unsigned w = __reduce_add_sync(0xffffffffu, cnt[c]);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&tally[c], (int)w);
  }
  __syncthreads();
  if (threadIdx.x < 8 && tally[threadIdx.x]) atomicAdd(&counters[threadIdx.x], tally[threadIdx.x]);
}

__global__ void k_escape_records(ParticlePtrs P, const int* flags, const int* pos, int n, double* out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || !flags[p]) return;
  double* r = out + 8 * (size_t)pos[p];
  r[0] = P.type[p];
  r[1] = P.px[p]; r[2] = P.py[p]; r[3] = P.pz[p];
  r[4] = P.vx[p]; r[5] = P.vy[p]; r[6] = P.vz[p];
  r[7] = P.vol[p];
}

// calibrateRhoTilde0: each of the 4096 lattice particles computes its
// normalised-weight contribution to u-face (4,4,4) in the reference's FP64
// order; one thread then sums them in particle order.
__device__ double cubic_d(double d2) {
  const double q = __ddiv_rn(d2, kR2);
  const double t = __dsub_rn(1.0, q);
  return t > 0.0 ? __dmul_rn(__dmul_rn(t, t), t) : 0.0;
}

__global__ void k_calib_contrib(double mp, double* contrib) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4096) return;
  const int s = q & 7, cell = q >> 3;
  const int i = cell & 7, j = (cell >> 3) & 7, k = cell >> 6;
  const double x = __dadd_rn(__dadd_rn((double)i, 0.25), __dmul_rn(0.5, (double)(s & 1)));
  const double y = __dadd_rn(__dadd_rn((double)j, 0.25), __dmul_rn(0.5, (double)((s >> 1) & 1)));
  const double z = __dadd_rn(__dadd_rn((double)k, 0.25), __dmul_rn(0.5, (double)((s >> 2) & 1)));
  const double gx = x, gy = __dsub_rn(y, 0.5), gz = __dsub_rn(z, 0.5);
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  double wsum = 0.0, w444 = 0.0;
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= 9 || b < 0 || b >= 8 || c < 0 || c >= 8) continue;
        const double ex = __dsub_rn(gx, (double)a), ey = __dsub_rn(gy, (double)b), ez = __dsub_rn(gz, (double)c);
        const double wv = cubic_d(__dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez)));
        wsum = __dadd_rn(wsum, wv);
        if (a == 4 && b == 4 && c == 4) w444 = wv;
      }
  double v = 0.0;
  if (wsum > 0.0) {
    const double w = __ddiv_rn(w444, wsum);
    if (w > 0.0) v = __dmul_rn(w, mp);
  }
  contrib[q] = v;
}

__global__ void k_calib_sum(const double* contrib, double rho_l, double* out) {
  double s = 0.0;
  for (int q = 0; q < 4096; ++q) s = __dadd_rn(s, contrib[q]);
  *out = s > 0.0 ? __ddiv_rn(s, rho_l) : 1.0;
}

ParticlePtrs particle_ptrs(pf_ctx* ctx) {
  return ParticlePtrs{ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->vol, ctx->type};
}

int slot_grid(const pf_ctx* ctx) { return slot_blocks(ctx, 16 * ctx->num_sms); }

// the pool may hold slots (its size is then on the device only)
bool pool_nonempty(const pf_ctx* ctx) { return ctx->pool_pending || ctx->nslots > 0; }

}  // namespace

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------

int mark_cells(pf_ctx* ctx) {
  StageScope stage(ctx, PF_STAGE_MARK);
  int rc = field_clear(ctx, PF_MK);
  if (rc) return rc;
  const int n = (int)ctx->np;
  DevGrid G = dev_grid(ctx);
  // request tiles: walls + particle cells
  rc = request_wall_tiles(ctx);
  if (rc) return rc;
  if (n > 0)
    (++ctx->launches), k_bin<false><<<nblocks(n, 256 * kBinPer), 256, 0, ctx->stream>>>(
        G, ctx->px, ctx->py, ctx->pz, n, nullptr, nullptr, nullptr, ctx->tile_need);
  PF_CUDA_TRY(cudaGetLastError());
  rc = pool_commit(ctx);
  if (rc) return rc;
  G = dev_grid(ctx);
  const uint32_t walls = (uint32_t)(2LL * ctx->g.ny * ctx->g.nz + 2LL * ctx->g.nx * ctx->g.nz + 2LL * ctx->g.nx * ctx->g.ny);
  (++ctx->launches), k_mark_walls<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(G, ctx->mk_first);
  if (n > 0)
    (++ctx->launches), k_mark_particles<<<nblocks(n, 256), 256, 0, ctx->stream>>>(G, ctx->px, ctx->py, ctx->pz, n,
                                                                                   ctx->mk_first, walls);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

static int p2g_core(pf_ctx* ctx, const pf_phase* ph, double Vp) {
  const int n = (int)ctx->np;
  const int nt = ctx->g.ntiles;
  ctx->bins_valid = false;
  ctx->splat_fresh = false;
  // with particles the normalisation overwrites every pooled node of these
  // fields from the splat's staging, so only their activity is reset
  for (int f = PF_U; f <= PF_MW; ++f) {
    int rc = field_clear(ctx, f, n == 0);
    if (rc) return rc;
  }
  int rc;
  {
    StageScope sc(ctx, PF_STAGE_BIN);
    PF_CUDA_TRY(cudaMemsetAsync(ctx->tile_count, 0, (size_t)(nt * PF_TV + 1) * sizeof(int), ctx->stream));
    DevGrid G = dev_grid(ctx);
    if (n > 0) {
      (++ctx->launches), k_bin<true><<<nblocks(n, 256 * kBinPer), 256, 0, ctx->stream>>>(
          G, ctx->px, ctx->py, ctx->pz, n, ctx->tile_count, ctx->pkey, ctx->prank, ctx->tile_need);
      // the tiles a particle's window can reach: the tiles holding particles
      // (and any requested before) and their neighbours
      const int nt0 = ctx->g.ntiles;
      (++ctx->launches), k_need_from_counts<<<nblocks((size_t)nt0 * 32, 256), 256, 0, ctx->stream>>>(
          ctx->tile_count, ctx->tile_need, ctx->tile_new, nt0);
      (++ctx->launches), k_need_dilate<<<nblocks(nt0, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->tile_new,
                                                                                   ctx->tile_need);
    }
    PF_CUDA_TRY(cudaGetLastError());
    rc = pool_commit(ctx);
    if (rc) return rc;
  }
  if (n == 0) return PF_OK;
  {
    StageScope sc(ctx, PF_STAGE_SORT);
    rc = scan_exclusive(ctx, ctx->tile_count, ctx->tile_start, nt * PF_TV + 1, nullptr);
    if (rc) return rc;
    (++ctx->launches), k_bin_scatter<<<nblocks(n, 256 * kBinPer), 256, 0, ctx->stream>>>(ctx->pkey, ctx->prank, ctx->tile_start, ctx->perm, n);
    PF_CUDA_TRY(cudaGetLastError());
    ctx->bins_valid = true;
  }
  {
    StageScope sc(ctx, PF_STAGE_SPLAT);
    const size_t smem = (size_t)kSplatGroups * kWarpBox * sizeof(float2);
    (++ctx->launches), k_splat<<<nt, kSplatThreads, smem, ctx->stream>>>(
        dev_grid(ctx), ctx->tile_start, ctx->perm, ctx->prank, ctx->splat_stage, ctx->px, ctx->py, ctx->pz, ctx->vx,
        ctx->vy, ctx->vz, ctx->type, ctx->vol, (float)(ph->rho_l * Vp), (float)(ph->rho_g * Vp));
    ctx->splat_fresh = true;
    PF_CUDA_TRY(cudaGetLastError());
  }
  return PF_OK;
}

int p2g(pf_ctx* ctx, const pf_phase* ph, double Vp) {
  int rc = p2g_core(ctx, ph, Vp);
  if (rc) return rc;
  return normalize_save_gravity(ctx, false, false, 0.0, 0.0);
}

int normalize_save_gravity(pf_ctx* ctx, bool save, bool gravity, double dt, double gval) {
  StageScope stage(ctx, PF_STAGE_NORMALIZE);
  if (pool_nonempty(ctx))
    (++ctx->launches), k_normalize<<<slot_grid(ctx), PF_TV, 0, ctx->stream>>>(
        dev_grid(ctx), ctx->splat_stage, ctx->tile_start, ctx->splat_fresh ? 1 : 0, ctx->d_nslots, save ? 1 : 0,
        gravity ? 1 : 0, (float)(dt * gval));
  ctx->splat_fresh = false;
  PF_CUDA_TRY(cudaGetLastError());
  if (save) ctx->saved_valid = true;
  return PF_OK;
}

int save_velocity(pf_ctx* ctx) {
  StageScope stage(ctx, PF_STAGE_BOUNDARY);
  if (pool_nonempty(ctx))
    (++ctx->launches), k_save<<<slot_grid(ctx), PF_TV, 0, ctx->stream>>>(dev_grid(ctx), ctx->d_nslots);
  PF_CUDA_TRY(cudaGetLastError());
  ctx->saved_valid = true;
  return PF_OK;
}

int apply_gravity(pf_ctx* ctx, double dt, double gval) {
  StageScope stage(ctx, PF_STAGE_BOUNDARY);
  if (pool_nonempty(ctx))
    (++ctx->launches), k_gravity<<<slot_grid(ctx), PF_TV, 0, ctx->stream>>>(dev_grid(ctx), ctx->d_nslots,
                                                                            (float)(dt * gval));
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int apply_walls(pf_ctx* ctx) {
  StageScope stage(ctx, PF_STAGE_BOUNDARY);
  int rc = request_wall_tiles(ctx);
  if (rc) return rc;
  rc = pool_commit(ctx);
  if (rc) return rc;
  (++ctx->launches), k_walls<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(dev_grid(ctx));
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int g2p(pf_ctx* ctx, const pf_ctx* saved, double aL, double aG) {
  StageScope stage(ctx, PF_STAGE_G2P);
  const int n = (int)ctx->np;
  if (n == 0) return PF_OK;
  DevGrid G = dev_grid(ctx);
  if (saved && saved != ctx) {
    DevGrid S = dev_grid(saved);
    (++ctx->launches), k_g2p<true><<<nblocks(n, 256), 256, 0, ctx->stream>>>(G, S, particle_ptrs(ctx), n, aL, aG);
  } else {
    if (!ctx->saved_valid) return set_error(ctx, PF_ERR_INVALID, "g2p: no saved velocity (call pf_save_velocity)");
    if (ctx->bins_valid)
      (++ctx->launches), k_g2p_tiles<<<ctx->g.ntiles, 256, 0, ctx->stream>>>(G, ctx->tile_start, ctx->perm,
                                                                               particle_ptrs(ctx), aL, aG);
    else
      (++ctx->launches), k_g2p<false><<<nblocks(n, 256), 256, 0, ctx->stream>>>(G, G, particle_ptrs(ctx), n, aL, aG);
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

static int read_clamp(pf_ctx* ctx, pf_clamp_stats* st) {
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints, ctx->d_clamp, 8 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (st) {
    const int* c = ctx->h_pinned_ints;
    st->clamped_liquid = c[0]; st->clamped_gas = c[1];
    st->x_lo = c[2]; st->x_hi = c[3]; st->y_lo = c[4]; st->y_hi = c[5]; st->z_lo = c[6]; st->z_hi = c[7];
  }
  return PF_OK;
}

int advect(pf_ctx* ctx, double dt, int order, pf_clamp_stats* st, double* esc, size_t* nesc) {
  StageScope stage(ctx, PF_STAGE_G2P);
  const int n = (int)ctx->np;
  ctx->bins_valid = false;  // particles move
  PF_CUDA_TRY(cudaMemsetAsync(ctx->d_clamp, 0, 8 * sizeof(int), ctx->stream));
  if (n > 0) {
    (++ctx->launches), k_advect<<<nblocks(n, 256), 256, 0, ctx->stream>>>(dev_grid(ctx), particle_ptrs(ctx), n, dt, order,
                                                        ctx->d_clamp, esc ? ctx->d_flags : nullptr, 0, 0.0, 0.0);
    PF_CUDA_TRY(cudaGetLastError());
  }
  if (esc) {
    int total = 0;
    if (n > 0) {
      int* pos = ctx->d_flags + ctx->cap;
      int rc = scan_exclusive(ctx, ctx->d_flags, pos, n, ctx->d_scalar);
      if (rc) return rc;
      PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints + 8, ctx->d_scalar, sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream));
      PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      total = ctx->h_pinned_ints[8];
      const size_t need_bytes = (size_t)(total > 0 ? total : 1) * 8 * sizeof(double);
      if (need_bytes > ctx->esc_bytes) {
        if (ctx->esc_buf) PF_CUDA_TRY(cudaFree(ctx->esc_buf));
        ctx->esc_buf = nullptr;
        ctx->esc_bytes = 0;
        PF_CUDA_TRY(cudaMalloc(&ctx->esc_buf, need_bytes));
        ctx->esc_bytes = need_bytes;
      }
      double* out = (double*)ctx->esc_buf;
      (++ctx->launches), k_escape_records<<<nblocks(n, 256), 256, 0, ctx->stream>>>(particle_ptrs(ctx), ctx->d_flags, pos, n, out);
      PF_CUDA_TRY(cudaGetLastError());
      if (total > 0)
        PF_CUDA_TRY(cudaMemcpyAsync(esc, out, (size_t)total * 8 * sizeof(double), cudaMemcpyDefault, ctx->stream));
    }
    if (nesc) *nesc = (size_t)total;
  }
  return read_clamp(ctx, st);
}

// With esc_flags the per-particle kernel also flags the clamped particles
// (the escape records' source); the tile kernel has no flags.
int g2p_advect(pf_ctx* ctx, double aL, double aG, double dt, int order, pf_clamp_stats* st, int* esc_flags) {
  StageScope stage(ctx, PF_STAGE_G2P);
  const int n = (int)ctx->np;
  PF_CUDA_TRY(cudaMemsetAsync(ctx->d_clamp, 0, 8 * sizeof(int), ctx->stream));
  if (n > 0) {
    if (ctx->bins_valid && !esc_flags)
      (++ctx->launches), k_g2p_advect_tiles<<<ctx->g.ntiles, 256, 0, ctx->stream>>>(
          dev_grid(ctx), ctx->tile_start, ctx->perm, particle_ptrs(ctx), dt, order, aL, aG, ctx->d_clamp);
    else
      (++ctx->launches), k_advect<<<nblocks(n, 256), 256, 0, ctx->stream>>>(dev_grid(ctx), particle_ptrs(ctx), n, dt,
                                                                             order, ctx->d_clamp, esc_flags, 1, aL, aG);
    PF_CUDA_TRY(cudaGetLastError());
  }
  ctx->bins_valid = false;  // particles moved
  if (st) return read_clamp(ctx, st);
  return PF_OK;
}

int calibrate(pf_ctx* ctx, const pf_phase* ph, double Vp, double* out) {
  double* contrib = (double*)ctx->staging;  // 4096 doubles + 1
  const double mp = ph->rho_l * Vp;
  (++ctx->launches), k_calib_contrib<<<16, 256, 0, ctx->stream>>>(mp, contrib);
  (++ctx->launches), k_calib_sum<<<1, 1, 0, ctx->stream>>>(contrib, ph->rho_l, contrib + 4096);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(out, contrib + 4096, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

}  // namespace pf
