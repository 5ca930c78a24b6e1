// pf_pool.cu -- the sparse tile pool: prefix scans, slot assignment by
// compaction, field clear/import/export, 4^3 activity, and the active-cell
// enumeration (collectCellsWithMarker, src/driver/sparse_ops3d_common.h:65-85).
#include <cstdio>
#include <cstring>

#include "pf_ctx.h"

namespace pf {

int set_cuda_error(pf_ctx* ctx, cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (ctx) ctx->err = buf;
  return PF_ERR_CUDA;
}

int set_error(pf_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

// ------------------------------------------------------------------------
// exclusive prefix scan (int32), 2048 items per 512-thread block, recursive
// over block totals
// ------------------------------------------------------------------------

constexpr int kScanNT = 512;
constexpr int kScanIPT = 4;
constexpr int kScanItems = kScanNT * kScanIPT;

__global__ void __launch_bounds__(kScanNT) k_scan_block(const int* in, int* out, int n, int* block_sums) {
  __shared__ int warp_tot[kScanNT / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * kScanItems;
  // coalesced load into registers: item q of this thread is base + q*NT + tid
  int v[kScanIPT];
  __shared__ int tile[kScanItems];
#pragma unroll
  for (int q = 0; q < kScanIPT; ++q) {
    const long long idx = base + q * kScanNT + threadIdx.x;
    tile[q * kScanNT + threadIdx.x] = idx < n ? in[idx] : 0;
  }
  __syncthreads();
  int sum = 0;
#pragma unroll
  for (int q = 0; q < kScanIPT; ++q) {
    v[q] = tile[threadIdx.x * kScanIPT + q];
    sum += v[q];
  }
  int xi = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, xi, o);
    if (lane >= o) xi += y;
  }
  if (lane == 31) warp_tot[wid] = xi;
  __syncthreads();
  if (wid == 0) {
    int t = lane < kScanNT / 32 ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kScanNT / 32) warp_tot[lane] = t;
  }
  __syncthreads();
  const int warp_off = wid > 0 ? warp_tot[wid - 1] : 0;
  int excl = warp_off + xi - sum;
#pragma unroll
  for (int q = 0; q < kScanIPT; ++q) {
    tile[threadIdx.x * kScanIPT + q] = excl;
    excl += v[q];
  }
  if (threadIdx.x == kScanNT - 1) block_sums[blockIdx.x] = warp_off + xi;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kScanIPT; ++q) {
    const long long idx = base + q * kScanNT + threadIdx.x;
    if (idx < n) out[idx] = tile[q * kScanNT + threadIdx.x];
  }
}

__global__ void k_scan_add(int* out, int n, const int* offs) {
  const int add = offs[blockIdx.x];
  const long long base = (long long)blockIdx.x * kScanItems;
  for (int q = threadIdx.x; q < kScanItems; q += blockDim.x) {
    const long long idx = base + q;
    if (idx < n) out[idx] += add;
  }
}

__global__ void k_copy_int(const int* src, int* dst) { *dst = *src; }

int scan_alloc(pf_ctx* ctx, size_t max_n) {
  size_t n = max_n;
  while (true) {
    const size_t nb = (n + kScanItems - 1) / kScanItems;
    int* buf = nullptr;
    PF_CUDA_TRY(cudaMalloc(&buf, (nb + 1) * sizeof(int)));
    ctx->scan_levels.push_back(buf);
    if (nb <= 1) break;
    n = nb;
  }
  return PF_OK;
}

static int scan_level(pf_ctx* ctx, const int* in, int* out, int n, int* total, size_t level) {
  if (level >= ctx->scan_levels.size()) return set_error(ctx, PF_ERR_INVALID, "scan too large");
  const int nb = (n + kScanItems - 1) / kScanItems;
  int* sums = ctx->scan_levels[level];
  if (n > 0) (++ctx->launches), k_scan_block<<<nb, kScanNT, 0, ctx->stream>>>(in, out, n, sums);
  if (nb > 1) {
    int rc = scan_level(ctx, sums, sums, nb, total, level + 1);
    if (rc) return rc;
    (++ctx->launches), k_scan_add<<<nb, 256, 0, ctx->stream>>>(out, n, sums);
  } else if (total) {
    if (n > 0) (++ctx->launches), k_copy_int<<<1, 1, 0, ctx->stream>>>(sums, total);
    else PF_CUDA_TRY(cudaMemsetAsync(total, 0, sizeof(int), ctx->stream));
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int scan_exclusive(pf_ctx* ctx, const int* in, int* out, int n, int* total_dev) {
  return scan_level(ctx, in, out, n, total_dev, 0);
}

// ------------------------------------------------------------------------
// pool
// ------------------------------------------------------------------------

DevGrid dev_grid(const pf_ctx* ctx) {
  DevGrid G;
  G.g = ctx->g;
  G.tile_slot = ctx->tile_slot;
  G.slot_tile = ctx->slot_tile;
  for (int f = 0; f < PF_NFIELDS; ++f) { G.fld[f] = ctx->fld[f]; G.act4[f] = ctx->act4[f]; }
  for (int a = 0; a < PF_NSAVED; ++a) G.saved[a] = ctx->saved[a];
  return G;
}

// Zero every field of slots [0, nslots) and unmap their tiles.
__global__ void k_pool_reset(DevGrid G, int* tile_slot, int nslots) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
#pragma unroll
    for (int f = 0; f < PF_NFIELDS; ++f) G.fld[f][o] = 0.0f;
#pragma unroll
    for (int a = 0; a < PF_NSAVED; ++a) G.saved[a][o] = 0.0f;
    if (threadIdx.x == 0) tile_slot[G.slot_tile[s]] = -1;
  }
}

int pool_reset(pf_ctx* ctx) {
  int rc = pool_sync(ctx);
  if (rc) return rc;
  if (ctx->nslots > 0) {
    const int nb = ctx->nslots < 4 * ctx->num_sms ? ctx->nslots : 4 * ctx->num_sms;
    (++ctx->launches), k_pool_reset<<<nb, PF_TV, 0, ctx->stream>>>(dev_grid(ctx), ctx->tile_slot, ctx->nslots);
    PF_CUDA_TRY(cudaGetLastError());
  }
  for (int f = 0; f < PF_NFIELDS; ++f)
    PF_CUDA_TRY(cudaMemsetAsync(ctx->act4[f], 0, ctx->act4_n[f], ctx->stream));
  ctx->nslots = 0;
  ctx->saved_valid = false;
  PF_CUDA_TRY(cudaMemsetAsync(ctx->d_nslots, 0, sizeof(int), ctx->stream));
  return PF_OK;
}

// new[t] = requested and not yet pooled
__global__ void k_need_flags(const uint8_t* need, const int* tile_slot, int* out, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (need[t] && tile_slot[t] < 0) ? 1 : 0;
}

// Assign slots nslots + rank in ascending tile order; clear requests.
__global__ void k_assign_slots(uint8_t* need, const int* flags, const int* rank, int* tile_slot,
                               int* slot_tile, const int* d_nslots, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (flags[t]) {
    const int s = *d_nslots + rank[t];
    tile_slot[t] = s;
    slot_tile[s] = t;
  }
  need[t] = 0;
}

__global__ void k_bump_nslots(int* d_nslots, const int* added) { *d_nslots += *added; }

int pool_commit(pf_ctx* ctx) {
  const int n = ctx->g.ntiles;
  int* flags = ctx->tile_new;
  int* rank = ctx->tile_rank;
  (++ctx->launches), k_need_flags<<<nblocks(n, 256), 256, 0, ctx->stream>>>(ctx->tile_need, ctx->tile_slot, flags, n);
  int rc = scan_exclusive(ctx, flags, rank, n, ctx->d_scalar);
  if (rc) return rc;
  (++ctx->launches), k_assign_slots<<<nblocks(n, 256), 256, 0, ctx->stream>>>(ctx->tile_need, flags, rank, ctx->tile_slot,
                                                          ctx->slot_tile, ctx->d_nslots, n);
  (++ctx->launches), k_bump_nslots<<<1, 1, 0, ctx->stream>>>(ctx->d_nslots, ctx->d_scalar);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_nslots, ctx->d_nslots, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaEventRecord(ctx->pool_ev, ctx->stream));
  ctx->pool_pending = true;
  return PF_OK;
}

int pool_sync(pf_ctx* ctx) {
  if (!ctx->pool_pending) return PF_OK;
  PF_CUDA_TRY(cudaEventSynchronize(ctx->pool_ev));
  ctx->pool_pending = false;
  ctx->nslots = *ctx->h_nslots;
  if (ctx->nslots < 0 || ctx->nslots > ctx->g.ntiles) return set_error(ctx, PF_ERR_INVALID, "pool size out of range");
  return PF_OK;
}

// A grid-stride slot loop that reads the pool size from d_nslots: the host's
// nslots when it is current, else `cap` CTAs (the pool may have grown).
int slot_blocks(const pf_ctx* ctx, int cap) {
  if (ctx->pool_pending) return cap;
  return ctx->nslots < cap ? ctx->nslots : cap;
}

__global__ void k_request_list(uint8_t* need, const int* tiles, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) need[tiles[q]] = 1;
}

int request_wall_tiles(pf_ctx* ctx) {
  const int n = (int)ctx->wall_tiles.size();
  if (n > 0) (++ctx->launches), k_request_list<<<nblocks(n, 256), 256, 0, ctx->stream>>>(ctx->tile_need, ctx->d_wall_tiles, n);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

__global__ void k_zero_field(float* f, int nslots) {
  const size_t n = (size_t)nslots * PF_TV;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    f[q] = 0.0f;
}

// SparseBlockGrid3D::clear (src/grid/sparse_block_grid3d.h:64-67) with the
// zero-fill that reactivation performs.
// With data == false only the activity is reset: the caller overwrites every
// pooled node of the field afterwards.
int field_clear(pf_ctx* ctx, int f, bool data) {
  if (data) {
    int rc = pool_sync(ctx);
    if (rc) return rc;
  }
  if (data && ctx->nslots > 0)
    PF_CUDA_TRY(cudaMemsetAsync(ctx->fld[f], 0, (size_t)ctx->nslots * PF_TV * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(ctx->act4[f], 0, ctx->act4_n[f], ctx->stream));
  if (f == PF_MK && ctx->mk_first)
    PF_CUDA_TRY(cudaMemsetAsync(ctx->mk_first, 0xff, ctx->act4_n[PF_MK] * sizeof(uint32_t), ctx->stream));
  return PF_OK;  // the saved copy is separate storage and stays valid
}

}  // namespace pf

// ------------------------------------------------------------------------
// field import / export (dense lattice arrays <-> pool)
// ------------------------------------------------------------------------
namespace {

using namespace pf;

// Request tiles holding any active 4^3 block of the imported field.
__global__ void k_request_from_act4(Geom g, int f, const uint8_t* act, uint8_t* need) {
  const int n = g.bdim[f][0] * g.bdim[f][1] * g.bdim[f][2];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n || !act[b]) return;
  const int bx = b % g.bdim[f][0];
  const int q = b / g.bdim[f][0];
  const int by = q % g.bdim[f][1];
  const int bz = q / g.bdim[f][1];
  need[tile_id(g, bx >> 1, by >> 1, bz >> 1)] = 1;
}

// An imported marker field's blocks count as activated in ascending block id,
// the order in which the reference's setCell loop over (k, j, i) touches them.
__global__ void k_first_from_act(const uint8_t* act, int n, uint32_t* first) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) first[b] = act[b] ? (uint32_t)b : 0xffffffffu;
}

__global__ void k_import_field(DevGrid G, int f, const float* dense, int nslots) {
  const int s = blockIdx.x;
  if (s >= nslots) return;
  const int t = G.slot_tile[s];
  const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
  const int l = threadIdx.x;
  const int i = tx * 8 + (l & 7), j = ty * 8 + ((l >> 3) & 7), k = tz * 8 + (l >> 6);
  float v = 0.0f;
  if (in_field(G.g, f, i, j, k) && G.act4[f][act4_index(G.g, f, i, j, k)]) {
    v = dense[(size_t)i + (size_t)G.g.fdim[f][0] * ((size_t)j + (size_t)G.g.fdim[f][1] * k)];
  }
  G.fld[f][(size_t)s * PF_TV + l] = v;
}

__global__ void k_export_field(DevGrid G, int f, float* dense, int nslots) {
  const int s = blockIdx.x;
  if (s >= nslots) return;
  const int t = G.slot_tile[s];
  const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
  const int l = threadIdx.x;
  const int i = tx * 8 + (l & 7), j = ty * 8 + ((l >> 3) & 7), k = tz * 8 + (l >> 6);
  if (in_field(G.g, f, i, j, k))
    dense[(size_t)i + (size_t)G.g.fdim[f][0] * ((size_t)j + (size_t)G.g.fdim[f][1] * k)] =
        G.fld[f][(size_t)s * PF_TV + l];
}

// dense flag per cell: marker == 1
__global__ void k_fluid_flags(DevGrid G, int32_t* flags) {
  const long long n = (long long)G.g.nx * G.g.ny * G.g.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.g.nx);
    const long long q = c / G.g.nx;
    const int j = (int)(q % G.g.ny), k = (int)(q / G.g.ny);
    flags[c] = cell_marker(G, i, j, k) == 1 ? 1 : 0;
  }
}

__global__ void k_compact_cells(const int32_t* flags, const int32_t* pos, long long n, int32_t* out) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    if (flags[c]) out[pos[c]] = (int32_t)c;
}

__global__ void k_compact_blocks(const uint8_t* act, int n, int* pos_scan, int32_t* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n && act[b]) out[pos_scan[b]] = b;
}

__global__ void k_u8_to_i32(const uint8_t* a, int32_t* o, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) o[b] = a[b] ? 1 : 0;
}

}  // namespace

namespace pf {

int grid_set_field(pf_ctx* ctx, int f, const float* dense, const uint8_t* act4) {
  const Geom& g = ctx->g;
  const size_t nn = (size_t)g.fdim[f][0] * g.fdim[f][1] * g.fdim[f][2];
  // staging: dense values after the act4 bytes, both on the device
  const size_t need_bytes = ctx->act4_n[f] + 16 + nn * sizeof(float);
  if (need_bytes > ctx->staging_bytes) return set_error(ctx, PF_ERR_INVALID, "field larger than staging");
  uint8_t* d_act = (uint8_t*)ctx->staging;
  float* d_dense = (float*)((char*)ctx->staging + ((ctx->act4_n[f] + 15) / 16) * 16);
  PF_CUDA_TRY(cudaMemcpyAsync(d_act, act4, ctx->act4_n[f], cudaMemcpyDefault, ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(d_dense, dense, nn * sizeof(float), cudaMemcpyDefault, ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->act4[f], d_act, ctx->act4_n[f], cudaMemcpyDeviceToDevice, ctx->stream));
  const int nb = (int)ctx->act4_n[f];
  (++ctx->launches), k_request_from_act4<<<nblocks(nb, 256), 256, 0, ctx->stream>>>(g, f, ctx->act4[f], ctx->tile_need);
  if (f == PF_MK) (++ctx->launches), k_first_from_act<<<nblocks(nb, 256), 256, 0, ctx->stream>>>(ctx->act4[f], nb, ctx->mk_first);
  PF_CUDA_TRY(cudaGetLastError());
  int rc = pool_commit(ctx);
  if (!rc) rc = pool_sync(ctx);
  if (rc) return rc;
  if (ctx->nslots > 0)
    (++ctx->launches), k_import_field<<<ctx->nslots, PF_TV, 0, ctx->stream>>>(dev_grid(ctx), f, d_dense, ctx->nslots);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int grid_get_field(pf_ctx* ctx, int f, float* dense, uint8_t* act4) {
  const Geom& g = ctx->g;
  const size_t nn = (size_t)g.fdim[f][0] * g.fdim[f][1] * g.fdim[f][2];
  if (nn * sizeof(float) > ctx->staging_bytes) return set_error(ctx, PF_ERR_INVALID, "field larger than staging");
  float* d_dense = (float*)ctx->staging;
  if (dense) {
    int rc = pool_sync(ctx);
    if (rc) return rc;
    PF_CUDA_TRY(cudaMemsetAsync(d_dense, 0, nn * sizeof(float), ctx->stream));
    if (ctx->nslots > 0)
      (++ctx->launches), k_export_field<<<ctx->nslots, PF_TV, 0, ctx->stream>>>(dev_grid(ctx), f, d_dense, ctx->nslots);
    PF_CUDA_TRY(cudaGetLastError());
    PF_CUDA_TRY(cudaMemcpyAsync(dense, d_dense, nn * sizeof(float), cudaMemcpyDefault, ctx->stream));
  }
  if (act4) PF_CUDA_TRY(cudaMemcpyAsync(act4, ctx->act4[f], ctx->act4_n[f], cudaMemcpyDefault, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int active_blocks4(pf_ctx* ctx, int f, int32_t* ids, size_t* n) {
  const int nb = (int)ctx->act4_n[f];
  int32_t* flags = ctx->cell_flags;
  int32_t* pos = ctx->cell_flags + ctx->act4_n[f] + 1;
  (++ctx->launches), k_u8_to_i32<<<nblocks(nb, 256), 256, 0, ctx->stream>>>(ctx->act4[f], flags, nb);
  int rc = scan_exclusive(ctx, flags, pos, nb, ctx->d_scalar);
  if (rc) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints, ctx->d_scalar, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int total = ctx->h_pinned_ints[0];
  if (ids) {
    if ((size_t)total > *n) return set_error(ctx, PF_ERR_INVALID, "ids buffer too small");
    int32_t* out = (int32_t*)ctx->staging;
    (++ctx->launches), k_compact_blocks<<<nblocks(nb, 256), 256, 0, ctx->stream>>>(ctx->act4[f], nb, pos, out);
    PF_CUDA_TRY(cudaGetLastError());
    PF_CUDA_TRY(cudaMemcpyAsync(ids, out, (size_t)total * sizeof(int32_t), cudaMemcpyDefault, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  *n = (size_t)total;
  return PF_OK;
}

// Active-cell enumeration: dense fluid flags in linear order, exclusive scan,
// scatter -> cells ascending in c = i + nx*(j + ny*k), the order std::sort
// gives in collectCellsWithMarker.
int active_cells(pf_ctx* ctx, int32_t* cells, size_t* n) {
  const long long nc = (long long)ctx->g.nx * ctx->g.ny * ctx->g.nz;
  int32_t* flags = ctx->cell_flags;
  int32_t* pos = ctx->cell_flags + nc;
  const int nb = (int)((nc + 255) / 256 < 65535 * 4 ? (nc + 255) / 256 : 65535 * 4);
  (++ctx->launches), k_fluid_flags<<<nb, 256, 0, ctx->stream>>>(dev_grid(ctx), flags);
  int rc = scan_exclusive(ctx, flags, pos, (int)nc, ctx->d_scalar);
  if (rc) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints, ctx->d_scalar, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int total = ctx->h_pinned_ints[0];
  if (cells) {
    if ((size_t)total > *n) return set_error(ctx, PF_ERR_INVALID, "cells buffer too small");
    int32_t* out = (int32_t*)ctx->staging;
    (++ctx->launches), k_compact_cells<<<nb, 256, 0, ctx->stream>>>(flags, pos, nc, out);
    PF_CUDA_TRY(cudaGetLastError());
    PF_CUDA_TRY(cudaMemcpyAsync(cells, out, (size_t)total * sizeof(int32_t), cudaMemcpyDefault, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  *n = (size_t)total;
  return PF_OK;
}

}  // namespace pf
