// pf_adapt.cu -- particle adaptivity on the device:
//
//   applyNarrowBandAir            src/driver/particle_adaptivity3d.h:111-166
//   applyTypedParticleCoarsening  src/driver/particle_adaptivity3d.h:168-248
//   applyLiquidParticleRefill     src/driver/particle_adaptivity3d.h:250-374
//   SparseSim3DTP::applyParticleAdaptivity  src/driver/sparse_sim3d_tp.cpp:843-848
//
// The reference walks the particles and cells sequentially; here every pass is
// a data-parallel kernel over particles or over the dense cell lattice:
//   * the particle's cell is the reference's truncating (int)((x - o) / dx) in
//     FP64, -1 outside the grid or at a non-finite position;
//   * per-cell particle lists come from a counting sort (atomic rank, scan,
//     place); the order the reference fixes inside a cell -- (score, index)
//     for coarsening, index for refill -- is each entry's rank within its cell,
//     counted against the cell's list;
//   * "any cell flag within r cells" is a separable max filter over x, y, z;
//   * erasure is a stable compaction (flag, scan, scatter into the second
//     particle set, swap), which keeps the survivors' order as eraseIf does;
//   * refill's budget, consumed in linear cell order, is an exclusive scan of
//     the per-cell requests: cell c gets clamp(budget - before(c), 0, wanted).
// FP64 expressions are written with explicit _rn intrinsics so that no FMA
// contraction changes a rounding against the reference.
#include <algorithm>
#include <climits>

#include "pf_ctx.h"

namespace pf {
namespace {

constexpr int kNT = 256;

// the context's current particle set (SoA, FP32)
struct PSet {
  float *px, *py, *pz, *vx, *vy, *vz, *vol;
  uint8_t* type;
};

struct AdaptScratch {
  size_t ncell = 0, cap = 0;
  int* cnt = nullptr;        // [ncell] particles per cell
  int* start = nullptr;      // [ncell] exclusive scan of cnt
  int* wanted = nullptr;     // [ncell] refill requests
  int* woff = nullptr;       // [ncell] exclusive scan of wanted
  uint8_t* fa = nullptr;     // [ncell] cell flags
  uint8_t* fb = nullptr;     // [ncell] dilated flags
  unsigned* score = nullptr; // [cap]
  int* sorted = nullptr;     // [cap] per-cell lists in the reference's order
  int* d_stats = nullptr;    // [16]
  int* h_stats = nullptr;    // [16] pinned
  // the step controls' two reductions (max speed, liquid volume), copied back
  // behind ctl_ev; a deferred read keeps the dt and settings it is for
  double* h_ctl = nullptr;   // [2] pinned
  cudaEvent_t ctl_ev = nullptr;
  bool ctl_pending = false;
  double ctl_dt = 0.0;
  pf_step_controls ctl_cfg{};
};

int scratch(pf_ctx* ctx, AdaptScratch** out) {
  AdaptScratch* s = static_cast<AdaptScratch*>(ctx->adapt);
  if (!s) {
    s = new AdaptScratch();
    ctx->adapt = s;
    const size_t nc = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    s->ncell = nc;
    s->cap = ctx->cap;
    int** iv[4] = {&s->cnt, &s->start, &s->wanted, &s->woff};
    for (int** q : iv) PF_CUDA_TRY(cudaMalloc(q, (nc + 1) * sizeof(int)));
    PF_CUDA_TRY(cudaMalloc(&s->fa, nc + 1));
    PF_CUDA_TRY(cudaMalloc(&s->fb, nc + 1));
    PF_CUDA_TRY(cudaMalloc(&s->score, (s->cap + 1) * sizeof(unsigned)));
    PF_CUDA_TRY(cudaMalloc(&s->sorted, (s->cap + 1) * sizeof(int)));
    PF_CUDA_TRY(cudaMalloc(&s->d_stats, 16 * sizeof(int)));
    PF_CUDA_TRY(cudaMallocHost(&s->h_stats, 16 * sizeof(int)));
    PF_CUDA_TRY(cudaMallocHost(&s->h_ctl, 2 * sizeof(double)));
    PF_CUDA_TRY(cudaEventCreateWithFlags(&s->ctl_ev, cudaEventDisableTiming));
  }
  *out = s;
  return PF_OK;
}

int read_stats(pf_ctx* ctx, AdaptScratch* s, int n) {
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_stats, s->d_stats, n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

// warp-aggregated add of v into *c
__device__ __forceinline__ void warp_add(int* c, int v) {
  const int s = __reduce_add_sync(__activemask(), v);
  if ((threadIdx.x & 31) == __ffs(__activemask()) - 1 && s) atomicAdd(c, s);
}

// ParticleCellDomain3D::particleCell (particle_adaptivity3d.h:36-47)
__device__ __forceinline__ int adapt_cell(const Geom& g, float x, float y, float z, int* ijk) {
  const double p[3] = {(double)x, (double)y, (double)z};
  const double o[3] = {g.ox, g.oy, g.oz};
  const int n[3] = {g.nx, g.ny, g.nz};
  if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) return -1;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ijk[a] = __double2int_rz(__ddiv_rn(__dsub_rn(p[a], o[a]), g.dx));
    if (ijk[a] < 0 || ijk[a] >= n[a]) return -1;
  }
  return ijk[0] + g.nx * (ijk[1] + g.ny * ijk[2]);
}

// mix32 (particle_adaptivity3d.h:75-82)
__device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// particleScore (particle_adaptivity3d.h:84-102)
__device__ unsigned particle_score(const Geom& g, float x, float y, float z, const int* ijk, unsigned seed) {
  const double p[3] = {(double)x, (double)y, (double)z};
  const double o[3] = {g.ox, g.oy, g.oz};
  int q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double lo = __dadd_rn(o[a], __dmul_rn((double)ijk[a], g.dx));
    q[a] = __double2int_rz(__dmul_rn(__ddiv_rn(__dsub_rn(p[a], lo), g.dx), 1024.0));
  }
  unsigned h = seed;
  h ^= mix32((unsigned)ijk[0] + 0x9e3779b9u);
  h ^= mix32((unsigned)ijk[1] + 0x85ebca6bu);
  h ^= mix32((unsigned)ijk[2] + 0xc2b2ae35u);
  h ^= mix32((unsigned)(q[0] & 2047) + 0x27d4eb2fu);
  h ^= mix32((unsigned)(q[1] & 2047) + 0x165667b1u);
  h ^= mix32((unsigned)(q[2] & 2047) + 0xd3a2646cu);
  return mix32(h);
}

// slotScore (particle_adaptivity3d.h:104-109)
__device__ __forceinline__ unsigned slot_score(unsigned cell, int slot, unsigned seed) {
  unsigned h = seed;
  h ^= mix32(cell + 0x68bc21ebu);
  h ^= mix32((unsigned)slot + 0x02e5be93u);
  return mix32(h);
}

// ---- shared passes --------------------------------------------------------

// count[c] += 1 where flag[c] != 0
__global__ void k_count_flags(const uint8_t* __restrict__ f, size_t n, int* count) {
  int v = 0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    v += f[c] != 0;
  warp_add(count, v);
}

// out[c] = any in[c + d * stride], |d| <= r, along one axis of extent `len`
__global__ void k_dilate(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, Geom g, int axis, int r) {
  const size_t nc = (size_t)g.nx * g.ny * g.nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((size_t)g.nx * g.ny));
    const int at = axis == 0 ? i : axis == 1 ? j : k;
    const int len = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
    const long long stride = axis == 0 ? 1 : axis == 1 ? g.nx : (long long)g.nx * g.ny;
    uint8_t any = 0;
    for (int d = max(-r, -at); d <= min(r, len - 1 - at) && !any; ++d) any = in[(long long)c + d * stride];
    out[c] = any;
  }
}

// the (2r+1)^3 box dilation (clipped to the grid) of fa; returns the buffer holding it
uint8_t* dilate_box(pf_ctx* ctx, AdaptScratch* s, int r) {
  if (r <= 0) return s->fa;
  const int nb = 8 * ctx->num_sms;
  (++ctx->launches), k_dilate<<<nb, kNT, 0, ctx->stream>>>(s->fa, s->fb, ctx->g, 0, r);
  (++ctx->launches), k_dilate<<<nb, kNT, 0, ctx->stream>>>(s->fb, s->fa, ctx->g, 1, r);
  (++ctx->launches), k_dilate<<<nb, kNT, 0, ctx->stream>>>(s->fa, s->fb, ctx->g, 2, r);
  return s->fb;
}

// every particle's cell (or -1)
__global__ void k_adapt_cells(Geom g, const float* __restrict__ px, const float* __restrict__ py,
                              const float* __restrict__ pz, int n, int* cell) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int ijk[3];
  cell[p] = adapt_cell(g, px[p], py[p], pz[p], ijk);
}

// keys[p] >= 0: rank[p] = its arrival in the cell, cnt[key] += 1
__global__ void k_count_keys(const int* __restrict__ key, int n, int* cnt, int* rank) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && key[p] >= 0) rank[p] = atomicAdd(&cnt[key[p]], 1);
}

__global__ void k_place(const int* __restrict__ key, const int* __restrict__ rank, const int* __restrict__ start,
                        int n, int* list) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && key[p] >= 0) list[start[key[p]] + rank[p]] = p;
}

// Stable compaction of the particles with keep[p] != 0 into the second
// particle set, which then becomes the current one.
__global__ void k_compact(const int* __restrict__ keep, const int* __restrict__ at, int n, PSet src,
                          PSet dst) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || !keep[p]) return;
  const int q = at[p];
  dst.px[q] = src.px[p];
  dst.py[q] = src.py[p];
  dst.pz[q] = src.pz[p];
  dst.vx[q] = src.vx[p];
  dst.vy[q] = src.vy[p];
  dst.vz[q] = src.vz[p];
  dst.vol[q] = src.vol[p];
  dst.type[q] = src.type[p];
}

int compact(pf_ctx* ctx, AdaptScratch* s, const int* keep) {
  const int n = (int)ctx->np;
  int* at = ctx->perm;
  int rc = scan_exclusive(ctx, keep, at, n, s->d_stats + 15);
  if (rc) return rc;
  rc = read_stats(ctx, s, 16);
  if (rc) return rc;
  const int m = s->h_stats[15];
  rc = ensure_back_set(ctx);
  if (rc) return rc;
  PSet src{ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->vol, ctx->type};
  PSet dst{ctx->bpx, ctx->bpy, ctx->bpz, ctx->bvx, ctx->bvy, ctx->bvz, ctx->bvol, ctx->btype};
  if (n > 0) (++ctx->launches), k_compact<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(keep, at, n, src, dst);
  PF_CUDA_TRY(cudaGetLastError());
  std::swap(ctx->px, ctx->bpx);
  std::swap(ctx->py, ctx->bpy);
  std::swap(ctx->pz, ctx->bpz);
  std::swap(ctx->vx, ctx->bvx);
  std::swap(ctx->vy, ctx->bvy);
  std::swap(ctx->vz, ctx->bvz);
  std::swap(ctx->vol, ctx->bvol);
  std::swap(ctx->type, ctx->btype);
  ctx->np = (size_t)m;
  ctx->bins_valid = false;
  // the old set was read by the compaction: a later asynchronous upload into it waits for that
  PF_CUDA_TRY(cudaEventRecord(ctx->back_free, ctx->stream));
  ctx->back_free_recorded = true;
  return PF_OK;
}

// ---- narrow-band air --------------------------------------------------------

__global__ void k_mark_liquid(const int* __restrict__ cell, const uint8_t* __restrict__ type, int n, uint8_t* f) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || type[p] != 0 || cell[p] < 0) return;
  if (!f[cell[p]]) f[cell[p]] = 1;  // stored only when it reads 0
}

// keep: every non-gas particle, and gas in a cell of the band
__global__ void k_band_keep(const int* __restrict__ cell, const uint8_t* __restrict__ type,
                            const uint8_t* __restrict__ band, int n, int* keep, int* stats) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool gas = type[p] == 1;
  const bool k = !gas || (cell[p] >= 0 && band[cell[p]]);
  keep[p] = k;
  warp_add(&stats[1], gas);
  warp_add(&stats[2], gas && k);
}

// ---- coarsening ---------------------------------------------------------------

__global__ void k_coarse_keys(Geom g, PSet P, int n, int ptype, unsigned seed, int* key, unsigned* score,
                              int* cnt, int* rank, int* stats) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool mine = P.type[p] == (uint8_t)ptype;
  warp_add(&stats[0], mine);
  int ijk[3];
  const int c = mine ? adapt_cell(g, P.px[p], P.py[p], P.pz[p], ijk) : -1;
  key[p] = c;
  if (c < 0) return;
  score[p] = particle_score(g, P.px[p], P.py[p], P.pz[p], ijk, seed);
  rank[p] = atomicAdd(&cnt[c], 1);
}

// each entry's rank by (score, index) in its cell -> sorted list; keep flags
__global__ void k_coarse_rank(const int* __restrict__ key, const unsigned* __restrict__ score,
                              const uint8_t* __restrict__ type, const int* __restrict__ cnt,
                              const int* __restrict__ start, const int* __restrict__ list, int n, int ptype,
                              int target, int* sorted, int* keep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = key[p];
  if (c < 0) {
    keep[p] = type[p] != (uint8_t)ptype;  // outside the grid: erased if of the coarsened type
    return;
  }
  const int s = start[c], m = cnt[c];
  const unsigned sp = score[p];
  int r = 0;
  for (int t = 0; t < m; ++t) {
    const int q = list[s + t];
    const unsigned sq = score[q];
    r += sq < sp || (sq == sp && q < p);
  }
  sorted[s + r] = p;
  keep[p] = r < target;
}

// one thread per occupied cell (its first entry): the cell's volume in sorted
// order, shared by the kept entries
__global__ void k_coarse_cells(const int* __restrict__ key, const int* __restrict__ cnt,
                               const int* __restrict__ start, const int* __restrict__ sorted, int n, int target,
                               float* vol, int* stats) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool lead = false;
  int c = -1;
  if (p < n) {
    c = key[p];
    lead = c >= 0 && sorted[start[c]] == p;
  }
  int m = 0, kc = 0;
  if (lead) {
    const int s = start[c];
    m = cnt[c];
    kc = min(m, target);
    double sum = 0.0;
    for (int t = 0; t < m; ++t) sum = __dadd_rn(sum, (double)vol[sorted[s + t]]);
    const float kept = kc > 0 ? (float)__ddiv_rn(sum, (double)kc) : 0.0f;
    for (int t = 0; t < kc; ++t) vol[sorted[s + t]] = kept;
  }
  if (p < n) {
    warp_add(&stats[1], lead);
    warp_add(&stats[2], lead && m > target);
    warp_add(&stats[3], kc);
  }
}

// ---- refill -------------------------------------------------------------------

__global__ void k_refill_keys(Geom g, PSet P, int n, int* key, int* cnt, int* rank, uint8_t* gas) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int ijk[3];
  const int c = adapt_cell(g, P.px[p], P.py[p], P.pz[p], ijk);
  const uint8_t t = P.type[p];
  key[p] = (c >= 0 && t == 0) ? c : -1;
  if (c < 0) return;
  if (t == 0) rank[p] = atomicAdd(&cnt[c], 1);
  else if (t == 1 && !gas[c]) gas[c] = 1;
}

// each liquid entry's rank by index in its cell -> sorted list
__global__ void k_index_rank(const int* __restrict__ key, const int* __restrict__ cnt,
                             const int* __restrict__ start, const int* __restrict__ list, int n, int* sorted) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || key[p] < 0) return;
  const int c = key[p], s = start[c], m = cnt[c];
  int r = 0;
  for (int t = 0; t < m; ++t) r += list[s + t] < p;
  sorted[s + r] = p;
}

// per cell: statistics and the request target - count of an underfull cell
__global__ void k_refill_want(const int* __restrict__ cnt, const uint8_t* __restrict__ near, size_t nc, int target,
                              int only, int* wanted, int* stats) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int m = cnt[c];
    int w = 0;
    bool under = false;
    const bool nr = m > 0 && near[c];
    if (m > 0 && !(only && !nr) && m < target) {
      under = true;
      w = target - m;
    }
    wanted[c] = w;
    warp_add(&stats[0], m > 0);
    warp_add(&stats[1], m);
    warp_add(&stats[2], nr);
    warp_add(&stats[3], under);
  }
}

// per cell with a grant: split volume, mean velocity, new particles at the
// sub-cell centres in slotScore order (appended after `n0`, cell by cell)
__global__ void k_refill_apply(Geom g, PSet P, size_t n0, const int* __restrict__ cnt,
                               const int* __restrict__ start, const int* __restrict__ sorted,
                               const int* __restrict__ wanted, const int* __restrict__ woff, long long budget,
                               unsigned seed) {
  const size_t nc = (size_t)g.nx * g.ny * g.nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int want = wanted[c];
    if (want <= 0) continue;
    const long long before = woff[c];
    const long long add = min((long long)want, max(0LL, budget - before));
    if (add <= 0) continue;
    const int m = cnt[c], s = start[c];
    double vs = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0;
    for (int t = 0; t < m; ++t) {
      const int p = sorted[s + t];
      vs = __dadd_rn(vs, (double)P.vol[p]);
      u0 = __dadd_rn(u0, (double)P.vx[p]);
      u1 = __dadd_rn(u1, (double)P.vy[p]);
      u2 = __dadd_rn(u2, (double)P.vz[p]);
    }
    const double inv = __ddiv_rn(1.0, (double)m);
    const float a0 = (float)__dmul_rn(u0, inv), a1 = (float)__dmul_rn(u1, inv), a2 = (float)__dmul_rn(u2, inv);
    const float split = (float)__ddiv_rn(vs, (double)(m + add));
    for (int t = 0; t < m; ++t) P.vol[sorted[s + t]] = split;
    int slots[8];
    for (int a = 0; a < 8; ++a) {  // insertion sort by (slotScore, slot)
      const unsigned sa = slot_score((unsigned)c, a, seed);
      int b = a - 1;
      while (b >= 0) {
        const unsigned sb = slot_score((unsigned)c, slots[b], seed);
        if (sb < sa || (sb == sa && slots[b] < a)) break;
        slots[b + 1] = slots[b];
        --b;
      }
      slots[b + 1] = a;
    }
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((size_t)g.nx * g.ny));
    const size_t out = n0 + (size_t)min(before, budget);
    for (int a = 0; a < add; ++a) {
      const int sl = slots[a & 7];
      const double sx = 0.25 + 0.5 * (double)(sl & 1), sy = 0.25 + 0.5 * (double)((sl >> 1) & 1),
                   sz = 0.25 + 0.5 * (double)((sl >> 2) & 1);
      const size_t q = out + a;
      P.px[q] = (float)__dadd_rn(g.ox, __dmul_rn(__dadd_rn((double)i, sx), g.dx));
      P.py[q] = (float)__dadd_rn(g.oy, __dmul_rn(__dadd_rn((double)j, sy), g.dx));
      P.pz[q] = (float)__dadd_rn(g.oz, __dmul_rn(__dadd_rn((double)k, sz), g.dx));
      P.vx[q] = a0;
      P.vy[q] = a1;
      P.vz[q] = a2;
      P.vol[q] = split;
      P.type[q] = 0;
    }
  }
}

PSet particles_of(pf_ctx* ctx) {
  return PSet{ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->vol, ctx->type};
}

}  // namespace

int narrow_band_air(pf_ctx* ctx, int radius, pf_band_stats* st) {
  StageScope stage(ctx, PF_STAGE_ADAPT);
  pf_band_stats out{};
  AdaptScratch* s = nullptr;
  int rc = scratch(ctx, &s);
  if (rc) return rc;
  const int n = (int)ctx->np;
  PF_CUDA_TRY(cudaMemsetAsync(s->d_stats, 0, 16 * sizeof(int), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(s->fa, 0, s->ncell, ctx->stream));
  int* cell = ctx->pkey;
  if (n > 0) {
    (++ctx->launches), k_adapt_cells<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(ctx->g, ctx->px, ctx->py, ctx->pz, n,
                                                                                cell);
    (++ctx->launches), k_mark_liquid<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(cell, ctx->type, n, s->fa);
  }
  (++ctx->launches), k_count_flags<<<8 * ctx->num_sms, kNT, 0, ctx->stream>>>(s->fa, s->ncell, s->d_stats);
  PF_CUDA_TRY(cudaGetLastError());
  rc = read_stats(ctx, s, 1);
  if (rc) return rc;
  out.liquid_cells = s->h_stats[0];
  if (out.liquid_cells > 0) {
    const uint8_t* band = dilate_box(ctx, s, radius);
    int* keep = ctx->d_flags;
    (++ctx->launches), k_band_keep<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(cell, ctx->type, band, n, keep,
                                                                              s->d_stats);
    PF_CUDA_TRY(cudaGetLastError());
    rc = compact(ctx, s, keep);
    if (rc) return rc;
    out.gas_before = s->h_stats[1];
    out.gas_after = s->h_stats[2];
    out.removed = n - (int)ctx->np;
  }
  if (st) *st = out;
  return PF_OK;
}

int coarsen_particles(pf_ctx* ctx, int ptype, int target, unsigned seed, pf_coarsen_stats* st) {
  StageScope stage(ctx, PF_STAGE_ADAPT);
  pf_coarsen_stats out{};
  AdaptScratch* s = nullptr;
  int rc = scratch(ctx, &s);
  if (rc) return rc;
  target = max(1, target);
  const int n = (int)ctx->np;
  PF_CUDA_TRY(cudaMemsetAsync(s->d_stats, 0, 16 * sizeof(int), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(s->cnt, 0, s->ncell * sizeof(int), ctx->stream));
  int *key = ctx->pkey, *rank = ctx->prank, *list = ctx->perm, *keep = ctx->d_flags;
  const PSet P = particles_of(ctx);
  if (n > 0)
    (++ctx->launches), k_coarse_keys<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(ctx->g, P, n, ptype, seed, key,
                                                                                s->score, s->cnt, rank, s->d_stats);
  rc = scan_exclusive(ctx, s->cnt, s->start, (int)s->ncell, nullptr);
  if (rc) return rc;
  if (n > 0) {
    (++ctx->launches), k_place<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(key, rank, s->start, n, list);
    (++ctx->launches), k_coarse_rank<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(
        key, s->score, ctx->type, s->cnt, s->start, list, n, ptype, target, s->sorted, keep);
    (++ctx->launches), k_coarse_cells<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(key, s->cnt, s->start, s->sorted,
                                                                                 n, target, ctx->vol, s->d_stats);
  }
  PF_CUDA_TRY(cudaGetLastError());
  rc = compact(ctx, s, keep);
  if (rc) return rc;
  out.before = s->h_stats[0];
  out.cells = s->h_stats[1];
  out.overfull_cells = s->h_stats[2];
  out.after = s->h_stats[3];
  out.removed = n - (int)ctx->np;
  if (st) *st = out;
  return PF_OK;
}

int refill_liquid(pf_ctx* ctx, int target, unsigned seed, int interface_only, int interface_radius, int max_added,
                  pf_refill_stats* st) {
  StageScope stage(ctx, PF_STAGE_ADAPT);
  pf_refill_stats out{};
  AdaptScratch* s = nullptr;
  int rc = scratch(ctx, &s);
  if (rc) return rc;
  target = max(1, target);
  const int n = (int)ctx->np;
  PF_CUDA_TRY(cudaMemsetAsync(s->d_stats, 0, 16 * sizeof(int), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(s->cnt, 0, s->ncell * sizeof(int), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(s->fa, 0, s->ncell, ctx->stream));
  int *key = ctx->pkey, *rank = ctx->prank, *list = ctx->perm;
  const PSet P = particles_of(ctx);
  if (n > 0)
    (++ctx->launches), k_refill_keys<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(ctx->g, P, n, key, s->cnt, rank, s->fa);
  rc = scan_exclusive(ctx, s->cnt, s->start, (int)s->ncell, nullptr);
  if (rc) return rc;
  if (n > 0) {
    (++ctx->launches), k_place<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(key, rank, s->start, n, list);
    (++ctx->launches), k_index_rank<<<nblocks(n, kNT), kNT, 0, ctx->stream>>>(key, s->cnt, s->start, list, n,
                                                                                s->sorted);
  }
  const uint8_t* near = dilate_box(ctx, s, interface_radius);
  (++ctx->launches), k_refill_want<<<8 * ctx->num_sms, kNT, 0, ctx->stream>>>(s->cnt, near, s->ncell, target,
                                                                               interface_only, s->wanted, s->d_stats);
  PF_CUDA_TRY(cudaGetLastError());
  rc = scan_exclusive(ctx, s->wanted, s->woff, (int)s->ncell, s->d_stats + 4);
  if (rc) return rc;
  rc = read_stats(ctx, s, 5);
  if (rc) return rc;
  const long long budget = max_added > 0 ? (long long)max_added : (long long)INT_MAX;
  const long long total = s->h_stats[4];
  const long long added = min(total, budget);
  if ((size_t)n + (size_t)added > ctx->cap) {
    if (st) *st = pf_refill_stats{(int)added, 0, 0, 0, 0, 0, 0};  // what it would add
    return set_error(ctx, PF_ERR_CAPACITY, "refill would exceed max_particles");
  }
  if (added > 0)
    (++ctx->launches), k_refill_apply<<<8 * ctx->num_sms, kNT, 0, ctx->stream>>>(
        ctx->g, P, (size_t)n, s->cnt, s->start, s->sorted, s->wanted, s->woff, budget, seed);
  PF_CUDA_TRY(cudaGetLastError());
  ctx->np = (size_t)n + (size_t)added;
  ctx->bins_valid = false;
  out.cells = s->h_stats[0];
  out.before = s->h_stats[1];
  out.interface_cells = s->h_stats[2];
  out.underfull_cells = s->h_stats[3];
  out.budget_limited = total > budget ? 1 : 0;
  out.added = (int)added;
  out.after = out.before + out.added;
  if (st) *st = out;
  return PF_OK;
}

// ---- the step's particle reductions: max speed and liquid volume -------------

constexpr int kRedBlocks = 8 * 148;

// per CTA: the largest finite |v| (sqrt(vx^2 + vy^2 + vz^2) in FP64, the
// reference's order) and the liquid volume sum * Vp; part[2b], part[2b + 1]
__global__ void __launch_bounds__(kNT) k_particle_reduce(PSet P, int n, double Vp, double* part) {
  __shared__ double smax[kNT], ssum[kNT];
  double vmax = 0.0, vol = 0.0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double x = P.vx[p], y = P.vy[p], z = P.vz[p];
    if (isfinite(x) && isfinite(y) && isfinite(z)) {
      const double s = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
      vmax = fmax(vmax, s);
    }
    if (P.type[p] == 0) vol = __dadd_rn(vol, __dmul_rn((double)P.vol[p], Vp));
  }
  smax[threadIdx.x] = vmax;
  ssum[threadIdx.x] = vol;
  __syncthreads();
  for (int s = kNT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
      ssum[threadIdx.x] = __dadd_rn(ssum[threadIdx.x], ssum[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = smax[0];
    part[2 * blockIdx.x + 1] = ssum[0];
  }
}

// the partials in a fixed order (one thread: kRedBlocks values)
__global__ void k_particle_reduce_total(const double* part, int nb, double* out) {
  double vmax = 0.0, vol = 0.0;
  for (int b = 0; b < nb; ++b) {
    vmax = fmax(vmax, part[2 * b]);
    vol = __dadd_rn(vol, part[2 * b + 1]);
  }
  out[0] = vmax;
  out[1] = vol;
}

// SparseSim3DTP::applyParticleAdaptivity (src/driver/sparse_sim3d_tp.cpp:843-848)
int apply_adaptivity(pf_ctx* ctx, const pf_adapt_cfg& a, pf_adapt_stats* st) {
  pf_adapt_stats out{};
  int rc = PF_OK;
  if (a.narrow_band_air) rc = narrow_band_air(ctx, a.narrow_band_radius, &out.band);
  if (!rc && a.gas_coarsening) rc = coarsen_particles(ctx, 1, a.gas_per_cell_target, a.gas_seed, &out.gas);
  if (!rc && a.liquid_coarsening)
    rc = coarsen_particles(ctx, 0, a.liquid_per_cell_target, a.liquid_seed, &out.liquid);
  if (!rc && a.liquid_refill)
    rc = refill_liquid(ctx, a.refill_per_cell_target, a.refill_seed, a.refill_interface_only,
                       a.refill_interface_radius, a.refill_max_added, &out.refill);
  if (st) *st = out;
  return rc;
}

// computeAdaptiveParticleTimestep3D (src/driver/timestep3d.h:16-50) and
// updateVolumeCorrectionStats (src/driver/sparse_sim3d_tp.cpp:368-379): the
// step's dt and divergence correction from two device reductions.  The max
// speed is exact; the liquid volume is an FP64 sum in another order than the
// reference's particle order.  With wait == false (neither control changes
// the step) the reductions are read back behind an event and turned into
// statistics by step_controls_finish.
int step_controls(pf_ctx* ctx, double dt, double Vp, const pf_step_controls& c, pf_step_control_stats* st,
                  bool wait) {
  AdaptScratch* s = nullptr;
  int rc = scratch(ctx, &s);
  if (rc) return rc;
  const int n = (int)ctx->np;
  double* part = reinterpret_cast<double*>(ctx->partials);  // kRedBlocks * 2 doubles fit the PCG partials
  static_assert(2 * kRedBlocks <= kMaxRedBlocks * kRedSlots, "partials buffer too small");
  double* out = reinterpret_cast<double*>(s->d_stats + 8);  // two doubles in the 16-int statistics buffer
  const int nb = kRedBlocks;
  (++ctx->launches), k_particle_reduce<<<nb, kNT, 0, ctx->stream>>>(particles_of(ctx), n, Vp, part);
  (++ctx->launches), k_particle_reduce_total<<<1, 1, 0, ctx->stream>>>(part, nb, out);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ctl, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaEventRecord(s->ctl_ev, ctx->stream));
  s->ctl_pending = true;
  s->ctl_dt = dt;
  s->ctl_cfg = c;
  if (!wait) {
    // the step goes on with the requested dt, which is what the statistics will say
    pf_step_control_stats o{};
    o.requested_dt = o.effective_dt = o.cfl_limit_dt = dt;
    if (st) *st = o;
    return PF_OK;
  }
  rc = step_controls_finish(ctx, st);
  return rc;
}

int step_controls_finish(pf_ctx* ctx, pf_step_control_stats* st) {
  AdaptScratch* s = static_cast<AdaptScratch*>(ctx->adapt);
  if (!s || !s->ctl_pending) return PF_OK;
  PF_CUDA_TRY(cudaEventSynchronize(s->ctl_ev));
  s->ctl_pending = false;
  const double* h = s->h_ctl;
  const double dt = s->ctl_dt;
  const pf_step_controls& c = s->ctl_cfg;
  pf_step_control_stats o{};
  o.requested_dt = o.effective_dt = o.cfl_limit_dt = dt;
  o.max_particle_speed = h[0];
  if (c.adaptive_timestep && dt > 0.0 && ctx->g.dx > 0.0 && c.adaptive_cfl > 0.0 && h[0] > 0.0) {
    o.cfl_limit_dt = c.adaptive_cfl * ctx->g.dx / h[0];
    double lim = std::min(dt, o.cfl_limit_dt);
    if (c.adaptive_min_dt > 0.0) lim = std::max(c.adaptive_min_dt, lim);
    o.effective_dt = std::min(dt, lim);
    o.limited = o.effective_dt < dt ? 1 : 0;
  }
  o.liquid_volume_current = h[1];
  o.liquid_volume_error = c.liquid_volume_target - h[1];
  o.c_div = 0.0;
  if (c.c_div_volume_correction && c.c_div_strength > 0.0 && c.liquid_volume_target > 0.0 && o.effective_dt > 0.0)
    o.c_div = c.c_div_strength * o.liquid_volume_error / (o.effective_dt * c.liquid_volume_target);
  if (st) *st = o;
  return PF_OK;
}

void adapt_free(pf_ctx* ctx) {
  AdaptScratch* s = static_cast<AdaptScratch*>(ctx->adapt);
  if (!s) return;
  cudaFree(s->cnt);
  cudaFree(s->start);
  cudaFree(s->wanted);
  cudaFree(s->woff);
  cudaFree(s->fa);
  cudaFree(s->fb);
  cudaFree(s->score);
  cudaFree(s->sorted);
  cudaFree(s->d_stats);
  cudaFreeHost(s->h_stats);
  cudaFreeHost(s->h_ctl);
  if (s->ctl_ev) cudaEventDestroy(s->ctl_ev);
  delete s;
  ctx->adapt = nullptr;
}

}  // namespace pf
