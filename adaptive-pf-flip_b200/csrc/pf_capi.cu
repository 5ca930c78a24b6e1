// pf_capi.cu -- the extern "C" entry points of libpfgpu (include/pfgpu.h):
// context set-up, particle exchange, grid access and the solver-step calls.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <utility>

#include "pf_coarse.cuh"
#include "pf_ctx.h"

using namespace pf;

namespace {

// AoS (n x 3) -> SoA, FP32 or FP64 input
template <typename T>
__global__ void k_unpack3(const T* aos, float* a, float* b, float* c, size_t n) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  a[p] = (float)aos[3 * p + 0];
  b[p] = (float)aos[3 * p + 1];
  c[p] = (float)aos[3 * p + 2];
}

template <typename T>
__global__ void k_pack3(const float* a, const float* b, const float* c, T* aos, size_t n) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  aos[3 * p + 0] = (T)a[p];
  aos[3 * p + 1] = (T)b[p];
  aos[3 * p + 2] = (T)c[p];
}

template <typename T>
__global__ void k_convert(const T* in, float* out, size_t n) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = (float)in[p];
}

template <typename T>
__global__ void k_convert_back(const float* in, T* out, size_t n) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = (T)in[p];
}

void free_all(pf_ctx* c) {
  auto F = [](void* p) { if (p) cudaFree(p); };
  pf::coarse_release(c);
  pf::adapt_free(c);
  pf::diag_free(c);
  pf::mr_free(c);
  pf::secondary_free(c);
  F(c->tile_slot); F(c->slot_tile); F(c->d_nslots); F(c->tile_need); F(c->tile_new); F(c->tile_rank);
  for (int f = 0; f < PF_NFIELDS; ++f) { F(c->fld[f]); F(c->act4[f]); }
  for (int a = 0; a < PF_NSAVED; ++a) F(c->saved[a]);
  F(c->d_wall_tiles);
  F(c->px); F(c->py); F(c->pz); F(c->vx); F(c->vy); F(c->vz); F(c->vol); F(c->type); F(c->staging);
  F(c->tile_count); F(c->tile_start); F(c->pkey); F(c->prank); F(c->perm); F(c->splat_stage);
  for (int* p : c->scan_levels) F(p);
  F(c->d_scalar);
  F(c->x); F(c->r); F(c->p); F(c->Ap); F(c->diag); F(c->cx); F(c->cy); F(c->cz); F(c->kind); F(c->z_plain);
  F(c->partials); F(c->ctl); F(c->ctl_outer); F(c->nbr_plain);
  F(c->xf); F(c->rf); F(c->pf32); F(c->Apf); F(c->diagf); F(c->cxf); F(c->cyf); F(c->czf); F(c->pbf); F(c->cbf);
  F(c->b64);
  F(c->d_clamp); F(c->d_flags); F(c->cell_flags); F(c->esc_buf); F(c->mk_first); F(c->rc_buf);
  if (c->up_stream) cudaStreamSynchronize(c->up_stream);
  F(c->bpx); F(c->bpy); F(c->bpz); F(c->bvx); F(c->bvy); F(c->bvz); F(c->bvol); F(c->btype); F(c->up_staging);
  if (c->up_done) cudaEventDestroy(c->up_done);
  if (c->back_free) cudaEventDestroy(c->back_free);
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  for (int q = 0; q < 2; ++q) {
    F(c->dl_staging[q]);
    if (c->dl_packed[q]) cudaEventDestroy(c->dl_packed[q]);
    if (c->dl_copied[q]) cudaEventDestroy(c->dl_copied[q]);
  }
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  for (const auto& t : c->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
  for (int s = 0; s < PF_NSTAGES; ++s) if (c->open_ev[s]) cudaEventDestroy(c->open_ev[s]);
  if (c->h_ctl) cudaFreeHost(c->h_ctl);
  if (c->h_pinned_ints) cudaFreeHost(c->h_pinned_ints);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->pool_ev) cudaEventDestroy(c->pool_ev);
  if (c->stream) cudaStreamDestroy(c->stream);
}

int create_impl(pf_ctx* ctx, const pf_grid_desc* d) {
  PF_CUDA_TRY(cudaSetDevice(d->device));
  cudaDeviceProp prop;
  PF_CUDA_TRY(cudaGetDeviceProperties(&prop, d->device));
  if (prop.major < 10) return set_error(ctx, PF_ERR_NO_DEVICE, "libpfgpu needs an sm_100 device");
  ctx->device = d->device;
  ctx->num_sms = prop.multiProcessorCount;
  PF_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  PF_CUDA_TRY(cudaEventCreate(&ctx->ev0));
  PF_CUDA_TRY(cudaEventCreate(&ctx->ev1));

  Geom& g = ctx->g;
  g.nx = d->nx; g.ny = d->ny; g.nz = d->nz;
  g.dx = d->dx; g.ox = d->ox; g.oy = d->oy; g.oz = d->oz;
  g.inv_dx = 1.0 / d->dx;
  {
    int e = 0;
    g.dx_pow2 = std::frexp(d->dx, &e) == 0.5 ? 1 : 0;
  }
  g.TX = (d->nx + 1 + 7) / 8; g.TY = (d->ny + 1 + 7) / 8; g.TZ = (d->nz + 1 + 7) / 8;
  g.ntiles = g.TX * g.TY * g.TZ;
  const int dims[PF_NFIELDS][3] = {{g.nx + 1, g.ny, g.nz}, {g.nx, g.ny + 1, g.nz}, {g.nx, g.ny, g.nz + 1},
                                   {g.nx + 1, g.ny, g.nz}, {g.nx, g.ny + 1, g.nz}, {g.nx, g.ny, g.nz + 1},
                                   {g.nx, g.ny, g.nz},     {g.nx, g.ny, g.nz}};
  size_t max_field_nodes = 0;
  for (int f = 0; f < PF_NFIELDS; ++f) {
    for (int a = 0; a < 3; ++a) {
      g.fdim[f][a] = dims[f][a];
      g.bdim[f][a] = (dims[f][a] + 3) / 4;
    }
    const size_t nn = (size_t)dims[f][0] * dims[f][1] * dims[f][2];
    if (nn > max_field_nodes) max_field_nodes = nn;
    ctx->act4_n[f] = (size_t)g.bdim[f][0] * g.bdim[f][1] * g.bdim[f][2];
  }
  const size_t nt = (size_t)g.ntiles;
  const size_t cells = nt * PF_TV;  // pool capacity = every tile
  ctx->cells_cap = cells;

  PF_CUDA_TRY(cudaMalloc(&ctx->tile_slot, nt * sizeof(int)));
  PF_CUDA_TRY(cudaMemset(ctx->tile_slot, 0xff, nt * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->slot_tile, nt * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->d_nslots, sizeof(int)));
  PF_CUDA_TRY(cudaMemset(ctx->d_nslots, 0, sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->tile_need, nt));
  PF_CUDA_TRY(cudaMemset(ctx->tile_need, 0, nt));
  PF_CUDA_TRY(cudaMalloc(&ctx->tile_new, nt * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->tile_rank, nt * sizeof(int)));
  for (int f = 0; f < PF_NFIELDS; ++f) {
    PF_CUDA_TRY(cudaMalloc(&ctx->fld[f], cells * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(ctx->fld[f], 0, cells * sizeof(float)));
    PF_CUDA_TRY(cudaMalloc(&ctx->act4[f], ctx->act4_n[f]));
    PF_CUDA_TRY(cudaMemset(ctx->act4[f], 0, ctx->act4_n[f]));
  }
  for (int a = 0; a < PF_NSAVED; ++a) {
    PF_CUDA_TRY(cudaMalloc(&ctx->saved[a], cells * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(ctx->saved[a], 0, cells * sizeof(float)));
  }
  // tiles touched by markCells walls and applyWallBoundary: every tile with
  // a node at index 0, 1, n-1 or n along some axis
  {
    std::vector<int>& wt = ctx->wall_tiles;
    auto on_wall = [](int t, int n) {
      const int lo = t * 8, hi = t * 8 + 7;
      const int cand[4] = {0, 1, n - 1, n};
      for (int q = 0; q < 4; ++q)
        if (cand[q] >= lo && cand[q] <= hi && cand[q] >= 0) return true;
      return false;
    };
    for (int tz = 0; tz < g.TZ; ++tz)
      for (int ty = 0; ty < g.TY; ++ty)
        for (int tx = 0; tx < g.TX; ++tx)
          if (on_wall(tx, g.nx) || on_wall(ty, g.ny) || on_wall(tz, g.nz)) wt.push_back(tile_id(g, tx, ty, tz));
    PF_CUDA_TRY(cudaMalloc(&ctx->d_wall_tiles, (wt.size() + 1) * sizeof(int)));
    if (!wt.empty())
      PF_CUDA_TRY(cudaMemcpy(ctx->d_wall_tiles, wt.data(), wt.size() * sizeof(int), cudaMemcpyHostToDevice));
  }

  // particles
  const size_t cap = d->max_particles > 0 ? d->max_particles : 1;
  ctx->cap = cap;
  float** pa[7] = {&ctx->px, &ctx->py, &ctx->pz, &ctx->vx, &ctx->vy, &ctx->vz, &ctx->vol};
  for (float** q : pa) PF_CUDA_TRY(cudaMalloc(q, cap * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->type, cap));
  const long long ncell = (long long)g.nx * g.ny * g.nz;
  size_t stg = cap * 3 * sizeof(double);
  const size_t fld_bytes = max_field_nodes * sizeof(float) + ctx->act4_n[0] + 64;
  if (fld_bytes > stg) stg = fld_bytes;
  if ((size_t)ncell * sizeof(int32_t) > stg) stg = (size_t)ncell * sizeof(int32_t);
  if ((size_t)(4096 + 16) * sizeof(double) > stg) stg = (4096 + 16) * sizeof(double);
  ctx->staging_bytes = stg;
  PF_CUDA_TRY(cudaMalloc(&ctx->staging, stg));

  // particle bins: one per pooled cell slot (tile * 512 + local cell)
  PF_CUDA_TRY(cudaMalloc(&ctx->tile_count, (cells + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->tile_start, (cells + 2) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->pkey, cap * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->prank, cap * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->perm, cap * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->splat_stage, nt * (size_t)pf::kSplatStageTile * sizeof(float2)));
  size_t scan_max = cells + 1;
  if ((size_t)ncell > scan_max) scan_max = (size_t)ncell;
  if (cap > scan_max) scan_max = cap;
  int rc = scan_alloc(ctx, scan_max);
  if (rc) return rc;
  PF_CUDA_TRY(cudaMalloc(&ctx->d_scalar, 16 * sizeof(int)));

  double** dv[9] = {&ctx->x, &ctx->r, &ctx->p, &ctx->Ap, &ctx->diag, &ctx->cx, &ctx->cy, &ctx->cz, &ctx->z_plain};
  for (double** q : dv) {
    PF_CUDA_TRY(cudaMalloc(q, cells * sizeof(double)));
    PF_CUDA_TRY(cudaMemset(*q, 0, cells * sizeof(double)));
  }
  PF_CUDA_TRY(cudaMalloc(&ctx->kind, cells));
  PF_CUDA_TRY(cudaMemset(ctx->kind, 0, cells));
  // per-CTA partials: up to kRedSlots doubles per reduction CTA
  PF_CUDA_TRY(cudaMalloc(&ctx->partials, (size_t)kMaxRedBlocks * kRedSlots * sizeof(double)));
  PF_CUDA_TRY(cudaMalloc(&ctx->nbr_plain, (cells / PF_TV + 1) * 6 * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->ctl, sizeof(SolveCtl)));
  PF_CUDA_TRY(cudaMemset(ctx->ctl, 0, sizeof(SolveCtl)));
  PF_CUDA_TRY(cudaMallocHost(&ctx->h_ctl, sizeof(SolveCtl)));
  PF_CUDA_TRY(cudaMalloc(&ctx->ctl_outer, sizeof(SolveCtl)));
  PF_CUDA_TRY(cudaMemset(ctx->ctl_outer, 0, sizeof(SolveCtl)));
  PF_CUDA_TRY(cudaMallocHost(&ctx->h_pinned_ints, 64 * sizeof(int)));
  ctx->h_nslots = ctx->h_pinned_ints + 32;  // the deferred pool-size read-back; no other use of that entry
  PF_CUDA_TRY(cudaEventCreateWithFlags(&ctx->pool_ev, cudaEventDisableTiming));
  PF_CUDA_TRY(cudaMalloc(&ctx->d_clamp, 8 * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&ctx->d_flags, 2 * cap * sizeof(int)));
  size_t cf = 2 * (size_t)ncell + 2;
  for (int f = 0; f < PF_NFIELDS; ++f)
    if (2 * ctx->act4_n[f] + 2 > cf) cf = 2 * ctx->act4_n[f] + 2;
  PF_CUDA_TRY(cudaMalloc(&ctx->cell_flags, cf * sizeof(int32_t)));
  PF_CUDA_TRY(cudaMalloc(&ctx->mk_first, ctx->act4_n[PF_MK] * sizeof(uint32_t)));
  PF_CUDA_TRY(cudaMemset(ctx->mk_first, 0xff, ctx->act4_n[PF_MK] * sizeof(uint32_t)));
  PF_CUDA_TRY(cudaDeviceSynchronize());
  return PF_OK;
}

bool valid_field(int f) { return f >= 0 && f < PF_NFIELDS; }

}  // namespace

namespace pf {
// The second particle set: filled by asynchronous uploads and by compaction,
// then swapped in.  Allocated on first use.
int ensure_back_set(pf_ctx* ctx) {
  if (ctx->up_stream) return PF_OK;
  const size_t cap = ctx->cap;
  PF_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->up_stream, cudaStreamNonBlocking));
  PF_CUDA_TRY(cudaEventCreateWithFlags(&ctx->up_done, cudaEventDisableTiming));
  PF_CUDA_TRY(cudaEventCreateWithFlags(&ctx->back_free, cudaEventDisableTiming));
  float** pa[7] = {&ctx->bpx, &ctx->bpy, &ctx->bpz, &ctx->bvx, &ctx->bvy, &ctx->bvz, &ctx->bvol};
  for (float** q : pa) PF_CUDA_TRY(cudaMalloc(q, cap * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->btype, cap));
  PF_CUDA_TRY(cudaMalloc(&ctx->up_staging, 6 * cap * sizeof(float)));
  return PF_OK;
}
}  // namespace pf

extern "C" {

int pf_create(const pf_grid_desc* desc, pf_ctx** out) {
  if (!desc || !out) return PF_ERR_INVALID;
  *out = nullptr;
  if (desc->nx <= 0 || desc->ny <= 0 || desc->nz <= 0 || !(desc->dx > 0.0)) return PF_ERR_INVALID;
  if ((long long)desc->nx * desc->ny * desc->nz > (1LL << 31) - 1) return PF_ERR_INVALID;
  if (desc->max_particles > (size_t)0x7fffffff) return PF_ERR_INVALID;
  pf_ctx* ctx = new (std::nothrow) pf_ctx();
  if (!ctx) return PF_ERR_INVALID;
  const int rc = create_impl(ctx, desc);
  if (rc) {
    fprintf(stderr, "pf_create: %s\n", ctx->err.c_str());
    free_all(ctx);
    delete ctx;
    return rc;
  }
  *out = ctx;
  return PF_OK;
}

int pf_destroy(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return PF_OK;
}

const char* pf_last_error(const pf_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pf_sync(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->copy_stream) PF_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
  if (ctx->up_stream) PF_CUDA_TRY(cudaStreamSynchronize(ctx->up_stream));
  return PF_OK;
}

void* pf_stream(pf_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

size_t pf_num_particles(const pf_ctx* ctx) { return ctx ? (ctx->up_pending ? ctx->np_next : ctx->np) : 0; }

// the pool size lives on the device until read back; reading it here waits
// for that copy (the only state this changes)
int pf_active_tiles(const pf_ctx* ctx) {
  if (!ctx) return -1;
  pf_ctx* c = const_cast<pf_ctx*>(ctx);
  cudaSetDevice(c->device);
  if (pool_sync(c)) return -1;
  return c->nslots;
}

// Swap in the particle set of a pending asynchronous upload: the context
// stream waits for it, and the set it replaces becomes free for the next
// upload once the work queued so far (which still reads it) is done.
static int take_upload(pf_ctx* ctx) {
  if (!ctx->up_pending) return PF_OK;
  PF_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->up_done, 0));
  std::swap(ctx->px, ctx->bpx);
  std::swap(ctx->py, ctx->bpy);
  std::swap(ctx->pz, ctx->bpz);
  std::swap(ctx->vx, ctx->bvx);
  std::swap(ctx->vy, ctx->bvy);
  std::swap(ctx->vz, ctx->bvz);
  std::swap(ctx->vol, ctx->bvol);
  std::swap(ctx->type, ctx->btype);
  ctx->np = ctx->np_next;
  ctx->bins_valid = false;
  PF_CUDA_TRY(cudaEventRecord(ctx->back_free, ctx->stream));
  ctx->back_free_recorded = true;
  ctx->up_pending = false;
  return PF_OK;
}

static int upload_impl(pf_ctx* ctx, size_t n, const void* pos, const void* vel, const uint8_t* type,
                       const void* vol, bool f64) {
  if (!ctx || (n && (!pos || !vel || !type || !vol))) return PF_ERR_INVALID;
  if (n > ctx->cap) return set_error(ctx, PF_ERR_CAPACITY, "more particles than max_particles");
  cudaSetDevice(ctx->device);
  int rc = take_upload(ctx);
  if (rc) return rc;
  ctx->np = n;
  ctx->bins_valid = false;
  if (n == 0) return PF_OK;
  const size_t es = f64 ? sizeof(double) : sizeof(float);
  const int nb = nblocks(n, 256);
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->staging, pos, 3 * n * es, cudaMemcpyDefault, ctx->stream));
  if (f64) (++ctx->launches), k_unpack3<double><<<nb, 256, 0, ctx->stream>>>((const double*)ctx->staging, ctx->px, ctx->py, ctx->pz, n);
  else (++ctx->launches), k_unpack3<float><<<nb, 256, 0, ctx->stream>>>((const float*)ctx->staging, ctx->px, ctx->py, ctx->pz, n);
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->staging, vel, 3 * n * es, cudaMemcpyDefault, ctx->stream));
  if (f64) (++ctx->launches), k_unpack3<double><<<nb, 256, 0, ctx->stream>>>((const double*)ctx->staging, ctx->vx, ctx->vy, ctx->vz, n);
  else (++ctx->launches), k_unpack3<float><<<nb, 256, 0, ctx->stream>>>((const float*)ctx->staging, ctx->vx, ctx->vy, ctx->vz, n);
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->type, type, n, cudaMemcpyDefault, ctx->stream));
  if (f64) {
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->staging, vol, n * es, cudaMemcpyDefault, ctx->stream));
    (++ctx->launches), k_convert<double><<<nb, 256, 0, ctx->stream>>>((const double*)ctx->staging, ctx->vol, n);
  } else {
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->vol, vol, n * es, cudaMemcpyDefault, ctx->stream));
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

static int download_impl(pf_ctx* ctx, void* pos, void* vel, uint8_t* type, void* vol, bool f64) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = take_upload(ctx);
  if (rc) return rc;
  const size_t n = ctx->np;
  if (n == 0) return PF_OK;
  const size_t es = f64 ? sizeof(double) : sizeof(float);
  const int nb = nblocks(n, 256);
  if (pos) {
    if (f64) (++ctx->launches), k_pack3<double><<<nb, 256, 0, ctx->stream>>>(ctx->px, ctx->py, ctx->pz, (double*)ctx->staging, n);
    else (++ctx->launches), k_pack3<float><<<nb, 256, 0, ctx->stream>>>(ctx->px, ctx->py, ctx->pz, (float*)ctx->staging, n);
    PF_CUDA_TRY(cudaMemcpyAsync(pos, ctx->staging, 3 * n * es, cudaMemcpyDefault, ctx->stream));
  }
  if (vel) {
    if (f64) (++ctx->launches), k_pack3<double><<<nb, 256, 0, ctx->stream>>>(ctx->vx, ctx->vy, ctx->vz, (double*)ctx->staging, n);
    else (++ctx->launches), k_pack3<float><<<nb, 256, 0, ctx->stream>>>(ctx->vx, ctx->vy, ctx->vz, (float*)ctx->staging, n);
    PF_CUDA_TRY(cudaMemcpyAsync(vel, ctx->staging, 3 * n * es, cudaMemcpyDefault, ctx->stream));
  }
  if (type) PF_CUDA_TRY(cudaMemcpyAsync(type, ctx->type, n, cudaMemcpyDefault, ctx->stream));
  if (vol) {
    if (f64) {
      (++ctx->launches), k_convert_back<double><<<nb, 256, 0, ctx->stream>>>(ctx->vol, (double*)ctx->staging, n);
      PF_CUDA_TRY(cudaMemcpyAsync(vol, ctx->staging, n * es, cudaMemcpyDefault, ctx->stream));
    } else {
      PF_CUDA_TRY(cudaMemcpyAsync(vol, ctx->vol, n * es, cudaMemcpyDefault, ctx->stream));
    }
  }
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int pf_upload_particles(pf_ctx* ctx, size_t n, const float* pos, const float* vel, const uint8_t* type,
                        const float* volume) {
  return upload_impl(ctx, n, pos, vel, type, volume, false);
}
int pf_download_particles(pf_ctx* ctx, float* pos, float* vel, uint8_t* type, float* volume) {
  return download_impl(ctx, pos, vel, type, volume, false);
}
// Asynchronous FP32 download: the arrays are packed into one of two device
// staging slots on the context stream, and the host copies run on a second
// stream, so they overlap the calls that follow (the next step's upload runs
// against the other direction of the link).  A slot is reused only after its
// previous host copy finished.
int pf_download_particles_async(pf_ctx* ctx, float* pos, float* vel, uint8_t* type, float* volume) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  {
    const int rc = take_upload(ctx);
    if (rc) return rc;
  }
  const size_t n = ctx->np;
  if (n == 0 || (!pos && !vel && !type && !volume)) return PF_OK;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b3 = up(3 * n * sizeof(float)), b1 = up(n * sizeof(float)), bt = up(n);
  const size_t need = 2 * b3 + b1 + bt;  // room for every array
  if (!ctx->copy_stream) {
    PF_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for (int q = 0; q < 2; ++q) {
      PF_CUDA_TRY(cudaEventCreateWithFlags(&ctx->dl_packed[q], cudaEventDisableTiming));
      PF_CUDA_TRY(cudaEventCreateWithFlags(&ctx->dl_copied[q], cudaEventDisableTiming));
    }
  }
  if (ctx->dl_bytes < need) {
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < 2; ++q) {
      if (ctx->dl_staging[q]) PF_CUDA_TRY(cudaFree(ctx->dl_staging[q]));
      ctx->dl_staging[q] = nullptr;
      ctx->dl_recorded[q] = false;
    }
    ctx->dl_bytes = 0;
    for (int q = 0; q < 2; ++q) PF_CUDA_TRY(cudaMalloc(&ctx->dl_staging[q], need));
    ctx->dl_bytes = need;
  }
  const int slot = ctx->dl_slot;
  ctx->dl_slot ^= 1;
  if (ctx->dl_recorded[slot]) PF_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->dl_copied[slot], 0));
  char* st = (char*)ctx->dl_staging[slot];
  float* s_pos = (float*)st;
  float* s_vel = (float*)(st + b3);
  float* s_vol = (float*)(st + 2 * b3);
  uint8_t* s_type = (uint8_t*)(st + 2 * b3 + b1);
  const int nb = nblocks(n, 256);
  if (pos) (++ctx->launches), k_pack3<float><<<nb, 256, 0, ctx->stream>>>(ctx->px, ctx->py, ctx->pz, s_pos, n);
  if (vel) (++ctx->launches), k_pack3<float><<<nb, 256, 0, ctx->stream>>>(ctx->vx, ctx->vy, ctx->vz, s_vel, n);
  if (type) PF_CUDA_TRY(cudaMemcpyAsync(s_type, ctx->type, n, cudaMemcpyDeviceToDevice, ctx->stream));
  if (volume) PF_CUDA_TRY(cudaMemcpyAsync(s_vol, ctx->vol, n * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaEventRecord(ctx->dl_packed[slot], ctx->stream));
  PF_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->dl_packed[slot], 0));
  if (pos) PF_CUDA_TRY(cudaMemcpyAsync(pos, s_pos, 3 * n * sizeof(float), cudaMemcpyDefault, ctx->copy_stream));
  if (vel) PF_CUDA_TRY(cudaMemcpyAsync(vel, s_vel, 3 * n * sizeof(float), cudaMemcpyDefault, ctx->copy_stream));
  if (type) PF_CUDA_TRY(cudaMemcpyAsync(type, s_type, n, cudaMemcpyDefault, ctx->copy_stream));
  if (volume) PF_CUDA_TRY(cudaMemcpyAsync(volume, s_vol, n * sizeof(float), cudaMemcpyDefault, ctx->copy_stream));
  PF_CUDA_TRY(cudaEventRecord(ctx->dl_copied[slot], ctx->copy_stream));
  ctx->dl_recorded[slot] = true;
  ctx->dl_last = slot;
  return PF_OK;
}

// The context stream waits (on the device) for every asynchronous download so
// far: work or events queued on it afterwards follow those host copies.
int pf_join_downloads(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->dl_last >= 0) PF_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->dl_copied[ctx->dl_last], 0));
  return PF_OK;
}

// Asynchronous FP32 upload into the second particle set: the host copies
// and the unpacking run on their own stream, overlapping the work already
// queued (the current step), and the next call that uses the particles swaps
// the set in.  A later upload before that call replaces this one.
int pf_upload_particles_async(pf_ctx* ctx, size_t n, const float* pos, const float* vel, const uint8_t* type,
                              const float* volume) {
  if (!ctx || (n && (!pos || !vel || !type || !volume))) return PF_ERR_INVALID;
  if (n > ctx->cap) return set_error(ctx, PF_ERR_CAPACITY, "more particles than max_particles");
  cudaSetDevice(ctx->device);
  const size_t cap = ctx->cap;
  {
    const int rc = pf::ensure_back_set(ctx);
    if (rc) return rc;
  }
  if (ctx->up_pending) PF_CUDA_TRY(cudaEventSynchronize(ctx->up_done));  // superseded; its copies must land first
  // the second set was the particles of earlier work: wait until that work is done
  if (ctx->back_free_recorded) PF_CUDA_TRY(cudaStreamWaitEvent(ctx->up_stream, ctx->back_free, 0));
  if (n > 0) {
    const int nb = nblocks(n, 256);
    float* sp = ctx->up_staging;
    float* sv = ctx->up_staging + 3 * cap;
    PF_CUDA_TRY(cudaMemcpyAsync(sp, pos, 3 * n * sizeof(float), cudaMemcpyDefault, ctx->up_stream));
    PF_CUDA_TRY(cudaMemcpyAsync(sv, vel, 3 * n * sizeof(float), cudaMemcpyDefault, ctx->up_stream));
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->btype, type, n, cudaMemcpyDefault, ctx->up_stream));
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->bvol, volume, n * sizeof(float), cudaMemcpyDefault, ctx->up_stream));
    (++ctx->launches), k_unpack3<float><<<nb, 256, 0, ctx->up_stream>>>(sp, ctx->bpx, ctx->bpy, ctx->bpz, n);
    (++ctx->launches), k_unpack3<float><<<nb, 256, 0, ctx->up_stream>>>(sv, ctx->bvx, ctx->bvy, ctx->bvz, n);
    PF_CUDA_TRY(cudaGetLastError());
  }
  PF_CUDA_TRY(cudaEventRecord(ctx->up_done, ctx->up_stream));
  ctx->np_next = n;
  ctx->up_pending = true;
  return PF_OK;
}

int pf_upload_particles_f64(pf_ctx* ctx, size_t n, const double* pos, const double* vel, const uint8_t* type,
                            const double* volume) {
  return upload_impl(ctx, n, pos, vel, type, volume, true);
}
int pf_download_particles_f64(pf_ctx* ctx, double* pos, double* vel, uint8_t* type, double* volume) {
  return download_impl(ctx, pos, vel, type, volume, true);
}

int pf_grid_set_field(pf_ctx* ctx, int field, const float* dense, const uint8_t* act4) {
  if (!ctx || !valid_field(field) || !dense || !act4) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::grid_set_field(ctx, field, dense, act4);
}

int pf_grid_get_field(pf_ctx* ctx, int field, float* dense, uint8_t* act4) {
  if (!ctx || !valid_field(field)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::grid_get_field(ctx, field, dense, act4);
}

int pf_grid_clear_field(pf_ctx* ctx, int field) {
  if (!ctx || !valid_field(field)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return field_clear(ctx, field);
}

int pf_grid_clear_all(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pool_reset(ctx);
}

int pf_grid_copy(pf_ctx* dst, const pf_ctx* src) {
  if (!dst || !src) return PF_ERR_INVALID;
  const Geom &a = dst->g, &b = src->g;
  if (a.nx != b.nx || a.ny != b.ny || a.nz != b.nz) return set_error(dst, PF_ERR_INVALID, "grid shapes differ");
  if (dst->device != src->device) return set_error(dst, PF_ERR_INVALID, "contexts on different devices");
  pf_ctx* ctx = dst;
  cudaSetDevice(ctx->device);
  PF_CUDA_TRY(cudaStreamSynchronize(src->stream));
  int rc = pool_sync(const_cast<pf_ctx*>(src));  // the source's pool size, read back
  if (!rc) rc = pool_reset(dst);
  if (rc) return rc;
  const size_t nt = (size_t)a.ntiles;
  const size_t cells = (size_t)src->nslots * PF_TV;
  PF_CUDA_TRY(cudaMemcpyAsync(dst->tile_slot, src->tile_slot, nt * sizeof(int), cudaMemcpyDeviceToDevice, dst->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(dst->slot_tile, src->slot_tile, nt * sizeof(int), cudaMemcpyDeviceToDevice, dst->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(dst->d_nslots, src->d_nslots, sizeof(int), cudaMemcpyDeviceToDevice, dst->stream));
  for (int f = 0; f < PF_NFIELDS; ++f) {
    if (cells) PF_CUDA_TRY(cudaMemcpyAsync(dst->fld[f], src->fld[f], cells * sizeof(float), cudaMemcpyDeviceToDevice, dst->stream));
    PF_CUDA_TRY(cudaMemcpyAsync(dst->act4[f], src->act4[f], dst->act4_n[f], cudaMemcpyDeviceToDevice, dst->stream));
  }
  for (int s = 0; s < PF_NSAVED; ++s)
    if (cells) PF_CUDA_TRY(cudaMemcpyAsync(dst->saved[s], src->saved[s], cells * sizeof(float), cudaMemcpyDeviceToDevice, dst->stream));
  dst->nslots = src->nslots;
  dst->saved_valid = src->saved_valid;
  PF_CUDA_TRY(cudaStreamSynchronize(dst->stream));
  return PF_OK;
}

int pf_active_blocks4(pf_ctx* ctx, int field, int32_t* ids, size_t* n) {
  if (!ctx || !valid_field(field) || !n) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::active_blocks4(ctx, field, ids, n);
}

int pf_active_cells(pf_ctx* ctx, int32_t* cells, size_t* n) {
  if (!ctx || !n) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::active_cells(ctx, cells, n);
}

int pf_mark_cells(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  {
    const int rc = take_upload(ctx);
    if (rc) return rc;
  }
  return pf::mark_cells(ctx);
}

int pf_p2g(pf_ctx* ctx, const pf_phase* phase, double Vp) {
  if (!ctx || !phase) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  {
    const int rc = take_upload(ctx);
    if (rc) return rc;
  }
  return pf::p2g(ctx, phase, Vp);
}

int pf_save_velocity(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::save_velocity(ctx);
}

int pf_apply_gravity(pf_ctx* ctx, double dt, double gravity) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::apply_gravity(ctx, dt, gravity);
}

int pf_apply_wall_boundary(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::apply_walls(ctx);
}

static int check_solve_cfg(const pf_solve_cfg* cfg) {
  if (!cfg) return PF_ERR_INVALID;
  if (cfg->mode < PF_SOLVER_PLAIN || cfg->mode > PF_SOLVER_LEARNED) return PF_ERR_INVALID;
  if (cfg->max_iter < 0 || !(cfg->abs_tol >= 0.0) || !(cfg->rel_tol >= 0.0)) return PF_ERR_INVALID;
  return PF_OK;
}

int pf_project(pf_ctx* ctx, const pf_phase* phase, double dt, const pf_solve_cfg* cfg, pf_solve_stats* stats) {
  if (!ctx || !phase || check_solve_cfg(cfg)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::project(ctx, phase, dt, cfg, stats);
}

int pf_g2p(pf_ctx* ctx, const pf_ctx* saved, double alpha_l, double alpha_g) {
  if (!ctx) return PF_ERR_INVALID;
  if (saved && saved != ctx) {
    const Geom &a = ctx->g, &b = saved->g;
    if (a.nx != b.nx || a.ny != b.ny || a.nz != b.nz || saved->device != ctx->device)
      return set_error(ctx, PF_ERR_INVALID, "saved grid differs in shape or device");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(saved->stream);
  }
  cudaSetDevice(ctx->device);
  const int rc = take_upload(ctx);
  if (rc) return rc;
  return pf::g2p(ctx, saved, alpha_l, alpha_g);
}

int pf_advect(pf_ctx* ctx, double dt, int order, pf_clamp_stats* stats, double* escape, size_t* n_escape) {
  if (!ctx || (order != 2 && order != 3)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  {
    const int rc = take_upload(ctx);
    if (rc) return rc;
  }
  return pf::advect(ctx, dt, order, stats, escape, n_escape);
}

// SparseSim3DTP::step() order (src/driver/sparse_sim3d_tp.cpp:854-884):
// markCells, P2G, saved copy, gravity, walls, projection, G2P, advection.
// The grid holds nothing across steps, so the pool is rebuilt from scratch.
// Up to the projection nothing waits for the device: the pool grows on the
// device, and the step-control and interface statistics are read back behind
// events once the solve has synchronised anyway (unless the adaptive timestep
// or the volume correction needs them first, or adaptivity is on).
static int step_impl(pf_ctx* ctx, const pf_step_cfg* cfg, pf_step_stats* stats) {
  int rc = take_upload(ctx);
  if (rc) return rc;
  // applyParticleAdaptivity comes first in SparseSim3DTP::step()
  if (ctx->adapt_on) {
    rc = pf::apply_adaptivity(ctx, ctx->adapt_cfg, &ctx->adapt_last);
    if (rc) return rc;
  }
  // then computeAdaptiveParticleTimestep3D and updateVolumeCorrectionStats
  const bool controls_now = ctx->controls.adaptive_timestep || ctx->controls.c_div_volume_correction;
  rc = pf::step_controls(ctx, cfg->dt, cfg->Vp, ctx->controls, &ctx->controls_last, controls_now);
  if (rc) return rc;
  const double dt = ctx->controls_last.effective_dt;
  // advanceSecondaryLifecycle, before updateVolumeCorrectionStats: when it
  // may move particles into the primary set the liquid volume is taken again
  const bool secondary = pf::secondary_active(ctx);
  if (secondary) {
    const bool reabsorbs = pf::secondary_reabsorbs(ctx);
    rc = pf::secondary_lifecycle(ctx, dt, cfg->gravity, cfg->Vp);
    if (rc) return rc;
    if (reabsorbs) {
      rc = pf::step_controls_finish(ctx, &ctx->controls_last);  // the timestep, from before the lifecycle
      if (rc) return rc;
      pf_step_controls vc = ctx->controls;
      vc.adaptive_timestep = 0;
      pf_step_control_stats vs{};
      rc = pf::step_controls(ctx, dt, cfg->Vp, vc, &vs, true);
      if (rc) return rc;
      ctx->controls_last.liquid_volume_current = vs.liquid_volume_current;
      ctx->controls_last.liquid_volume_error = vs.liquid_volume_error;
      ctx->controls_last.c_div = vs.c_div;
    }
  }
  pf_solve_cfg solve = cfg->solve;
  if (ctx->controls.c_div_volume_correction) solve.c_div = ctx->controls_last.c_div;
  rc = pool_reset(ctx);
  if (rc) return rc;
  rc = pf::mark_cells(ctx);
  if (rc) return rc;
  rc = pf::p2g(ctx, &cfg->phase, cfg->Vp);  // normalisation without the fused extras
  if (rc) return rc;
  rc = pf::interface_diagnostics(ctx, &cfg->phase, nullptr, false);  // diagnoseSparseInterface3D after P2G
  if (rc) return rc;
  rc = pf::save_velocity(ctx);
  if (rc) return rc;
  rc = pf::apply_gravity(ctx, dt, cfg->gravity);
  if (rc) return rc;
  if (ctx->st_strength > 0.0) {  // applySparseSurfaceTension3D between gravity and the walls
    rc = pf::surface_tension(ctx, &cfg->phase, dt, ctx->st_strength, ctx->st_max_dv, ctx->st_radius, nullptr);
    if (rc) return rc;
  } else {
    ctx->surface_last = pf_surface_stats{};
  }
  rc = pf::apply_walls(ctx);
  if (rc) return rc;
  pf_solve_stats sst{};
  rc = pf::project(ctx, &cfg->phase, dt, &solve, &sst);
  if (rc) return rc;
  pf_clamp_stats cst{};
  int* esc = secondary ? pf::secondary_escape_flags(ctx) : nullptr;
  rc = pf::g2p_advect(ctx, cfg->alpha_l, cfg->alpha_g, dt, cfg->advect_order, &cst, esc);
  if (rc) return rc;
  if (secondary) {  // storeEscapedParticles and emitSecondarySpray
    rc = pf::interface_diagnostics_finish(ctx);
    if (rc) return rc;
    rc = pf::secondary_after_advect(ctx, esc, cfg->Vp, ctx->diag_last);
    if (rc) return rc;
  }
  rc = pool_sync(ctx);
  if (rc) return rc;
  if (stats) {
    stats->solve = sst;
    stats->clamp = cst;
    stats->active_tiles = ctx->nslots;
  }
  return PF_OK;
}

int pf_step(pf_ctx* ctx, const pf_step_cfg* cfg, pf_step_stats* stats) {
  if (!ctx || !cfg || check_solve_cfg(&cfg->solve)) return PF_ERR_INVALID;
  if (cfg->advect_order != 2 && cfg->advect_order != 3) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = step_impl(ctx, cfg, stats);
  // the deferred read-backs complete on every path
  const int r1 = pf::step_controls_finish(ctx, &ctx->controls_last);
  const int r2 = pf::interface_diagnostics_finish(ctx);
  const int r3 = pool_sync(ctx);
  if (!rc) rc = r1 ? r1 : r2 ? r2 : r3;
  return rc;
}

int pf_calibrate_rho_tilde0(pf_ctx* ctx, const pf_phase* phase, double Vp, double* out) {
  if (!ctx || !phase || !out) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::calibrate(ctx, phase, Vp, out);
}

// ---- particle adaptivity --------------------------------------------------

int pf_narrow_band_air(pf_ctx* ctx, int radius, pf_band_stats* stats) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const int rc = take_upload(ctx);
  if (rc) return rc;
  return pf::narrow_band_air(ctx, radius, stats);
}

int pf_coarsen_particles(pf_ctx* ctx, int type, int per_cell_target, unsigned seed, pf_coarsen_stats* stats) {
  if (!ctx || type < 0 || type > 255) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const int rc = take_upload(ctx);
  if (rc) return rc;
  return pf::coarsen_particles(ctx, type, per_cell_target, seed, stats);
}

int pf_refill_liquid(pf_ctx* ctx, int per_cell_target, unsigned seed, int interface_only, int interface_radius,
                     int max_added, pf_refill_stats* stats) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const int rc = take_upload(ctx);
  if (rc) return rc;
  return pf::refill_liquid(ctx, per_cell_target, seed, interface_only, interface_radius, max_added, stats);
}

int pf_interface_diagnostics(pf_ctx* ctx, const pf_phase* phase, pf_interface_stats* stats) {
  if (!ctx || !phase) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::interface_diagnostics(ctx, phase, stats);
}

int pf_get_interface_stats(const pf_ctx* ctx, pf_interface_stats* out) {
  if (!ctx || !out) return PF_ERR_INVALID;
  *out = ctx->diag_last;
  return PF_OK;
}

int pf_surface_tension(pf_ctx* ctx, const pf_phase* phase, double dt, double strength, double max_delta_speed,
                       int smoothing_radius, pf_surface_stats* stats) {
  if (!ctx || !phase) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::surface_tension(ctx, phase, dt, strength, max_delta_speed, smoothing_radius, stats);
}

int pf_set_surface_tension(pf_ctx* ctx, double strength, double max_delta_speed, int smoothing_radius) {
  if (!ctx) return PF_ERR_INVALID;
  ctx->st_strength = strength;
  ctx->st_max_dv = max_delta_speed;
  ctx->st_radius = smoothing_radius;
  return PF_OK;
}

int pf_get_surface_stats(const pf_ctx* ctx, pf_surface_stats* out) {
  if (!ctx || !out) return PF_ERR_INVALID;
  *out = ctx->surface_last;
  return PF_OK;
}

int pf_set_step_controls(pf_ctx* ctx, const pf_step_controls* controls) {
  if (!ctx) return PF_ERR_INVALID;
  ctx->controls = controls ? *controls : pf_step_controls{0, 0.5, 1e-5, 0, 1.0, 0.0};
  return PF_OK;
}

int pf_get_step_control_stats(const pf_ctx* ctx, pf_step_control_stats* out) {
  if (!ctx || !out) return PF_ERR_INVALID;
  *out = ctx->controls_last;
  return PF_OK;
}

int pf_set_adaptivity(pf_ctx* ctx, const pf_adapt_cfg* cfg) {
  if (!ctx) return PF_ERR_INVALID;
  ctx->adapt_on = cfg != nullptr;
  if (cfg) ctx->adapt_cfg = *cfg;
  ctx->adapt_last = pf_adapt_stats{};
  return PF_OK;
}

int pf_get_adaptivity_stats(const pf_ctx* ctx, pf_adapt_stats* out) {
  if (!ctx || !out) return PF_ERR_INVALID;
  *out = ctx->adapt_last;
  return PF_OK;
}

}  // extern "C"

namespace pf {
// the pending asynchronous upload, swapped in before another producer of the
// particle set (pf_seed_scene) overwrites it
int take_upload_for(pf_ctx* ctx) { return take_upload(ctx); }
}  // namespace pf
