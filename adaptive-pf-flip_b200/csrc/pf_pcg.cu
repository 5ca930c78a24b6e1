// pf_pcg.cu -- pressure solvers over the pool-layout 7-point system.
//
// PLAIN: FP64 Jacobi-PCG with the reference's recurrences and stopping rule
//   (src/driver/sparse_ops3d_tp.cpp:315-364); three kernels per iteration:
//   SpMV + p.Ap, x/r update + r.z + max|r|, direction update.
// MIXED: FP64 outer iterative refinement r = b - A x with the exact FP64
//   operator, inner Jacobi-PCG with FP32 vectors and FP32 (or BF16) scaled
//   face coefficients, FP64 inner products and norms.  The BF16 operator keeps
//   its diagonal equal to the sum of the rounded face weights, so it stays a
//   weighted graph Laplacian within a factor (1 +- 2^-8) of the exact one and
//   the refinement contracts by about that factor per sweep whatever the
//   conditioning.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "pf_ctx.h"
#include "pf_solver.cuh"

namespace pf {
namespace {

// ------------------------------ PLAIN -------------------------------------

__global__ void __launch_bounds__(PF_TV) k_spmv_plain(DevGrid G, int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                      PcgVec<double> v, double scale, double* partials) {
  if (ctl->done) return;
  __shared__ int nbs[6];
  double acc = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    __syncthreads();
    neighbor_slots(G, s, nbs);
    __syncthreads();
    const int l = threadIdx.x;
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kind[o];
    if (!kd) continue;
    const double p0 = v.p[o];
    double ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets(s, l, nbs, no);
      // +x -x +y -y +z -z, the reference's face order
      const double c[6] = {no[0] >= 0 ? v.cx[no[0]] : 0.0, v.cx[o], no[2] >= 0 ? v.cy[no[2]] : 0.0, v.cy[o],
                           no[4] >= 0 ? v.cz[no[4]] : 0.0, v.cz[o]};
      double off = 0.0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (c[d] != 0.0 && no[d] >= 0) off = __dadd_rn(off, __dmul_rn(c[d], v.p[no[d]]));
      }
      ap = __dmul_rn(scale, __dsub_rn(__dmul_rn(v.diag[o], p0), off));
    }
    v.Ap[o] = ap;
    acc = __dadd_rn(acc, __dmul_rn(p0, ap));
  }
  block_reduce_2(acc, 0.0, partials, ctl, kStagePAp);
}

// Every pooled tile's six neighbour slots, nbr[6 s + d] in neighbor_slots'
// order (+x -x +y -y +z -z; -1 outside the lattice or unpooled).
__global__ void k_plain_nbr(DevGrid G, int nslots, int* nbr) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 6 * nslots) return;
  const int s = q / 6, d = q - 6 * s;
  const int t = G.slot_tile[s];
  int tx = t % G.g.TX, r = t / G.g.TX, ty = r % G.g.TY, tz = r / G.g.TY;
  tx += d == 0 ? 1 : d == 1 ? -1 : 0;
  ty += d == 2 ? 1 : d == 3 ? -1 : 0;
  tz += d == 4 ? 1 : d == 5 ? -1 : 0;
  nbr[q] = (tx >= 0 && ty >= 0 && tz >= 0 && tx < G.g.TX && ty < G.g.TY && tz < G.g.TZ)
               ? G.tile_slot[tile_id(G.g, tx, ty, tz)]
               : -1;
}

// k_spmv_plain with the cross-tile neighbours read from the table: no shared
// memory or barriers per tile, so a CTA's loads of one tile do not wait on a
// neighbour-slot round trip.  Same arithmetic and order as k_spmv_plain.
__global__ void __launch_bounds__(PF_TV, 4) k_spmv_plain_tab(int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                          const int* __restrict__ nbr, PcgVec<double> v,
                                                          double scale, double* partials) {
  if (ctl->done) return;
  const int l = threadIdx.x;
  double acc = 0.0;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, l);
  int nb_next = nbr_lane(nbr, blockIdx.x, nslots);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kd_next;
    const int nb = nb_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, l);
    nb_next = nbr_lane(nbr, s + gridDim.x, nslots);
    const int3 nt = neighbor_lanes(nb, l);
    if (!kd) continue;
    const double p0 = v.p[o];
    double ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets_sel(nt, s, l, no);
      // +x -x +y -y +z -z, the reference's face order
      const double c[6] = {no[0] >= 0 ? v.cx[no[0]] : 0.0, v.cx[o], no[2] >= 0 ? v.cy[no[2]] : 0.0, v.cy[o],
                           no[4] >= 0 ? v.cz[no[4]] : 0.0, v.cz[o]};
      double off = 0.0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (c[d] != 0.0 && no[d] >= 0) off = __dadd_rn(off, __dmul_rn(c[d], v.p[no[d]]));
      }
      ap = __dmul_rn(scale, __dsub_rn(__dmul_rn(v.diag[o], p0), off));
    }
    v.Ap[o] = ap;
    acc = __dadd_rn(acc, __dmul_rn(p0, ap));
  }
  block_reduce_2(acc, 0.0, partials, ctl, kStagePAp);
}

__global__ void __launch_bounds__(PF_TV, 4) k_update_plain(int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                        PcgVec<double> v, double scale, double* partials) {
  if (ctl->done) return;
  const double alpha = ctl->alpha;
  double rz = 0.0, rmax = 0.0;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, threadIdx.x);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, threadIdx.x);
    if (!kd) continue;
    const double pp = v.p[o], x = v.x[o], r_old = v.r[o], ap = v.Ap[o], dg = v.diag[o];
    v.x[o] = __dadd_rn(x, __dmul_rn(alpha, pp));
    const double r = __dsub_rn(r_old, __dmul_rn(alpha, ap));
    v.r[o] = r;
    const double d = kd == 2 ? 1.0 : __dmul_rn(scale, dg);
    const double z = d > 0.0 ? __ddiv_rn(r, d) : 0.0;
    if (v.z) v.z[o] = z;
    rz = __dadd_rn(rz, __dmul_rn(r, z));
    rmax = fmax(rmax, fabs(r));
  }
  block_reduce_2(rz, rmax, partials, ctl, kStageUpdate);
}

__global__ void __launch_bounds__(PF_TV) k_direction_plain(int nslots, const SolveCtl* ctl, const uint8_t* kind,
                                                           PcgVec<double> v, double scale) {
  if (ctl->done) return;
  const double beta = ctl->beta;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, threadIdx.x);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, threadIdx.x);
    if (!kd) continue;
    double z;
    if (v.z) {
      z = v.z[o];  // the update's r / diag
    } else {
      const double d = kd == 2 ? 1.0 : __dmul_rn(scale, v.diag[o]);
      z = d > 0.0 ? __ddiv_rn(v.r[o], d) : 0.0;
    }
    v.p[o] = __dadd_rn(z, __dmul_rn(beta, v.p[o]));
  }
}

// ------------------------------ MIXED -------------------------------------

__device__ __forceinline__ float ldc(const float* a, long long i) { return a[i]; }
__device__ __forceinline__ float ldc(const __nv_bfloat16* a, long long i) { return __bfloat162float(a[i]); }
__device__ __forceinline__ void stc(float* a, long long i, float v) { a[i] = v; }
__device__ __forceinline__ void stc(__nv_bfloat16* a, long long i, float v) { a[i] = __float2bfloat16_rn(v); }
__device__ __forceinline__ float rnd(float v, const float*) { return v; }
__device__ __forceinline__ float rnd(float v, const __nv_bfloat16*) { return __bfloat162float(__float2bfloat16_rn(v)); }

template <typename CC, typename CP>
struct MixVec {
  float *e, *r, *Ap, *d;  // correction, inner residual, A'p, diagonal of A'
  CP* p;                  // search direction (FP32 or BF16)
  CC *cx, *cy, *cz;       // scaled low-face couplings (FP32 or BF16)
};

// Inner operator A': couplings w = round(scale*beta), diagonal = sum of the
// rounded weights of all non-solid faces (air faces keep their exact-scaled
// weight rounded the same way).
template <typename CC, typename CP>
__global__ void __launch_bounds__(PF_TV) k_mixed_setup(DevGrid G, int nslots, const uint8_t* kind, PcgVec<double> v,
                                                       MixVec<CC, CP> m, double scale) {
  __shared__ int nbs[6];
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    __syncthreads();
    neighbor_slots(G, s, nbs);
    __syncthreads();
    const int l = threadIdx.x;
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kind[o];
    const float wx = (float)(scale * v.cx[o]), wy = (float)(scale * v.cy[o]), wz = (float)(scale * v.cz[o]);
    stc(m.cx, o, wx);
    stc(m.cy, o, wy);
    stc(m.cz, o, wz);
    float dgf = 0.0f;
    if (kd == 2) {
      dgf = 1.0f;
    } else if (kd == 1) {
      long long no[6];
      neighbor_offsets(s, l, nbs, no);
      const double cexact[6] = {no[0] >= 0 ? v.cx[no[0]] : 0.0, v.cx[o], no[2] >= 0 ? v.cy[no[2]] : 0.0, v.cy[o],
                                no[4] >= 0 ? v.cz[no[4]] : 0.0, v.cz[o]};
      // exact scaled diagonal minus exact couplings = exact air-face weight sum
      double dd = scale * v.diag[o];
      double corr = 0.0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const double w = scale * cexact[d];
        corr += (double)rnd((float)w, m.cx) - w;
      }
      dgf = (float)(dd + corr);
    }
    m.d[o] = dgf;
  }
}

// start an inner solve: r' = r64 (FP32), e = 0, p = z = r'/d'; r.z, max|r'|
template <typename CC, typename CP>
__global__ void __launch_bounds__(PF_TV) k_mixed_start(int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                       const double* r64, MixVec<CC, CP> m, double* partials) {
  double rz = 0.0, rmax = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kind[o];
    float r = 0.0f, z = 0.0f;
    if (kd) {
      r = (float)r64[o];
      const float d = m.d[o];
      z = d > 0.0f ? r / d : 0.0f;
      rz += (double)r * (double)z;
      rmax = fmax(rmax, (double)fabsf(r));
    }
    m.r[o] = r;
    m.e[o] = 0.0f;
    stc(m.p, o, z);
  }
  block_reduce_2(rz, rmax, partials, ctl, kStageInit);
}

template <typename CC, typename CP>
__global__ void __launch_bounds__(PF_TV) k_mixed_spmv(DevGrid G, int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                      MixVec<CC, CP> m, double* partials) {
  if (ctl->done) return;
  __shared__ int nbs[6];
  const int l = threadIdx.x;
  double acc = 0.0;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, l);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    __syncthreads();
    neighbor_slots(G, s, nbs);
    __syncthreads();
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, l);
    if (!kd) continue;
    const float p0 = ldc(m.p, o);
    float ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets(s, l, nbs, no);
      float off = 0.0f;
      if (no[0] >= 0) off += ldc(m.cx, no[0]) * ldc(m.p, no[0]);
      if (no[1] >= 0) off += ldc(m.cx, o) * ldc(m.p, no[1]);
      if (no[2] >= 0) off += ldc(m.cy, no[2]) * ldc(m.p, no[2]);
      if (no[3] >= 0) off += ldc(m.cy, o) * ldc(m.p, no[3]);
      if (no[4] >= 0) off += ldc(m.cz, no[4]) * ldc(m.p, no[4]);
      if (no[5] >= 0) off += ldc(m.cz, o) * ldc(m.p, no[5]);
      ap = m.d[o] * p0 - off;
    }
    m.Ap[o] = ap;
    acc += (double)p0 * (double)ap;
  }
  block_reduce_2(acc, 0.0, partials, ctl, kStagePAp);
}

template <typename CC, typename CP>
__global__ void __launch_bounds__(PF_TV) k_mixed_update(int nslots, SolveCtl* ctl, const uint8_t* kind, MixVec<CC, CP> m,
                                                        double* partials) {
  if (ctl->done) return;
  const float alpha = (float)ctl->alpha;
  double rz = 0.0, rmax = 0.0;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, threadIdx.x);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, threadIdx.x);
    if (!kd) continue;
    m.e[o] += alpha * ldc(m.p, o);
    const float r = m.r[o] - alpha * m.Ap[o];
    m.r[o] = r;
    const float d = m.d[o];
    const float z = d > 0.0f ? r / d : 0.0f;
    rz += (double)r * (double)z;
    rmax = fmax(rmax, (double)fabsf(r));
  }
  block_reduce_2(rz, rmax, partials, ctl, kStageUpdate);
}

template <typename CC, typename CP>
__global__ void __launch_bounds__(PF_TV) k_mixed_direction(int nslots, const SolveCtl* ctl, const uint8_t* kind,
                                                           MixVec<CC, CP> m) {
  if (ctl->done) return;
  const float beta = (float)ctl->beta;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, threadIdx.x);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, threadIdx.x);
    if (!kd) continue;
    const float d = m.d[o];
    const float z = d > 0.0f ? m.r[o] / d : 0.0f;
    stc(m.p, o, z + beta * ldc(m.p, o));
  }
}

__global__ void k_set_inner(SolveCtl* ctl, double tol_abs, double tol_rel, int max_iter) {
  ctl->tol_abs = tol_abs;
  ctl->tol_rel = tol_rel;
  ctl->max_iter = max_iter;
  ctl->done = 0;
  ctl->it = 0;
  ctl->counter = 0;
}

}  // namespace

// Poll the control block; returns done code and fills it/res.
static int poll(pf_ctx* ctx, SolveCtl* out) {
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *ctx->h_ctl;
  return PF_OK;
}

int pcg_plain(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, PcgVec<double> vec, double scale,
              const pf_solve_cfg* cfg, SolveResult* res) {
  StageScope stage(ctx, PF_STAGE_PCG);
  DevGrid G = dev_grid(ctx);
  SolveCtl c{};
  int rc = poll(ctx, &c);
  if (rc) return rc;
  res->res0 = c.res0;
  res->tol = c.tol;
  int launched = 0;
  int batch = cfg->check_every > 0 ? cfg->check_every : 4;
  // the update hands z to the direction pass: one division per cell and
  // iteration instead of two, the same bytes (z is read where r and diag
  // were), the same values
  vec.z = ctx->z_plain;
  if (nslots > 0)
    (++ctx->launches), k_plain_nbr<<<nblocks((size_t)6 * nslots, 256), 256, 0, ctx->stream>>>(G, nslots, ctx->nbr_plain);
  while (!c.done && launched < cfg->max_iter) {
    const int nb = std::min(batch, cfg->max_iter - launched);
    for (int q = 0; q < nb; ++q) {
      (++ctx->launches), k_spmv_plain_tab<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, ctx->nbr_plain, vec,
                                                                          scale, ctx->partials);
      (++ctx->launches), k_update_plain<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, vec, scale, ctx->partials);
      (++ctx->launches), k_direction_plain<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, vec, scale);
    }
    PF_CUDA_TRY(cudaGetLastError());
    launched += nb;
    rc = poll(ctx, &c);
    if (rc) return rc;
    if (cfg->check_every <= 0) batch = std::min(batch * 2, 64);
  }
  res->iterations = c.it;
  res->res_final = c.it > 0 ? c.res : c.res0;
  res->converged = c.done == 1 ? 1 : 0;
  res->breakdown = c.done == 2 ? 1 : 0;
  res->nonfinite = c.done == 4 ? 1 : 0;
  return PF_OK;
}

int ensure_solver_buffers(pf_ctx* ctx, int mode) {
  if (mode == PF_SOLVER_PLAIN || ctx->rf) return PF_OK;
  const size_t n = ctx->cells_cap;
  PF_CUDA_TRY(cudaMalloc(&ctx->xf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->rf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->pf32, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->Apf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->diagf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->cxf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->cyf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->czf, n * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&ctx->pbf, n * sizeof(uint16_t)));
  PF_CUDA_TRY(cudaMalloc(&ctx->cbf, 3 * n * sizeof(uint16_t)));
  PF_CUDA_TRY(cudaMalloc(&ctx->b64, n * sizeof(double)));
  return PF_OK;
}

template <typename CC, typename CP>
static int mixed_inner(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, MixVec<CC, CP> m, double tol_abs,
                       double tol_rel, int max_iter, int check_every, int* iters, SolveCtl* out) {
  DevGrid G = dev_grid(ctx);
  (++ctx->launches), k_set_inner<<<1, 1, 0, ctx->stream>>>(ctx->ctl, tol_abs, tol_rel, max_iter);
  (++ctx->launches), k_mixed_start<CC, CP><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, ctx->r, m, ctx->partials);
  PF_CUDA_TRY(cudaGetLastError());
  SolveCtl c{};
  int rc = poll(ctx, &c);
  if (rc) return rc;
  int launched = 0;
  int batch = check_every > 0 ? check_every : 4;
  while (!c.done && launched < max_iter) {
    const int nb = std::min(batch, max_iter - launched);
    for (int q = 0; q < nb; ++q) {
      (++ctx->launches), k_mixed_spmv<CC, CP><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, ctx->ctl, kind, m, ctx->partials);
      (++ctx->launches), k_mixed_update<CC, CP><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, m, ctx->partials);
      (++ctx->launches), k_mixed_direction<CC, CP><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, m);
    }
    PF_CUDA_TRY(cudaGetLastError());
    launched += nb;
    rc = poll(ctx, &c);
    if (rc) return rc;
    if (check_every <= 0) batch = std::min(batch * 2, 64);
  }
  *iters += c.it;
  *out = c;
  return PF_OK;
}

// The inner solver of MIXED: Jacobi-PCG on A' with FP32 vectors (and FP32 or
// BF16 couplings and direction), FP64 inner products, from e = 0.
template <typename CC, typename CP>
struct MixedInner final : InnerSolver {
  int nslots = 0, nred = 0, check_every = 0;
  const uint8_t* kind = nullptr;
  MixVec<CC, CP> m{};
  int solve(pf_ctx* ctx, double eta, int max_iter, bool, const float** z, int* iters) override {
    SolveCtl ic{};
    // one poll in the middle of the budget, one at its end
    const int poll_at = check_every > 0 ? check_every : std::max(1, max_iter / 2);
    int before = 0;
    const int rc = mixed_inner<CC, CP>(ctx, nslots, nred, kind, m, 0.0, eta, max_iter, poll_at, &before, &ic);
    if (rc) return rc;
    *iters = ic.it;
    *z = m.e;
    return ic.done == 4 ? set_error(ctx, PF_ERR_NONFINITE, "non-finite value in the inner solve") : PF_OK;
  }
};

// MIXED: FP64 flexible CG on the exact operator (pf_outer.cu), preconditioned
// by the inner Jacobi-PCG on A' in reduced precision.
template <typename CC, typename CP>
static int solve_mixed_t(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale,
                         const pf_solve_cfg* cfg, MixVec<CC, CP> m, SolveResult* res) {
  DevGrid G = dev_grid(ctx);
  PcgVec<double> v{ctx->x, ctx->r, ctx->p, ctx->Ap, ctx->diag, ctx->cx, ctx->cy, ctx->cz};
  (++ctx->launches), k_mixed_setup<CC, CP><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, kind, v, m, scale);
  if (nslots > 0)
    (++ctx->launches), k_plain_nbr<<<nblocks((size_t)6 * nslots, 256), 256, 0, ctx->stream>>>(G, nslots, ctx->nbr_plain);
  PF_CUDA_TRY(cudaGetLastError());
  MixedInner<CC, CP> inner;
  inner.nslots = nslots;
  inner.nred = nred;
  inner.kind = kind;
  inner.m = m;
  inner.check_every = cfg->check_every;
  const double eta = cfg->inner_rel_tol > 0.0 ? cfg->inner_rel_tol : 1e-3;
  const int inner_max = cfg->inner_max_iter > 0 ? cfg->inner_max_iter : 200;
  return solve_inner_outer(ctx, nslots, nred, kind, ctx->nbr_plain, scale, cfg, inner, eta, inner_max, res);
}

int solve_mixed(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale, const pf_solve_cfg* cfg,
                const void* /*phase_consts*/, SolveResult* res) {
  StageScope stage(ctx, PF_STAGE_PCG);
  int rc = ensure_solver_buffers(ctx, cfg->mode);
  if (rc) return rc;
  // FP64 assembly first: exact operator, rhs, tolerance (shared with PLAIN)
  typedef __nv_bfloat16 bf16;
  bf16* cb = (bf16*)ctx->cbf;
  if (cfg->bf16_storage >= 2) {  // BF16 couplings and search direction
    MixVec<bf16, bf16> m{ctx->xf, ctx->rf, ctx->Apf, ctx->diagf, (bf16*)ctx->pbf, cb, cb + ctx->cells_cap,
                         cb + 2 * ctx->cells_cap};
    return solve_mixed_t(ctx, nslots, nred, kind, scale, cfg, m, res);
  }
  if (cfg->bf16_storage == 1) {  // BF16 couplings, FP32 search direction
    MixVec<bf16, float> m{ctx->xf, ctx->rf, ctx->Apf, ctx->diagf, ctx->pf32, cb, cb + ctx->cells_cap,
                          cb + 2 * ctx->cells_cap};
    return solve_mixed_t(ctx, nslots, nred, kind, scale, cfg, m, res);
  }
  MixVec<float, float> m{ctx->xf, ctx->rf, ctx->Apf, ctx->diagf, ctx->pf32, ctx->cxf, ctx->cyf, ctx->czf};
  return solve_mixed_t(ctx, nslots, nred, kind, scale, cfg, m, res);
}

}  // namespace pf

namespace pf {

// One PLAIN Jacobi-PCG iteration (the three kernels pcg_plain launches), for
// the allocation-free projection (pf_noalloc.cu).
void launch_pcg_plain_iteration(const DevGrid& G, int nslots, int nred, SolveCtl* ctl, const uint8_t* kind,
                                PcgVec<double> v, double scale, double* partials, cudaStream_t s) {
  k_spmv_plain<<<nred, PF_TV, 0, s>>>(G, nslots, ctl, kind, v, scale, partials);
  k_update_plain<<<nred, PF_TV, 0, s>>>(nslots, ctl, kind, v, scale, partials);
  k_direction_plain<<<nred, PF_TV, 0, s>>>(nslots, ctl, kind, v, scale);
}

}  // namespace pf
