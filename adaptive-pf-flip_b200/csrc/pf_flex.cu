// pf_flex.cu -- LEARNED mode: flexible PCG with the two-level preconditioner
//   M^-1 r = D^-1 r + P c(P^T r)
// where c is the learned coarse solve (or, for ablation and for training
// targets, the exact Galerkin coarse solve; or nothing, plain Jacobi).
//
// Polak-Ribiere beta r.(z - z_prev)/rz as the reference's flexible option
// (src/pressure/multires_pressure3d.cpp:1425-1434).  Each iteration forms
// both candidates z_j = D^-1 r and z_c = z_j + P c; z_c is accepted only when
// r.z_c >= r.z_j (1 + min_gain) (the rz-gain guard of
// src/pressure/multires_pressure3d.cpp:1322-1334), and after kDisableAfter
// consecutive rejections the solve continues with Jacobi alone (the
// auto-disable of :1172).  Whatever the coarse term does, convergence is
// judged on the residual of the exact FP64 operator: directly in the FP64
// variant, through FP64 iterative refinement in the FP32 variant.
#include <algorithm>
#include <cmath>

#include "pf_coarse.cuh"
#include "pf_solver.cuh"

namespace pf {
namespace {

constexpr int kDisableAfter = 8;

template <typename V>
struct FlexVec {
  V *e, *r, *Ap, *z, *p;  // solution (correction), residual, A p, stored M^-1 r, direction
  V *d, *cx, *cy, *cz;    // operator: diagonal and low-face couplings, times scale
  const uint8_t* cls;     // coarse class of each unknown (255: none)
  V scale;
};

__global__ void k_fx_set(SolveCtl* ctl, double tol_abs, double tol_rel, int max_iter, double offered, int reset) {
  ctl->tol_abs = tol_abs;
  ctl->tol_rel = tol_rel;
  ctl->max_iter = max_iter;
  ctl->done = 0;
  ctl->it = 0;
  ctl->counter = 0;
  ctl->aux[2] = offered;
  if (reset) {
    ctl->aux[1] = 0.0;
    ctl->aux[3] = 0.0;
    ctl->accepted = 0;
    ctl->rejected = 0;
  }
}

// FP32 copy of the operator times scale, and the FP64 right-hand side kept
__global__ void __launch_bounds__(PF_TV) k_fx_setup32(int nslots, const uint8_t* kind, const double* diag,
                                                      const double* cx, const double* cy, const double* cz,
                                                      const double* r, double scale, float* df, float* cxf,
                                                      float* cyf, float* czf, double* b) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const bool fl = kind[o] == 1;
    df[o] = fl ? (float)(scale * diag[o]) : (kind[o] == 2 ? 1.0f : 0.0f);
    cxf[o] = (float)(scale * cx[o]);
    cyf[o] = (float)(scale * cy[o]);
    czf[o] = (float)(scale * cz[o]);
    b[o] = r[o];
  }
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_start(int nslots, SolveCtl* ctl, const uint8_t* kind, const double* r64,
                                                    FlexVec<V> m, double* partials) {
  double rmax = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const V r = kind[o] ? (V)r64[o] : (V)0;
    m.r[o] = r;
    m.e[o] = (V)0;
    m.z[o] = (V)0;
    m.p[o] = (V)0;
    rmax = fmax(rmax, fabs((double)r));
  }
  block_reduce_2(0.0, rmax, partials, ctl, kStageInit);  // sets res0, tol, done
}

template <typename V>
__device__ __forceinline__ V jacobi(const FlexVec<V>& m, uint8_t kd, size_t o) {
  const V d = kd == 1 ? m.scale * m.d[o] : (V)0;
  return d > (V)0 ? m.r[o] / d : (V)0;
}

template <typename V>
__device__ __forceinline__ V coarse_term(const FlexVec<V>& m, const int* slot_tile, int s, size_t o,
                                         const float* ec) {
  const uint8_t c = m.cls[o];
  return c != 255 ? (V)ec[coarse_index(slot_tile[s], c)] : (V)0;
}

// Dots of both candidates: r.zc, r.zj, r.(zc - z_prev), r.(zj - z_prev); the
// last CTA applies the guard, picks the preconditioner and the flexible beta.
template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_precond(const int* slot_tile, int nslots, SolveCtl* ctl,
                                                      const uint8_t* kind, FlexVec<V> m, const float* ec, int first,
                                                      double min_gain, double* partials) {
  if (ctl->done) return;
  const bool offered = ctl->aux[2] != 0.0 && ctl->aux[1] == 0.0;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kind[o];
    if (!kd) continue;
    const double r = (double)m.r[o];
    const double zj = (double)jacobi(m, kd, o);
    const double zc = offered ? zj + (double)coarse_term(m, slot_tile, s, o, ec) : zj;
    const double zp = (double)m.z[o];
    a[0] += r * zc;
    a[1] += r * zj;
    a[2] += r * (zc - zp);
    a[3] += r * (zj - zp);
  }
  __shared__ double sh[4][32];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double v = warp_sum(a[q]);
    if (lane == 0) sh[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < 4; ++q) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += sh[q][w];
      partials[kRedSlots * blockIdx.x + q] = v;
    }
    __threadfence();
    am_last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // the last CTA sums the partials with all its threads, in a fixed order
  double S[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 4; ++q) S[q] += __ldcg(&partials[kRedSlots * b + q]);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double v = warp_sum(S[q]);
    __syncthreads();
    if (lane == 0) sh[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += sh[q][w];
    S[q] = v;
  }
  ctl->counter = 0;
  bool use_c = false;
  if (offered) {
    use_c = isfinite(S[0]) && S[0] > 0.0 && S[0] >= S[1] * (1.0 + min_gain);
    if (use_c) {
      ctl->accepted += 1;
      ctl->aux[3] = 0.0;
    } else {
      ctl->rejected += 1;
      ctl->aux[3] += 1.0;  // rejection streak
      if (ctl->aux[3] >= kDisableAfter) ctl->aux[1] = 1.0;
    }
  }
  ctl->aux[0] = use_c ? 1.0 : 0.0;
  const double rzn = use_c ? S[0] : S[1];
  if (!isfinite(rzn)) {
    ctl->done = 4;
    return;
  }
  double b = 0.0;
  if (!first && ctl->rz != 0.0) {
    b = (use_c ? S[2] : S[3]) / ctl->rz;
    if (!isfinite(b) || b < 0.0) b = 0.0;
  }
  ctl->beta = b;
  ctl->rz = rzn;
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_dir(const int* slot_tile, int nslots, const SolveCtl* ctl,
                                                  const uint8_t* kind, FlexVec<V> m, const float* ec) {
  if (ctl->done) return;
  const V beta = (V)ctl->beta;
  const bool use_c = ctl->aux[0] != 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kind[o];
    if (!kd) continue;
    V z = jacobi(m, kd, o);
    if (use_c) z += coarse_term(m, slot_tile, s, o, ec);
    m.z[o] = z;
    m.p[o] = z + beta * m.p[o];
  }
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_spmv(DevGrid G, int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                   FlexVec<V> m, double* partials) {
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
    const V p0 = m.p[o];
    V ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets(s, l, nbs, no);
      V off = (V)0;
      if (no[0] >= 0) off += m.cx[no[0]] * m.p[no[0]];
      if (no[1] >= 0) off += m.cx[o] * m.p[no[1]];
      if (no[2] >= 0) off += m.cy[no[2]] * m.p[no[2]];
      if (no[3] >= 0) off += m.cy[o] * m.p[no[3]];
      if (no[4] >= 0) off += m.cz[no[4]] * m.p[no[4]];
      if (no[5] >= 0) off += m.cz[o] * m.p[no[5]];
      ap = m.scale * (m.d[o] * p0 - off);
    }
    m.Ap[o] = ap;
    acc += (double)p0 * (double)ap;
  }
  block_reduce_2(acc, 0.0, partials, ctl, kStagePAp);
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_update(int nslots, SolveCtl* ctl, const uint8_t* kind, FlexVec<V> m,
                                                     double* partials) {
  if (ctl->done) return;
  const V alpha = (V)ctl->alpha;
  double rmax = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (!kind[o]) continue;
    m.e[o] += alpha * m.p[o];
    const V r = m.r[o] - alpha * m.Ap[o];
    m.r[o] = r;
    rmax = fmax(rmax, fabs((double)r));
  }
  block_reduce_2(0.0, rmax, partials, ctl, kStageFlex);
}

__global__ void k_fx_add(int nslots, const uint8_t* kind, double* x, const float* e) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (kind[o]) x[o] += (double)e[o];
  }
}

// r = b - A x with the exact FP64 operator; max|r| -> ctl->res
__global__ void __launch_bounds__(PF_TV) k_fx_residual(DevGrid G, int nslots, SolveCtl* ctl, const uint8_t* kind,
                                                       const double* x, const double* diag, const double* cx,
                                                       const double* cy, const double* cz, const double* b,
                                                       double scale, double* r, double* partials) {
  __shared__ int nbs[6];
  double rmax = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    __syncthreads();
    neighbor_slots(G, s, nbs);
    __syncthreads();
    const int l = threadIdx.x;
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kind[o];
    if (!kd) continue;
    double ax;
    if (kd == 2) {
      ax = x[o];
    } else {
      long long no[6];
      neighbor_offsets(s, l, nbs, no);
      double off = 0.0;
      if (no[0] >= 0) off += cx[no[0]] * x[no[0]];
      if (no[1] >= 0) off += cx[o] * x[no[1]];
      if (no[2] >= 0) off += cy[no[2]] * x[no[2]];
      if (no[3] >= 0) off += cy[o] * x[no[3]];
      if (no[4] >= 0) off += cz[no[4]] * x[no[4]];
      if (no[5] >= 0) off += cz[o] * x[no[5]];
      ax = scale * (diag[o] * x[o] - off);
    }
    const double rr = b[o] - ax;
    r[o] = rr;
    rmax = fmax(rmax, fabs(rr));
  }
  block_reduce_2(0.0, rmax, partials, ctl, kStageResid);
}

int poll_ctl(pf_ctx* ctx, SolveCtl* out) {
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *ctx->h_ctl;
  return PF_OK;
}

template <typename V>
int apply_coarse(pf_ctx* ctx, int nslots, const uint8_t* kind, const V* r, int precond) {
  int rc = coarse_restrict(ctx, nslots, kind, r, ctx->ctl);
  if (rc) return rc;
  if (precond == PF_PRECOND_EXACT_COARSE) return coarse_solve_exact(ctx, 400, 1e-6, ctx->ctl);
  return coarse_solve_net(ctx, ctx->ctl);
}

// Flexible PCG from x = 0 on r_init until max|r| < max(tol_abs, tol_rel max|r0|).
template <typename V>
int flex_solve(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, FlexVec<V> m, const double* r_init,
               double tol_abs, double tol_rel, int max_iter, int check_every, int precond, double min_gain,
               int reset_guard, SolveCtl* out) {
  DevGrid G = dev_grid(ctx);
  const float* ec = ((CoarseCtx*)ctx->learned)->op.ec;
  const bool coarse = precond != PF_PRECOND_JACOBI;
  (++ctx->launches), k_fx_set<<<1, 1, 0, ctx->stream>>>(ctx->ctl, tol_abs, tol_rel, max_iter, coarse ? 1.0 : 0.0,
                                                        reset_guard);
  (++ctx->launches), k_fx_start<V><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, r_init, m, ctx->partials);
  int rc = PF_OK;
  if (coarse) rc = apply_coarse<V>(ctx, nslots, kind, m.r, precond);
  if (rc) return rc;
  (++ctx->launches), k_fx_precond<V><<<nred, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, ctx->ctl, kind, m, ec, 1,
                                                                      min_gain, ctx->partials);
  (++ctx->launches), k_fx_dir<V><<<nred, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, ctx->ctl, kind, m, ec);
  PF_CUDA_TRY(cudaGetLastError());
  SolveCtl c{};
  rc = poll_ctl(ctx, &c);
  if (rc) return rc;
  int launched = 0;
  int batch = check_every > 0 ? check_every : 4;
  while (!c.done && launched < max_iter) {
    const int nb = std::min(batch, max_iter - launched);
    for (int q = 0; q < nb; ++q) {
      (++ctx->launches), k_fx_spmv<V><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, ctx->ctl, kind, m, ctx->partials);
      (++ctx->launches), k_fx_update<V><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, m, ctx->partials);
      if (coarse) {
        rc = apply_coarse<V>(ctx, nslots, kind, m.r, precond);
        if (rc) return rc;
      }
      (++ctx->launches), k_fx_precond<V><<<nred, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, ctx->ctl, kind, m,
                                                                          ec, 0, min_gain, ctx->partials);
      (++ctx->launches), k_fx_dir<V><<<nred, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, ctx->ctl, kind, m, ec);
    }
    PF_CUDA_TRY(cudaGetLastError());
    launched += nb;
    rc = poll_ctl(ctx, &c);
    if (rc) return rc;
    if (check_every <= 0) batch = std::min(batch * 2, 64);
  }
  *out = c;
  return PF_OK;
}

int ensure_z64(pf_ctx* ctx, double** z) {
  CoarseCtx* cc = (CoarseCtx*)ctx->learned;
  if (cc->z64_cap < ctx->cells_cap) {
    if (cc->z64) cudaFree(cc->z64);
    cc->z64 = nullptr;
    PF_CUDA_TRY(cudaMalloc(&cc->z64, ctx->cells_cap * sizeof(double)));
    cc->z64_cap = ctx->cells_cap;
  }
  *z = cc->z64;
  return PF_OK;
}

}  // namespace

int solve_learned(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale, const pf_solve_cfg* cfg,
                  SolveResult* res) {
  StageScope stage(ctx, PF_STAGE_PCG);
  int rc = coarse_ensure(ctx);
  if (rc) return rc;
  const int precond = cfg->precond;
  if (precond != PF_PRECOND_NETWORK && precond != PF_PRECOND_EXACT_COARSE && precond != PF_PRECOND_JACOBI)
    return set_error(ctx, PF_ERR_INVALID, "unknown preconditioner");
  if (precond == PF_PRECOND_NETWORK && !coarse_net_ready(ctx))
    return set_error(ctx, PF_ERR_INVALID, "learned preconditioner: no network loaded (pf_learned_load/train)");
  if (precond != PF_PRECOND_JACOBI) {
    rc = coarse_assemble(ctx, nslots, kind, ctx->diag, ctx->cx, ctx->cy, ctx->cz, scale);
    if (rc) return rc;
  }
  if (precond == PF_PRECOND_NETWORK) {
    rc = coarse_prepare_net(ctx);
    if (rc) return rc;
  }
  const uint8_t* cls = ((CoarseCtx*)ctx->learned)->op.cls;
  SolveCtl c{};
  rc = poll_ctl(ctx, &c);  // the assembly's initial residual and tolerance
  if (rc) return rc;
  res->res0 = c.res0;
  res->tol = c.tol;
  if (!(c.res0 >= c.tol)) {
    res->converged = 1;
    res->res_final = c.res0;
    return PF_OK;
  }
  DevGrid G = dev_grid(ctx);

  if (!cfg->inner_fp32) {
    // FP64 flexible PCG on the exact operator
    double* z64 = nullptr;
    rc = ensure_z64(ctx, &z64);
    if (rc) return rc;
    FlexVec<double> m{ctx->x, ctx->r, ctx->Ap, z64, ctx->p, ctx->diag, ctx->cx, ctx->cy, ctx->cz, cls, scale};
    SolveCtl o{};
    rc = flex_solve<double>(ctx, nslots, nred, kind, m, ctx->r, cfg->abs_tol, cfg->rel_tol, cfg->max_iter,
                            cfg->check_every, precond, cfg->accept_min_gain, 1, &o);
    if (rc) return rc;
    res->iterations = o.it;
    res->refinements = 0;
    res->res_final = o.res;
    res->converged = o.done == 1 ? 1 : 0;
    res->breakdown = o.done == 2 ? 1 : 0;
    res->nonfinite = o.done == 4 ? 1 : 0;
    res->precond_applied = o.accepted;
    res->precond_rejected = o.rejected;
    return PF_OK;
  }

  // FP32 flexible PCG inside FP64 iterative refinement
  rc = ensure_solver_buffers(ctx, PF_SOLVER_MIXED);
  if (rc) return rc;
  (++ctx->launches), k_fx_setup32<<<nred, PF_TV, 0, ctx->stream>>>(nslots, kind, ctx->diag, ctx->cx, ctx->cy, ctx->cz,
                                                                    ctx->r, scale, ctx->diagf, ctx->cxf, ctx->cyf,
                                                                    ctx->czf, ctx->b64);
  PF_CUDA_TRY(cudaGetLastError());
  // z needs its own FP32 array: the BF16 coupling buffer (6 bytes per cell) is unused here
  FlexVec<float> m{ctx->xf, ctx->rf, ctx->Apf, (float*)ctx->cbf, ctx->pf32, ctx->diagf,
                   ctx->cxf, ctx->cyf, ctx->czf, cls, 1.0f};
  const double tol = c.tol;
  double resid = c.res0;
  int iters = 0, sweeps = 0;
  const int max_sweeps = cfg->max_refine > 0 ? cfg->max_refine : 8;
  const double inner_rel = cfg->inner_rel_tol > 0.0 ? cfg->inner_rel_tol : 1e-5;
  bool converged = false, nonfinite = false;
  while (!converged && sweeps < max_sweeps && iters < cfg->max_iter) {
    SolveCtl ic{};
    rc = flex_solve<float>(ctx, nslots, nred, kind, m, ctx->r, 0.0, inner_rel, cfg->max_iter - iters,
                           cfg->check_every, precond, cfg->accept_min_gain, sweeps == 0, &ic);
    if (rc) return rc;
    ++sweeps;
    iters += ic.it;
    res->precond_applied = ic.accepted;
    res->precond_rejected = ic.rejected;
    (++ctx->launches), k_fx_add<<<nred, PF_TV, 0, ctx->stream>>>(nslots, kind, ctx->x, m.e);
    (++ctx->launches), k_fx_residual<<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, ctx->ctl, kind, ctx->x, ctx->diag,
                                                                      ctx->cx, ctx->cy, ctx->cz, ctx->b64, scale,
                                                                      ctx->r, ctx->partials);
    PF_CUDA_TRY(cudaGetLastError());
    rc = poll_ctl(ctx, &c);
    if (rc) return rc;
    resid = c.res;
    if (!std::isfinite(resid) || ic.done == 4) {
      nonfinite = true;
      break;
    }
    converged = resid < tol;
    if (ic.it == 0) break;
  }
  res->iterations = iters;
  res->refinements = sweeps;
  res->res_final = resid;
  res->converged = converged ? 1 : 0;
  res->nonfinite = nonfinite ? 1 : 0;
  return PF_OK;
}

}  // namespace pf
