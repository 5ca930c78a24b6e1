// pf_outer.cu -- reduced-precision pressure solves that still reach the FP64
// tolerance: an FP64 flexible conjugate gradient on the exact operator whose
// preconditioner is a truncated inner solve run in FP32 (or with BF16
// storage).
//
// At a density ratio of 1000:1 on a 256^3 grid the Jacobi-preconditioned
// operator has kappa * eps_FP32 of order one: FP32 recurrences cannot resolve
// a 1e-6 residual, and restarting them from an FP64 residual (iterative
// refinement) stalls.  Here the FP32 solve is only a preconditioner: each
// outer iteration hands the FP64 residual to the inner solver, which reduces
// it by a factor eta (or stops after a fixed number of iterations) from a zero
// start and returns z.  Because that z depends nonlinearly on r, the outer
// iteration is flexible CG with one stored direction (FCG(1), Notay, SIAM J.
// Sci. Comput. 22 (2000); the inner-outer analysis of Golub & Ye, SIAM J. Sci.
// Comput. 21 (1999)):
//   p_k = z_k - beta p_{k-1},  beta = z_k . q_{k-1} / p_{k-1} . q_{k-1}
//   q_k = A p_k,  alpha = r_k . p_k / p_k . q_k
//   x += alpha p_k,  r -= alpha q_k
// All outer vectors, the operator and the inner products are FP64, so the
// outer Krylov space keeps converging to the FP64 residual even when an inner
// solve only cuts its residual by 10-100x.  Convergence is judged on max|r|
// with the same rule as PLAIN (src/pressure/multires_pressure3d.cpp:858-863).
#include <algorithm>
#include <cmath>

#include "pf_solver.cuh"

namespace pf {
namespace {

__global__ void k_oc_set(SolveCtl* ctl, double tol, double res0, int max_iter) {
  *ctl = SolveCtl{};
  ctl->tol = tol;
  ctl->res0 = res0;
  ctl->res = res0;
  ctl->max_iter = max_iter;
  ctl->pin = -1;
}

// x = 0, p = q = 0 (the first direction is z itself)
__global__ void k_oc_zero(int nslots, double* x, double* p, double* q) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    x[o] = 0.0;
    p[o] = 0.0;
    q[o] = 0.0;
  }
}

// z . q_{k-1} -> beta
__global__ void __launch_bounds__(PF_TV) k_oc_beta(int nslots, SolveCtl* ctl, const uint8_t* kind, const float* z,
                                                   const double* q, double* partials) {
  if (ctl->done) return;
  double zq = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (kind[o]) zq += (double)z[o] * q[o];
  }
  block_reduce_3(zq, 0.0, 0.0, partials, ctl, kStageOuterBeta);
}

// p = z - beta p
__global__ void k_oc_dir(int nslots, const SolveCtl* ctl, const uint8_t* kind, const float* z, double* p) {
  if (ctl->done) return;
  const double beta = ctl->beta;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (kind[o]) p[o] = (double)z[o] - beta * p[o];
  }
}

// q = A p with the exact FP64 operator; p . q and r . p -> alpha
__global__ void __launch_bounds__(PF_TV) k_oc_spmv(const int* __restrict__ nbr, int nslots, SolveCtl* ctl,
                                                   const uint8_t* kind, const double* p, const double* r,
                                                   const double* diag, const double* cx, const double* cy,
                                                   const double* cz, double scale, double* q, double* partials) {
  if (ctl->done) return;
  double pq = 0.0, rp = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const int l = threadIdx.x;
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kind[o];
    if (!kd) continue;
    const double p0 = p[o];
    double ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets_tab(nbr, s, l, no);
      double off = 0.0;
      if (no[0] >= 0) off += cx[no[0]] * p[no[0]];
      if (no[1] >= 0) off += cx[o] * p[no[1]];
      if (no[2] >= 0) off += cy[no[2]] * p[no[2]];
      if (no[3] >= 0) off += cy[o] * p[no[3]];
      if (no[4] >= 0) off += cz[no[4]] * p[no[4]];
      if (no[5] >= 0) off += cz[o] * p[no[5]];
      ap = scale * (diag[o] * p0 - off);
    }
    q[o] = ap;
    pq += p0 * ap;
    rp += r[o] * p0;
  }
  block_reduce_3(pq, 0.0, rp, partials, ctl, kStageOuterPAp);
}

// x += alpha p, r -= alpha q; max|r| -> convergence
__global__ void __launch_bounds__(PF_TV) k_oc_update(int nslots, SolveCtl* ctl, const uint8_t* kind, double* x,
                                                     double* r, const double* p, const double* q, double* partials) {
  if (ctl->done) return;
  const double alpha = ctl->alpha;
  double rmax = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (!kind[o]) continue;
    x[o] += alpha * p[o];
    const double rn = r[o] - alpha * q[o];
    r[o] = rn;
    rmax = fmax(rmax, fabs(rn));
  }
  block_reduce_3(0.0, rmax, 0.0, partials, ctl, kStageOuterUpdate);
}

int poll_outer(pf_ctx* ctx, SolveCtl* out) {
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl_outer, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *ctx->h_ctl;
  return PF_OK;
}

}  // namespace

int solve_inner_outer(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, const int* nbr, double scale,
                      const pf_solve_cfg* cfg, InnerSolver& inner, double eta, int inner_max, SolveResult* res) {
  // the assembly's initial residual and tolerance (ctx->ctl, kStageInit); r = b, x = 0
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const SolveCtl c0 = *ctx->h_ctl;
  res->res0 = c0.res0;
  res->tol = c0.tol;
  res->res_final = c0.res0;
  if (c0.done == 4) {
    res->nonfinite = 1;
    return PF_OK;
  }
  (++ctx->launches), k_oc_zero<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->x, ctx->p, ctx->Ap);
  PF_CUDA_TRY(cudaGetLastError());
  if (!(c0.res0 >= c0.tol)) {
    res->converged = 1;
    return PF_OK;
  }
  (++ctx->launches), k_oc_set<<<1, 1, 0, ctx->stream>>>(ctx->ctl_outer, c0.tol, c0.res0, cfg->max_iter);
  PF_CUDA_TRY(cudaGetLastError());
  int inner_total = 0, outer = 0;
  SolveCtl c{};
  while (inner_total + outer < cfg->max_iter) {
    const float* z = nullptr;
    int its = 0;
    const int budget = std::min(inner_max, cfg->max_iter - inner_total - outer);
    int rc = inner.solve(ctx, eta, std::max(budget, 1), outer == 0, &z, &its);
    if (rc) return rc;
    inner_total += its;
    double* partials = ctx->partials;
    (++ctx->launches), k_oc_beta<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl_outer, kind, z, ctx->Ap, partials);
    (++ctx->launches), k_oc_dir<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl_outer, kind, z, ctx->p);
    (++ctx->launches), k_oc_spmv<<<nred, PF_TV, 0, ctx->stream>>>(nbr, nslots, ctx->ctl_outer, kind, ctx->p, ctx->r,
                                                                  ctx->diag, ctx->cx, ctx->cy, ctx->cz, scale,
                                                                  ctx->Ap, partials);
    (++ctx->launches), k_oc_update<<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl_outer, kind, ctx->x, ctx->r,
                                                                    ctx->p, ctx->Ap, partials);
    PF_CUDA_TRY(cudaGetLastError());
    ++outer;
    rc = poll_outer(ctx, &c);
    if (rc) return rc;
    if (c.done) break;
    if (its == 0) break;  // the inner solver made no progress: nothing left to offer
  }
  res->iterations = inner_total;
  res->refinements = outer;
  res->res_final = outer > 0 ? c.res : c0.res0;
  res->converged = c.done == 1 ? 1 : 0;
  res->breakdown = c.done == 2 ? 1 : 0;
  res->nonfinite = c.done == 4 ? 1 : 0;
  return PF_OK;
}

}  // namespace pf
