// pf_coarse.cu -- two-class aggregation on the tile lattice: classification,
// Galerkin coarse operator, restriction, and an exact coarse solve
// (Jacobi-PCG in one CTA).  The exact solve is the target the learned coarse
// solve is trained against and the method it is ablated with.
#include <cmath>

#include "pf_coarse.cuh"
#include "pf_solver.cuh"

namespace pf {
namespace {

// Sums of n values over the block, fixed order, result in warp 0 lane 0.
template <int N>
__device__ __forceinline__ void block_sums(double* v) {
  __shared__ double sh[32][N];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) v[q] = warp_sum(v[q]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < N; ++q) sh[wid][q] = v[q];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = warp_sum(lane < nw ? sh[lane][q] : 0.0);
  }
}

__global__ void k_range_init(unsigned long long* drange) {
  drange[0] = (unsigned long long)__double_as_longlong(INFINITY);
  drange[1] = 0ull;
}

// min / max of the fine diagonal over fluid unknowns; positive doubles order
// like their bit patterns, so integer atomics give an order-free result
__global__ void __launch_bounds__(PF_TV) k_diag_range(int nslots, const uint8_t* kind, const double* diag,
                                                      unsigned long long* drange) {
  double lo = INFINITY, hi = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (kind[o] == 1 && diag[o] > 0.0) {
      lo = fmin(lo, diag[o]);
      hi = fmax(hi, diag[o]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0 && hi > 0.0) {
    atomicMin(&drange[0], (unsigned long long)__double_as_longlong(lo));
    atomicMax(&drange[1], (unsigned long long)__double_as_longlong(hi));
  }
}

// class split threshold: geometric mean of the diagonal range, or no split
// (everything class 0) when the coefficients vary by less than 16x
__device__ __forceinline__ double class_threshold(const unsigned long long* drange) {
  const double lo = __longlong_as_double((long long)drange[0]);
  const double hi = __longlong_as_double((long long)drange[1]);
  if (!(hi > 0.0) || !(lo > 0.0) || hi < 16.0 * lo) return INFINITY;
  return sqrt(lo * hi);
}

__device__ __forceinline__ int cell_class(uint8_t kd, double d, double tau) {
  if (kd != 1) return -1;
  return d >= tau ? 1 : 0;
}

// One CTA per pooled tile: classes of its unknowns and its coarse record.
__global__ void __launch_bounds__(PF_TV) k_coarse_assemble(DevGrid G, int nslots, const uint8_t* kind,
                                                           const double* diag, const double* cx, const double* cy,
                                                           const double* cz, double scale,
                                                           const unsigned long long* drange, uint8_t* cls,
                                                           float* cop) {
  const int s = blockIdx.x;
  if (s >= nslots) return;
  __shared__ int nbs[6];
  neighbor_slots(G, s, nbs);
  __syncthreads();
  const double tau = class_threshold(drange);
  const int t = G.slot_tile[s];
  const int l = threadIdx.x;
  const size_t o = (size_t)s * PF_TV + l;
  double v[kCopStride];
#pragma unroll
  for (int q = 0; q < kCopStride; ++q) v[q] = 0.0;
  const int c = cell_class(kind[o], diag[o], tau);
  cls[o] = c < 0 ? 255 : (uint8_t)c;
  if (c >= 0) {
    v[kCopD + c] = scale * diag[o];
    v[kCopN + c] = 1.0;
    long long no[6];
    neighbor_offsets(s, l, nbs, no);
    const double w3[3] = {scale * cx[o], scale * cy[o], scale * cz[o]};
    const int inner[3] = {(l & 7) > 0, ((l >> 3) & 7) > 0, (l >> 6) > 0};
    const int base[3] = {kCopX, kCopY, kCopZ};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double w = w3[a];
      if (w == 0.0) continue;
      const long long j = no[2 * a + 1];  // the low-side neighbour of this face
      if (j < 0) continue;
      const int cj = cell_class(kind[j], diag[j], tau);
      if (cj < 0) continue;
      if (inner[a]) {
        if (cj == c) v[kCopD + c] -= 2.0 * w;
        else v[kCopE] += w;
      } else {
        v[base[a] + 2 * c + cj] += w;
      }
    }
  }
  block_sums<kCopStride>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < kCopStride; ++q) cop[(size_t)t * kCopStride + q] = (float)v[q];
  }
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_coarse_restrict(const int* slot_tile, int nslots, const uint8_t* cls,
                                                           const V* r, float* rc, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const int s = blockIdx.x;
  if (s >= nslots) return;
  const size_t o = (size_t)s * PF_TV + threadIdx.x;
  const uint8_t c = cls[o];
  const double rr = c != 255 ? (double)r[o] : 0.0;
  double v[2] = {c == 0 ? rr : 0.0, c == 1 ? rr : 0.0};
  block_sums<2>(v);
  if (threadIdx.x == 0) {
    const int t = slot_tile[s];
    rc[2 * t] = (float)v[0];
    rc[2 * t + 1] = (float)v[1];
  }
}

__device__ __forceinline__ double coarse_apply(const CoarseOp& A, const double* x, int t, int c) {
  const int tx = t % A.TX, q = t / A.TX, ty = q % A.TY, tz = q / A.TY;
  const float* R = A.cop + (size_t)t * kCopStride;
  double y = (double)R[kCopD + c] * x[2 * t + c] - (double)R[kCopE] * x[2 * t + 1 - c];
  const int step[3] = {1, A.TX, A.TX * A.TY};
  const int has_lo[3] = {tx > 0, ty > 0, tz > 0};
  const int has_hi[3] = {tx + 1 < A.TX, ty + 1 < A.TY, tz + 1 < A.TZ};
  const int base[3] = {kCopX, kCopY, kCopZ};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (has_lo[a]) {
      const int u = t - step[a];
      y -= (double)R[base[a] + 2 * c] * x[2 * u] + (double)R[base[a] + 2 * c + 1] * x[2 * u + 1];
    }
    if (has_hi[a]) {
      const int u = t + step[a];
      const float* Ru = A.cop + (size_t)u * kCopStride;
      y -= (double)Ru[base[a] + c] * x[2 * u] + (double)Ru[base[a] + 2 + c] * x[2 * u + 1];
    }
  }
  return y;
}

__device__ __forceinline__ bool coarse_live(const CoarseOp& A, int u) {
  const int t = u >> 1, c = u & 1;
  return A.cop[(size_t)t * kCopStride + kCopN + c] > 0.0f && A.cop[(size_t)t * kCopStride + kCopD + c] > 0.0f;
}

__device__ __forceinline__ double block_sum1(double v) {
  double a[1] = {v};
  block_sums<1>(a);
  __shared__ double out;
  if (threadIdx.x == 0) out = a[0];
  __syncthreads();
  const double r = out;
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_max1(double v) {
  __shared__ double sh[32];
  __shared__ double out;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double a = lane < nw ? sh[lane] : 0.0;
    a = warp_max(a);
    if (lane == 0) out = a;
  }
  __syncthreads();
  const double r = out;
  __syncthreads();
  return r;
}

// Jacobi-PCG on the coarse unknowns in one CTA; iterations bounded by max_iter.
__global__ void __launch_bounds__(1024) k_coarse_cg(CoarseOp A, int max_iter, double rel_tol, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const int nu = 2 * A.nt;
  double* x = A.work;
  double* r = A.work + nu;
  double* p = A.work + 2 * (size_t)nu;
  double* Ap = A.work + 3 * (size_t)nu;
  auto dinv = [&](int u) -> double {
    return coarse_live(A, u) ? 1.0 / (double)A.cop[(size_t)(u >> 1) * kCopStride + kCopD + (u & 1)] : 0.0;
  };
  double rz = 0.0, rmax = 0.0;
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    const double di = dinv(u);
    const double rr = di > 0.0 ? (double)A.rc[u] : 0.0;
    x[u] = 0.0;
    r[u] = rr;
    p[u] = rr * di;
    rz += rr * rr * di;
    rmax = fmax(rmax, fabs(rr));
  }
  rz = block_sum1(rz);
  const double r0 = block_max1(rmax);
  const double tol = rel_tol * r0;
  if (r0 > 0.0) {
    for (int it = 0; it < max_iter; ++it) {
      double pAp = 0.0;
      for (int u = threadIdx.x; u < nu; u += blockDim.x) {
        const double y = coarse_live(A, u) ? coarse_apply(A, p, u >> 1, u & 1) : 0.0;
        Ap[u] = y;
        pAp += p[u] * y;
      }
      pAp = block_sum1(pAp);
      if (!(fabs(pAp) > 1e-300)) break;
      const double alpha = rz / pAp;
      double rzn = 0.0, rm = 0.0;
      for (int u = threadIdx.x; u < nu; u += blockDim.x) {
        x[u] += alpha * p[u];
        const double rr = r[u] - alpha * Ap[u];
        r[u] = rr;
        rzn += rr * rr * dinv(u);
        rm = fmax(rm, fabs(rr));
      }
      rzn = block_sum1(rzn);
      rm = block_max1(rm);
      if (rm < tol) break;
      const double beta = rzn / rz;
      rz = rzn;
      for (int u = threadIdx.x; u < nu; u += blockDim.x) p[u] = r[u] * dinv(u) + beta * p[u];
      __syncthreads();
    }
  }
  __syncthreads();
  for (int u = threadIdx.x; u < nu; u += blockDim.x) A.ec[u] = (float)x[u];
}

}  // namespace

int coarse_ensure(pf_ctx* ctx) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c) {
    c = new CoarseCtx();
    ctx->learned = c;
    CoarseOp& A = c->op;
    A.TX = ctx->g.TX;
    A.TY = ctx->g.TY;
    A.TZ = ctx->g.TZ;
    A.nt = ctx->g.ntiles;
    const size_t nt = (size_t)A.nt;
    PF_CUDA_TRY(cudaMalloc(&A.cop, nt * kCopStride * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(A.cop, 0, nt * kCopStride * sizeof(float)));
    PF_CUDA_TRY(cudaMalloc(&A.rc, 2 * nt * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(A.rc, 0, 2 * nt * sizeof(float)));
    PF_CUDA_TRY(cudaMalloc(&A.ec, 2 * nt * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(A.ec, 0, 2 * nt * sizeof(float)));
    PF_CUDA_TRY(cudaMalloc(&A.drange, 2 * sizeof(unsigned long long)));
    PF_CUDA_TRY(cudaMalloc(&A.work, 8 * nt * sizeof(double)));
  }
  if (c->cls_cap < ctx->cells_cap) {
    if (c->op.cls) cudaFree(c->op.cls);
    c->op.cls = nullptr;
    PF_CUDA_TRY(cudaMalloc(&c->op.cls, ctx->cells_cap));
    PF_CUDA_TRY(cudaMemset(c->op.cls, 255, ctx->cells_cap));
    c->cls_cap = ctx->cells_cap;
  }
  return PF_OK;
}

void coarse_release(pf_ctx* ctx) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c) return;
  learned_release(c);
  CoarseOp& A = c->op;
  void* ptrs[] = {A.cop, A.rc, A.ec, A.cls, A.drange, A.work, c->nbr, c->rc_part, c->inv_d};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete c;
  ctx->learned = nullptr;
}

int coarse_assemble(pf_ctx* ctx, int nslots, const uint8_t* kind, const double* diag, const double* cx,
                    const double* cy, const double* cz, double scale) {
  int rc = coarse_ensure(ctx);
  if (rc) return rc;
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  const size_t nt = (size_t)A.nt;
  PF_CUDA_TRY(cudaMemsetAsync(A.cop, 0, nt * kCopStride * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(A.rc, 0, 2 * nt * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(A.ec, 0, 2 * nt * sizeof(float), ctx->stream));
  (++ctx->launches), k_range_init<<<1, 1, 0, ctx->stream>>>(A.drange);
  if (nslots > 0) {
    const int nred = nslots < kMaxRedBlocks ? nslots : kMaxRedBlocks;
    (++ctx->launches), k_diag_range<<<nred, PF_TV, 0, ctx->stream>>>(nslots, kind, diag, A.drange);
    (++ctx->launches), k_coarse_assemble<<<nslots, PF_TV, 0, ctx->stream>>>(dev_grid(ctx), nslots, kind, diag, cx, cy,
                                                                          cz, scale, A.drange, A.cls, A.cop);
  }
  PF_CUDA_TRY(cudaGetLastError());
  coarse_new_system(ctx);
  return PF_OK;
}

template <typename V>
static int restrict_impl(pf_ctx* ctx, int nslots, const V* r, const SolveCtl* skip) {
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  if (nslots > 0)
    (++ctx->launches), k_coarse_restrict<V><<<nslots, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, A.cls, r, A.rc,
                                                                             skip);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int coarse_restrict(pf_ctx* ctx, int nslots, const uint8_t*, const float* r, const SolveCtl* skip) {
  return restrict_impl(ctx, nslots, r, skip);
}

int coarse_restrict(pf_ctx* ctx, int nslots, const uint8_t*, const double* r, const SolveCtl* skip) {
  return restrict_impl(ctx, nslots, r, skip);
}

int coarse_solve_exact(pf_ctx* ctx, int max_iter, double rel_tol, const SolveCtl* skip) {
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  (++ctx->launches), k_coarse_cg<<<1, 1024, 0, ctx->stream>>>(A, max_iter, rel_tol, skip);
  PF_CUDA_TRY(cudaGetLastError());
  return coarse_harvest(ctx, skip);
}

}  // namespace pf
