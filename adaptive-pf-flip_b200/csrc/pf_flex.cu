// pf_flex.cu -- LEARNED mode: flexible PCG with the two-level preconditioner
//   M^-1 r = D^-1 r + P c(P^T r)
// where c is the learned coarse solve (or, for ablation and for training
// targets, the exact Galerkin coarse solve; or nothing, plain Jacobi).
//
// Polak-Ribiere beta r.(z - z_prev)/rz as the reference's flexible option
// (src/pressure/multires_pressure3d.cpp:1425-1434).  Each iteration has both
// candidates z_j = D^-1 r and z_c = z_j + P c; z_c is accepted only when
// r.z_c >= r.z_j (1 + min_gain) (the rz-gain guard of
// src/pressure/multires_pressure3d.cpp:1322-1334), and after kDisableAfter
// consecutive rejections the solve continues with Jacobi alone (the
// auto-disable of :1172).  Whatever the coarse term does, convergence is
// judged on the residual of the exact FP64 operator: directly in the FP64
// variant, through FP64 iterative refinement in the FP32 variant.
//
// Three fine-grid passes per iteration:
//   spmv    Ap, p.Ap -> alpha
//   update  x += alpha p, r -= alpha Ap, max|r|, r.D^-1 r, r.z_prev and the
//           per-warp partial sums of the restriction rc = P^T r (z_prev is
//           recomputed from the old r, so z is never stored)
//   [coarse solve on the tile lattice: rc from the partials, ec = c(rc)]
//   guard   r.P ec = rc.ec on the coarse lattice, so r.z_c = r.D^-1 r + rc.ec
//           without another fine pass; accept or reject, beta
//   dir     p = z + beta p
// The iteration body can be captured once into a CUDA graph and replayed.
#include <algorithm>
#include <cmath>

#include "pf_coarse.cuh"
#include "pf_solver.cuh"

namespace pf {
namespace {

constexpr int kDisableAfter = 8;

template <typename V>
struct FlexVec {
  V *e, *r, *Ap, *p;    // solution (correction), residual, A p, direction
  V *d, *cx, *cy, *cz;  // operator: diagonal and low-face couplings, times scale
  const uint8_t* cls;   // coarse class of each unknown (255: none)
  V scale;
  // FP64 solves: inv_diag of every cell, formed once per solve (the passes
  // then load it where they would load d, and divide nowhere)
  const double* di;
};

__global__ void k_fx_set(SolveCtl* ctl, double tol_abs, double tol_rel, int max_iter, double offered, int reset) {
  ctl->tol_abs = tol_abs;
  ctl->tol_rel = tol_rel;
  ctl->max_iter = max_iter;
  ctl->done = 0;
  ctl->it = 0;
  ctl->counter = 0;
  ctl->aux[0] = 0.0;
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
__device__ __forceinline__ double inv_diag(const FlexVec<V>& m, uint8_t kd, size_t o) {
  const double d = kd == 1 ? (double)m.scale * (double)m.d[o] : 0.0;
  return d > 0.0 ? 1.0 / d : 0.0;
}

// The passes round exactly as written: every multiply-add is an explicit fused
// fma (or an explicit product and sum), so the results do not depend on which
// products the compiler would contract in a given code layout.
__device__ __forceinline__ double fmav(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmav(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// r d^-1 + c (Jacobi term plus the coarse term), a product then a sum
__device__ __forceinline__ double coarse_add(double r, double di, double c) { return __dadd_rn(__dmul_rn(r, di), c); }

// 1 / (scale diag) of cell o: from the per-solve array in FP64 solves, else
// formed here
template <typename V>
__device__ __forceinline__ double inv_diag_at(const FlexVec<V>& m, uint8_t kd, size_t o) {
  if constexpr (sizeof(V) == 8) return m.di[o];
  else return inv_diag(m, kd, o);
}

constexpr int kWarpsPerSlot = PF_TV / 32;

// Per-warp class sums of r (32 cells of slot s) into part[(s * 16 + warp) * 2 + class];
// k_rc_reduce folds them into rc.  No block synchronisation.
__device__ __forceinline__ void restrict_warp(const uint8_t* cls, size_t o, double r, int s, float* part) {
  // FP32 suffices for the coarse residual (the preconditioner's input)
  const uint8_t c = cls[o];
  const float rf = (float)r;
  float a0 = c == 0 ? rf : 0.0f, a1 = c == 1 ? rf : 0.0f;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, d);
    a1 += __shfl_down_sync(0xffffffffu, a1, d);
  }
  if ((threadIdx.x & 31) == 0) {
    float* q = part + ((size_t)s * kWarpsPerSlot + (threadIdx.x >> 5)) * 2;
    q[0] = a0;
    q[1] = a1;
  }
}

// restrict_warp with the cell's class already loaded
__device__ __forceinline__ void restrict_warp_c(uint8_t c, double r, int s, float* part) {
  const float rf = (float)r;
  float a0 = c == 0 ? rf : 0.0f, a1 = c == 1 ? rf : 0.0f;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, d);
    a1 += __shfl_down_sync(0xffffffffu, a1, d);
  }
  if ((threadIdx.x & 31) == 0) {
    float* q = part + ((size_t)s * kWarpsPerSlot + (threadIdx.x >> 5)) * 2;
    q[0] = a0;
    q[1] = a1;
  }
}

// rc[2 tile + c] = sum of the 16 warp partials of the tile's slot, in order
__global__ void k_rc_reduce(const float* part, const int* slot_tile, int nslots, float* rc, const SolveCtl* skip) {
  pdl_wait();
  pdl_launch_dependents();
  if (skip && skip->done) return;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * nslots; q += gridDim.x * blockDim.x) {
    const int s = q >> 1, c = q & 1;
    double t = 0.0;
    for (int w = 0; w < kWarpsPerSlot; ++w) t += (double)part[((size_t)s * kWarpsPerSlot + w) * 2 + c];
    rc[coarse_index(slot_tile[s], (uint8_t)c)] = (float)t;
  }
}

// r = r_init (on unknowns), x = p = 0; max|r| -> res0 / tolerance; r.D^-1 r;
// rc = P^T r when rc != nullptr
template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_start(int nslots, SolveCtl* ctl, const uint8_t* kind, const double* r64,
                                                    FlexVec<V> m, float* rc_part, double* partials) {
  double rmax = 0.0, rzj = 0.0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const uint8_t kd = kind[o];
    const V r = kd ? (V)r64[o] : (V)0;
    m.r[o] = r;
    m.e[o] = (V)0;
    m.p[o] = (V)0;
    rmax = fmax(rmax, fabs((double)r));
    rzj += (double)r * (double)r * inv_diag(m, kd, o);
    if (rc_part) restrict_warp(m.cls, o, (double)r, s, rc_part);
  }
  block_reduce_3(rzj, rmax, 0.0, partials, ctl, kStageInit);  // res0, tol, done; flex = {r.D^-1 r, 0}
}

// inv_diag of every cell of the pooled slots (0 off the unknowns), once per
// FP64 solve
template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_inv_diag(int nslots, const uint8_t* kind, FlexVec<V> m, double* di) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    di[o] = inv_diag(m, kind[o], o);
  }
}

__global__ void k_build_nbr(DevGrid G, int nslots, int* nbr) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 6 * nslots; q += gridDim.x * blockDim.x) {
    const int s = q / 6, d = q - 6 * s;
    const int t = G.slot_tile[s];
    int tx = t % G.g.TX, r = t / G.g.TX, ty = r % G.g.TY, tz = r / G.g.TY;
    tx += d == 0 ? 1 : d == 1 ? -1 : 0;
    ty += d == 2 ? 1 : d == 3 ? -1 : 0;
    tz += d == 4 ? 1 : d == 5 ? -1 : 0;
    int v = -1;
    if (tx >= 0 && ty >= 0 && tz >= 0 && tx < G.g.TX && ty < G.g.TY && tz < G.g.TZ)
      v = G.tile_slot[tile_id(G.g, tx, ty, tz)];
    nbr[q] = v;
  }
}

template <typename V>
__global__ void __launch_bounds__(PF_TV, 4) k_fx_spmv(const int* __restrict__ nbr, int nslots, SolveCtl* ctl,
                                                   const uint8_t* kind, FlexVec<V> m, double* partials) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const int l = threadIdx.x;
  double acc = 0.0;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, l);
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kd_next;
    kd_next = next_kind(kind, s + gridDim.x, nslots, l);
    if (!kd) continue;
    const V p0 = m.p[o];
    V ap;
    if (kd == 2) {
      ap = p0;
    } else {
      long long no[6];
      neighbor_offsets_tab(nbr, s, l, no);
      V off = (V)0;
      if (no[0] >= 0) off = fmav(m.cx[no[0]], m.p[no[0]], off);
      if (no[1] >= 0) off = fmav(m.cx[o], m.p[no[1]], off);
      if (no[2] >= 0) off = fmav(m.cy[no[2]], m.p[no[2]], off);
      if (no[3] >= 0) off = fmav(m.cy[o], m.p[no[3]], off);
      if (no[4] >= 0) off = fmav(m.cz[no[4]], m.p[no[4]], off);
      if (no[5] >= 0) off = fmav(m.cz[o], m.p[no[5]], off);
      ap = m.scale * fmav(m.d[o], p0, -off);
    }
    m.Ap[o] = ap;
    acc = fmav((double)p0, (double)ap, acc);
  }
  block_reduce_2(acc, 0.0, partials, ctl, kStagePAp);
}

// x/r update with max|r| (convergence), r.D^-1 r and r.z_prev of the new r,
// where z_prev = D^-1 r_old (+ P ec_old if the last direction used it); and
// the warp partials of rc = P^T r_new when rc_part != nullptr
template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_update(int nslots, SolveCtl* ctl, const uint8_t* kind, FlexVec<V> m,
                                                     const int* slot_tile, const float* ec, float* rc_part,
                                                     double* partials) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const V alpha = (V)ctl->alpha;
  const bool used_c = ctl->aux[0] != 0.0;
  double rmax = 0.0, rzj = 0.0, rzp = 0.0;
  const int l = threadIdx.x;
  const bool want_cls = used_c || rc_part != nullptr;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, l);
  uint8_t cl_next = want_cls ? next_kind(m.cls, blockIdx.x, nslots, l) : (uint8_t)255;
  int tile_next = used_c && blockIdx.x < nslots ? slot_tile[blockIdx.x] : 0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kd_next, cl = cl_next;
    const int tile = tile_next;
    const int sn = s + gridDim.x;
    kd_next = next_kind(kind, sn, nslots, l);
    if (want_cls) cl_next = next_kind(m.cls, sn, nslots, l);
    if (used_c && sn < nslots) tile_next = slot_tile[sn];
    double rn = 0.0;
    if (kd) {
      const float ev = used_c && cl != 255 ? ec[coarse_index(tile, cl)] : 0.0f;
      const V e = m.e[o], p = m.p[o], r_old = m.r[o], ap = m.Ap[o];
      const double di = inv_diag_at(m, kd, o);
      m.e[o] = fmav(alpha, p, e);
      const V r = fmav(-alpha, ap, r_old);
      m.r[o] = r;
      rn = (double)r;
      const double zp = used_c ? coarse_add((double)r_old, di, cl != 255 ? (double)ev : 0.0) : (double)r_old * di;
      rmax = fmax(rmax, fabs(rn));
      rzj = fmav(rn * rn, di, rzj);
      rzp = fmav(rn, zp, rzp);
    }
    if (rc_part) restrict_warp_c(cl, rn, s, rc_part);
  }
  block_reduce_3(rzj, rmax, rzp, partials, ctl, kStageFlex);
}

// rc.ec over the coarse unknowns (grid-stride partials; the last CTA sums
// them in order), then the guard and beta:
//   r.z_j = flex[0], r.z_prev = flex[1], r.z_c = r.z_j + rc.ec
constexpr int kGuardThreads = 256;

__global__ void __launch_bounds__(kGuardThreads) k_fx_guard(SolveCtl* ctl, const float* rc, const float* ec, int nu,
                                                            int first, double min_gain, double* partials) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const bool offered = ctl->aux[2] != 0.0 && ctl->aux[1] == 0.0;
  double d = 0.0;
  if (offered)
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nu; u += gridDim.x * blockDim.x)
      d += (double)rc[u] * (double)ec[u];
  __shared__ double sh[kGuardThreads / 32];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  d = warp_sum(d);
  if (lane == 0) sh[wid] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += sh[w];
    partials[kRedSlots * blockIdx.x] = v;
    __threadfence();
    am_last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last || threadIdx.x != 0) return;
  __threadfence();
  double D = 0.0;
  for (int b = 0; b < (int)gridDim.x; ++b) D += __ldcg(&partials[kRedSlots * b]);
  ctl->counter = 0;
  const double S1 = ctl->flex[0], Q = ctl->flex[1];
  const double S0 = S1 + D;
  bool use_c = false;
  if (offered) {
    use_c = isfinite(S0) && S0 > 0.0 && S0 >= S1 * (1.0 + min_gain);
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
  const double rzn = use_c ? S0 : S1;
  if (!isfinite(rzn)) {
    ctl->done = 4;
    return;
  }
  double b = 0.0;
  if (!first && ctl->rz != 0.0) {
    b = (rzn - Q) / ctl->rz;  // Polak-Ribiere: r.(z - z_prev) / r_prev.z_prev
    if (!isfinite(b) || b < 0.0) b = 0.0;
  }
  ctl->beta = b;
  ctl->rz = rzn;
}

template <typename V>
__global__ void __launch_bounds__(PF_TV) k_fx_dir(const int* slot_tile, int nslots, const SolveCtl* ctl,
                                                  const uint8_t* kind, FlexVec<V> m, const float* ec) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const V beta = (V)ctl->beta;
  const bool use_c = ctl->aux[0] != 0.0;
  const int l = threadIdx.x;
  uint8_t kd_next = next_kind(kind, blockIdx.x, nslots, l);
  uint8_t cl_next = use_c ? next_kind(m.cls, blockIdx.x, nslots, l) : (uint8_t)255;
  int tile_next = use_c && blockIdx.x < nslots ? slot_tile[blockIdx.x] : 0;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + l;
    const uint8_t kd = kd_next, cl = cl_next;
    const int tile = tile_next;
    const int sn = s + gridDim.x;
    kd_next = next_kind(kind, sn, nslots, l);
    if (use_c) {
      cl_next = next_kind(m.cls, sn, nslots, l);
      if (sn < nslots) tile_next = slot_tile[sn];
    }
    if (!kd) continue;
    const float ev = use_c && cl != 255 ? ec[coarse_index(tile, cl)] : 0.0f;
    const double di = inv_diag_at(m, kd, o);
    if (use_c) {
      const double z = coarse_add((double)m.r[o], di, cl != 255 ? (double)ev : 0.0);
      m.p[o] = fmav(beta, m.p[o], (V)z);
    } else {  // Jacobi only: one fma of r d^-1 over beta p
      m.p[o] = (V)fmav((double)m.r[o], di, (double)(beta * m.p[o]));
    }
  }
}

int poll_ctl(pf_ctx* ctx, SolveCtl* out) {
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *ctx->h_ctl;
  return PF_OK;
}

}  // namespace

int build_neighbor_table(pf_ctx* ctx, int nslots, int** nbr) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  const size_t cap = ctx->cells_cap / PF_TV;
  if (c->nbr_cap < cap) {
    if (c->nbr) cudaFree(c->nbr);
    if (c->rc_part) cudaFree(c->rc_part);
    if (c->inv_d) cudaFree(c->inv_d);
    c->nbr = nullptr;
    c->rc_part = nullptr;
    c->inv_d = nullptr;
    PF_CUDA_TRY(cudaMalloc(&c->nbr, 6 * cap * sizeof(int)));
    PF_CUDA_TRY(cudaMalloc(&c->inv_d, cap * PF_TV * sizeof(double)));
    PF_CUDA_TRY(cudaMalloc(&c->rc_part, cap * kWarpsPerSlot * 2 * sizeof(float)));
    c->nbr_cap = cap;
  }
  if (nslots > 0) {
    const int blocks = std::min((6 * nslots + 255) / 256, 148 * 16);
    (++ctx->launches), k_build_nbr<<<blocks, 256, 0, ctx->stream>>>(dev_grid(ctx), nslots, c->nbr);
    PF_CUDA_TRY(cudaGetLastError());
  }
  *nbr = c->nbr;
  return PF_OK;
}

namespace {

// rc from the warp partials, then the coarse correction ec
int coarse_solve(pf_ctx* ctx, int nslots, int precond) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  const int blocks = std::max(1, std::min((2 * nslots + 255) / 256, 148 * 8));
  ++ctx->launches;
  PF_CUDA_TRY(launch_pdl(k_rc_reduce, dim3(blocks), dim3(256), ctx->stream, (const float*)c->rc_part,
                         (const int*)ctx->slot_tile, nslots, c->op.rc, (const SolveCtl*)ctx->ctl));
  if (precond == PF_PRECOND_EXACT_COARSE) return coarse_solve_exact(ctx, 400, 1e-6, ctx->ctl);
  return coarse_solve_net(ctx, ctx->ctl);
}

int launch_guard(pf_ctx* ctx, bool coarse, int first, double min_gain) {
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  const int nu = coarse ? 2 * A.nt : 0;
  const int blocks = std::max(1, std::min((nu + kGuardThreads - 1) / kGuardThreads, 64));
  ++ctx->launches;
  PF_CUDA_TRY(launch_pdl(k_fx_guard, dim3(blocks), dim3(kGuardThreads), ctx->stream, ctx->ctl, (const float*)A.rc,
                         (const float*)A.ec, nu, first, min_gain, ctx->partials));
  return PF_OK;
}

// spmv, update, [coarse solve], guard, dir
template <typename V>
int launch_iteration(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, const FlexVec<V>& m, int precond,
                     double min_gain) {
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  const bool coarse = precond != PF_PRECOND_JACOBI;
  const int* nbr = ((CoarseCtx*)ctx->learned)->nbr;
  ++ctx->launches;
  PF_CUDA_TRY(launch_pdl(k_fx_spmv<V>, dim3(nred), dim3(PF_TV), ctx->stream, nbr, nslots, ctx->ctl, kind, m,
                         ctx->partials));
  float* rc_part = coarse ? ((CoarseCtx*)ctx->learned)->rc_part : nullptr;
  ++ctx->launches;
  PF_CUDA_TRY(launch_pdl(k_fx_update<V>, dim3(nred), dim3(PF_TV), ctx->stream, nslots, ctx->ctl, kind, m,
                         (const int*)ctx->slot_tile, (const float*)A.ec, rc_part, ctx->partials));
  if (coarse) {
    int rc = coarse_solve(ctx, nslots, precond);
    if (rc) return rc;
  }
  int rcg = launch_guard(ctx, coarse, 0, min_gain);
  if (rcg) return rcg;
  ++ctx->launches;
  PF_CUDA_TRY(launch_pdl(k_fx_dir<V>, dim3(nred), dim3(PF_TV), ctx->stream, (const int*)ctx->slot_tile, nslots,
                         (const SolveCtl*)ctx->ctl, kind, m, (const float*)A.ec));
  return PF_OK;
}

// The iteration body captured once; replays are launched like one kernel.
struct IterGraph {
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;  // kernels per replay
  ~IterGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

template <typename V>
int capture_iteration(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, const FlexVec<V>& m, int precond,
                      double min_gain, IterGraph* g) {
  const long long before = ctx->launches;
  PF_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = launch_iteration<V>(ctx, nslots, nred, kind, m, precond, min_gain);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  PF_CUDA_TRY(e);
  const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
  cudaGraphDestroy(graph);
  PF_CUDA_TRY(ei);
  g->launches = ctx->launches - before;
  ctx->launches = before;
  return PF_OK;
}

// Flexible PCG from x = 0 on r_init until max|r| < max(tol_abs, tol_rel max|r0|).
// `keep`, when given, holds the captured iteration body across calls with
// the same vectors (the inner solves of one inner-outer solve).
template <typename V>
int flex_solve(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, FlexVec<V> m, const double* r_init,
               double tol_abs, double tol_rel, int max_iter, int check_every, int precond, double min_gain,
               int reset_guard, SolveCtl* out, IterGraph* keep = nullptr) {
  CoarseOp& A = ((CoarseCtx*)ctx->learned)->op;
  const bool coarse = precond != PF_PRECOND_JACOBI;
  (++ctx->launches), k_fx_set<<<1, 1, 0, ctx->stream>>>(ctx->ctl, tol_abs, tol_rel, max_iter, coarse ? 1.0 : 0.0,
                                                        reset_guard);
  float* rc_part = coarse ? ((CoarseCtx*)ctx->learned)->rc_part : nullptr;
  (++ctx->launches), k_fx_start<V><<<nred, PF_TV, 0, ctx->stream>>>(nslots, ctx->ctl, kind, r_init, m, rc_part,
                                                                    ctx->partials);
  int rc = PF_OK;
  if (coarse) rc = coarse_solve(ctx, nslots, precond);
  if (rc) return rc;
  rc = launch_guard(ctx, coarse, 1, min_gain);
  if (rc) return rc;
  (++ctx->launches), k_fx_dir<V><<<nred, PF_TV, 0, ctx->stream>>>(ctx->slot_tile, nslots, ctx->ctl, kind, m, A.ec);
  PF_CUDA_TRY(cudaGetLastError());
  // the exact coarse solve records training pairs on the host side, so it is
  // launched directly; the other bodies are replayed from a graph
  IterGraph local;
  IterGraph& graph = keep ? *keep : local;
  if (precond != PF_PRECOND_EXACT_COARSE && !graph.exec) {
    rc = capture_iteration<V>(ctx, nslots, nred, kind, m, precond, min_gain, &graph);
    if (rc) return rc;
  }
  SolveCtl c{};
  rc = poll_ctl(ctx, &c);
  if (rc) return rc;
  int launched = 0;
  int batch = check_every > 0 ? check_every : 4;
  while (!c.done && launched < max_iter) {
    const int nb = std::min(batch, max_iter - launched);
    for (int q = 0; q < nb; ++q) {
      if (graph.exec) {
        PF_CUDA_TRY(cudaGraphLaunch(graph.exec, ctx->stream));
        ctx->launches += graph.launches;
      } else {
        rc = launch_iteration<V>(ctx, nslots, nred, kind, m, precond, min_gain);
        if (rc) return rc;
      }
    }
    launched += nb;
    rc = poll_ctl(ctx, &c);
    if (rc) return rc;
    if (check_every <= 0) batch = std::min(batch * 2, 64);
  }
  *out = c;
  return PF_OK;
}

// The inner solver of LEARNED with FP32 vectors: the flexible PCG with the
// two-level preconditioner on the FP32 copy of the operator, from e = 0.
struct LearnedInner final : InnerSolver {
  int nslots = 0, nred = 0, check_every = 0, precond = 0;
  const uint8_t* kind = nullptr;
  double min_gain = 0.0;
  FlexVec<float> m{};
  IterGraph graph;
  int accepted = 0, rejected = 0;
  int solve(pf_ctx* ctx, double eta, int max_iter, bool first, const float** z, int* iters) override {
    SolveCtl ic{};
    const int poll_at = check_every > 0 ? check_every : std::max(1, max_iter / 2);
    const int rc = flex_solve<float>(ctx, nslots, nred, kind, m, ctx->r, 0.0, eta, max_iter, poll_at, precond,
                                     min_gain, first ? 1 : 0, &ic, &graph);
    if (rc) return rc;
    *iters = ic.it;
    *z = m.e;
    accepted = ic.accepted;
    rejected = ic.rejected;
    return ic.done == 4 ? set_error(ctx, PF_ERR_NONFINITE, "non-finite value in the inner solve") : PF_OK;
  }
};

}  // namespace

int solve_learned(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale, const pf_solve_cfg* cfg,
                  SolveResult* res) {
  StageScope stage(ctx, PF_STAGE_PCG);
  StageScope setup_stage(ctx, PF_STAGE_PRECOND_SETUP);
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
  int* nbr = nullptr;
  rc = build_neighbor_table(ctx, nslots, &nbr);
  if (rc) return rc;
  stage_end(ctx, PF_STAGE_PRECOND_SETUP);

  if (!cfg->inner_fp32) {
    // FP64 flexible PCG on the exact operator
    FlexVec<double> m{ctx->x, ctx->r, ctx->Ap, ctx->p, ctx->diag, ctx->cx, ctx->cy, ctx->cz, cls, scale};
    double* di = ((CoarseCtx*)ctx->learned)->inv_d;
    (++ctx->launches), k_fx_inv_diag<double><<<nred, PF_TV, 0, ctx->stream>>>(nslots, kind, m, di);
    PF_CUDA_TRY(cudaGetLastError());
    m.di = di;
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

  // FP64 flexible CG preconditioned by the learned flexible PCG in FP32
  rc = ensure_solver_buffers(ctx, PF_SOLVER_MIXED);
  if (rc) return rc;
  (++ctx->launches), k_fx_setup32<<<nred, PF_TV, 0, ctx->stream>>>(nslots, kind, ctx->diag, ctx->cx, ctx->cy, ctx->cz,
                                                                    ctx->r, scale, ctx->diagf, ctx->cxf, ctx->cyf,
                                                                    ctx->czf, ctx->b64);
  PF_CUDA_TRY(cudaGetLastError());
  LearnedInner inner;
  inner.nslots = nslots;
  inner.nred = nred;
  inner.kind = kind;
  inner.check_every = cfg->check_every;
  inner.precond = precond;
  inner.min_gain = cfg->accept_min_gain;
  inner.m = FlexVec<float>{ctx->xf, ctx->rf, ctx->Apf, ctx->pf32, ctx->diagf, ctx->cxf, ctx->cyf, ctx->czf, cls, 1.0f};
  const double eta = cfg->inner_rel_tol > 0.0 ? cfg->inner_rel_tol : 1e-3;
  const int inner_max = cfg->inner_max_iter > 0 ? cfg->inner_max_iter : 200;
  rc = solve_inner_outer(ctx, nslots, nred, kind, nbr, scale, cfg, inner, eta, inner_max, res);
  res->precond_applied = inner.accepted;
  res->precond_rejected = inner.rejected;
  return rc;
}

}  // namespace pf
