// pf_solver.cuh -- building blocks of the pressure solvers: pool-layout
// vectors, fixed-order two-level reductions that finish in the producing
// kernel's last CTA, and the scalar recurrences of (flexible) PCG kept in
// device memory.
#pragma once

#include <cmath>

#include "pf_ctx.h"

namespace pf {

template <typename V>
struct PcgVec {
  V *x, *r, *p, *Ap, *diag, *cx, *cy, *cz;
  V* z;  // PLAIN: z = r / diag from the update to the direction pass (null: formed in both)
  __device__ __forceinline__ void store_p(size_t o, double v) const { p[o] = (V)v; }
};

struct SolveResult {
  int iterations = 0, refinements = 0, converged = 0, breakdown = 0, nonfinite = 0;
  int precond_applied = 0, precond_rejected = 0;
  double res0 = 0.0, res_final = 0.0, tol = 0.0;
};

// reduction stages finished by the last CTA
enum RedStage {
  kStageInit = 0,    // after assembly: rz, max|r0| -> tolerance, early exit
  kStagePAp = 1,     // after SpMV: p.Ap -> alpha (breakdown check)
  kStageUpdate = 2,  // after x/r update: r.z, max|r| -> convergence, beta
  kStageResid = 3,   // outer refinement: max|b - A x| (FP64)
  kStageFlex = 4,    // flexible PCG x/r update: max|r| -> convergence; r.D^-1 r, r.z_prev kept for the guard
  kStageOuterBeta = 5,    // inner-outer FCG(1): z.q_prev -> beta (0 on the first outer iteration)
  kStageOuterPAp = 6,     // inner-outer FCG(1): p.q, r.p -> alpha (breakdown check)
  kStageOuterUpdate = 7,  // inner-outer FCG(1): max|r| -> convergence
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Sum of a and max of b over the block, in a fixed order (result in thread 0).
__device__ __forceinline__ void block_sum_max(double& a, double& b) {
  __shared__ double sa[32], sb[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_sum(a);
  b = warp_max(b);
  __syncthreads();
  if (lane == 0) { sa[wid] = a; sb[wid] = b; }
  __syncthreads();
  if (wid == 0) {
    a = lane < nw ? sa[lane] : 0.0;
    b = lane < nw ? sb[lane] : 0.0;
    a = warp_sum(a);
    b = warp_max(b);
  }
}

__device__ __forceinline__ void finalize_stage(SolveCtl* ctl, int stage, double S, double M, double S2) {
  switch (stage) {
    case kStageInit: {
      ctl->rz = S;
      ctl->flex[0] = S;
      ctl->flex[1] = S2;
      ctl->res0 = M;
      ctl->res = M;
      double tol = ctl->tol_abs;
      if (ctl->tol_rel > 0.0 && ctl->tol_rel * M > tol) tol = ctl->tol_rel * M;
      ctl->tol = tol;
      ctl->it = 0;
      if (!isfinite(S) || !isfinite(M)) ctl->done = 4;
      else if (!(M >= tol)) ctl->done = 1;
      else ctl->done = 0;
      break;
    }
    case kStagePAp: {
      ctl->pAp = S;
      if (!isfinite(S)) ctl->done = 4;
      else if (fabs(S) < 1e-30 || !isfinite(ctl->rz / S)) ctl->done = 2;
      else ctl->alpha = ctl->rz / S;
      break;
    }
    case kStageUpdate: {
      ctl->it += 1;
      ctl->res = M;
      if (!isfinite(M) || !isfinite(S)) ctl->done = 4;
      else if (M < ctl->tol) ctl->done = 1;
      else if (ctl->it >= ctl->max_iter) ctl->done = 3;
      else {
        ctl->beta = S / ctl->rz;
        ctl->rz = S;
      }
      break;
    }
    case kStageResid: {
      ctl->res = M;
      if (!isfinite(M)) ctl->done = 4;
      break;
    }
    case kStageOuterBeta: {
      double b = ctl->it > 0 && ctl->pAp != 0.0 ? S / ctl->pAp : 0.0;
      if (!isfinite(b)) b = 0.0;
      ctl->beta = b;
      break;
    }
    case kStageOuterPAp: {
      ctl->pAp = S;
      if (!isfinite(S) || !isfinite(S2)) ctl->done = 4;
      else if (!(S > 0.0) || !isfinite(S2 / S)) ctl->done = 2;
      else ctl->alpha = S2 / S;
      break;
    }
    case kStageOuterUpdate: {
      ctl->it += 1;
      ctl->res = M;
      if (!isfinite(M)) ctl->done = 4;
      else if (M < ctl->tol) ctl->done = 1;
      else if (ctl->it >= ctl->max_iter) ctl->done = 3;
      break;
    }
    case kStageFlex: {
      ctl->it += 1;
      ctl->res = M;
      ctl->flex[0] = S;
      ctl->flex[1] = S2;
      if (!isfinite(M) || !isfinite(S) || !isfinite(S2)) ctl->done = 4;
      else if (M < ctl->tol) ctl->done = 1;
      else if (ctl->it >= ctl->max_iter) ctl->done = 3;
      break;
    }
  }
}

// Per-CTA partial (sum a, max b, sum c) -> partials; the last CTA reduces all
// partials in index order and finishes the stage.  Every CTA of the grid must
// call this exactly once.
__device__ __forceinline__ void block_reduce_3(double a, double b, double c, double* partials, SolveCtl* ctl,
                                               int stage) {
  __shared__ bool am_last;
  double c2 = c, z0 = 0.0;
  block_sum_max(a, b);
  block_sum_max(c2, z0);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = a;
    partials[3 * blockIdx.x + 1] = b;
    partials[3 * blockIdx.x + 2] = c2;
    __threadfence();
    const unsigned t = atomicAdd(&ctl->counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double S = 0.0, M = 0.0, S2 = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) {
    S += __ldcg(&partials[3 * q + 0]);
    M = fmax(M, __ldcg(&partials[3 * q + 1]));
    S2 += __ldcg(&partials[3 * q + 2]);
  }
  block_sum_max(S, M);
  double z1 = 0.0;
  block_sum_max(S2, z1);
  if (threadIdx.x == 0) {
    finalize_stage(ctl, stage, S, M, S2);
    ctl->counter = 0;
  }
}

__device__ __forceinline__ void block_reduce_2(double a, double b, double* partials, SolveCtl* ctl, int stage,
                                               double /*unused*/ = 0.0) {
  block_reduce_3(a, b, 0.0, partials, ctl, stage);
}

// The streaming passes of the solvers walk their slots with a grid stride
// and read each cell's kind before its operands.  They load the kind of the
// next slot one trip ahead, so a trip waits for one round of memory latency
// (the operands) instead of two (kind, then operands).  The same holds for
// every other value an operand's address depends on (a cell's coarse class,
// the slot's tile, the neighbour table), and a pass issues all loads of a
// cell before its first store: the vectors may alias as far as the compiler
// knows, so a load after a store waits for the store's operands.
__device__ __forceinline__ uint8_t next_kind(const uint8_t* kind, int s, int nslots, int l) {
  return s < nslots ? kind[(size_t)s * PF_TV + l] : (uint8_t)0;
}

// Neighbour slots of the tile of slot s, order +x -x +y -y +z -z (-1 if none).
__device__ __forceinline__ void neighbor_slots(const DevGrid& G, int s, int* nbs) {
  if (threadIdx.x < 6) {
    const int t = G.slot_tile[s];
    int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
    const int d = threadIdx.x;
    tx += d == 0 ? 1 : d == 1 ? -1 : 0;
    ty += d == 2 ? 1 : d == 3 ? -1 : 0;
    tz += d == 4 ? 1 : d == 5 ? -1 : 0;
    int v = -1;
    if (tx >= 0 && ty >= 0 && tz >= 0 && tx < G.g.TX && ty < G.g.TY && tz < G.g.TZ)
      v = G.tile_slot[tile_id(G.g, tx, ty, tz)];
    nbs[d] = v;
  }
}

// Offsets of the six neighbours of local cell l within slot s: element index
// into a pool-layout array, or -1 when the neighbour tile is not pooled.
__device__ __forceinline__ void neighbor_offsets(int s, int l, const int* nbs, long long* off) {
  const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
  const long long base = (long long)s * PF_TV;
  off[0] = lx < 7 ? base + l + 1 : (nbs[0] >= 0 ? (long long)nbs[0] * PF_TV + (l & ~7) : -1);
  off[1] = lx > 0 ? base + l - 1 : (nbs[1] >= 0 ? (long long)nbs[1] * PF_TV + (l | 7) : -1);
  off[2] = ly < 7 ? base + l + 8 : (nbs[2] >= 0 ? (long long)nbs[2] * PF_TV + (l & ~56) : -1);
  off[3] = ly > 0 ? base + l - 8 : (nbs[3] >= 0 ? (long long)nbs[3] * PF_TV + (l | 56) : -1);
  off[4] = lz < 7 ? base + l + 64 : (nbs[4] >= 0 ? (long long)nbs[4] * PF_TV + (l & ~448) : -1);
  off[5] = lz > 0 ? base + l - 64 : (nbs[5] >= 0 ? (long long)nbs[5] * PF_TV + (l | 448) : -1);
}

// The same offsets from a neighbour-slot table nbr[6 s + d] (order as
// neighbor_slots), read only by the threads on a tile face: the stencil then
// needs no per-slot shared memory or synchronisation.
__device__ __forceinline__ void neighbor_offsets_tab(const int* __restrict__ nbr, int s, int l, long long* off) {
  const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
  const long long base = (long long)s * PF_TV;
  const int* nb = nbr + 6 * (size_t)s;
  int t;
  off[0] = lx < 7 ? base + l + 1 : ((t = __ldg(nb + 0)) >= 0 ? (long long)t * PF_TV + (l & ~7) : -1);
  off[1] = lx > 0 ? base + l - 1 : ((t = __ldg(nb + 1)) >= 0 ? (long long)t * PF_TV + (l | 7) : -1);
  off[2] = ly < 7 ? base + l + 8 : ((t = __ldg(nb + 2)) >= 0 ? (long long)t * PF_TV + (l & ~56) : -1);
  off[3] = ly > 0 ? base + l - 8 : ((t = __ldg(nb + 3)) >= 0 ? (long long)t * PF_TV + (l | 56) : -1);
  off[4] = lz < 7 ? base + l + 64 : ((t = __ldg(nb + 4)) >= 0 ? (long long)t * PF_TV + (l & ~448) : -1);
  off[5] = lz > 0 ? base + l - 64 : ((t = __ldg(nb + 5)) >= 0 ? (long long)t * PF_TV + (l | 448) : -1);
}

// The table entries of slot s held one per lane: lane d < 6 of every warp
// holds nbr[6 s + d] (-1 past the last slot).  A pass loads them one trip of
// its slot loop ahead, so the neighbour gathers of a trip need no table round
// trip.
__device__ __forceinline__ int nbr_lane(const int* __restrict__ nbr, int s, int nslots) {
  const int lane = threadIdx.x & 31;
  return s < nslots && lane < 6 ? __ldg(nbr + 6 * (size_t)s + lane) : -1;
}

// The neighbour slot a cell needs per axis, from the entries nbr_lane gave:
// the +side slot for a cell on the tile's high face, the -side slot
// otherwise (only a cell on the low face uses it).  Every lane of the warp
// must call it (shuffles).
__device__ __forceinline__ int3 neighbor_lanes(int nbl, int l) {
  const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
  return make_int3(__shfl_sync(0xffffffffu, nbl, lx == 7 ? 0 : 1), __shfl_sync(0xffffffffu, nbl, ly == 7 ? 2 : 3),
                   __shfl_sync(0xffffffffu, nbl, lz == 7 ? 4 : 5));
}

// neighbor_offsets_tab from the slots neighbor_lanes gave
__device__ __forceinline__ void neighbor_offsets_sel(int3 t, int s, int l, long long* off) {
  const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
  const long long base = (long long)s * PF_TV;
  off[0] = lx < 7 ? base + l + 1 : (t.x >= 0 ? (long long)t.x * PF_TV + (l & ~7) : -1);
  off[1] = lx > 0 ? base + l - 1 : (t.x >= 0 ? (long long)t.x * PF_TV + (l | 7) : -1);
  off[2] = ly < 7 ? base + l + 8 : (t.y >= 0 ? (long long)t.y * PF_TV + (l & ~56) : -1);
  off[3] = ly > 0 ? base + l - 8 : (t.y >= 0 ? (long long)t.y * PF_TV + (l | 56) : -1);
  off[4] = lz < 7 ? base + l + 64 : (t.z >= 0 ? (long long)t.z * PF_TV + (l & ~448) : -1);
  off[5] = lz > 0 ? base + l - 64 : (t.z >= 0 ? (long long)t.z * PF_TV + (l | 448) : -1);
}

// nbr[6 s + d] for every pooled slot (pf_flex.cu)
int build_neighbor_table(pf_ctx* ctx, int nslots, int** nbr);

// A truncated inner solve in reduced precision, the preconditioner of the
// inner-outer solver: from z = 0 it reduces the FP64 residual ctx->r by the
// factor eta (max-norm) or stops after max_iter iterations, and returns z in
// FP32 pool layout (zero off the unknowns) and its iteration count.  `first`
// marks the first inner solve of an outer solve.
struct InnerSolver {
  virtual int solve(pf_ctx* ctx, double eta, int max_iter, bool first, const float** z, int* iters) = 0;
  virtual ~InnerSolver() = default;
};

// FP64 flexible CG with one stored direction on the exact operator, each
// outer iteration preconditioned by inner.solve (pf_outer.cu).  Reports the
// inner iterations in res->iterations and the outer ones in res->refinements.
int solve_inner_outer(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, const int* nbr, double scale,
                      const pf_solve_cfg* cfg, InnerSolver& inner, double eta, int inner_max, SolveResult* res);

// solver drivers (pf_pcg.cu)
int pcg_plain(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, PcgVec<double> vec, double scale,
              const pf_solve_cfg* cfg, SolveResult* res);
int solve_mixed(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale, const pf_solve_cfg* cfg,
                const void* phase_consts, SolveResult* res);
int ensure_solver_buffers(pf_ctx* ctx, int mode);
int solve_learned(pf_ctx* ctx, int nslots, int nred, const uint8_t* kind, double scale, const pf_solve_cfg* cfg,
                  SolveResult* res);

}  // namespace pf
