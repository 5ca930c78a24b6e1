// pf_coarse.cuh -- the coarse space of the two-level preconditioners.
//
// Two coarse unknowns per 8^3 tile, one per coefficient class: the fine
// unknowns of a tile are split by their diagonal (sum of face beta) at the
// geometric mean of the system's smallest and largest diagonal, so the
// light phase (beta = 1/rho_g, a gas bubble) and the heavy phase
// (beta = 1/rho_l) aggregate separately.  A bubble's constant-pressure mode,
// the near-null mode that makes the 1000:1 system hard for Jacobi, is then a
// sum of coarse basis vectors.  P is piecewise constant over each aggregate
// (the pinned cell belongs to none), the coarse operator is the Galerkin
// product A_c = P^T A P, and the preconditioner is
//   M^-1 r = D^-1 r + P c(P^T r)
// with c the exact coarse solve or the learned network (pf_learned.cu).
// Coarse arrays are dense over the whole tile lattice; tiles that are not
// pooled (or hold no unknowns of a class) have empty aggregates.
#pragma once

#include "pf_ctx.h"

namespace pf {

// Per-tile record of the coarse operator (kCopStride floats).  Couplings are
// stored as non-negative weights w; the operator entry is -w.
//   kCopD + c             diagonal of aggregate (t, c)
//   kCopE                 coupling between (t, 0) and (t, 1)
//   kCopX/Y/Z + 2*c + c2  coupling between (t, c) and (t - e_axis, c2)
//   kCopN + c             number of fine unknowns in (t, c)
enum : int { kCopD = 0, kCopE = 2, kCopX = 3, kCopY = 7, kCopZ = 11, kCopN = 15, kCopStride = 17 };
constexpr int kCoarseClasses = 2;

struct CoarseOp {
  int TX, TY, TZ, nt;
  float* cop;                   // [nt * kCopStride]
  float *rc, *ec;               // [nt * 2] restricted residual, coarse correction
  uint8_t* cls;                 // [pool cells] class of each fine unknown (255: none)
  unsigned long long* drange;   // [2] min / max fine diagonal (bit patterns of positive doubles)
  double* work;                 // [8 * nt] scratch of the exact coarse CG
};

struct LearnedState;  // network weights, optimiser, activations, training set (pf_learned.cu)

struct CoarseCtx {
  CoarseOp op{};
  LearnedState* net = nullptr;
  size_t cls_cap = 0;
  int* nbr = nullptr;       // neighbour-slot table of the pool (6 per slot)
  double* inv_d = nullptr;  // 1 / (scale diag) per cell of an FP64 flexible solve, 0 off the unknowns
  float* rc_part = nullptr; // per-warp restriction partials (16 warps x 2 classes per slot)
  size_t nbr_cap = 0;       // slots
};

int coarse_ensure(pf_ctx* ctx);
void coarse_release(pf_ctx* ctx);
// Classes and the Galerkin operator from the exact FP64 fine couplings
// (unscaled beta sums) times scale.
int coarse_assemble(pf_ctx* ctx, int nslots, const uint8_t* kind, const double* diag, const double* cx,
                    const double* cy, const double* cz, double scale);
// rc = P^T r (fine residual in pool layout); skipped when skip->done
int coarse_restrict(pf_ctx* ctx, int nslots, const uint8_t* kind, const float* r, const SolveCtl* skip);
int coarse_restrict(pf_ctx* ctx, int nslots, const uint8_t* kind, const double* r, const SolveCtl* skip);
// ec = A_c^-1 rc by Jacobi-PCG on the coarse lattice (one CTA); skipped when skip->done
int coarse_solve_exact(pf_ctx* ctx, int max_iter, double rel_tol, const SolveCtl* skip);
// once per solve, after coarse_assemble: the network's gates for this A_c
int coarse_prepare_net(pf_ctx* ctx);
// ec = learned correction of rc; returns PF_ERR_INVALID when no network is loaded
int coarse_solve_net(pf_ctx* ctx, const SolveCtl* skip);
bool coarse_net_ready(const pf_ctx* ctx);
// After a coarse solve: append (rc, ec) to the training set when harvesting
int coarse_harvest(pf_ctx* ctx, const SolveCtl* skip);
// A new coarse operator was assembled (starts a new system in the training set)
void coarse_new_system(pf_ctx* ctx);
void learned_release(CoarseCtx* c);

// device helpers shared by the solver kernels
__device__ __forceinline__ int coarse_index(int tile, uint8_t cls) { return 2 * tile + cls; }

}  // namespace pf
