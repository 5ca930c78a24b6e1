// pf_project.cu -- beta = 1/rho variable-coefficient projection (Eq. 8),
// restating spProjectStepVC3D (src/driver/sparse_ops3d_tp.cpp:234-423) for
// the tile pool.
//
// Unknowns are the fluid cells of the pooled tiles, kept in pool layout
// (slot*512 + local) so the 7-point stencil needs no index arrays: in-tile
// neighbours are +-1/+-8/+-64, cross-tile ones go through the dense
// tile->slot array.  Off-diagonal couplings are stored once per cell for its
// low x/y/z faces (already masked: nonzero only between two non-pinned fluid
// cells, as the reference's nbr[] test at :309), so the SpMV reads 3 own
// coefficients + 3 neighbours' coefficients.
//
// PLAIN mode is the reference-equivalent FP64 Jacobi-PCG: rows, the
// preconditioner and every vector update round exactly as the reference
// (explicit _rn intrinsics, no FMA contraction); only the order of the inner
// products differs (a fixed-order two-level reduction, so results are
// reproducible run to run).  Each reduction finishes in the last CTA of the
// producing kernel, which also advances the scalar recurrences (alpha, beta,
// convergence) in device memory; the host only polls a done flag every few
// iterations.
#include <cmath>

#include "pf_ctx.h"
#include "pf_solver.cuh"

namespace pf {
namespace {

// Eq. 7 phase field -> beta (src/physics/phasefield.h:10-18), FP64 with the
// reference's operation order; rmin and the denominator come from the host,
// computed in the reference's order as well.
struct PhaseK {
  double rmin, den, rho_l, rho_g;
};

__device__ __forceinline__ double beta_of_raw(double raw, const PhaseK& P) {
  double phi;
  if (raw < P.rmin) {
    phi = 0.0;
  } else {
    double e = __dsub_rn(raw, P.rmin);
    if (e < 0.0) e = 0.0;
    phi = sqrt(__ddiv_rn(e, P.den));
    if (!(phi < 1.0)) phi = 1.0;
  }
  const double rho = __dadd_rn(__dmul_rn(phi, P.rho_l), __dmul_rn(__dsub_rn(1.0, phi), P.rho_g));
  return __ddiv_rn(1.0, rho);
}

__device__ __forceinline__ bool is_solid(const DevGrid& G, int i, int j, int k) {
  return !in_cells(G.g, i, j, k) || cell_marker(G, i, j, k) == 2;
}
__device__ __forceinline__ bool is_fluid(const DevGrid& G, int i, int j, int k) {
  return in_cells(G.g, i, j, k) && cell_marker(G, i, j, k) == 1;
}
__device__ __forceinline__ bool is_air(const DevGrid& G, int i, int j, int k) {
  return in_cells(G.g, i, j, k) && cell_marker(G, i, j, k) == 0;
}

__device__ __forceinline__ void slot_coords(const DevGrid& G, int s, int l, int& i, int& j, int& k) {
  const int t = G.slot_tile[s];
  const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
  i = tx * 8 + (l & 7);
  j = ty * 8 + ((l >> 3) & 7);
  k = tz * 8 + (l >> 6);
}

// request the tiles of every face of every fluid cell (the reference's
// g.u()/g.v()/g.w() writes activate them, :386-421)
__global__ void k_request_faces(DevGrid G, int nslots, uint8_t* need) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    int i, j, k;
    slot_coords(G, s, threadIdx.x, i, j, k);
    if (!in_cells(G.g, i, j, k) || cell_marker(G, i, j, k) != 1) continue;
    const int t1 = tile_id(G.g, (i + 1) >> 3, j >> 3, k >> 3);
    const int t2 = tile_id(G.g, i >> 3, (j + 1) >> 3, k >> 3);
    const int t3 = tile_id(G.g, i >> 3, j >> 3, (k + 1) >> 3);
    if (!need[t1]) need[t1] = 1;
    if (!need[t2]) need[t2] = 1;
    if (!need[t3]) need[t3] = 1;
  }
}

// fluid count, smallest fluid linear index, "some fluid cell touches air"
// (:250-264)
__global__ void k_classify(DevGrid G, int nslots, SolveCtl* ctl, uint8_t* kind) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    int i, j, k;
    slot_coords(G, s, threadIdx.x, i, j, k);
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    const bool fl = in_cells(G.g, i, j, k) && cell_marker(G, i, j, k) == 1;
    kind[o] = fl ? 1 : 0;
    const unsigned m = __ballot_sync(0xffffffffu, fl);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&ctl->n_cells, __popc(m));
    if (!fl) continue;
    const int c = i + G.g.nx * (j + G.g.ny * k);
    atomicMin(&ctl->min_fluid, c);
    if (is_air(G, i + 1, j, k) || is_air(G, i - 1, j, k) || is_air(G, i, j + 1, k) ||
        is_air(G, i, j - 1, k) || is_air(G, i, j, k + 1) || is_air(G, i, j, k - 1))
      atomicOr(&ctl->touches_air, 1);
  }
}

__global__ void k_pick_pin(SolveCtl* ctl) {
  ctl->pin = (ctl->n_cells > 0 && !ctl->touches_air) ? ctl->min_fluid : -1;
}

// Assembly (:266-313) and the first preconditioned direction.
template <typename V>
__global__ void __launch_bounds__(PF_TV) k_assemble(DevGrid G, int nslots, SolveCtl* ctl, uint8_t* kind,
                                                    PcgVec<V> vec, double scale, double cdiv, PhaseK ph,
                                                    double* partials) {
  double rz = 0.0, rmax = 0.0;
  const int pin = ctl->pin;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    int i, j, k;
    slot_coords(G, s, threadIdx.x, i, j, k);
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    double dg = 0.0, clx = 0.0, cly = 0.0, clz = 0.0, rr = 0.0;
    if (kind[o]) {
      const int c = i + G.g.nx * (j + G.g.ny * k);
      const bool pinned = c == pin;
      if (pinned) kind[o] = 2;
      const bool sol[6] = {is_solid(G, i + 1, j, k), is_solid(G, i - 1, j, k), is_solid(G, i, j + 1, k),
                           is_solid(G, i, j - 1, k), is_solid(G, i, j, k + 1), is_solid(G, i, j, k - 1)};
      const double fb[6] = {beta_of_raw(fget(G, PF_MU, i + 1, j, k), ph), beta_of_raw(fget(G, PF_MU, i, j, k), ph),
                            beta_of_raw(fget(G, PF_MV, i, j + 1, k), ph), beta_of_raw(fget(G, PF_MV, i, j, k), ph),
                            beta_of_raw(fget(G, PF_MW, i, j, k + 1), ph), beta_of_raw(fget(G, PF_MW, i, j, k), ph)};
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if (!sol[d]) dg = __dadd_rn(dg, fb[d]);
      auto nonpin_fluid = [&](int a, int b, int cc) {
        return is_fluid(G, a, b, cc) && (a + G.g.nx * (b + G.g.ny * cc)) != pin;
      };
      if (!pinned) {
        if (nonpin_fluid(i - 1, j, k)) clx = fb[1];
        if (nonpin_fluid(i, j - 1, k)) cly = fb[3];
        if (nonpin_fluid(i, j, k - 1)) clz = fb[5];
        const double uR = sol[0] ? 0.0 : (double)fget(G, PF_U, i + 1, j, k);
        const double uL = sol[1] ? 0.0 : (double)fget(G, PF_U, i, j, k);
        const double vT = sol[2] ? 0.0 : (double)fget(G, PF_V, i, j + 1, k);
        const double vB = sol[3] ? 0.0 : (double)fget(G, PF_V, i, j, k);
        const double wU = sol[4] ? 0.0 : (double)fget(G, PF_W, i, j, k + 1);
        const double wD = sol[5] ? 0.0 : (double)fget(G, PF_W, i, j, k);
        const double div = __dadd_rn(__dadd_rn(__dsub_rn(uR, uL), __dsub_rn(vT, vB)), __dsub_rn(wU, wD));
        rr = __dadd_rn(__ddiv_rn(-div, G.g.dx), cdiv);
      }
      const double dd = pinned ? 1.0 : __dmul_rn(scale, dg);
      const double z = dd > 0.0 ? __ddiv_rn(rr, dd) : 0.0;
      rz = __dadd_rn(rz, __dmul_rn(rr, z));
      rmax = fmax(rmax, fabs(rr));
      vec.store_p(o, z);
    } else {
      vec.store_p(o, 0.0);
    }
    vec.diag[o] = (V)dg;
    vec.cx[o] = (V)clx;
    vec.cy[o] = (V)cly;
    vec.cz[o] = (V)clz;
    vec.r[o] = (V)rr;
    vec.x[o] = (V)0.0;
  }
  block_reduce_2(rz, rmax, partials, ctl, /*stage=*/0, scale);
}

}  // namespace

// ---------------------------------------------------------------------------

static PhaseK phase_consts(const pf_phase* ph) {
  // the reference's order: rmin = (eta*rho_g)*rho_tilde_0, den = (alpha*rt0)*rho_l
  const double eta = std::log(ph->rho_l / ph->rho_g);
  PhaseK k;
  k.rmin = eta * ph->rho_g * ph->rho_tilde_0;
  k.den = ph->alpha_phi * ph->rho_tilde_0 * ph->rho_l;
  k.rho_l = ph->rho_l;
  k.rho_g = ph->rho_g;
  return k;
}

namespace {

// pressure write-back (:366-372): p field = (float)x on fluid cells
template <typename V>
__global__ void k_write_pressure(DevGrid G, int nslots, const uint8_t* kind, const V* x) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
    if (!kind[o]) continue;
    int i, j, k;
    slot_coords(G, s, threadIdx.x, i, j, k);
    G.fld[PF_P][o] = (float)(double)x[o];
    activate4(G, PF_P, i, j, k);
  }
}

// velocity update on faces adjacent to fluid cells (:374-422)
__global__ void k_velocity_update(DevGrid G, int nslots, double s_dt, PhaseK ph) {
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    int i, j, k;
    slot_coords(G, s, threadIdx.x, i, j, k);
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int f = PF_U + a;
      const int n_a = a == 0 ? G.g.nx : a == 1 ? G.g.ny : G.g.nz;
      const int ia = a == 0 ? i : a == 1 ? j : k;
      if (ia < 1 || ia > n_a - 1) continue;
      if (!in_field(G.g, f, i, j, k)) continue;
      const int li = i - (a == 0), lj = j - (a == 1), lk = k - (a == 2);
      const bool lf = is_fluid(G, li, lj, lk), hf = is_fluid(G, i, j, k);
      if (!lf && !hf) continue;
      if (is_solid(G, li, lj, lk) || is_solid(G, i, j, k)) {
        G.fld[f][o] = 0.0f;
      } else {
        const double pl = lf ? (double)fget(G, PF_P, li, lj, lk) : 0.0;
        const double ph_ = hf ? (double)fget(G, PF_P, i, j, k) : 0.0;
        const double bet = beta_of_raw((double)G.fld[PF_MU + a][o], ph);
        const float du = (float)__dmul_rn(__dmul_rn(s_dt, bet), __dsub_rn(ph_, pl));
        G.fld[f][o] = G.fld[f][o] - du;
      }
      activate4(G, f, i, j, k);
    }
  }
}

}  // namespace

int project(pf_ctx* ctx, const pf_phase* ph, double dt, const pf_solve_cfg* cfg, pf_solve_stats* st) {
  StageScope stage(ctx, PF_STAGE_PROJECT);
  pf_solve_stats local{};
  local.pin_cell = -1;
  int rc = field_clear(ctx, PF_P);  // waits for any pending pool growth
  if (rc) return rc;
  // pool the tiles of every fluid-cell face (no-op inside a step)
  if (ctx->nslots > 0) {
    (++ctx->launches), k_request_faces<<<ctx->nslots, PF_TV, 0, ctx->stream>>>(dev_grid(ctx), ctx->nslots, ctx->tile_need);
    PF_CUDA_TRY(cudaGetLastError());
  }
  rc = pool_commit(ctx);
  if (!rc) rc = pool_sync(ctx);
  if (rc) return rc;
  const int nslots = ctx->nslots;
  if (nslots == 0) { if (st) *st = local; return PF_OK; }
  DevGrid G = dev_grid(ctx);

  // reset the control block
  SolveCtl init{};
  init.min_fluid = 0x7fffffff;
  init.pin = -1;
  init.max_iter = cfg->max_iter;
  init.tol_abs = cfg->abs_tol;
  init.tol_rel = cfg->rel_tol;
  *ctx->h_ctl = init;
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->ctl, ctx->h_ctl, sizeof(SolveCtl), cudaMemcpyHostToDevice, ctx->stream));
  uint8_t* kind = ctx->kind;
  const int nred = nslots < kMaxRedBlocks ? nslots : kMaxRedBlocks;
  (++ctx->launches), k_classify<<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, ctx->ctl, kind);
  (++ctx->launches), k_pick_pin<<<1, 1, 0, ctx->stream>>>(ctx->ctl);
  PF_CUDA_TRY(cudaGetLastError());

  const PhaseK phk = phase_consts(ph);
  const double scale = dt / (ctx->g.dx * ctx->g.dx);
  PF_CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  SolveResult res{};
  PcgVec<double> vec{ctx->x, ctx->r, ctx->p, ctx->Ap, ctx->diag, ctx->cx, ctx->cy, ctx->cz};
  (++ctx->launches), k_assemble<double><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, ctx->ctl, kind, vec, scale, cfg->c_div, phk,
                                                      ctx->partials);
  PF_CUDA_TRY(cudaGetLastError());
  if (cfg->mode == PF_SOLVER_PLAIN) {
    rc = pcg_plain(ctx, nslots, nred, kind, vec, scale, cfg, &res);
    if (rc) return rc;
    (++ctx->launches), k_write_pressure<double><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, kind, ctx->x);
  } else if (cfg->mode == PF_SOLVER_LEARNED) {
    rc = solve_learned(ctx, nslots, nred, kind, scale, cfg, &res);
    if (rc) return rc;
    (++ctx->launches), k_write_pressure<double><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, kind, ctx->x);
  } else {
    rc = solve_mixed(ctx, nslots, nred, kind, scale, cfg, (const void*)&phk, &res);
    if (rc) return rc;
    (++ctx->launches), k_write_pressure<double><<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, kind, ctx->x);
  }
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  (++ctx->launches), k_velocity_update<<<nred, PF_TV, 0, ctx->stream>>>(G, nslots, dt / ctx->g.dx, phk);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  const SolveCtl& c = *ctx->h_ctl;
  local.iterations = res.iterations;
  local.refinements = res.refinements;
  local.n_cells = c.n_cells;
  local.pin_cell = c.pin;
  local.res0 = res.res0;
  local.res_final = res.res_final;
  local.tol_effective = res.tol;
  local.converged = res.converged;
  local.breakdown = res.breakdown;
  local.precond_applied = res.precond_applied;
  local.precond_rejected = res.precond_rejected;
  local.solve_ms = ms;
  if (st) *st = local;
  if (res.nonfinite) return set_error(ctx, PF_ERR_NONFINITE, "non-finite value in the pressure solve");
  return PF_OK;
}

}  // namespace pf

namespace pf {

// Launchers for the allocation-free projection (pf_noalloc.cu): the kernels of
// project() above, on caller-provided buffers and stream.
void launch_project_setup(const DevGrid& G, int nslots, int nred, SolveCtl* ctl, uint8_t* kind,
                          PcgVec<double> vec, double scale, double cdiv, const pf_phase* ph, double* partials,
                          cudaStream_t s) {
  k_classify<<<nred, PF_TV, 0, s>>>(G, nslots, ctl, kind);
  k_pick_pin<<<1, 1, 0, s>>>(ctl);
  k_assemble<double><<<nred, PF_TV, 0, s>>>(G, nslots, ctl, kind, vec, scale, cdiv, phase_consts(ph), partials);
}

void launch_project_finish(const DevGrid& G, int nslots, int nred, const uint8_t* kind, const double* x,
                           double dt_over_dx, const pf_phase* ph, cudaStream_t s) {
  k_write_pressure<double><<<nred, PF_TV, 0, s>>>(G, nslots, kind, x);
  k_velocity_update<<<nred, PF_TV, 0, s>>>(G, nslots, dt_over_dx, phase_consts(ph));
}

}  // namespace pf
