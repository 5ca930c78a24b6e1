/*
 * pf_oracle.h -- CPU restatement of the adaptive-pf-flip sparse 3D two-phase
 * solver step (P2G, marker/boundary passes, beta=1/rho PCG projection, G2P,
 * RK2/RK3 advection).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the GPU path is
 * compared against; it is never linked into, loaded by, or called from the
 * product library (libpfgpu).  Only tests, the smoke check and the CPU-baseline
 * leg of bench.py use it.
 *
 * Every function states the reference file:line it restates (paths relative to
 * the adaptive-pf-flip source tree).  The floating-point operation order of the
 * reference is kept wherever the result is compared bit-for-bit (activation
 * tests, per-node accumulation order, PCG reductions in ascending cell order),
 * so the oracle reproduces the reference's own outputs exactly on the same
 * inputs; the parity tests check that against the compiled reference.
 *
 * Grid representation: every field is a dense float array over its own node
 * lattice (u: (nx+1,ny,nz), v: (nx,ny+1,nz), w: (nx,ny,nz+1), mu/mv/mw alike,
 * p and the marker: (nx,ny,nz)), index i + X*(j + Y*k), plus a byte per 4^3
 * block (bid = bx + nbx*(by + nby*bz)) recording whether the reference's
 * SparseBlockGrid3D<4> would hold that block active.  Values inside inactive
 * blocks are kept at zero, which is what SparseBlockGrid3D::get returns for
 * them (src/grid/sparse_block_grid3d.h:50-55).
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PFO_U = 0, PFO_V, PFO_W, PFO_MU, PFO_MV, PFO_MW, PFO_P, PFO_MK, PFO_NFIELDS };

typedef struct pfo_grid pfo_grid;

typedef struct {
  double rho_l, rho_g, alpha_phi, rho_tilde_0; /* PhaseParams, src/physics/phasefield.h:4-9 */
} pfo_phase;

typedef struct {
  int max_iter;     /* cg_iters */
  double abs_tol;   /* reference cg_tol: stop when max|r| < tol */
  double rel_tol;   /* 0 = reference behaviour; else tol = max(abs, rel*max|r0|) */
  double c_div;     /* divergenceCorrection */
} pfo_solve_cfg;

typedef struct {
  int iterations;
  int n_cells;
  long long pin_cell; /* linear cell index or -1 */
  double res0, res_final, tol_effective;
  int converged;
  int breakdown;
} pfo_solve_stats;

typedef struct {
  int clamped_liquid, clamped_gas;
  int x_lo, x_hi, y_lo, y_hi, z_lo, z_hi;
} pfo_clamp_stats;

typedef struct {
  double dt, gravity, Vp, alpha_l, alpha_g;
  int cg_iters;
  double cg_tol, cg_rel_tol, c_div;
  int advect_order;
} pfo_step_cfg;

pfo_grid* pfo_grid_create(int nx, int ny, int nz, double dx, double ox, double oy, double oz);
void pfo_grid_destroy(pfo_grid* g);
int pfo_grid_copy(pfo_grid* dst, const pfo_grid* src);
int pfo_field_dims(const pfo_grid* g, int f, int* dims3, int* bdims3);
int pfo_get_field(const pfo_grid* g, int f, float* dense, unsigned char* act);
int pfo_set_field(pfo_grid* g, int f, const float* dense, const unsigned char* act);
int pfo_clear_field(pfo_grid* g, int f);
int pfo_clear_all(pfo_grid* g);

double pfo_phi_from_raw(double raw, const pfo_phase* pp);
double pfo_beta_from_raw(double raw, const pfo_phase* pp);
double pfo_calibrate_rho_tilde0(const pfo_phase* pp, double Vp);

int pfo_mark_cells(pfo_grid* g, size_t n, const double* pos);
int pfo_p2g(pfo_grid* g, size_t n, const double* pos, const double* vel,
            const unsigned char* type, const double* vol, const pfo_phase* pp, double Vp);
int pfo_apply_gravity(pfo_grid* g, double dt, double gravity);
int pfo_apply_wall_boundary(pfo_grid* g);
int pfo_project(pfo_grid* g, const pfo_phase* pp, double dt, const pfo_solve_cfg* cfg,
                pfo_solve_stats* st);
int pfo_g2p(const pfo_grid* g, const pfo_grid* saved, size_t n, const double* pos, double* vel,
            const unsigned char* type, double aL, double aG);
int pfo_advect(const pfo_grid* g, size_t n, double* pos, const unsigned char* type,
               const double* vel, const double* vol, double dt, int order,
               pfo_clamp_stats* st, double* escape_out, size_t* n_escape);
int pfo_collect_cells(const pfo_grid* g, int marker, int* out, size_t* n);
int pfo_step(pfo_grid* g, pfo_grid* saved, size_t n, double* pos, double* vel,
             const unsigned char* type, const double* vol, const pfo_phase* pp,
             const pfo_step_cfg* cfg, pfo_solve_stats* sst, pfo_clamp_stats* cst);

/* ---- particle adaptivity (src/driver/particle_adaptivity3d.h) ---------- */
/* Particles are the caller's arrays (pos, vel: 3 doubles each, type, vol);
 * every function updates them in place and *n with the new count.  Erasures
 * keep the survivors' order (Particles3DTP::eraseIf); refill appends at the
 * end and fails (-1, nothing changed) if *n would exceed cap. */
typedef struct { int removed, liquid_cells, gas_before, gas_after; } pfo_band_stats;
typedef struct { int removed, cells, overfull_cells, before, after; } pfo_coarsen_stats;
typedef struct { int added, cells, interface_cells, underfull_cells, budget_limited, before, after; } pfo_refill_stats;

unsigned pfo_particle_score(const pfo_grid* g, const double* x, int i, int j, int k, unsigned seed);
unsigned pfo_slot_score(size_t cell, int slot, unsigned seed);
int pfo_narrow_band_air(const pfo_grid* g, size_t* n, double* pos, double* vel, unsigned char* type, double* vol,
                        int radius, pfo_band_stats* st);
int pfo_coarsen_particles(const pfo_grid* g, size_t* n, double* pos, double* vel, unsigned char* type, double* vol,
                          int ptype, int target, unsigned seed, pfo_coarsen_stats* st);
int pfo_refill_liquid(const pfo_grid* g, size_t* n, size_t cap, double* pos, double* vel, unsigned char* type,
                      double* vol, int target, unsigned seed, int interface_only, int interface_radius, int max_added,
                      pfo_refill_stats* st);

/* ---- interface diagnostics (src/driver/interface_diagnostics3d.cpp:363-379) ---- */
typedef struct {
  int sample_cells, interface_cells, finite, surface_tension_candidate;
  double phi_min, phi_max, phi_mean, grad_mean, grad_max, curvature_abs_mean, curvature_abs_max;
} pfo_interface_stats;
int pfo_interface_diagnostics(const pfo_grid* g, const pfo_phase* pp, pfo_interface_stats* st);

/* ---- surface tension (src/driver/interface_diagnostics3d.cpp:405-447) ---- */
typedef struct {
  int enabled, applied_cells, finite, curvature_smoothing_radius, capillary_stable;
  double strength, max_delta_speed_limit, mean_delta_speed, max_delta_speed, raw_curvature_abs_mean,
      raw_curvature_abs_max, smoothed_curvature_abs_mean, smoothed_curvature_abs_max, capillary_dt_limit;
} pfo_surface_stats;
int pfo_surface_tension(pfo_grid* g, const pfo_phase* pp, double dt, double strength, double max_delta_speed,
                        int smoothing_radius, pfo_surface_stats* st);

/* ---- 2-level multires step (pf_oracle_mr.c) ------------------------------
 * src/grid/multires_layout3d.h, src/driver/multires_ops3d_tp.cpp,
 * src/driver/multires_sim3d_tp.cpp:23-227, 577-733,
 * src/pressure/multires_pressure3d.cpp.  The layout is one flag per level-1
 * block of 8^3 fine cells (1: split into level-0 blocks), x fastest.  Face
 * fields are dense over the fine face lattice; 0..5 = u v w mu mv mw, 6..8 =
 * the step's saved u v w.  Markers and pressure are per fine cell (the value
 * of the leaf cell holding it). */
enum { PFO_MR_NFACE = 9 };
typedef struct pfo_mr pfo_mr;
typedef struct {
  int enabled, particle_padding, gas_padding, hysteresis_cells, max_fine_leaves;
} pfo_mr_dynamic;
typedef struct {
  int max_iter;
  double abs_tol, rel_tol;
  int jacobi, flexible_beta, adaptive_restart;
  double restart_growth, c_div;
} pfo_mr_solve_cfg;
typedef struct {
  int active_cells, pinned_cell, max_iterations, iterations, restarts, beta_resets, converged, breakdown;
  double initial_residual, final_residual, effective_tolerance, min_positive_diag, max_diag;
} pfo_mr_solve_stats;
typedef struct {
  double dt, gravity, Vp, alpha_l, alpha_g;
  int advect_order;
  pfo_mr_solve_cfg solve;
} pfo_mr_step_cfg;

/* ---- secondary particles (pf_oracle_sec.c) --------------------------------
 * src/driver/secondary_particles3d.h:9-467.  A set is caller storage:
 * positions and velocities (3 doubles each), volumes and ages, n of cap. */
typedef struct {
  size_t n, cap;
  double *pos, *vel, *vol;
  int* age;
} pfo_sec_set;
typedef struct {
  int nx, ny, nz;
  double dx, ox, oy, oz;
} pfo_sec_domain;
typedef struct { /* SecondaryParticleLifecycleConfig3D */
  int enabled, droplet_lifetime_steps, bubble_lifetime_steps;
  double velocity_damping, reabsorb_margin_cells, gravity, droplet_gravity_scale, bubble_buoyancy_scale,
      droplet_drag, bubble_drag, particle_volume_scale;
} pfo_sec_cfg;
typedef struct { /* SecondaryParticleLifecycleStats3D */
  int enabled, finite, advected_droplets, advected_bubbles, reabsorbed_droplets, reabsorbed_bubbles,
      expired_droplets, expired_bubbles, dragged_droplets, dragged_bubbles, reabsorbed_droplets_to_primary,
      reabsorbed_bubbles_to_primary;
  double current_droplet_volume, current_bubble_volume, reabsorbed_droplet_volume, reabsorbed_bubble_volume,
      expired_droplet_volume, expired_bubble_volume, reabsorbed_droplet_volume_to_primary,
      reabsorbed_bubble_volume_to_primary;
} pfo_sec_stats;
typedef struct { /* SecondarySprayEmissionConfig3D */
  int enabled, requested_particles;
  double droplet_fraction, droplet_volume, bubble_volume, particle_volume_scale;
  int interface_gate, interface_cells;
  double interface_grad_max, interface_curvature_abs_max;
  int min_interface_cells;
  double min_interface_grad_max, min_interface_curvature_abs_max;
  int impact_splash_candidates;
  double impact_region_fraction, impact_downward_speed_min, impact_foam_fraction;
} pfo_spray_cfg;
typedef struct { /* SecondarySprayEmissionStats3D */
  int enabled, finite, requested_particles, effective_requested_particles, interface_gate_enabled,
      interface_gate_passed, interface_cells, candidate_liquid_particles, impact_candidate_liquid_particles,
      foam_ready_droplets, emitted_droplets, emitted_bubbles;
  double interface_grad_max, interface_curvature_abs_max, emitted_droplet_volume, emitted_bubble_volume;
} pfo_spray_stats;
double pfo_sec_volume_sum(const pfo_sec_set* s, double scale);
/* advanceSecondaryParticles3D; reab_* NULL unless reabsorbed particles go back
 * to the primary set.  -1 when a set's capacity is exceeded. */
int pfo_sec_advance(const pfo_sec_domain* d, const pfo_sec_cfg* c, double dt, pfo_sec_set* droplets,
                    pfo_sec_set* bubbles, pfo_sec_set* reab_droplets, pfo_sec_set* reab_bubbles, pfo_sec_stats* st);
/* emitSecondarySpraySeeds3D on a primary particle set */
int pfo_spray_emit(size_t n, const double* pos, const double* vel, const unsigned char* type, const double* vol,
                   const pfo_spray_cfg* c, int frame_index, pfo_sec_set* droplets, pfo_sec_set* bubbles,
                   pfo_spray_stats* st);

pfo_mr* pfo_mr_create(int nx, int ny, int nz, double dx);
void pfo_mr_destroy(pfo_mr* m);
void pfo_mr_dims(const pfo_mr* m, int* blocks3);
int pfo_mr_set_layout(pfo_mr* m, const int* boxes, int nbox); /* coarse everywhere, then refine each box */
int pfo_mr_set_levels(pfo_mr* m, const unsigned char* refined);
int pfo_mr_get_levels(const pfo_mr* m, unsigned char* refined);
int pfo_mr_count_fine_leaves(const pfo_mr* m);
int pfo_mr_update_refinement(pfo_mr* m, const pfo_mr_dynamic* dyn, size_t n, const double* pos,
                             const unsigned char* type);
void pfo_mr_refinement_state(const pfo_mr* m, int* out8);
int pfo_mr_face_valid(const pfo_mr* m, int axis, unsigned char* out);
int pfo_mr_get_face(const pfo_mr* m, int field, float* out);
int pfo_mr_set_face(pfo_mr* m, int field, const float* in);
int pfo_mr_get_cells(const pfo_mr* m, float* marker, float* pressure);
int pfo_mr_mark_cells(pfo_mr* m, size_t n, const double* pos);
int pfo_mr_p2g(pfo_mr* m, size_t n, const double* pos, const double* vel, const unsigned char* type,
               const double* vol, const pfo_phase* pp, double Vp);
int pfo_mr_apply_gravity(pfo_mr* m, double dt, double gravity);
int pfo_mr_apply_walls(pfo_mr* m);
int pfo_mr_project(pfo_mr* m, const pfo_phase* pp, double dt, const pfo_mr_solve_cfg* cfg, pfo_mr_solve_stats* st);
int pfo_mr_g2p(const pfo_mr* m, size_t n, const double* pos, double* vel, const unsigned char* type, double aL,
               double aG);
int pfo_mr_advect(const pfo_mr* m, size_t n, double* pos, const unsigned char* type, double dt, int order,
                  pfo_clamp_stats* st);
int pfo_mr_step(pfo_mr* m, const pfo_mr_dynamic* dyn, size_t n, double* pos, double* vel,
                const unsigned char* type, const double* vol, const pfo_phase* pp, const pfo_mr_step_cfg* cfg,
                pfo_mr_solve_stats* sst, pfo_clamp_stats* cst);

#ifdef __cplusplus
}
#endif
#endif
