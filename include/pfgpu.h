/*
 * pfgpu.h -- C ABI of the B200 (sm_100a) solver-step library for the sparse
 * 3D two-phase Phase-Field-FLIP step of adaptive-pf-flip.
 *
 * One context owns one sparse MAC grid (a pool of 8^3-cell tiles behind a
 * dense tile->slot array, with 4^3-block activity kept per field exactly as
 * the reference's SparseBlockGrid3D<4> tracks it) and one particle set, both
 * resident in device memory.  Every entry point is stream-ordered on the
 * context's own CUDA stream, returns 0 on success or a negative PF_ERR_* code,
 * and is not thread-safe per context.  Entry points that return statistics
 * synchronise the stream before returning.
 *
 * Reference interfaces replaced (paths relative to the adaptive-pf-flip tree):
 *   spP2G3D_tp         src/driver/sparse_ops3d_tp.h:9   -> pf_p2g
 *   spProjectStepVC3D  src/driver/sparse_ops3d_tp.h:10  -> pf_project
 *   spG2P3D_tp         src/driver/sparse_ops3d_tp.h:12  -> pf_g2p
 *   spAdvect3D_tp      src/driver/sparse_ops3d_tp.h:13  -> pf_advect
 *   SparseSim3DTP::step (markCells, applyGravity, applyWallBoundary and the
 *     call order of src/driver/sparse_sim3d_tp.cpp:22-97, 854-884)
 *                                                       -> pf_mark_cells,
 *        pf_apply_gravity, pf_apply_wall_boundary, pf_save_velocity, pf_step
 *   MRSim3DTP::step, 2-level multires (src/driver/multires_sim3d_tp.cpp:671-733),
 *     mrP2G3D_tp (src/driver/multires_ops3d_tp.h:8)   -> pf_mr_step, pf_mr_p2g,
 *        pf_mr_set_layout, pf_mr_set_dynamic, pf_mr_update_refinement
 *   SparseMacGrid3D<4> / SparseBlockGrid3D<4> storage
 *     (src/grid/sparse_mac_grid3d.h:6-47, src/grid/sparse_block_grid3d.h:10-68)
 *                                                       -> pf_grid_set_field,
 *        pf_grid_get_field, pf_grid_clear_field, pf_active_blocks4
 *   collectCellsWithMarker (src/driver/sparse_ops3d_common.h:65-85)
 *                                                       -> pf_active_cells
 *   Particles3DTP storage (src/particles/particles3d_tp.h:4-35)
 *                                                       -> pf_upload_particles*,
 *        pf_download_particles*
 *   advanceSecondaryParticles3D, emitSecondarySpraySeeds3D
 *     (src/driver/secondary_particles3d.h:136-467) and the step's escape
 *     branching (src/driver/sparse_sim3d_tp.cpp:185-337)
 *                                                       -> pf_set_secondary,
 *        pf_secondary_advance, pf_secondary_spray, pf_get_secondary
 */
#ifndef PFGPU_H
#define PFGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFGPU_ABI_VERSION 1

#if defined(__GNUC__)
#define PFGPU_API __attribute__((visibility("default")))
#else
#define PFGPU_API
#endif

/* status codes */
#define PF_OK 0
#define PF_ERR_INVALID (-1)   /* bad argument or size */
#define PF_ERR_CUDA (-2)      /* CUDA runtime error (message via pf_last_error) */
#define PF_ERR_CAPACITY (-3)  /* more particles than the context was created for */
#define PF_ERR_NONFINITE (-4) /* NaN/Inf met in the solve */
#define PF_ERR_NO_DEVICE (-5) /* no usable sm_100 device */

/* field ids: the eight SparseMacGrid3D<4> fields */
enum pf_field { PF_U = 0, PF_V, PF_W, PF_MU, PF_MV, PF_MW, PF_P, PF_MK, PF_NFIELDS };

typedef struct pf_ctx pf_ctx;

typedef struct {
  int nx, ny, nz;        /* cells */
  double dx;             /* cell size */
  double ox, oy, oz;     /* origin */
  size_t max_particles;  /* particle capacity */
  int device;            /* CUDA device ordinal */
} pf_grid_desc;

/* PhaseParams (src/physics/phasefield.h:4-9) */
typedef struct {
  double rho_l, rho_g, alpha_phi, rho_tilde_0;
} pf_phase;

/* pressure solver modes */
#define PF_SOLVER_PLAIN 0   /* FP64 Jacobi-PCG, the reference-equivalent drop-in */
#define PF_SOLVER_MIXED 1   /* FP64 flexible CG preconditioned by FP32/BF16-storage Jacobi-PCG (FP64 dots) */
#define PF_SOLVER_LEARNED 2 /* flexible PCG, Jacobi + learned two-level coarse correction */

typedef struct {
  int mode;             /* PF_SOLVER_* */
  int max_iter;         /* reference cg_iters */
  double abs_tol;       /* reference cg_tol: stop when max|r| < tol */
  double rel_tol;       /* 0: reference rule; else tol = max(abs_tol, rel_tol*max|r0|) */
  double c_div;         /* divergenceCorrection */
  int bf16_storage;     /* mixed: 1 store the inner solve's couplings (beta) in BF16; 2 also its search
                           direction */
  int check_every;      /* host convergence poll interval in iterations (0 = default) */
  int max_refine;       /* unused (kept for the struct layout) */
  double inner_rel_tol; /* mixed / learned FP32: an inner solve stops at max|r| <= inner_rel_tol max|r_0|
                           (0 = default: 1e-3) */
  int precond;          /* learned: PF_PRECOND_* */
  double accept_min_gain; /* learned: keep the coarse term only if r.z >= (1+gain) r.D^-1 r */
  int inner_fp32;       /* learned: 0 FP64 flexible PCG; 1 FP64 flexible CG preconditioned by the learned
                           flexible PCG in FP32 */
  int inner_max_iter;   /* mixed / learned FP32: iteration cap of one inner solve (0 = default: 200) */
} pf_solve_cfg;

/* preconditioner of the LEARNED mode's flexible PCG */
#define PF_PRECOND_NETWORK 0      /* Jacobi + learned coarse correction (the default) */
#define PF_PRECOND_EXACT_COARSE 1 /* Jacobi + exact Galerkin coarse solve (training target, ablation) */
#define PF_PRECOND_JACOBI 2       /* Jacobi alone: the same solver without the network */

typedef struct {
  int iterations;        /* total inner PCG iterations */
  int refinements;       /* mixed / learned FP32: outer FP64 iterations (iterations counts the inner ones) */
  int n_cells;           /* fluid cells (unknowns incl. the pin) */
  int converged;
  int breakdown;         /* |p.Ap| < 1e-30 or non-finite */
  long long pin_cell;    /* linear index of the pinned cell or -1 */
  double res0;           /* max|r0| */
  double res_final;      /* max|r| at exit (FP64 residual) */
  double tol_effective;
  int precond_applied;   /* learned: network applications accepted */
  int precond_rejected;  /* learned: applications that fell back to Jacobi */
  double solve_ms;       /* device time of the solve */
} pf_solve_stats;

/* ParticleEscapeStats3D (src/driver/particle_escape3d.h:38-80) */
typedef struct {
  int clamped_liquid, clamped_gas;
  int x_lo, x_hi, y_lo, y_hi, z_lo, z_hi;
} pf_clamp_stats;

typedef struct {
  double dt, gravity, Vp, alpha_l, alpha_g;
  pf_phase phase;
  pf_solve_cfg solve;
  int advect_order;      /* 2 (midpoint) or 3 */
} pf_step_cfg;

typedef struct {
  pf_solve_stats solve;
  pf_clamp_stats clamp;
  int active_tiles;      /* pooled 8^3 tiles */
} pf_step_stats;

/* SurfaceTensionStats3D (src/driver/interface_diagnostics3d.h:21-36) */
typedef struct {
  int enabled, applied_cells, finite, curvature_smoothing_radius, capillary_stable;
  double strength, max_delta_speed_limit, mean_delta_speed, max_delta_speed, raw_curvature_abs_mean,
      raw_curvature_abs_max, smoothed_curvature_abs_mean, smoothed_curvature_abs_max, capillary_dt_limit;
} pf_surface_stats;

/* The step's own controls (src/driver/sparse_sim3d_tp.h:13-26): the adaptive
 * timestep (computeAdaptiveParticleTimestep3D, src/driver/timestep3d.h:16-50)
 * and the volume-correcting divergence target (updateVolumeCorrectionStats,
 * src/driver/sparse_sim3d_tp.cpp:368-379).  The reference's defaults: both
 * off, cfl 0.5, min_dt 1e-5, strength 1, target 0. */
typedef struct {
  int adaptive_timestep;
  double adaptive_cfl, adaptive_min_dt;
  int c_div_volume_correction;
  double c_div_strength, liquid_volume_target;
} pf_step_controls;
/* TimestepStats3D (src/driver/timestep3d.h:8-14) and the volume statistics */
typedef struct {
  double requested_dt, effective_dt, max_particle_speed, cfl_limit_dt;
  int limited;
  double liquid_volume_current, liquid_volume_error, c_div;
} pf_step_control_stats;

/* InterfaceDiagnostics3D (src/driver/interface_diagnostics3d.h:7-19) */
typedef struct {
  int sample_cells, interface_cells, finite, surface_tension_candidate;
  double phi_min, phi_max, phi_mean, grad_mean, grad_max, curvature_abs_mean, curvature_abs_max;
} pf_interface_stats;

/* Particle adaptivity results (src/driver/particle_adaptivity3d.h:49-72:
 * NarrowBandAirResult3D, GasParticleCoarseningResult3D,
 * LiquidParticleRefillResult3D). */
typedef struct { int removed, liquid_cells, gas_before, gas_after; } pf_band_stats;
typedef struct { int removed, cells, overfull_cells, before, after; } pf_coarsen_stats;
typedef struct { int added, cells, interface_cells, underfull_cells, budget_limited, before, after; } pf_refill_stats;

/* The adaptivity switches of SparseSim3DTP (src/driver/sparse_sim3d_tp.h:29-66),
 * applied at the start of every pf_step in the order of
 * SparseSim3DTP::applyParticleAdaptivity (src/driver/sparse_sim3d_tp.cpp:843-848).
 * The reference's defaults: all off; radius 2; targets 4; seeds 0x9e3779b9
 * (gas), 0x7f4a7c15 (liquid coarsening), 0x6a09e667 (refill); refill
 * interface radius 1, budget 0 (none). */
typedef struct {
  int narrow_band_air, narrow_band_radius;
  int gas_coarsening, gas_per_cell_target;
  unsigned gas_seed;
  int liquid_coarsening, liquid_per_cell_target;
  unsigned liquid_seed;
  int liquid_refill, refill_per_cell_target;
  unsigned refill_seed;
  int refill_interface_only, refill_interface_radius, refill_max_added;
} pf_adapt_cfg;
typedef struct {
  pf_band_stats band;
  pf_coarsen_stats gas, liquid;
  pf_refill_stats refill;
} pf_adapt_stats;

/* ---- context ---------------------------------------------------------- */
PFGPU_API int pf_create(const pf_grid_desc* desc, pf_ctx** out);
PFGPU_API int pf_destroy(pf_ctx* ctx);
PFGPU_API const char* pf_last_error(const pf_ctx* ctx);
/* Wait for the context's stream and its asynchronous uploads and downloads. */
PFGPU_API int pf_sync(pf_ctx* ctx);
/* The context's stream as an opaque handle (a cudaStream_t). */
PFGPU_API void* pf_stream(pf_ctx* ctx);

/* ---- particles (pointers may be host or device memory) ---------------- */
/* FP32: pos/vel are n x 3 interleaved xyz, type 0 liquid / 1 gas, volume. */
PFGPU_API int pf_upload_particles(pf_ctx* ctx, size_t n, const float* pos, const float* vel,
                        const uint8_t* type, const float* volume);
PFGPU_API int pf_download_particles(pf_ctx* ctx, float* pos, float* vel, uint8_t* type, float* volume);
/* The same upload without waiting: the copies (host buffers should be pinned
 * and stay unchanged until pf_sync) and the unpacking run on a second stream
 * into a second particle set, overlapping the work already queued, e.g. the
 * current step.  The next call that uses the particles (P2G, markCells, G2P,
 * advection, a step, a download, another upload) swaps the set in. */
PFGPU_API int pf_upload_particles_async(pf_ctx* ctx, size_t n, const float* pos, const float* vel,
                                        const uint8_t* type, const float* volume);
/* The same copy without waiting for it: the arrays are staged on the device
 * in stream order and copied to the host on a second stream, overlapping the
 * calls that follow (e.g. the next step's upload).  Host buffers should be
 * pinned (a pageable buffer makes the copy synchronous).  The host may read
 * them after pf_sync; pf_join_downloads makes the context stream wait for
 * them on the device (for events recorded after it). */
PFGPU_API int pf_download_particles_async(pf_ctx* ctx, float* pos, float* vel, uint8_t* type, float* volume);
PFGPU_API int pf_join_downloads(pf_ctx* ctx);
/* FP64: the reference's Particles3DTP layout (std::vector<Vec3> = n x 3 doubles). */
PFGPU_API int pf_upload_particles_f64(pf_ctx* ctx, size_t n, const double* pos, const double* vel,
                            const uint8_t* type, const double* volume);
PFGPU_API int pf_download_particles_f64(pf_ctx* ctx, double* pos, double* vel, uint8_t* type,
                              double* volume);
PFGPU_API size_t pf_num_particles(const pf_ctx* ctx);

/* ---- grid access (dense host/device arrays over the field's own lattice:
 *      u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1), mu/mv/mw alike,
 *      p and mk (nx,ny,nz); index i + X*(j + Y*k); act4 holds one byte per
 *      4^3 block, bid = bx + nbx*(by + nby*bz), nbx = ceil(X/4)).  The
 *      marker field mk is exchanged as float 0 air / 1 fluid / 2 solid. --- */
PFGPU_API int pf_grid_set_field(pf_ctx* ctx, int field, const float* dense, const uint8_t* act4);
PFGPU_API int pf_grid_get_field(pf_ctx* ctx, int field, float* dense, uint8_t* act4);
PFGPU_API int pf_grid_clear_field(pf_ctx* ctx, int field);
PFGPU_API int pf_grid_clear_all(pf_ctx* ctx);
/* Copy every field (values and activity) of src into dst (same lattice). */
PFGPU_API int pf_grid_copy(pf_ctx* dst, const pf_ctx* src);
/* Sorted 4^3 block ids active in a field; ids may be NULL to query *n. */
PFGPU_API int pf_active_blocks4(pf_ctx* ctx, int field, int32_t* ids, size_t* n);
/* Cells with marker 1 as ascending linear indices i + nx*(j + ny*k). */
PFGPU_API int pf_active_cells(pf_ctx* ctx, int32_t* cells, size_t* n);
PFGPU_API int pf_active_tiles(const pf_ctx* ctx);

/* ---- solver step pieces ------------------------------------------------ */
PFGPU_API int pf_mark_cells(pf_ctx* ctx);
PFGPU_API int pf_p2g(pf_ctx* ctx, const pf_phase* phase, double Vp);
PFGPU_API int pf_save_velocity(pf_ctx* ctx);
PFGPU_API int pf_apply_gravity(pf_ctx* ctx, double dt, double gravity);
PFGPU_API int pf_apply_wall_boundary(pf_ctx* ctx);
PFGPU_API int pf_project(pf_ctx* ctx, const pf_phase* phase, double dt, const pf_solve_cfg* cfg,
               pf_solve_stats* stats);
/* saved: context holding the pre-force grid, or NULL for the copy taken by
 * pf_save_velocity on ctx itself. */
PFGPU_API int pf_g2p(pf_ctx* ctx, const pf_ctx* saved, double alpha_l, double alpha_g);
/* escape (optional, host or device, capacity n x 8 doubles): per clamped
 * particle {type, x, y, z, vx, vy, vz, volume} in particle order. */
PFGPU_API int pf_advect(pf_ctx* ctx, double dt, int order, pf_clamp_stats* stats, double* escape,
              size_t* n_escape);
/* One full step in the reference's step() order, device-resident. */
PFGPU_API int pf_step(pf_ctx* ctx, const pf_step_cfg* cfg, pf_step_stats* stats);

/* diagnoseSparseInterface3D (src/driver/interface_diagnostics3d.cpp:363-379)
 * on the context's grid: phase field, gradient and curvature statistics over
 * the fluid cells.  Counts, minima and maxima equal the reference's; the
 * means agree to rounding (summed in another order).  pf_step computes them
 * after P2G, as SparseSim3DTP::step() does; pf_get_interface_stats returns
 * the last step's. */
PFGPU_API int pf_interface_diagnostics(pf_ctx* ctx, const pf_phase* phase, pf_interface_stats* stats);
/* Controls pf_step applies after the adaptivity (NULL: both off).  Every step
 * computes the statistics (max particle speed, liquid volume), as the
 * reference's does; with the adaptive timestep on, the step runs with
 * effective_dt instead of cfg->dt, and with the volume correction on, the
 * projection uses c_div instead of cfg->solve.c_div. */
PFGPU_API int pf_set_step_controls(pf_ctx* ctx, const pf_step_controls* controls);
/* applySparseSurfaceTension3D (src/driver/interface_diagnostics3d.cpp:405-447)
 * on the context's grid: every fluid interface cell adds half its capillary
 * velocity change -strength*curvature*grad(phi)*dt (limited to max_delta_speed
 * when that is > 0; curvature averaged over a radius of 0..3 cells) to its
 * six faces that hold mass.  Face velocities equal the reference's exactly;
 * the statistics' means agree to rounding. */
PFGPU_API int pf_surface_tension(pf_ctx* ctx, const pf_phase* phase, double dt, double strength,
                                 double max_delta_speed, int smoothing_radius, pf_surface_stats* stats);
/* pf_step applies it between gravity and the walls when strength > 0
 * (the reference's surface_tension switch; 0 = off, the default). */
PFGPU_API int pf_set_surface_tension(pf_ctx* ctx, double strength, double max_delta_speed, int smoothing_radius);
PFGPU_API int pf_get_surface_stats(const pf_ctx* ctx, pf_surface_stats* out);
PFGPU_API int pf_get_step_control_stats(const pf_ctx* ctx, pf_step_control_stats* out);
PFGPU_API int pf_get_interface_stats(const pf_ctx* ctx, pf_interface_stats* out);

/* ---- particle adaptivity (src/driver/particle_adaptivity3d.h) ----------
 * Each call rewrites the context's particle set on the device; erasures keep
 * the survivors' order, refill appends after the last particle.  Particle
 * order, positions, types, velocities and volumes equal the reference's
 * (FP64 results rounded to the FP32 storage). */
/* pa3d::applyNarrowBandAir (:111-166): gas particles farther than `radius`
 * cells (Chebyshev) from every cell holding liquid are erased. */
PFGPU_API int pf_narrow_band_air(pf_ctx* ctx, int radius, pf_band_stats* stats);
/* pa3d::applyTypedParticleCoarsening (:168-248): per cell, the
 * per_cell_target particles of `type` with the lowest hash score stay and
 * share the cell's volume (type 1 is applyGasParticleCoarsening). */
PFGPU_API int pf_coarsen_particles(pf_ctx* ctx, int type, int per_cell_target, unsigned seed,
                                   pf_coarsen_stats* stats);
/* pa3d::applyLiquidParticleRefill (:250-374): underfull liquid cells get new
 * particles at sub-cell centres.  PF_ERR_CAPACITY, with nothing changed, when
 * the result would exceed max_particles; stats->added then holds the number
 * of particles the call would have added. */
PFGPU_API int pf_refill_liquid(pf_ctx* ctx, int per_cell_target, unsigned seed, int interface_only,
                               int interface_radius, int max_added, pf_refill_stats* stats);
/* Adaptivity run by pf_step (NULL: none, the default); the results of the
 * last step's adaptivity. */
PFGPU_API int pf_set_adaptivity(pf_ctx* ctx, const pf_adapt_cfg* cfg);
PFGPU_API int pf_get_adaptivity_stats(const pf_ctx* ctx, pf_adapt_stats* out);

/* ---- secondary particles (src/driver/secondary_particles3d.h) -----------
 * Two FP64 sets beside the primary particles: droplets (set 0) and bubbles
 * (set 1), each particle with an age in steps.  pf_step runs, at the places
 * SparseSim3DTP::step does (src/driver/sparse_sim3d_tp.cpp:854-884): the
 * lifecycle after the step controls, the escape branching (every particle the
 * advection clamps to the domain is copied into the set of its type, age 0)
 * and the spray seeds after the advection.  Sets and statistics equal the
 * reference's arithmetic on the same inputs; spray candidates with equal
 * scores are ranked in particle order. */
/* SparseSim3DTP's settings (src/driver/sparse_sim3d_tp.h:82-137);
 * pf_secondary_default_cfg gives the reference's defaults (all switches off,
 * lifetimes 48 steps, damping 0.98, margin 1 cell, gravity scale 1, buoyancy
 * scale 0.25, spray droplet fraction 0.9, volumes 0.55 / 0.45, gate minima
 * 1 cell and 1e-5, impact region 0.55, impact speed 1, foam fraction 0.3). */
typedef struct {
  int escaped_particle_branching;
  int lifecycle;                                       /* secondary_particle_lifecycle */
  int droplet_lifetime_steps, bubble_lifetime_steps;   /* < 0: no expiry */
  double velocity_damping, reabsorb_margin_cells;
  double droplet_gravity_scale, bubble_buoyancy_scale;
  double droplet_drag, bubble_drag;                    /* per second; 0: none */
  int reabsorb_to_primary;                             /* reabsorbed particles rejoin the primary set */
  int spray_emission, spray_particles_per_step;
  double spray_droplet_fraction, spray_droplet_volume, spray_bubble_volume;
  int spray_interface_gate, spray_min_interface_cells;
  double spray_min_interface_grad_max, spray_min_interface_curvature_abs_max;
  int spray_impact_candidates;
  double spray_impact_region_fraction, spray_impact_downward_speed_min, spray_impact_foam_fraction;
} pf_secondary_cfg;
/* The last step's SecondaryParticleLifecycleStats3D (:33-54; volumes scaled
 * by Vp; lifecycle_*_volume are the sets' volumes after the lifecycle),
 * SecondarySprayEmissionStats3D (:76-93), the particles and volume added to
 * each set by the escapes and the spray together, the spray step index after
 * the step, and the sets' volumes at the end of the step. */
typedef struct {
  int lifecycle_enabled, lifecycle_finite;
  int advected_droplets, advected_bubbles, reabsorbed_droplets, reabsorbed_bubbles;
  int expired_droplets, expired_bubbles, dragged_droplets, dragged_bubbles;
  int reabsorbed_droplets_to_primary, reabsorbed_bubbles_to_primary;
  double lifecycle_droplet_volume, lifecycle_bubble_volume;
  double reabsorbed_droplet_volume, reabsorbed_bubble_volume, expired_droplet_volume, expired_bubble_volume;
  double reabsorbed_droplet_volume_to_primary, reabsorbed_bubble_volume_to_primary;
  int spray_enabled, spray_finite, spray_requested_particles, spray_effective_requested_particles;
  int spray_interface_gate_enabled, spray_interface_gate_passed, spray_interface_cells;
  int spray_candidate_liquid_particles, spray_impact_candidate_liquid_particles, spray_foam_ready_droplets;
  int spray_emitted_droplets, spray_emitted_bubbles;
  double spray_interface_grad_max, spray_interface_curvature_abs_max;
  double spray_emitted_droplet_volume, spray_emitted_bubble_volume;
  int escaped_droplets_added, escaped_bubbles_added;
  double escaped_droplet_volume_added, escaped_bubble_volume_added;
  double escape_droplet_volume, escape_bubble_volume; /* the escaped particles' share of the two above */
  int spray_step_index;
  double droplet_volume_current, bubble_volume_current;
} pf_secondary_stats;
PFGPU_API int pf_secondary_default_cfg(pf_secondary_cfg* out);
/* Settings pf_step uses (NULL: all switches off; the sets are kept). */
PFGPU_API int pf_set_secondary(pf_ctx* ctx, const pf_secondary_cfg* cfg);
PFGPU_API int pf_get_secondary_stats(const pf_ctx* ctx, pf_secondary_stats* out);
/* Set `which` (0 droplets, 1 bubbles): its size, and its particles as host
 * arrays (pos/vel n x 3 interleaved; any pointer may be NULL). */
PFGPU_API int pf_secondary_count(const pf_ctx* ctx, int which, size_t* n);
PFGPU_API int pf_get_secondary(pf_ctx* ctx, int which, double* pos, double* vel, double* vol, int* age);
PFGPU_API int pf_set_secondary_particles(pf_ctx* ctx, int which, size_t n, const double* pos, const double* vel,
                                         const double* vol, const int* age);
/* The step's pieces on their own: advanceSecondaryLifecycle (reabsorbed
 * particles appended to the primary set when reabsorb_to_primary is on;
 * PF_ERR_CAPACITY when they would not fit) and emitSecondarySpray on the
 * current particles with the given interface statistics. */
PFGPU_API int pf_secondary_advance(pf_ctx* ctx, double dt, double gravity, double Vp);
PFGPU_API int pf_secondary_spray(pf_ctx* ctx, double Vp, const pf_interface_stats* iface);

/* ---- per-stage device timing (CUDA events on the context stream) -------
 * Off by default.  When on, every solver-step entry point brackets its
 * stages with events; pf_get_timing synchronises and returns the summed
 * device milliseconds and launch counts per stage since the last reset.
 * pf_mr_step reports its refinement as ADAPT, markCells as MARK, P2G as
 * SPLAT, the saved copy, gravity and walls as BOUNDARY, the projection as
 * PROJECT (its PCG iterations as PCG) and G2P with advection as G2P. */
enum pf_stage {
  PF_STAGE_BIN = 0,      /* particle binning + exact 4^3 activation + pool growth */
  PF_STAGE_SORT,         /* tile offsets scan + particle permutation */
  PF_STAGE_SPLAT,        /* P2G splat kernel */
  PF_STAGE_NORMALIZE,    /* momentum / mass (+ saved copy, gravity) */
  PF_STAGE_MARK,         /* markCells */
  PF_STAGE_BOUNDARY,     /* gravity, walls, saved copy */
  PF_STAGE_PROJECT,      /* whole projection */
  PF_STAGE_PCG,          /* iterative solve only */
  PF_STAGE_G2P,          /* G2P and/or advection */
  PF_STAGE_PRECOND_SETUP, /* LEARNED solves: coarse operator, gate network, neighbour table */
  PF_STAGE_ADAPT,        /* particle adaptivity: narrow band, coarsening, refill */
  PF_STAGE_DIAG,         /* interface diagnostics */
  PF_NSTAGES
};
typedef struct {
  double ms[PF_NSTAGES];
  long long count[PF_NSTAGES];
} pf_timing;
PFGPU_API int pf_set_timing(pf_ctx* ctx, int enable);
/* Number of kernels this context has launched since it was created. */
PFGPU_API long long pf_launch_count(const pf_ctx* ctx);
PFGPU_API int pf_get_timing(pf_ctx* ctx, pf_timing* out, int reset);

/* ---- allocation-free projection ----------------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory: hosts that reserve the whole device budget themselves and hand out
 * buffers from their own allocator (and plug-ins running inside such hosts),
 * or fixed-rate loops that must never wait on the driver's allocator.  It
 * does what pf_project does in PLAIN mode (the same set-up, Jacobi-PCG
 * recurrences and velocity update; its SpMV looks cross-tile neighbours up
 * through the tile map instead of a per-solve table; results agree to
 * rounding of the inner products) on dense device arrays the caller owns:
 * mk (nx,ny,nz) markers 0/1/2, face raw masses mu/mv/mw and face velocities
 * u/v/w on the field lattices of pf_grid_set_field (index i + X*(j + Y*k)),
 * all treated as fully active.  u, v, w are updated in place and p
 * (nx,ny,nz) receives the pressure (0 outside fluid cells).
 *
 * All working memory sits in one fixed __device__ array inside the library
 * (about 6.3 MB on every GPU that loads it, held until the process exits);
 * the call makes no cudaMalloc/cudaFree or other allocating call.  With CUDA's
 * lazy module loading (the default) the first call in a context loads the
 * library's module, which is when that array is allocated; later calls
 * allocate nothing.  Limit:
 * ceil((nx+1)/8)*ceil((ny+1)/8)*ceil((nz+1)/8) <= PF_NOALLOC_MAX_TILES, e.g.
 * grids up to 39^3 cells; larger grids return PF_ERR_INVALID without running.
 * Every call looks the array's device address up in the current context
 * (cudaGetSymbolAddress), so it stays valid after a device reset or when the
 * caller makes a context of its own current; make the first call in a context
 * before any stream capture.  Every call uses the same array and leaves its
 * contents behind (each call re-initialises what it reads), so calls whose
 * work overlaps on the GPU -- on different streams, or from different host
 * threads -- race and must be serialised by the caller.  `stream` is a
 * cudaStream_t (NULL: the default stream); the call returns after its work on
 * that stream has finished. */
#define PF_NOALLOC_MAX_TILES 125
PFGPU_API int pf_project_noalloc(int nx, int ny, int nz, double dx, const float* mk, const float* mu,
                                 const float* mv, const float* mw, float* u, float* v, float* w, float* p,
                                 const pf_phase* phase, double dt, int max_iter, double abs_tol,
                                 double rel_tol, double c_div, pf_solve_stats* stats, void* stream);

/* ---- synthetic scenes of the benchmark configurations -------------------
 * Seeds the context's particle set on the device (replacing it) with 8
 * jittered particles per seeded cell, in the layouts of the reference's
 * SparseSim3DTP::initRayleighTaylor / initBubbleTank
 * (src/driver/sparse_sim3d_tp.cpp:739-776) at the benchmark densities:
 *   PF_SCENE_RAYLEIGH_TAYLOR: every interior cell; type 0 (heavy) above
 *     y = 0.5 + 0.05 cos(2 pi x) cos(2 pi z), type 1 below; zero velocity;
 *   PF_SCENE_BUBBLE_TANK: interior cells whose centre lies below y = 0.7;
 *     type 1 inside the sphere of radius 0.15 at (0.5, 0.3, 0.5), type 0
 *     elsewhere; velocities N(0, 0.1^2) per component;
 *   PF_SCENE_DAM_BREAK: a water column (interior cells whose centre has
 *     x < 0.4 and y < 0.6), then a pool beside it (y < 0.15); type 0, zero
 *     velocity, the air empty (the multires configuration's scene).
 * Volumes are 1.  Positions are bit-identical to the host generator of the
 * same seed (adaptive-pf-flip_b200/scenes.py).  *n_out receives the count;
 * PF_ERR_CAPACITY if it exceeds max_particles. */
#define PF_SCENE_RAYLEIGH_TAYLOR 0
#define PF_SCENE_BUBBLE_TANK 1
#define PF_SCENE_DAM_BREAK 2
PFGPU_API int pf_seed_scene(pf_ctx* ctx, int scene, unsigned long long seed, size_t* n_out);

/* calibrateRhoTilde0 (src/transfer/transfer3d_tp.cpp:29-36), on the device. */
PFGPU_API int pf_calibrate_rho_tilde0(pf_ctx* ctx, const pf_phase* phase, double Vp, double* out);

/* ---- 2-level multires step (MRSim3DTP) ------------------------------------
 * The reference's multires solver step (src/driver/multires_sim3d_tp.cpp:
 * 671-733) on the context's particle set, with its own grid on the same
 * nx, ny, nz and dx (the origin must be 0).  The layout holds level-1 blocks
 * of 8^3 fine cells (x fastest), each coarse (4^3 cells of 2 dx) or refined
 * into fine cells (src/grid/multires_layout3d.h:25-162).
 *
 * pf_mr_set_layout: setCoarseEverywhere(1), then refineFineCellBox of each
 *   box clamped to the domain (the static layouts of
 *   src/driver/multires_sim3d_tp.cpp:158-180).  Before any layout is set every
 *   block is coarse.
 * pf_mr_set_levels / pf_mr_get_levels: one byte per level-1 block, 1 where it
 *   is refined; blocks3 receives the block counts ceil(n / 8).
 * pf_mr_set_dynamic: updateDynamicRefinement's settings (enabled, particle and
 *   gas padding, hysteresis, fine-leaf budget; MRSim3DTP's defaults are
 *   {1, 1, 2, 1, 0}).  pf_mr_update_refinement runs it alone (state8: the
 *   retained box's valid flag and x0 y0 z0 x1 y1 z1, the budget flag);
 *   pf_mr_reset_refinement forgets the retained box.
 * pf_mr_step: updateDynamicRefinement (when enabled), markCells, mrP2G3D_tp,
 *   the saved copy, gravity, walls, projectMR3D with the Jacobi PCG (adaptive
 *   restart, optional flexible beta; the coarse-correction and coarse
 *   preconditioner options are not available), mrG2P3D_tp, mrAdvect3D_tp.
 * pf_mr_p2g: mrP2G3D_tp (src/driver/multires_ops3d_tp.cpp:209-274) alone.
 * pf_mr_get_face: a face field on the dense fine face lattice (0..5 = u v w mu
 *   mv mw, 6..8 = the last step's saved u v w); patches off the leaf-cell
 *   boundaries read 0.  pf_mr_get_cells: marker (0 empty, 1 fluid, 2 solid)
 *   and pressure per fine cell, the value of the leaf cell holding it. */
typedef struct {
  int x0, y0, z0, x1, y1, z1; /* fine cells [x0, x1) x [y0, y1) x [z0, z1) */
} pf_mr_box;
typedef struct {
  int enabled, particle_padding, gas_padding, hysteresis_cells, max_fine_leaves;
} pf_mr_dynamic;
typedef struct {
  double dt, gravity, Vp, alpha_l, alpha_g;
  pf_phase phase;
  int advect_order;     /* 2 or 3 */
  int cg_iters;         /* max_iterations */
  double cg_tol;        /* absolute_tolerance */
  double cg_rel_tol;    /* relative_tolerance */
  int jacobi, flexible_beta, adaptive_restart;
  double restart_growth;
  double c_div;         /* divergence_correction */
} pf_mr_step_cfg;
typedef struct {
  /* MRPressureSolveStats3D (src/pressure/multires_pressure3d.h:60-133) */
  int active_cells, pinned_cell, iterations, restarts, beta_resets, converged, breakdown;
  double initial_residual, final_residual, effective_tolerance;
  int fine_leaves;     /* level-0 blocks of the step's layout */
  pf_clamp_stats clamp;
  double solve_ms;     /* device time of assembly and PCG */
} pf_mr_step_stats;
PFGPU_API int pf_mr_set_layout(pf_ctx* ctx, const pf_mr_box* boxes, int n);
PFGPU_API int pf_mr_set_levels(pf_ctx* ctx, const uint8_t* refined);
PFGPU_API int pf_mr_get_levels(pf_ctx* ctx, uint8_t* refined, int* blocks3);
PFGPU_API int pf_mr_set_dynamic(pf_ctx* ctx, const pf_mr_dynamic* dyn);
PFGPU_API int pf_mr_reset_refinement(pf_ctx* ctx);
PFGPU_API int pf_mr_update_refinement(pf_ctx* ctx, int* state8);
PFGPU_API int pf_mr_step(pf_ctx* ctx, const pf_mr_step_cfg* cfg, pf_mr_step_stats* stats);
PFGPU_API int pf_mr_p2g(pf_ctx* ctx, const pf_phase* phase, double Vp);
PFGPU_API int pf_mr_get_face(pf_ctx* ctx, int field, float* dense);
PFGPU_API int pf_mr_get_cells(pf_ctx* ctx, uint8_t* marker, float* pressure);

/* ---- learned coarse solve (PF_SOLVER_LEARNED with PF_PRECOND_NETWORK) ----
 * New in this library (the reference's sparse path has no learned solver; its
 * flexible-PCG / guarded-preconditioner pattern is
 * src/pressure/multires_pressure3d.cpp:1301-1447).  The network maps the
 * tile-lattice coarse residual and operator to the coarse correction; its
 * parameters are one flat FP32 vector of pf_learned_num_params() floats
 * (per layer: weights [27][C_in][C_out], then biases [C_out]). */
PFGPU_API size_t pf_learned_num_params(void);
/* Fresh He-normal weights from a seed; resets the optimiser. */
PFGPU_API int pf_learned_init(pf_ctx* ctx, unsigned long long seed);
/* Load / read the parameter vector (n must equal pf_learned_num_params()). */
PFGPU_API int pf_learned_load(pf_ctx* ctx, const float* params, size_t n);
PFGPU_API int pf_learned_params(pf_ctx* ctx, float* out, size_t n);
/* Training data: while enabled, every EXACT_COARSE solve stores its coarse
 * operator and up to max_per_system (r_c, A_c^-1 r_c) pairs, one every
 * `stride` coarse solves, into a device pool of capacity_floats floats. */
PFGPU_API int pf_learned_harvest(pf_ctx* ctx, int enable, int stride, int max_per_system, size_t capacity_floats);
PFGPU_API int pf_learned_dataset(pf_ctx* ctx, int* systems, int* pairs);
PFGPU_API int pf_learned_clear_dataset(pf_ctx* ctx);
/* Append src's training set to dst's (same device): one optimiser can then
 * train on pairs harvested on grids of several sizes. */
PFGPU_API int pf_learned_merge_dataset(pf_ctx* dst, pf_ctx* src);
/* `steps` Adam steps on batches of `batch` pairs of one system each; losses
 * (optional, [steps]) receives each step's mean energy-norm error. */
PFGPU_API int pf_learned_train(pf_ctx* ctx, int steps, int batch, double lr, unsigned long long seed,
                               double* losses);
/* The network on a caller-given coarse system: cop [X*Y*Z][17], rc and
 * target [B][X*Y*Z][2] (target may be NULL), e_out [B][X*Y*Z][2]; with a
 * target also the mean loss and the parameter gradient (grad_out may be NULL). */
PFGPU_API int pf_learned_eval(pf_ctx* ctx, int X, int Y, int Z, const float* cop, const float* rc,
                              const float* target, int B, float* e_out, double* loss_out, float* grad_out);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) with a caller-given gradient. */
PFGPU_API int pf_learned_adam(pf_ctx* ctx, const float* grad, size_t n, double lr);

/* ---- render-cache export (src/driver/render_cache3d.h) ---- */

/* RenderCacheCamera3D (src/driver/render_cache3d.h:19-27) */
typedef struct pf_render_camera {
  double position[3], target[3], up[3];
  double fov_degrees, near_clip, far_clip, focal_length_mm;
} pf_render_camera;

/* defaultRenderCacheCamera3D (src/driver/render_cache3d.h:47-61). */
PFGPU_API int pf_default_render_camera(int nx, int ny, int nz, double dx, pf_render_camera* cam);

/* writeSparseRenderCache3D (src/driver/render_cache3d.h:551-600): the JSONL
 * frame (header, camera, water_volume, secondary_channels,
 * cinematic_metadata, phase_field cells, particles) of the context's current
 * grid and particles.  The phase cells are selected and compacted on the
 * device; the text uses the reference's number format (17 significant
 * digits).  dt is the step's effective dt, Vp the particle volume scale, cam
 * NULL for the default camera.  Cells are listed as the reference lists
 * them: marker blocks in the order markCells first activated them, cells in
 * each block in lattice order.  No secondary particles exist here, so their
 * sections are empty.  PF_ERR_INVALID for an empty path, a file that cannot
 * be written or the reference's invalid metadata. */
PFGPU_API int pf_write_render_cache(pf_ctx* ctx, const char* path, int frame, double time, double dt, const pf_phase* ph,
                          double Vp, const pf_render_camera* cam, long long* bytes_written);

/* writeRenderCacheManifest3D (src/driver/render_cache3d.h:711-755): the JSON
 * manifest of a sequence of render-cache frames, text identical to the
 * reference's (17 significant digits, its string escaping).  Host only: no
 * context or device is needed.  PF_ERR_INVALID for an empty path or sim_kind,
 * non-positive dims or dx, a non-finite dx, a frame with a negative frame,
 * step or byte count, an empty path or a non-finite time (the reference's
 * checks), or a file that cannot be written. */
typedef struct {
  int frame, step;
  double time;
  const char* path;
  long long bytes;
} pf_render_manifest_frame;
PFGPU_API int pf_write_render_manifest(const char* path, const char* sim_kind, int nx, int ny, int nz, double dx,
                                       const pf_render_manifest_frame* frames, int n_frames);

#ifdef __cplusplus
}
#endif
#endif /* PFGPU_H */
