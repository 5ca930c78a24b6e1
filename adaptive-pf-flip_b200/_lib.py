"""ctypes binding of libpfgpu.so (the C ABI declared in include/pfgpu.h).

The library is the only compute path: if it is missing, or no sm_100 GPU is
usable, calls raise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libpfgpu.so")

PF_OK = 0
PF_ERR_INVALID = -1
PF_ERR_CUDA = -2
PF_ERR_CAPACITY = -3
PF_ERR_NONFINITE = -4
PF_ERR_NO_DEVICE = -5
ERR_NAMES = {PF_ERR_INVALID: "PF_ERR_INVALID", PF_ERR_CUDA: "PF_ERR_CUDA", PF_ERR_CAPACITY: "PF_ERR_CAPACITY",
             PF_ERR_NONFINITE: "PF_ERR_NONFINITE", PF_ERR_NO_DEVICE: "PF_ERR_NO_DEVICE"}

PF_U, PF_V, PF_W, PF_MU, PF_MV, PF_MW, PF_P, PF_MK = range(8)
PF_SOLVER_PLAIN, PF_SOLVER_MIXED, PF_SOLVER_LEARNED = 0, 1, 2
PF_PRECOND_NETWORK, PF_PRECOND_EXACT_COARSE, PF_PRECOND_JACOBI = 0, 1, 2
PF_SCENE_RAYLEIGH_TAYLOR, PF_SCENE_BUBBLE_TANK, PF_SCENE_DAM_BREAK = 0, 1, 2

# every entry point include/pfgpu.h declares
EXPORTS = (
    "pf_create", "pf_destroy", "pf_last_error", "pf_sync", "pf_stream",
    "pf_upload_particles", "pf_download_particles", "pf_upload_particles_f64", "pf_download_particles_f64",
    "pf_download_particles_async", "pf_join_downloads", "pf_upload_particles_async",
    "pf_num_particles", "pf_grid_set_field", "pf_grid_get_field", "pf_grid_clear_field", "pf_grid_clear_all",
    "pf_grid_copy", "pf_active_blocks4", "pf_active_cells", "pf_active_tiles", "pf_mark_cells", "pf_p2g",
    "pf_save_velocity", "pf_apply_gravity", "pf_apply_wall_boundary", "pf_project", "pf_g2p", "pf_advect",
    "pf_step", "pf_calibrate_rho_tilde0", "pf_set_timing", "pf_get_timing", "pf_launch_count",
    "pf_project_noalloc", "pf_learned_num_params", "pf_learned_init", "pf_learned_load", "pf_learned_params",
    "pf_learned_harvest", "pf_learned_dataset", "pf_learned_clear_dataset", "pf_learned_merge_dataset",
    "pf_learned_train",
    "pf_learned_eval", "pf_learned_adam",
    "pf_narrow_band_air", "pf_coarsen_particles", "pf_refill_liquid", "pf_set_adaptivity", "pf_get_adaptivity_stats",
    "pf_interface_diagnostics", "pf_get_interface_stats", "pf_set_step_controls", "pf_get_step_control_stats",
    "pf_surface_tension", "pf_set_surface_tension", "pf_get_surface_stats",
    "pf_default_render_camera", "pf_write_render_cache", "pf_seed_scene",
    "pf_mr_set_layout", "pf_mr_set_levels", "pf_mr_get_levels", "pf_mr_set_dynamic", "pf_mr_reset_refinement",
    "pf_mr_update_refinement", "pf_mr_step", "pf_mr_p2g", "pf_mr_get_face", "pf_mr_get_cells",
    "pf_write_render_manifest",
    "pf_secondary_default_cfg", "pf_set_secondary", "pf_get_secondary_stats", "pf_secondary_count",
    "pf_get_secondary", "pf_set_secondary_particles", "pf_secondary_advance", "pf_secondary_spray",
)

STAGES = ("bin", "sort", "splat", "normalize", "mark", "boundary", "project", "pcg", "g2p", "precond_setup",
          "adapt", "diag")


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("ox", C.c_double),
                ("oy", C.c_double), ("oz", C.c_double), ("max_particles", C.c_size_t), ("device", C.c_int)]


class Phase(C.Structure):
    _fields_ = [("rho_l", C.c_double), ("rho_g", C.c_double), ("alpha_phi", C.c_double),
                ("rho_tilde_0", C.c_double)]


class SolveCfg(C.Structure):
    _fields_ = [("mode", C.c_int), ("max_iter", C.c_int), ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("c_div", C.c_double), ("bf16_storage", C.c_int), ("check_every", C.c_int),
                ("max_refine", C.c_int), ("inner_rel_tol", C.c_double), ("precond", C.c_int),
                ("accept_min_gain", C.c_double), ("inner_fp32", C.c_int), ("inner_max_iter", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("n_cells", C.c_int), ("converged", C.c_int),
                ("breakdown", C.c_int), ("pin_cell", C.c_longlong), ("res0", C.c_double),
                ("res_final", C.c_double), ("tol_effective", C.c_double), ("precond_applied", C.c_int),
                ("precond_rejected", C.c_int), ("solve_ms", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class ClampStats(C.Structure):
    _fields_ = [("clamped_liquid", C.c_int), ("clamped_gas", C.c_int), ("x_lo", C.c_int), ("x_hi", C.c_int),
                ("y_lo", C.c_int), ("y_hi", C.c_int), ("z_lo", C.c_int), ("z_hi", C.c_int)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class StepCfg(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double), ("Vp", C.c_double), ("alpha_l", C.c_double),
                ("alpha_g", C.c_double), ("phase", Phase), ("solve", SolveCfg), ("advect_order", C.c_int)]


class RenderManifestFrame(C.Structure):
    _fields_ = [("frame", C.c_int), ("step", C.c_int), ("time", C.c_double), ("path", C.c_char_p),
                ("bytes", C.c_longlong)]


class MRBox(C.Structure):
    _fields_ = [("x0", C.c_int), ("y0", C.c_int), ("z0", C.c_int), ("x1", C.c_int), ("y1", C.c_int), ("z1", C.c_int)]


class MRDynamic(C.Structure):
    _fields_ = [("enabled", C.c_int), ("particle_padding", C.c_int), ("gas_padding", C.c_int),
                ("hysteresis_cells", C.c_int), ("max_fine_leaves", C.c_int)]


class MRStepCfg(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double), ("Vp", C.c_double), ("alpha_l", C.c_double),
                ("alpha_g", C.c_double), ("phase", Phase), ("advect_order", C.c_int), ("cg_iters", C.c_int),
                ("cg_tol", C.c_double), ("cg_rel_tol", C.c_double), ("jacobi", C.c_int), ("flexible_beta", C.c_int),
                ("adaptive_restart", C.c_int), ("restart_growth", C.c_double), ("c_div", C.c_double)]


class MRStepStats(C.Structure):
    _fields_ = [("active_cells", C.c_int), ("pinned_cell", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("beta_resets", C.c_int), ("converged", C.c_int), ("breakdown", C.c_int),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("effective_tolerance", C.c_double), ("fine_leaves", C.c_int), ("clamp", ClampStats),
                ("solve_ms", C.c_double)]


class StepStats(C.Structure):
    _fields_ = [("solve", SolveStats), ("clamp", ClampStats), ("active_tiles", C.c_int)]


class _Stats(C.Structure):
    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class BandStats(_Stats):
    """pf_band_stats: NarrowBandAirResult3D (src/driver/particle_adaptivity3d.h:49-54)"""
    _fields_ = [("removed", C.c_int), ("liquid_cells", C.c_int), ("gas_before", C.c_int), ("gas_after", C.c_int)]


class CoarsenStats(_Stats):
    """pf_coarsen_stats: GasParticleCoarseningResult3D (src/driver/particle_adaptivity3d.h:56-62)"""
    _fields_ = [("removed", C.c_int), ("cells", C.c_int), ("overfull_cells", C.c_int), ("before", C.c_int),
                ("after", C.c_int)]


class RefillStats(_Stats):
    """pf_refill_stats: LiquidParticleRefillResult3D (src/driver/particle_adaptivity3d.h:64-72)"""
    _fields_ = [("added", C.c_int), ("cells", C.c_int), ("interface_cells", C.c_int), ("underfull_cells", C.c_int),
                ("budget_limited", C.c_int), ("before", C.c_int), ("after", C.c_int)]


class AdaptCfg(C.Structure):
    """pf_adapt_cfg: SparseSim3DTP's adaptivity switches (src/driver/sparse_sim3d_tp.h:29-66), with its defaults."""
    _fields_ = [("narrow_band_air", C.c_int), ("narrow_band_radius", C.c_int),
                ("gas_coarsening", C.c_int), ("gas_per_cell_target", C.c_int), ("gas_seed", C.c_uint),
                ("liquid_coarsening", C.c_int), ("liquid_per_cell_target", C.c_int), ("liquid_seed", C.c_uint),
                ("liquid_refill", C.c_int), ("refill_per_cell_target", C.c_int), ("refill_seed", C.c_uint),
                ("refill_interface_only", C.c_int), ("refill_interface_radius", C.c_int),
                ("refill_max_added", C.c_int)]

    def __init__(self, **kw):
        d = dict(narrow_band_radius=2, gas_per_cell_target=4, gas_seed=0x9e3779b9, liquid_per_cell_target=4,
                 liquid_seed=0x7f4a7c15, refill_per_cell_target=4, refill_seed=0x6a09e667,
                 refill_interface_radius=1)
        d.update(kw)
        super().__init__(**d)


class InterfaceStats(_Stats):
    """pf_interface_stats: InterfaceDiagnostics3D (src/driver/interface_diagnostics3d.h:7-19)"""
    _fields_ = [("sample_cells", C.c_int), ("interface_cells", C.c_int), ("finite", C.c_int),
                ("surface_tension_candidate", C.c_int), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("phi_mean", C.c_double), ("grad_mean", C.c_double), ("grad_max", C.c_double),
                ("curvature_abs_mean", C.c_double), ("curvature_abs_max", C.c_double)]


class SurfaceStats(_Stats):
    """pf_surface_stats: SurfaceTensionStats3D (src/driver/interface_diagnostics3d.h:21-36)"""
    _fields_ = [("enabled", C.c_int), ("applied_cells", C.c_int), ("finite", C.c_int),
                ("curvature_smoothing_radius", C.c_int), ("capillary_stable", C.c_int), ("strength", C.c_double),
                ("max_delta_speed_limit", C.c_double), ("mean_delta_speed", C.c_double),
                ("max_delta_speed", C.c_double), ("raw_curvature_abs_mean", C.c_double),
                ("raw_curvature_abs_max", C.c_double), ("smoothed_curvature_abs_mean", C.c_double),
                ("smoothed_curvature_abs_max", C.c_double), ("capillary_dt_limit", C.c_double)]


class StepControls(C.Structure):
    """pf_step_controls: SparseSim3DTP's adaptive timestep and volume correction (src/driver/sparse_sim3d_tp.h:13-26)"""
    _fields_ = [("adaptive_timestep", C.c_int), ("adaptive_cfl", C.c_double), ("adaptive_min_dt", C.c_double),
                ("c_div_volume_correction", C.c_int), ("c_div_strength", C.c_double),
                ("liquid_volume_target", C.c_double)]


class RenderCamera(C.Structure):
    """pf_render_camera: RenderCacheCamera3D (src/driver/render_cache3d.h:19-27)."""
    _fields_ = [("position", C.c_double * 3), ("target", C.c_double * 3), ("up", C.c_double * 3),
                ("fov_degrees", C.c_double), ("near_clip", C.c_double), ("far_clip", C.c_double),
                ("focal_length_mm", C.c_double)]


class StepControlStats(_Stats):
    """pf_step_control_stats: TimestepStats3D (src/driver/timestep3d.h:8-14) and the volume statistics"""
    _fields_ = [("requested_dt", C.c_double), ("effective_dt", C.c_double), ("max_particle_speed", C.c_double),
                ("cfl_limit_dt", C.c_double), ("limited", C.c_int), ("liquid_volume_current", C.c_double),
                ("liquid_volume_error", C.c_double), ("c_div", C.c_double)]


class SecondaryCfg(C.Structure):
    """pf_secondary_cfg: SparseSim3DTP's secondary-particle settings (src/driver/sparse_sim3d_tp.h:82-137)."""
    _fields_ = [("escaped_particle_branching", C.c_int), ("lifecycle", C.c_int),
                ("droplet_lifetime_steps", C.c_int), ("bubble_lifetime_steps", C.c_int),
                ("velocity_damping", C.c_double), ("reabsorb_margin_cells", C.c_double),
                ("droplet_gravity_scale", C.c_double), ("bubble_buoyancy_scale", C.c_double),
                ("droplet_drag", C.c_double), ("bubble_drag", C.c_double), ("reabsorb_to_primary", C.c_int),
                ("spray_emission", C.c_int), ("spray_particles_per_step", C.c_int),
                ("spray_droplet_fraction", C.c_double), ("spray_droplet_volume", C.c_double),
                ("spray_bubble_volume", C.c_double), ("spray_interface_gate", C.c_int),
                ("spray_min_interface_cells", C.c_int), ("spray_min_interface_grad_max", C.c_double),
                ("spray_min_interface_curvature_abs_max", C.c_double), ("spray_impact_candidates", C.c_int),
                ("spray_impact_region_fraction", C.c_double), ("spray_impact_downward_speed_min", C.c_double),
                ("spray_impact_foam_fraction", C.c_double)]


class SecondaryStats(_Stats):
    """pf_secondary_stats: SecondaryParticleLifecycleStats3D and SecondarySprayEmissionStats3D
    (src/driver/secondary_particles3d.h:33-54, 76-93), the step's additions and the sets' volumes."""
    _fields_ = [(n, C.c_int) for n in (
        "lifecycle_enabled", "lifecycle_finite", "advected_droplets", "advected_bubbles", "reabsorbed_droplets",
        "reabsorbed_bubbles", "expired_droplets", "expired_bubbles", "dragged_droplets", "dragged_bubbles",
        "reabsorbed_droplets_to_primary", "reabsorbed_bubbles_to_primary")] + \
        [(n, C.c_double) for n in (
            "lifecycle_droplet_volume", "lifecycle_bubble_volume", "reabsorbed_droplet_volume",
            "reabsorbed_bubble_volume", "expired_droplet_volume", "expired_bubble_volume",
            "reabsorbed_droplet_volume_to_primary", "reabsorbed_bubble_volume_to_primary")] + \
        [(n, C.c_int) for n in (
            "spray_enabled", "spray_finite", "spray_requested_particles", "spray_effective_requested_particles",
            "spray_interface_gate_enabled", "spray_interface_gate_passed", "spray_interface_cells",
            "spray_candidate_liquid_particles", "spray_impact_candidate_liquid_particles",
            "spray_foam_ready_droplets", "spray_emitted_droplets", "spray_emitted_bubbles")] + \
        [(n, C.c_double) for n in (
            "spray_interface_grad_max", "spray_interface_curvature_abs_max", "spray_emitted_droplet_volume",
            "spray_emitted_bubble_volume")] + \
        [("escaped_droplets_added", C.c_int), ("escaped_bubbles_added", C.c_int),
         ("escaped_droplet_volume_added", C.c_double), ("escaped_bubble_volume_added", C.c_double),
         ("escape_droplet_volume", C.c_double), ("escape_bubble_volume", C.c_double),
         ("spray_step_index", C.c_int), ("droplet_volume_current", C.c_double),
         ("bubble_volume_current", C.c_double)]


class AdaptStats(C.Structure):
    _fields_ = [("band", BandStats), ("gas", CoarsenStats), ("liquid", CoarsenStats), ("refill", RefillStats)]


class Timing(C.Structure):
    _fields_ = [("ms", C.c_double * len(STAGES)), ("count", C.c_longlong * len(STAGES))]

    def as_dict(self):
        return {name: (self.ms[i], self.count[i]) for i, name in enumerate(STAGES)}


class PfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libpfgpu.so and declare its signatures (no GPU needed)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"libpfgpu.so not built at {path}: run `python adaptive-pf-flip_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    vp, sz, i, d = C.c_void_p, C.c_size_t, C.c_int, C.c_double
    P = C.POINTER
    sig = {
        "pf_create": (i, [P(GridDesc), P(vp)]),
        "pf_destroy": (i, [vp]),
        "pf_last_error": (C.c_char_p, [vp]),
        "pf_sync": (i, [vp]),
        "pf_stream": (vp, [vp]),
        "pf_upload_particles": (i, [vp, sz, vp, vp, vp, vp]),
        "pf_download_particles": (i, [vp, vp, vp, vp, vp]),
        "pf_download_particles_async": (i, [vp, vp, vp, vp, vp]),
        "pf_join_downloads": (i, [vp]),
        "pf_upload_particles_async": (i, [vp, C.c_size_t, vp, vp, vp, vp]),
        "pf_upload_particles_f64": (i, [vp, sz, vp, vp, vp, vp]),
        "pf_download_particles_f64": (i, [vp, vp, vp, vp, vp]),
        "pf_num_particles": (sz, [vp]),
        "pf_grid_set_field": (i, [vp, i, vp, vp]),
        "pf_grid_get_field": (i, [vp, i, vp, vp]),
        "pf_grid_clear_field": (i, [vp, i]),
        "pf_grid_clear_all": (i, [vp]),
        "pf_grid_copy": (i, [vp, vp]),
        "pf_active_blocks4": (i, [vp, i, vp, P(sz)]),
        "pf_active_cells": (i, [vp, vp, P(sz)]),
        "pf_active_tiles": (i, [vp]),
        "pf_mark_cells": (i, [vp]),
        "pf_p2g": (i, [vp, P(Phase), d]),
        "pf_save_velocity": (i, [vp]),
        "pf_apply_gravity": (i, [vp, d, d]),
        "pf_apply_wall_boundary": (i, [vp]),
        "pf_project": (i, [vp, P(Phase), d, P(SolveCfg), P(SolveStats)]),
        "pf_g2p": (i, [vp, vp, d, d]),
        "pf_advect": (i, [vp, d, i, P(ClampStats), vp, P(sz)]),
        "pf_step": (i, [vp, P(StepCfg), P(StepStats)]),
        "pf_calibrate_rho_tilde0": (i, [vp, P(Phase), d, P(d)]),
        "pf_seed_scene": (i, [vp, i, C.c_ulonglong, P(sz)]),
        "pf_mr_set_layout": (i, [vp, vp, i]),
        "pf_mr_set_levels": (i, [vp, vp]),
        "pf_mr_get_levels": (i, [vp, vp, vp]),
        "pf_mr_set_dynamic": (i, [vp, P(MRDynamic)]),
        "pf_mr_reset_refinement": (i, [vp]),
        "pf_mr_update_refinement": (i, [vp, vp]),
        "pf_mr_step": (i, [vp, P(MRStepCfg), P(MRStepStats)]),
        "pf_mr_p2g": (i, [vp, P(Phase), d]),
        "pf_mr_get_face": (i, [vp, i, vp]),
        "pf_mr_get_cells": (i, [vp, vp, vp]),
        "pf_write_render_manifest": (i, [C.c_char_p, C.c_char_p, i, i, i, d, P(RenderManifestFrame), i]),
        "pf_set_timing": (i, [vp, i]),
        "pf_get_timing": (i, [vp, P(Timing), i]),
        "pf_launch_count": (C.c_longlong, [vp]),
        "pf_project_noalloc": (i, [i, i, i, d, vp, vp, vp, vp, vp, vp, vp, vp, P(Phase), d, i, d, d, d,
                                   P(SolveStats), vp]),
        "pf_learned_num_params": (sz, []),
        "pf_learned_init": (i, [vp, C.c_ulonglong]),
        "pf_learned_load": (i, [vp, vp, sz]),
        "pf_learned_params": (i, [vp, vp, sz]),
        "pf_learned_harvest": (i, [vp, i, i, i, sz]),
        "pf_learned_dataset": (i, [vp, P(i), P(i)]),
        "pf_learned_clear_dataset": (i, [vp]),
        "pf_learned_merge_dataset": (i, [vp, vp]),
        "pf_learned_train": (i, [vp, i, i, d, C.c_ulonglong, vp]),
        "pf_learned_eval": (i, [vp, i, i, i, vp, vp, vp, i, vp, P(d), vp]),
        "pf_learned_adam": (i, [vp, vp, sz, d]),
        "pf_narrow_band_air": (i, [vp, i, P(BandStats)]),
        "pf_coarsen_particles": (i, [vp, i, i, C.c_uint, P(CoarsenStats)]),
        "pf_refill_liquid": (i, [vp, i, C.c_uint, i, i, i, P(RefillStats)]),
        "pf_set_adaptivity": (i, [vp, P(AdaptCfg)]),
        "pf_get_adaptivity_stats": (i, [vp, P(AdaptStats)]),
        "pf_interface_diagnostics": (i, [vp, P(Phase), P(InterfaceStats)]),
        "pf_get_interface_stats": (i, [vp, P(InterfaceStats)]),
        "pf_set_step_controls": (i, [vp, P(StepControls)]),
        "pf_surface_tension": (i, [vp, P(Phase), d, d, d, i, P(SurfaceStats)]),
        "pf_set_surface_tension": (i, [vp, d, d, i]),
        "pf_get_surface_stats": (i, [vp, P(SurfaceStats)]),
        "pf_get_step_control_stats": (i, [vp, P(StepControlStats)]),
        "pf_default_render_camera": (i, [i, i, i, d, P(RenderCamera)]),
        "pf_write_render_cache": (i, [vp, C.c_char_p, i, d, d, P(Phase), d, P(RenderCamera), P(C.c_longlong)]),
        "pf_secondary_default_cfg": (i, [P(SecondaryCfg)]),
        "pf_set_secondary": (i, [vp, P(SecondaryCfg)]),
        "pf_get_secondary_stats": (i, [vp, P(SecondaryStats)]),
        "pf_secondary_count": (i, [vp, i, P(sz)]),
        "pf_get_secondary": (i, [vp, i, vp, vp, vp, vp]),
        "pf_set_secondary_particles": (i, [vp, i, sz, vp, vp, vp, vp]),
        "pf_secondary_advance": (i, [vp, d, d, d]),
        "pf_secondary_spray": (i, [vp, d, P(InterfaceStats)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int, ctx=None, what: str = ""):
    if rc != PF_OK:
        msg = what
        if ctx:
            m = load().pf_last_error(ctx)
            if m:
                msg = f"{what}: {m.decode(errors='replace')}"
        raise PfError(rc, msg)
