"""CPU checkers for the 2-level multires step -- TEST INFRASTRUCTURE ONLY.

* ``OracleMR``    -- the C restatement (``pf_oracle_mr.c``);
* ``ReferenceMR`` -- the reference's own ``MRSim3DTP`` (src/driver/
                     multires_sim3d_tp.h:10-191), compiled into
                     ``_ref/libpfref.so`` and driven through ``ref_capi.cpp``.

Both hold a particle set (float64, the reference's layout) and a layout, take
the same settings and return the same dense views: face fields over the fine
face lattice shaped (Z, Y, X) (u: X = nx + 1, ...), markers and pressure per
fine cell (the value of the leaf cell holding it) and one byte per level-1
block (8^3 fine cells, 1 where it is split into level-0 blocks).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import ClampStats, PhaseParams, _Phase, _dp, _fp, _ip, _up, oracle_lib, ref_lib

FACE_NAMES = ("u", "v", "w", "mu", "mv", "mw")


class _Dynamic(C.Structure):
    _fields_ = [("enabled", C.c_int), ("particle_padding", C.c_int), ("gas_padding", C.c_int),
                ("hysteresis_cells", C.c_int), ("max_fine_leaves", C.c_int)]


class _SolveCfg(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("abs_tol", C.c_double), ("rel_tol", C.c_double), ("jacobi", C.c_int),
                ("flexible_beta", C.c_int), ("adaptive_restart", C.c_int), ("restart_growth", C.c_double),
                ("c_div", C.c_double)]


class MRSolveStats(C.Structure):
    """The fields of MRPressureSolveStats3D (src/pressure/multires_pressure3d.h:60-133) this path sets."""
    _fields_ = [("active_cells", C.c_int), ("pinned_cell", C.c_int), ("max_iterations", C.c_int),
                ("iterations", C.c_int), ("restarts", C.c_int), ("beta_resets", C.c_int), ("converged", C.c_int),
                ("breakdown", C.c_int), ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("effective_tolerance", C.c_double), ("min_positive_diag", C.c_double), ("max_diag", C.c_double)]


class _StepCfg(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double), ("Vp", C.c_double), ("alpha_l", C.c_double),
                ("alpha_g", C.c_double), ("advect_order", C.c_int), ("solve", _SolveCfg)]


@dataclass
class MRSettings:
    """MRSim3DTP's settings on this path, with its defaults
    (src/driver/multires_sim3d_tp.h:15-67)."""
    dt: float = 0.02
    gravity: float = -9.81
    Vp: float = 1.0
    alpha_liquid: float = 0.95
    alpha_gas: float = 0.95
    advection_order: int = 2
    cg_iters: int = 160
    cg_tol: float = 1e-7
    cg_rel_tol: float = 1e-6
    cg_jacobi_preconditioner: bool = True
    cg_flexible_beta: bool = False
    cg_adaptive_restart: bool = True
    cg_restart_growth: float = 10.0
    dynamic_refinement: bool = True
    dynamic_particle_padding: int = 1
    dynamic_gas_padding: int = 2
    dynamic_hysteresis_cells: int = 1
    dynamic_max_fine_leaves: int = 0
    phase: PhaseParams = field(default_factory=PhaseParams)


def _typed_oracle():
    lib = oracle_lib()
    if getattr(lib, "_mr_typed", False):
        return lib
    vp = C.c_void_p
    lib.pfo_mr_create.restype = vp
    lib.pfo_mr_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
    lib.pfo_mr_destroy.argtypes = [vp]
    lib.pfo_mr_dims.argtypes = [vp, _ip]
    lib.pfo_mr_set_layout.argtypes = [vp, _ip, C.c_int]
    lib.pfo_mr_set_levels.argtypes = [vp, _up]
    lib.pfo_mr_get_levels.argtypes = [vp, _up]
    lib.pfo_mr_count_fine_leaves.argtypes = [vp]
    lib.pfo_mr_update_refinement.argtypes = [vp, C.POINTER(_Dynamic), C.c_size_t, _dp, _up]
    lib.pfo_mr_refinement_state.argtypes = [vp, _ip]
    lib.pfo_mr_face_valid.argtypes = [vp, C.c_int, _up]
    lib.pfo_mr_get_face.argtypes = [vp, C.c_int, _fp]
    lib.pfo_mr_set_face.argtypes = [vp, C.c_int, _fp]
    lib.pfo_mr_get_cells.argtypes = [vp, _fp, _fp]
    lib.pfo_mr_mark_cells.argtypes = [vp, C.c_size_t, _dp]
    lib.pfo_mr_p2g.argtypes = [vp, C.c_size_t, _dp, _dp, _up, _dp, C.POINTER(_Phase), C.c_double]
    lib.pfo_mr_step.argtypes = [vp, C.POINTER(_Dynamic), C.c_size_t, _dp, _dp, _up, _dp, C.POINTER(_Phase),
                                C.POINTER(_StepCfg), C.POINTER(MRSolveStats), C.POINTER(ClampStats)]
    lib._mr_typed = True
    return lib


def _typed_ref():
    lib = ref_lib()
    if getattr(lib, "_mr_typed", False):
        return lib
    vp = C.c_void_p
    lib.pfr_mr_create.restype = vp
    lib.pfr_mr_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
    lib.pfr_mr_destroy.argtypes = [vp]
    lib.pfr_mr_configure.argtypes = [vp, _dp, _dp, _ip]
    lib.pfr_mr_set_layout.argtypes = [vp, _ip, C.c_int]
    lib.pfr_mr_get_levels.argtypes = [vp, _up]
    lib.pfr_mr_count_level.argtypes = [vp, C.c_int]
    lib.pfr_mr_set_particles.argtypes = [vp, C.c_size_t, _dp, _dp, _up, _dp]
    lib.pfr_mr_num_particles.restype = C.c_size_t
    lib.pfr_mr_num_particles.argtypes = [vp]
    lib.pfr_mr_get_particles.argtypes = [vp, _dp, _dp, _up, _dp]
    lib.pfr_mr_init_bubble_tank.argtypes = [vp]
    lib.pfr_mr_update_refinement.argtypes = [vp, _ip]
    lib.pfr_mr_p2g.argtypes = [vp]
    lib.pfr_mr_step.argtypes = [vp, _ip, _dp]
    lib.pfr_mr_get_face.argtypes = [vp, C.c_int, _fp]
    lib.pfr_mr_face_valid.argtypes = [vp, C.c_int, _up]
    lib.pfr_mr_get_cells.argtypes = [vp, _fp, _fp]
    lib._mr_typed = True
    return lib


def face_shape(nx, ny, nz, axis):
    return (nz + (axis == 2), ny + (axis == 1), nx + (axis == 0))


def block_counts(nx, ny, nz):
    return ((nx + 7) // 8, (ny + 7) // 8, (nz + 7) // 8)


def _boxes(boxes):
    b = np.ascontiguousarray(np.asarray(boxes, np.int32).reshape(-1, 6))
    return (b if len(b) else np.zeros((1, 6), np.int32)), len(b)


class _MRBase:
    def __init__(self, nx, ny, nz, dx, settings: MRSettings | None = None):
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(dx)
        self.settings = settings or MRSettings()
        self.n = 0
        self.pos = np.zeros((0, 3))
        self.vel = np.zeros((0, 3))
        self.type = np.zeros(0, np.uint8)
        self.volume = np.zeros(0)

    def set_particles(self, pos, vel, type, volume=None):
        n = len(pos)
        self.n = n
        self.pos = np.ascontiguousarray(pos, np.float64).reshape(n, 3).copy()
        self.vel = np.ascontiguousarray(vel, np.float64).reshape(n, 3).copy()
        self.type = np.ascontiguousarray(type, np.uint8).reshape(n).copy()
        self.volume = np.ascontiguousarray(np.ones(n) if volume is None else volume, np.float64).reshape(n).copy()

    def face(self, f):
        out = np.zeros(face_shape(self.nx, self.ny, self.nz, f % 3), np.float32)
        self._get_face(f, out)
        return out

    def fine_cells(self):
        return int(np.count_nonzero(self.levels())) * 512


class OracleMR(_MRBase):
    """The C restatement, stepping particles it keeps in float64."""

    def __init__(self, nx, ny, nz, dx, settings=None):
        super().__init__(nx, ny, nz, dx, settings)
        self.lib = _typed_oracle()
        self.h = self.lib.pfo_mr_create(self.nx, self.ny, self.nz, self.dx)
        if not self.h:
            raise MemoryError("pfo_mr_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.pfo_mr_destroy(self.h)
            self.h = None

    def _dyn(self):
        s = self.settings
        return _Dynamic(int(s.dynamic_refinement), s.dynamic_particle_padding, s.dynamic_gas_padding,
                        s.dynamic_hysteresis_cells, s.dynamic_max_fine_leaves)

    def _cfg(self):
        s = self.settings
        solve = _SolveCfg(s.cg_iters, s.cg_tol, s.cg_rel_tol, int(s.cg_jacobi_preconditioner), int(s.cg_flexible_beta),
                          int(s.cg_adaptive_restart), s.cg_restart_growth, 0.0)
        return _StepCfg(s.dt, s.gravity, s.Vp, s.alpha_liquid, s.alpha_gas, s.advection_order, solve)

    def set_layout(self, boxes):
        b, n = _boxes(boxes)
        self.lib.pfo_mr_set_layout(self.h, b, n)

    def set_levels(self, refined):
        self.lib.pfo_mr_set_levels(self.h, np.ascontiguousarray(refined, np.uint8).ravel())

    def levels(self):
        MX, MY, MZ = block_counts(self.nx, self.ny, self.nz)
        out = np.zeros((MZ, MY, MX), np.uint8)
        self.lib.pfo_mr_get_levels(self.h, out.ravel())
        return out

    def fine_leaves(self):
        return int(self.lib.pfo_mr_count_fine_leaves(self.h))

    def update_refinement(self):
        self.lib.pfo_mr_update_refinement(self.h, C.byref(self._dyn()), self.n, self.pos.ravel(), self.type)
        st = np.zeros(8, np.int32)
        self.lib.pfo_mr_refinement_state(self.h, st)
        return st

    def face_valid(self, axis):
        out = np.zeros(face_shape(self.nx, self.ny, self.nz, axis), np.uint8)
        self.lib.pfo_mr_face_valid(self.h, axis, out.ravel())
        return out

    def _get_face(self, f, out):
        self.lib.pfo_mr_get_face(self.h, f, out.ravel())

    def cells(self):
        mk = np.zeros((self.nz, self.ny, self.nx), np.float32)
        p = np.zeros_like(mk)
        self.lib.pfo_mr_get_cells(self.h, mk.ravel(), p.ravel())
        return mk, p

    def mark_cells(self):
        self.lib.pfo_mr_mark_cells(self.h, self.n, self.pos.ravel())

    def p2g(self):
        ph = self.settings.phase.as_struct()
        pos, vel = self.pos.ravel(), self.vel.ravel()
        self.lib.pfo_mr_p2g(self.h, self.n, pos, vel, self.type, self.volume, C.byref(ph), self.settings.Vp)

    def step(self):
        ph = self.settings.phase.as_struct()
        sst, cst = MRSolveStats(), ClampStats()
        pos, vel = self.pos.reshape(-1), self.vel.reshape(-1)
        self.lib.pfo_mr_step(self.h, C.byref(self._dyn()), self.n, pos, vel, self.type, self.volume, C.byref(ph),
                             C.byref(self._cfg()), C.byref(sst), C.byref(cst))
        return sst, cst


class ReferenceMR(_MRBase):
    """The reference's MRSim3DTP itself; particles live in the reference."""

    def __init__(self, nx, ny, nz, dx, settings=None):
        super().__init__(nx, ny, nz, dx, settings)
        self.lib = _typed_ref()
        self.h = self.lib.pfr_mr_create(self.nx, self.ny, self.nz, self.dx)
        if not self.h:
            raise MemoryError("pfr_mr_create failed")
        self.configure()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.pfr_mr_destroy(self.h)
            self.h = None

    def configure(self):
        s = self.settings
        d = np.array([s.dt, s.gravity, s.Vp, s.alpha_liquid, s.alpha_gas, s.cg_tol, s.cg_rel_tol, s.cg_restart_growth],
                     np.float64)
        i = np.array([s.advection_order, s.cg_iters, int(s.cg_jacobi_preconditioner), int(s.cg_flexible_beta),
                      int(s.cg_adaptive_restart), int(s.dynamic_refinement), s.dynamic_particle_padding,
                      s.dynamic_gas_padding, s.dynamic_hysteresis_cells, s.dynamic_max_fine_leaves], np.int32)
        self.lib.pfr_mr_configure(self.h, s.phase.as_array(), d, i)

    def set_layout(self, boxes):
        b, n = _boxes(boxes)
        self.lib.pfr_mr_set_layout(self.h, b, n)

    def levels(self):
        MX, MY, MZ = block_counts(self.nx, self.ny, self.nz)
        out = np.zeros((MZ, MY, MX), np.uint8)
        self.lib.pfr_mr_get_levels(self.h, out.ravel())
        return out

    def fine_leaves(self):
        return int(self.lib.pfr_mr_count_level(self.h, 0))

    def set_particles(self, pos, vel, type, volume=None):
        super().set_particles(pos, vel, type, volume)
        self.lib.pfr_mr_set_particles(self.h, self.n, self.pos.ravel(), self.vel.ravel(), self.type, self.volume)

    def pull_particles(self):
        self.n = int(self.lib.pfr_mr_num_particles(self.h))
        self.pos = np.zeros((self.n, 3))
        self.vel = np.zeros((self.n, 3))
        self.type = np.zeros(self.n, np.uint8)
        self.volume = np.zeros(self.n)
        self.lib.pfr_mr_get_particles(self.h, self.pos.ravel(), self.vel.ravel(), self.type, self.volume)

    def init_bubble_tank(self):
        """MRSim3DTP::initBubbleTankInterfaceBand (src/driver/multires_sim3d_tp.cpp:457-503)."""
        self.lib.pfr_mr_init_bubble_tank(self.h)
        self.pull_particles()

    def update_refinement(self):
        st = np.zeros(8, np.int32)
        self.lib.pfr_mr_update_refinement(self.h, st)
        return st

    def face_valid(self, axis):
        out = np.zeros(face_shape(self.nx, self.ny, self.nz, axis), np.uint8)
        self.lib.pfr_mr_face_valid(self.h, axis, out.ravel())
        return out

    def _get_face(self, f, out):
        rc = self.lib.pfr_mr_get_face(self.h, f, out.ravel())
        if rc:
            raise RuntimeError(f"pfr_mr_get_face: {rc}")

    def cells(self):
        mk = np.zeros((self.nz, self.ny, self.nx), np.float32)
        p = np.zeros_like(mk)
        self.lib.pfr_mr_get_cells(self.h, mk.ravel(), p.ravel())
        return mk, p

    def p2g(self):
        self.lib.pfr_mr_p2g(self.h)

    def step(self):
        iv = np.zeros(10, np.int32)
        dv = np.zeros(3, np.float64)
        self.lib.pfr_mr_step(self.h, iv, dv)
        self.pull_particles()
        sst = MRSolveStats()
        sst.active_cells, sst.pinned_cell, sst.iterations, sst.restarts, sst.beta_resets = (int(v) for v in iv[:5])
        sst.converged, sst.breakdown = int(iv[5]), int(iv[6])
        sst.initial_residual, sst.final_residual, sst.effective_tolerance = (float(v) for v in dv)
        cst = ClampStats()
        cst.clamped_liquid, cst.clamped_gas = int(iv[8]), int(iv[9])
        return sst, cst
