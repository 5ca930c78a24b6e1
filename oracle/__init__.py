"""CPU checkers for the sparse 3D two-phase solver step -- TEST INFRASTRUCTURE ONLY.

Two interchangeable backends with one Python interface:

* ``Oracle``    -- ``lib/libpforacle.so``, the C restatement in ``pf_oracle.c``
                   (each function cites the reference file:line it follows);
* ``Reference`` -- ``_ref/libpfref.so``, the unmodified adaptive-pf-flip
                   sources compiled by ``oracle/Makefile`` and driven through
                   ``ref_capi.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` import this package.  The product
library (``adaptive-pf-flip_b200``) never does.

Layouts match the reference: particle positions/velocities are AoS float64
``(n, 3)`` (``std::vector<Vec3>``), ``type`` uint8 (0 liquid, 1 gas),
``volume`` float64.  A grid field comes back as a dense float32 array shaped
``(Z, Y, X)`` over that field's node lattice plus a uint8 array shaped
``(nbz, nby, nbx)`` with one activity flag per 4^3 block.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "libpforacle.so")
REF_SO = os.path.join(HERE, "_ref", "libpfref.so")

U, V, W, MU, MV, MW, P, MK = range(8)
FIELD_NAMES = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class _Phase(C.Structure):
    _fields_ = [("rho_l", C.c_double), ("rho_g", C.c_double),
                ("alpha_phi", C.c_double), ("rho_tilde_0", C.c_double)]


class _SolveCfg(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("abs_tol", C.c_double),
                ("rel_tol", C.c_double), ("c_div", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("n_cells", C.c_int), ("pin_cell", C.c_longlong),
                ("res0", C.c_double), ("res_final", C.c_double), ("tol_effective", C.c_double),
                ("converged", C.c_int), ("breakdown", C.c_int)]


class BandStats(C.Structure):
    """NarrowBandAirResult3D (src/driver/particle_adaptivity3d.h:49-54)"""
    _fields_ = [("removed", C.c_int), ("liquid_cells", C.c_int), ("gas_before", C.c_int), ("gas_after", C.c_int)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class CoarsenStats(C.Structure):
    """GasParticleCoarseningResult3D (src/driver/particle_adaptivity3d.h:56-62)"""
    _fields_ = [("removed", C.c_int), ("cells", C.c_int), ("overfull_cells", C.c_int), ("before", C.c_int),
                ("after", C.c_int)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class RefillStats(C.Structure):
    """LiquidParticleRefillResult3D (src/driver/particle_adaptivity3d.h:64-72)"""
    _fields_ = [("added", C.c_int), ("cells", C.c_int), ("interface_cells", C.c_int), ("underfull_cells", C.c_int),
                ("budget_limited", C.c_int), ("before", C.c_int), ("after", C.c_int)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class InterfaceStats(C.Structure):
    """InterfaceDiagnostics3D (src/driver/interface_diagnostics3d.h:7-19)"""
    _fields_ = [("sample_cells", C.c_int), ("interface_cells", C.c_int), ("finite", C.c_int),
                ("surface_tension_candidate", C.c_int), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("phi_mean", C.c_double), ("grad_mean", C.c_double), ("grad_max", C.c_double),
                ("curvature_abs_mean", C.c_double), ("curvature_abs_max", C.c_double)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class SurfaceStats(C.Structure):
    """SurfaceTensionStats3D (src/driver/interface_diagnostics3d.h:21-36)"""
    _fields_ = [("enabled", C.c_int), ("applied_cells", C.c_int), ("finite", C.c_int),
                ("curvature_smoothing_radius", C.c_int), ("capillary_stable", C.c_int), ("strength", C.c_double),
                ("max_delta_speed_limit", C.c_double), ("mean_delta_speed", C.c_double),
                ("max_delta_speed", C.c_double), ("raw_curvature_abs_mean", C.c_double),
                ("raw_curvature_abs_max", C.c_double), ("smoothed_curvature_abs_mean", C.c_double),
                ("smoothed_curvature_abs_max", C.c_double), ("capillary_dt_limit", C.c_double)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class ClampStats(C.Structure):
    _fields_ = [("clamped_liquid", C.c_int), ("clamped_gas", C.c_int),
                ("x_lo", C.c_int), ("x_hi", C.c_int), ("y_lo", C.c_int),
                ("y_hi", C.c_int), ("z_lo", C.c_int), ("z_hi", C.c_int)]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class _StepCfg(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double), ("Vp", C.c_double),
                ("alpha_l", C.c_double), ("alpha_g", C.c_double), ("cg_iters", C.c_int),
                ("cg_tol", C.c_double), ("cg_rel_tol", C.c_double), ("c_div", C.c_double),
                ("advect_order", C.c_int)]


@dataclass
class PhaseParams:
    """Mirror of the reference's PhaseParams (src/physics/phasefield.h:4-9)."""
    rho_l: float = 1.0
    rho_g: float = 0.01
    alpha_phi: float = 1.0
    rho_tilde_0: float = 1.0

    def as_array(self):
        return np.array([self.rho_l, self.rho_g, self.alpha_phi, self.rho_tilde_0], np.float64)

    def as_struct(self):
        return _Phase(self.rho_l, self.rho_g, self.alpha_phi, self.rho_tilde_0)


class Particles:
    """SoA-of-AoS particle set in the reference's layout (Particles3DTP)."""

    def __init__(self, pos=None, vel=None, type=None, volume=None):
        pos = np.zeros((0, 3)) if pos is None else pos
        n = len(pos)
        self.pos = np.ascontiguousarray(pos, np.float64).reshape(n, 3)
        self.vel = np.ascontiguousarray(np.zeros((n, 3)) if vel is None else vel, np.float64).reshape(n, 3)
        self.type = np.ascontiguousarray(np.zeros(n) if type is None else type, np.uint8).reshape(n)
        self.volume = np.ascontiguousarray(np.ones(n) if volume is None else volume, np.float64).reshape(n)

    def __len__(self):
        return len(self.pos)

    def add(self, p, v, t, vol=1.0):
        self.pos = np.vstack([self.pos, np.asarray(p, np.float64).reshape(1, 3)])
        self.vel = np.vstack([self.vel, np.asarray(v, np.float64).reshape(1, 3)])
        self.type = np.append(self.type, np.uint8(t)).astype(np.uint8)
        self.volume = np.append(self.volume, float(vol))

    def copy(self):
        return Particles(self.pos.copy(), self.vel.copy(), self.type.copy(), self.volume.copy())


def field_dims(nx, ny, nz, f):
    return [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1),
            (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1),
            (nx, ny, nz), (nx, ny, nz)][f]


def block_dims(nx, ny, nz, f):
    X, Y, Z = field_dims(nx, ny, nz, f)
    return ((X + 3) // 4, (Y + 3) // 4, (Z + 3) // 4)


_LIBS = {}


def _load(path, kind):
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{kind} library missing: {path} (run `make -C oracle`)")
    lib = C.CDLL(path)
    _LIBS[path] = lib
    return lib


def oracle_lib():
    lib = _load(ORACLE_SO, "oracle")
    if getattr(lib, "_typed", False):
        return lib
    vp = C.c_void_p
    lib.pfo_grid_create.restype = vp
    lib.pfo_grid_create.argtypes = [C.c_int] * 3 + [C.c_double] * 4
    lib.pfo_grid_destroy.argtypes = [vp]
    lib.pfo_grid_copy.argtypes = [vp, vp]
    lib.pfo_get_field.argtypes = [vp, C.c_int, _fp, _up]
    lib.pfo_set_field.argtypes = [vp, C.c_int, _fp, _up]
    lib.pfo_clear_field.argtypes = [vp, C.c_int]
    lib.pfo_phi_from_raw.restype = C.c_double
    lib.pfo_phi_from_raw.argtypes = [C.c_double, C.POINTER(_Phase)]
    lib.pfo_beta_from_raw.restype = C.c_double
    lib.pfo_beta_from_raw.argtypes = [C.c_double, C.POINTER(_Phase)]
    lib.pfo_calibrate_rho_tilde0.restype = C.c_double
    lib.pfo_calibrate_rho_tilde0.argtypes = [C.POINTER(_Phase), C.c_double]
    lib.pfo_mark_cells.argtypes = [vp, C.c_size_t, _dp]
    lib.pfo_p2g.argtypes = [vp, C.c_size_t, _dp, _dp, _up, _dp, C.POINTER(_Phase), C.c_double]
    lib.pfo_apply_gravity.argtypes = [vp, C.c_double, C.c_double]
    lib.pfo_apply_wall_boundary.argtypes = [vp]
    lib.pfo_project.argtypes = [vp, C.POINTER(_Phase), C.c_double, C.POINTER(_SolveCfg),
                                C.POINTER(SolveStats)]
    lib.pfo_g2p.argtypes = [vp, vp, C.c_size_t, _dp, _dp, _up, C.c_double, C.c_double]
    lib.pfo_advect.argtypes = [vp, C.c_size_t, _dp, _up, _dp, _dp, C.c_double, C.c_int,
                               C.POINTER(ClampStats), C.c_void_p, C.POINTER(C.c_size_t)]
    lib.pfo_collect_cells.argtypes = [vp, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]
    lib.pfo_step.argtypes = [vp, vp, C.c_size_t, _dp, _dp, _up, _dp, C.POINTER(_Phase),
                             C.POINTER(_StepCfg), C.POINTER(SolveStats), C.POINTER(ClampStats)]
    sp = C.POINTER(C.c_size_t)
    lib.pfo_particle_score.restype = C.c_uint
    lib.pfo_particle_score.argtypes = [vp, _dp, C.c_int, C.c_int, C.c_int, C.c_uint]
    lib.pfo_slot_score.restype = C.c_uint
    lib.pfo_slot_score.argtypes = [C.c_size_t, C.c_int, C.c_uint]
    lib.pfo_narrow_band_air.argtypes = [vp, sp, _dp, _dp, _up, _dp, C.c_int, C.POINTER(BandStats)]
    lib.pfo_coarsen_particles.argtypes = [vp, sp, _dp, _dp, _up, _dp, C.c_int, C.c_int, C.c_uint,
                                          C.POINTER(CoarsenStats)]
    lib.pfo_refill_liquid.argtypes = [vp, sp, C.c_size_t, _dp, _dp, _up, _dp, C.c_int, C.c_uint, C.c_int, C.c_int,
                                      C.c_int, C.POINTER(RefillStats)]
    lib.pfo_interface_diagnostics.argtypes = [vp, C.POINTER(_Phase), C.POINTER(InterfaceStats)]
    lib.pfo_surface_tension.argtypes = [vp, C.POINTER(_Phase), C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.POINTER(SurfaceStats)]
    lib._typed = True
    return lib


def ref_lib():
    lib = _load(REF_SO, "reference")
    if getattr(lib, "_typed", False):
        return lib
    vp = C.c_void_p
    lib.pfr_create.restype = vp
    lib.pfr_create.argtypes = [C.c_int] * 3 + [C.c_double] * 4
    lib.pfr_destroy.argtypes = [vp]
    lib.pfr_copy_grid.argtypes = [vp, vp]
    lib.pfr_get_field.argtypes = [vp, C.c_int, _fp, _up]
    lib.pfr_set_field.argtypes = [vp, C.c_int, _fp, _up]
    lib.pfr_active_block_ids.argtypes = [vp, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]
    lib.pfr_collect_cells.argtypes = [vp, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]
    lib.pfr_write_render_cache.argtypes = [vp, C.c_char_p, C.c_int, C.c_double, C.c_double, _dp, C.c_double, _dp]
    lib.pfr_set_particles.argtypes = [vp, C.c_size_t, _dp, _dp, _up, _dp]
    lib.pfr_num_particles.restype = C.c_size_t
    lib.pfr_num_particles.argtypes = [vp]
    lib.pfr_get_particles.argtypes = [vp, _dp, _dp, _up, _dp]
    lib.pfr_p2g.argtypes = [vp, _dp, C.c_double]
    lib.pfr_project.argtypes = [vp, _dp, C.c_double, C.c_int, C.c_double, C.c_double]
    lib.pfr_g2p.argtypes = [vp, vp, C.c_double, C.c_double]
    lib.pfr_advect.argtypes = [vp, C.c_double, C.c_int, _ip, C.c_void_p, C.POINTER(C.c_size_t)]
    lib.pfr_step.argtypes = [vp, _dp, _dp]
    lib.pfr_calibrate_rho_tilde0.restype = C.c_double
    lib.pfr_calibrate_rho_tilde0.argtypes = [_dp, C.c_double]
    lib.pfr_phi_from_raw.restype = C.c_double
    lib.pfr_phi_from_raw.argtypes = [C.c_double, _dp]
    lib.pfr_beta_from_raw.restype = C.c_double
    lib.pfr_beta_from_raw.argtypes = [C.c_double, _dp]
    lib.pfr_narrow_band_air.argtypes = [vp, C.c_int, _ip]
    lib.pfr_coarsen_particles.argtypes = [vp, C.c_int, C.c_int, C.c_uint, _ip]
    lib.pfr_refill_liquid.argtypes = [vp, C.c_int, C.c_uint, C.c_int, C.c_int, C.c_int, _ip]
    lib.pfr_interface_diagnostics.argtypes = [vp, _dp, _ip, _dp]
    lib.pfr_surface_tension.argtypes = [vp, _dp, C.c_double, C.c_double, C.c_double, C.c_int, _ip, _dp]
    lib.pfr_write_render_manifest.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                              _ip, _ip, _dp, C.POINTER(C.c_char_p),
                                              np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
    lib._typed = True
    return lib


def reference_available():
    return os.path.exists(REF_SO)


class _GridBase:
    def __init__(self, nx, ny, nz, dx, origin=(0.0, 0.0, 0.0)):
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(dx)
        self.origin = tuple(float(o) for o in origin)

    def dims(self, f):
        return field_dims(self.nx, self.ny, self.nz, f)

    def bdims(self, f):
        return block_dims(self.nx, self.ny, self.nz, f)

    def _bufs(self, f):
        X, Y, Z = self.dims(f)
        bx, by, bz = self.bdims(f)
        return np.zeros((Z, Y, X), np.float32), np.zeros((bz, by, bx), np.uint8)

    def active_blocks(self, f):
        """Sorted 4^3 block ids (bx + nbx*(by + nby*bz)) active in field f."""
        _, act = self.get_field(f)
        return np.flatnonzero(act.ravel()).astype(np.int64)

    def fields(self):
        return {FIELD_NAMES[f]: self.get_field(f) for f in range(8)}

    def cell_markers(self):
        vals, _ = self.get_field(MK)
        return (vals + np.float32(0.5)).astype(np.int32)

    def fluid_cells(self):
        """Fluid cells as ascending linear indices c = i + nx*(j + ny*k)."""
        return np.flatnonzero(self.cell_markers().ravel() == 1).astype(np.int64)

    def set_cells(self, markers):
        """Set the marker field from a dense (Z,Y,X) int array; cells with a
        nonzero marker activate their block (SparseMacGrid3D::setCell)."""
        m = np.asarray(markers)
        X, Y, Z = self.dims(MK)
        act = np.zeros(self.bdims(MK)[::-1], np.uint8)
        kk, jj, ii = np.nonzero(m)
        act[kk // 4, jj // 4, ii // 4] = 1
        self.set_field(MK, m.astype(np.float32), act)


class OracleGrid(_GridBase):
    """Grid of the C restatement."""

    def __init__(self, nx, ny, nz, dx, origin=(0.0, 0.0, 0.0)):
        super().__init__(nx, ny, nz, dx, origin)
        self.lib = oracle_lib()
        self.h = self.lib.pfo_grid_create(self.nx, self.ny, self.nz, self.dx, *self.origin)
        if not self.h:
            raise MemoryError("pfo_grid_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.pfo_grid_destroy(self.h)
            self.h = None

    def get_field(self, f):
        d, a = self._bufs(f)
        self.lib.pfo_get_field(self.h, f, d, a)
        return d, a

    def set_field(self, f, dense, act):
        self.lib.pfo_set_field(self.h, f, np.ascontiguousarray(dense, np.float32),
                               np.ascontiguousarray(act, np.uint8))

    def copy(self):
        g = OracleGrid(self.nx, self.ny, self.nz, self.dx, self.origin)
        self.lib.pfo_grid_copy(g.h, self.h)
        return g


class ReferenceGrid(_GridBase):
    """Grid (and particle store) of the compiled reference (SparseSim3DTP)."""

    def __init__(self, nx, ny, nz, dx, origin=(0.0, 0.0, 0.0)):
        super().__init__(nx, ny, nz, dx, origin)
        self.lib = ref_lib()
        self.h = self.lib.pfr_create(self.nx, self.ny, self.nz, self.dx, *self.origin)
        if not self.h:
            raise MemoryError("pfr_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.pfr_destroy(self.h)
            self.h = None

    def get_field(self, f):
        d, a = self._bufs(f)
        self.lib.pfr_get_field(self.h, f, d, a)
        return d, a

    def set_field(self, f, dense, act):
        self.lib.pfr_set_field(self.h, f, np.ascontiguousarray(dense, np.float32),
                               np.ascontiguousarray(act, np.uint8))

    def copy(self):
        g = ReferenceGrid(self.nx, self.ny, self.nz, self.dx, self.origin)
        self.lib.pfr_copy_grid(g.h, self.h)
        return g

    def allocation_order(self, f):
        n = C.c_size_t()
        self.lib.pfr_active_block_ids(self.h, f, None, C.byref(n))
        out = np.zeros(n.value, np.int32)
        self.lib.pfr_active_block_ids(self.h, f, out.ctypes.data, C.byref(n))
        return out

    def collect_cells(self, marker=1):
        """sparse3d::collectCellsWithMarker (src/driver/sparse_ops3d_common.h:65-85): the cells
        with `marker`, ascending linear index, from the reference's own code."""
        n = C.c_size_t()
        self.lib.pfr_collect_cells(self.h, int(marker), None, C.byref(n))
        out = np.zeros(max(n.value, 1), np.int32)
        if self.lib.pfr_collect_cells(self.h, int(marker), out.ctypes.data, C.byref(n)) != 0:
            raise RuntimeError("pfr_collect_cells failed")
        return out[: n.value].astype(np.int64)

    def write_render_cache(self, path, frame, time, dt, pp: PhaseParams, Vp, camera):
        """writeSparseRenderCache3D (src/driver/render_cache3d.h:617-663) of this grid and its particles;
        camera: 13 doubles (position, target, up, fov, near, far, focal length)."""
        cam = np.ascontiguousarray(camera, np.float64)
        rc = self.lib.pfr_write_render_cache(self.h, str(path).encode(), int(frame), float(time), float(dt),
                                             pp.as_array(), float(Vp), cam)
        if rc != 0:
            raise RuntimeError("writeSparseRenderCache3D failed")

    def _put(self, ps: Particles):
        self.lib.pfr_set_particles(self.h, len(ps), ps.pos, ps.vel, ps.type, ps.volume)

    def _take(self, ps: Particles):
        n = int(self.lib.pfr_num_particles(self.h))
        if n != len(ps):
            ps.pos, ps.vel = np.zeros((n, 3)), np.zeros((n, 3))
            ps.type, ps.volume = np.zeros(n, np.uint8), np.zeros(n)
        self.lib.pfr_get_particles(self.h, ps.pos, ps.vel, ps.type, ps.volume)


class Oracle:
    """Per-call API of the C restatement, named after the reference functions."""
    Grid = OracleGrid
    name = "oracle"

    def __init__(self):
        self.lib = oracle_lib()

    def phi_from_raw(self, raw, pp: PhaseParams):
        return self.lib.pfo_phi_from_raw(float(raw), C.byref(pp.as_struct()))

    def beta_from_raw(self, raw, pp: PhaseParams):
        return self.lib.pfo_beta_from_raw(float(raw), C.byref(pp.as_struct()))

    def calibrate_rho_tilde0(self, pp: PhaseParams, Vp):
        return self.lib.pfo_calibrate_rho_tilde0(C.byref(pp.as_struct()), float(Vp))

    def mark_cells(self, g: OracleGrid, ps: Particles):
        self.lib.pfo_mark_cells(g.h, len(ps), ps.pos)

    def p2g(self, g: OracleGrid, ps: Particles, pp: PhaseParams, Vp):
        self.lib.pfo_p2g(g.h, len(ps), ps.pos, ps.vel, ps.type, ps.volume,
                         C.byref(pp.as_struct()), float(Vp))

    def apply_gravity(self, g, dt, gravity):
        self.lib.pfo_apply_gravity(g.h, float(dt), float(gravity))

    def apply_wall_boundary(self, g):
        self.lib.pfo_apply_wall_boundary(g.h)

    def project(self, g, pp: PhaseParams, dt, cg_iters, cg_tol, c_div=0.0, rel_tol=0.0):
        st = SolveStats()
        cfg = _SolveCfg(int(cg_iters), float(cg_tol), float(rel_tol), float(c_div))
        self.lib.pfo_project(g.h, C.byref(pp.as_struct()), float(dt), C.byref(cfg), C.byref(st))
        return st

    def g2p(self, g, ps: Particles, saved, aL, aG):
        self.lib.pfo_g2p(g.h, saved.h, len(ps), ps.pos, ps.vel, ps.type, float(aL), float(aG))

    def advect(self, ps: Particles, g, dt, order=2, escape=False):
        st = ClampStats()
        n_esc = C.c_size_t()
        buf = np.zeros((max(len(ps), 1), 8), np.float64) if escape else None
        self.lib.pfo_advect(g.h, len(ps), ps.pos, ps.type, ps.vel, ps.volume, float(dt), int(order),
                            C.byref(st), buf.ctypes.data if escape else None, C.byref(n_esc))
        if escape:
            return st, buf[: n_esc.value].copy()
        return st

    def step(self, g, saved, ps: Particles, pp: PhaseParams, cfg: dict):
        sst, cst = SolveStats(), ClampStats()
        sc = _StepCfg(cfg["dt"], cfg["gravity"], cfg["Vp"], cfg["alpha_l"], cfg["alpha_g"],
                      int(cfg["cg_iters"]), cfg["cg_tol"], cfg.get("cg_rel_tol", 0.0),
                      cfg.get("c_div", 0.0), int(cfg.get("advect_order", 2)))
        rc = self.lib.pfo_step(g.h, saved.h, len(ps), ps.pos, ps.vel, ps.type, ps.volume,
                               C.byref(pp.as_struct()), C.byref(sc), C.byref(sst), C.byref(cst))
        if rc != 0:
            raise RuntimeError("pfo_step failed")
        return sst, cst


    # ---- particle adaptivity (src/driver/particle_adaptivity3d.h:111-374) ----
    def narrow_band_air(self, g, ps: Particles, radius=2):
        n = C.c_size_t(len(ps))
        st = BandStats()
        if self.lib.pfo_narrow_band_air(g.h, C.byref(n), ps.pos, ps.vel, ps.type, ps.volume, int(radius),
                                        C.byref(st)):
            raise MemoryError("pfo_narrow_band_air")
        _truncate(ps, n.value)
        return st

    def coarsen_particles(self, g, ps: Particles, ptype, target, seed):
        n = C.c_size_t(len(ps))
        st = CoarsenStats()
        if self.lib.pfo_coarsen_particles(g.h, C.byref(n), ps.pos, ps.vel, ps.type, ps.volume, int(ptype),
                                          int(target), int(seed) & 0xffffffff, C.byref(st)):
            raise MemoryError("pfo_coarsen_particles")
        _truncate(ps, n.value)
        return st

    def refill_liquid(self, g, ps: Particles, target, seed, interface_only=False, interface_radius=1,
                      max_added=0):
        n0 = len(ps)
        cap = n0 + int(np.count_nonzero(ps.type == 0)) * max(int(target), 1)
        pos, vel = np.zeros((cap, 3)), np.zeros((cap, 3))
        typ, vol = np.zeros(cap, np.uint8), np.zeros(cap)
        pos[:n0], vel[:n0], typ[:n0], vol[:n0] = ps.pos, ps.vel, ps.type, ps.volume
        n = C.c_size_t(n0)
        st = RefillStats()
        if self.lib.pfo_refill_liquid(g.h, C.byref(n), cap, pos, vel, typ, vol, int(target),
                                      int(seed) & 0xffffffff, int(bool(interface_only)), int(interface_radius),
                                      int(max_added), C.byref(st)):
            raise MemoryError("pfo_refill_liquid")
        m = n.value
        ps.pos, ps.vel, ps.type, ps.volume = pos[:m].copy(), vel[:m].copy(), typ[:m].copy(), vol[:m].copy()
        return st


    def interface_diagnostics(self, g, pp: PhaseParams):
        """diagnoseSparseInterface3D (src/driver/interface_diagnostics3d.cpp:363-379)"""
        st = InterfaceStats()
        self.lib.pfo_interface_diagnostics(g.h, C.byref(pp.as_struct()), C.byref(st))
        return st


    def surface_tension(self, g, pp: PhaseParams, dt, strength, max_delta_speed, smoothing_radius):
        """applySparseSurfaceTension3D (src/driver/interface_diagnostics3d.cpp:405-447)"""
        st = SurfaceStats()
        self.lib.pfo_surface_tension(g.h, C.byref(pp.as_struct()), float(dt), float(strength),
                                     float(max_delta_speed), int(smoothing_radius), C.byref(st))
        return st


def _truncate(ps: Particles, n):
    ps.pos, ps.vel = ps.pos[:n].copy(), ps.vel[:n].copy()
    ps.type, ps.volume = ps.type[:n].copy(), ps.volume[:n].copy()


class Reference:
    """Per-call API of the compiled, unmodified reference."""
    Grid = ReferenceGrid
    name = "reference"

    def __init__(self):
        self.lib = ref_lib()

    def phi_from_raw(self, raw, pp: PhaseParams):
        return self.lib.pfr_phi_from_raw(float(raw), pp.as_array())

    def beta_from_raw(self, raw, pp: PhaseParams):
        return self.lib.pfr_beta_from_raw(float(raw), pp.as_array())

    def calibrate_rho_tilde0(self, pp: PhaseParams, Vp):
        return self.lib.pfr_calibrate_rho_tilde0(pp.as_array(), float(Vp))

    def p2g(self, g: ReferenceGrid, ps: Particles, pp: PhaseParams, Vp):
        g._put(ps)
        self.lib.pfr_p2g(g.h, pp.as_array(), float(Vp))

    def project(self, g, pp: PhaseParams, dt, cg_iters, cg_tol, c_div=0.0):
        self.lib.pfr_project(g.h, pp.as_array(), float(dt), int(cg_iters), float(cg_tol), float(c_div))

    def g2p(self, g, ps: Particles, saved, aL, aG):
        g._put(ps)
        self.lib.pfr_g2p(g.h, saved.h, float(aL), float(aG))
        g._take(ps)

    def advect(self, ps: Particles, g, dt, order=2, escape=False):
        g._put(ps)
        st = np.zeros(8, np.int32)
        n_esc = C.c_size_t()
        buf = np.zeros((max(len(ps), 1), 8), np.float64) if escape else None
        self.lib.pfr_advect(g.h, float(dt), int(order), st, buf.ctypes.data if escape else None,
                            C.byref(n_esc))
        g._take(ps)
        cs = ClampStats(*[int(v) for v in st])
        if escape:
            return cs, buf[: n_esc.value].copy()
        return cs

    def step(self, g: ReferenceGrid, ps: Particles, pp: PhaseParams, cfg: dict, put=True, take=True):
        if put:
            g._put(ps)
        arr = np.array([cfg["dt"], cfg["gravity"], cfg["Vp"], cfg["alpha_l"], cfg["alpha_g"],
                        cfg["cg_iters"], cfg["cg_tol"], cfg.get("advect_order", 2)], np.float64)
        self.lib.pfr_step(g.h, pp.as_array(), arr)
        if take:
            g._take(ps)

    def interface_diagnostics(self, g: ReferenceGrid, pp: PhaseParams):
        iv, dv = np.zeros(4, np.int32), np.zeros(7, np.float64)
        self.lib.pfr_interface_diagnostics(g.h, pp.as_array(), iv, dv)
        return InterfaceStats(*[int(v) for v in iv], *[float(v) for v in dv])

    def surface_tension(self, g: ReferenceGrid, pp: PhaseParams, dt, strength, max_delta_speed, smoothing_radius):
        iv, dv = np.zeros(5, np.int32), np.zeros(9, np.float64)
        self.lib.pfr_surface_tension(g.h, pp.as_array(), float(dt), float(strength), float(max_delta_speed),
                                     int(smoothing_radius), iv, dv)
        return SurfaceStats(*[int(v) for v in iv], *[float(v) for v in dv])

    # ---- particle adaptivity, the reference's own pa3d functions ----
    def narrow_band_air(self, g: ReferenceGrid, ps: Particles, radius=2):
        g._put(ps)
        out = np.zeros(4, np.int32)
        self.lib.pfr_narrow_band_air(g.h, int(radius), out)
        g._take(ps)
        return BandStats(*[int(v) for v in out])

    def coarsen_particles(self, g: ReferenceGrid, ps: Particles, ptype, target, seed):
        g._put(ps)
        out = np.zeros(5, np.int32)
        self.lib.pfr_coarsen_particles(g.h, int(ptype), int(target), int(seed) & 0xffffffff, out)
        g._take(ps)
        return CoarsenStats(*[int(v) for v in out])

    def refill_liquid(self, g: ReferenceGrid, ps: Particles, target, seed, interface_only=False,
                      interface_radius=1, max_added=0):
        g._put(ps)
        out = np.zeros(7, np.int32)
        self.lib.pfr_refill_liquid(g.h, int(target), int(seed) & 0xffffffff, int(bool(interface_only)),
                                   int(interface_radius), int(max_added), out)
        g._take(ps)
        return RefillStats(*[int(v) for v in out])


def build(quiet=True):
    """Compile the checkers (make -C oracle)."""
    import subprocess
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def build_reference_tests(quiet=True):
    """Build the reference's doctest cases against the GPU drop-in
    (make -C oracle ref_tests; needs libpfgpu.so built first)."""
    import subprocess
    out = subprocess.run(["make", "-C", HERE, "ref_tests"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("reference test build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)
