"""Host-side mirror of the reference's sparse 3D two-phase interface over libpfgpu.

Names, argument meaning and argument order follow the reference:
  spP2G3D_tp / spProjectStepVC3D / spG2P3D_tp / spAdvect3D_tp
    (src/driver/sparse_ops3d_tp.h:8-15), SparseMacGrid3D<4>
    (src/grid/sparse_mac_grid3d.h:6-47), Particles3DTP
    (src/particles/particles3d_tp.h:4-35), PhaseParams and the Eq. 7 helpers
    (src/physics/phasefield.h:4-18), ParticleEscapeStats3D/Buffer3D
    (src/driver/particle_escape3d.h), SparseSim3DTP::step
    (src/driver/sparse_sim3d_tp.cpp:854-884).

A SparseMacGrid3D owns one libpfgpu context (device-resident tile pool and a
particle buffer).  The per-call functions move the caller's FP64 particle
arrays in and out of that context around each call, as the reference's
in-place mutation of Particles3DTP implies; SparseSim3DTP keeps the particles
on the device across steps.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

FIELD_NAMES = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")


# ---------------------------------------------------------------------------
# phase field (src/physics/phasefield.h)
# ---------------------------------------------------------------------------

@dataclass
class PhaseParams:
    """PhaseParams (src/physics/phasefield.h:4-9)."""
    rho_l: float = 1.0
    rho_g: float = 0.01
    alpha_phi: float = 1.0
    rho_tilde_0: float = 1.0

    def _c(self):
        return L.Phase(self.rho_l, self.rho_g, self.alpha_phi, self.rho_tilde_0)


def etaPhi(pp: PhaseParams) -> float:
    return math.log(pp.rho_l / pp.rho_g)


def phiFromRawDensity(rt: float, pp: PhaseParams) -> float:
    rmin = etaPhi(pp) * pp.rho_g * pp.rho_tilde_0
    if rt < rmin:
        return 0.0
    v = math.sqrt(max(rt - rmin, 0.0) / (pp.alpha_phi * pp.rho_tilde_0 * pp.rho_l))
    return min(v, 1.0)


def densityFromPhi(phi: float, pp: PhaseParams) -> float:
    return phi * pp.rho_l + (1.0 - phi) * pp.rho_g


def betaFromPhi(phi: float, pp: PhaseParams) -> float:
    return 1.0 / densityFromPhi(phi, pp)


# ---------------------------------------------------------------------------
# particles (src/particles/particles3d_tp.h)
# ---------------------------------------------------------------------------

class Particles3DTP:
    """Particles3DTP: pos/vel (n,3) float64, type uint8 (0 liquid, 1 gas), volume float64."""

    def __init__(self, pos=None, vel=None, type=None, volume=None):
        n = 0 if pos is None else len(pos)
        self.pos = np.ascontiguousarray(np.zeros((n, 3)) if pos is None else pos, np.float64).reshape(n, 3)
        self.vel = np.ascontiguousarray(np.zeros((n, 3)) if vel is None else vel, np.float64).reshape(n, 3)
        self.type = np.ascontiguousarray(np.zeros(n) if type is None else type, np.uint8).reshape(n)
        self.volume = np.ascontiguousarray(np.ones(n) if volume is None else volume, np.float64).reshape(n)

    def size(self):
        return len(self.pos)

    __len__ = size

    def add(self, p, v, t, vol=1.0):
        self.pos = np.vstack([self.pos, np.asarray(p, np.float64).reshape(1, 3)])
        self.vel = np.vstack([self.vel, np.asarray(v, np.float64).reshape(1, 3)])
        self.type = np.append(self.type, np.uint8(t)).astype(np.uint8)
        self.volume = np.append(self.volume, float(vol))

    def copy(self):
        return Particles3DTP(self.pos.copy(), self.vel.copy(), self.type.copy(), self.volume.copy())


@dataclass
class ParticleEscapeStats3D:
    """ParticleEscapeStats3D (src/driver/particle_escape3d.h:38-80)."""
    clamped_liquid: int = 0
    clamped_gas: int = 0
    clamped_x_lo: int = 0
    clamped_x_hi: int = 0
    clamped_y_lo: int = 0
    clamped_y_hi: int = 0
    clamped_z_lo: int = 0
    clamped_z_hi: int = 0

    def clamped_total(self):
        return self.clamped_liquid + self.clamped_gas

    def droplet_candidates(self):
        return self.clamped_liquid

    def bubble_candidates(self):
        return self.clamped_gas


@dataclass
class ParticleEscapeBuffer3D:
    """ParticleEscapeBuffer3D: records (type, pos, vel, volume) of clamped particles in order."""
    records: list = field(default_factory=list)

    def droplet_count(self):
        return sum(1 for r in self.records if r["type"] == 0)

    def bubble_count(self):
        return sum(1 for r in self.records if r["type"] == 1)


@dataclass
class SolverConfig:
    """Pressure solver selection beyond the reference's (cg_iters, cg_tol)."""
    mode: int = L.PF_SOLVER_PLAIN
    rel_tol: float = 0.0
    bf16_storage: int = 0  # 1: BF16 couplings in the mixed inner solve; 2: also its search direction
    check_every: int = 0
    max_refine: int = 0
    inner_rel_tol: float = 0.0
    precond: int = L.PF_PRECOND_NETWORK
    accept_min_gain: float = 0.0
    inner_fp32: bool = False
    inner_max_iter: int = 0

    def _c(self, cg_iters, cg_tol, c_div) -> L.SolveCfg:
        return L.SolveCfg(int(self.mode), int(cg_iters), float(cg_tol), float(self.rel_tol), float(c_div),
                          int(self.bf16_storage), int(self.check_every), int(self.max_refine),
                          float(self.inner_rel_tol), int(self.precond), float(self.accept_min_gain),
                          int(bool(self.inner_fp32)), int(self.inner_max_iter))


# ---------------------------------------------------------------------------
# grid (src/grid/sparse_mac_grid3d.h)
# ---------------------------------------------------------------------------

def _field_dims(nx, ny, nz, f):
    return [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1), (nx + 1, ny, nz), (nx, ny + 1, nz),
            (nx, ny, nz + 1), (nx, ny, nz), (nx, ny, nz)][f]


class SparseMacGrid3D:
    """GPU-resident SparseMacGrid3D<4>: eight sparse fields in a pool of 8^3
    tiles, reference-granular (4^3) activity per field."""

    def __init__(self, nx, ny, nz, dx, origin=(0.0, 0.0, 0.0), max_particles=1 << 16, device=0):
        self.lib = L.load()
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(dx)
        self.ox, self.oy, self.oz = (float(o) for o in origin)
        self.device = int(device)
        self.max_particles = int(max_particles)
        d = L.GridDesc(self.nx, self.ny, self.nz, self.dx, self.ox, self.oy, self.oz, self.max_particles,
                       self.device)
        h = C.c_void_p()
        rc = self.lib.pf_create(C.byref(d), C.byref(h))
        L.check(rc, None, "pf_create")
        self.ctx = h.value

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.pf_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- shape helpers --
    def dims(self, f):
        return _field_dims(self.nx, self.ny, self.nz, f)

    def bdims(self, f):
        X, Y, Z = self.dims(f)
        return ((X + 3) // 4, (Y + 3) // 4, (Z + 3) // 4)

    def inBounds(self, i, j, k):
        return 0 <= i < self.nx and 0 <= j < self.ny and 0 <= k < self.nz

    # -- field exchange --
    def get_field(self, f):
        X, Y, Z = self.dims(f)
        bx, by, bz = self.bdims(f)
        dense = np.zeros((Z, Y, X), np.float32)
        act = np.zeros((bz, by, bx), np.uint8)
        rc = self.lib.pf_grid_get_field(self.ctx, f, dense.ctypes.data, act.ctypes.data)
        L.check(rc, self.ctx, "pf_grid_get_field")
        return dense, act

    def set_field(self, f, dense, act):
        X, Y, Z = self.dims(f)
        dense = np.ascontiguousarray(dense, np.float32).reshape(Z, Y, X)
        act = np.ascontiguousarray(act, np.uint8).reshape(self.bdims(f)[::-1])
        rc = self.lib.pf_grid_set_field(self.ctx, f, dense.ctypes.data, act.ctypes.data)
        L.check(rc, self.ctx, "pf_grid_set_field")

    def set_values(self, f, values):
        """Write a dense (Z,Y,X) array; nonzero nodes activate their 4^3 block
        (the reference's ref() on every written node)."""
        v = np.asarray(values, np.float32)
        X, Y, Z = self.dims(f)
        act = np.zeros(self.bdims(f)[::-1], np.uint8)
        kk, jj, ii = np.nonzero(v)
        act[kk // 4, jj // 4, ii // 4] = 1
        self.set_field(f, v, act)

    def set_cells(self, markers):
        """Marker field from a dense (nz,ny,nx) int array (SparseMacGrid3D::setCell)."""
        self.set_values(L.PF_MK, np.asarray(markers, np.float32))

    def field(self, f):
        return self.get_field(f)[0]

    def clear_field(self, f):
        L.check(self.lib.pf_grid_clear_field(self.ctx, f), self.ctx, "pf_grid_clear_field")

    def clearAll(self):
        L.check(self.lib.pf_grid_clear_all(self.ctx), self.ctx, "pf_grid_clear_all")

    def copy(self):
        g = SparseMacGrid3D(self.nx, self.ny, self.nz, self.dx, (self.ox, self.oy, self.oz),
                            max_particles=1, device=self.device)
        L.check(self.lib.pf_grid_copy(g.ctx, self.ctx), g.ctx, "pf_grid_copy")
        return g

    def active_blocks(self, f):
        """Sorted ids (bx + nbx*(by + nby*bz)) of the active 4^3 blocks of field f."""
        n = C.c_size_t()
        L.check(self.lib.pf_active_blocks4(self.ctx, f, None, C.byref(n)), self.ctx, "pf_active_blocks4")
        out = np.zeros(max(n.value, 1), np.int32)
        L.check(self.lib.pf_active_blocks4(self.ctx, f, out.ctypes.data, C.byref(n)), self.ctx, "pf_active_blocks4")
        return out[: n.value].astype(np.int64)

    def activeBlockCount(self, f):
        return len(self.active_blocks(f))

    def activeCellBlocks(self):
        return self.activeBlockCount(L.PF_P)

    def fluid_cells(self):
        """collectCellsWithMarker(g, 1): fluid cells ascending in i + nx*(j + ny*k)."""
        n = C.c_size_t()
        L.check(self.lib.pf_active_cells(self.ctx, None, C.byref(n)), self.ctx, "pf_active_cells")
        out = np.zeros(max(n.value, 1), np.int32)
        L.check(self.lib.pf_active_cells(self.ctx, out.ctypes.data, C.byref(n)), self.ctx, "pf_active_cells")
        return out[: n.value].astype(np.int64)

    def active_tiles(self):
        return int(self.lib.pf_active_tiles(self.ctx))

    def cell_markers(self):
        return (self.field(L.PF_MK) + np.float32(0.5)).astype(np.int32)

    # -- particle exchange --
    def _ensure_capacity(self, n):
        if n > self.max_particles:
            raise L.PfError(L.PF_ERR_CAPACITY, f"{n} particles > max_particles={self.max_particles}")

    def upload(self, ps):
        n = len(ps.pos)
        self._ensure_capacity(n)
        pos = np.ascontiguousarray(ps.pos, np.float64)
        vel = np.ascontiguousarray(ps.vel, np.float64)
        typ = np.ascontiguousarray(ps.type, np.uint8)
        vol = np.ascontiguousarray(ps.volume, np.float64)
        rc = self.lib.pf_upload_particles_f64(self.ctx, n, pos.ctypes.data, vel.ctypes.data, typ.ctypes.data,
                                              vol.ctypes.data)
        L.check(rc, self.ctx, "pf_upload_particles_f64")

    def take_particles(self, ps):
        """Download the whole device particle set into ps (its count may have changed)."""
        n = int(self.lib.pf_num_particles(self.ctx))
        P, V = np.empty((n, 3), np.float64), np.empty((n, 3), np.float64)
        T, W = np.empty(n, np.uint8), np.empty(n, np.float64)
        if n:
            rc = self.lib.pf_download_particles_f64(self.ctx, P.ctypes.data, V.ctypes.data, T.ctypes.data,
                                                    W.ctypes.data)
            L.check(rc, self.ctx, "pf_download_particles_f64")
        ps.pos, ps.vel, ps.type, ps.volume = P, V, T, W

    def download(self, ps, pos=True, vel=True):
        n = len(ps.pos)
        if n == 0:
            return
        P = np.empty((n, 3), np.float64) if pos else None
        V = np.empty((n, 3), np.float64) if vel else None
        rc = self.lib.pf_download_particles_f64(self.ctx, P.ctypes.data if pos else None,
                                                V.ctypes.data if vel else None, None, None)
        L.check(rc, self.ctx, "pf_download_particles_f64")
        if pos:
            ps.pos = P
        if vel:
            ps.vel = V


# ---------------------------------------------------------------------------
# per-call drop-ins (src/driver/sparse_ops3d_tp.h:8-15)
# ---------------------------------------------------------------------------

def calibrateRhoTilde0(pp: PhaseParams, Vp: float, grid: SparseMacGrid3D | None = None) -> float:
    """calibrateRhoTilde0 (src/transfer/transfer3d_tp.cpp:29-36) on the GPU."""
    g = grid or SparseMacGrid3D(8, 8, 8, 1.0, max_particles=1)
    out = C.c_double()
    L.check(g.lib.pf_calibrate_rho_tilde0(g.ctx, C.byref(pp._c()), float(Vp), C.byref(out)), g.ctx,
            "pf_calibrate_rho_tilde0")
    return out.value


def spP2G3D_tp(g: SparseMacGrid3D, ps, pp: PhaseParams, Vp: float):
    g.upload(ps)
    L.check(g.lib.pf_p2g(g.ctx, C.byref(pp._c()), float(Vp)), g.ctx, "pf_p2g")


def spProjectStepVC3D(g: SparseMacGrid3D, pp: PhaseParams, dt, cg_iters, cg_tol, divergenceCorrection=0.0,
                      solver: SolverConfig | None = None) -> L.SolveStats:
    s = solver or SolverConfig()
    cfg = s._c(cg_iters, cg_tol, divergenceCorrection)
    st = L.SolveStats()
    L.check(g.lib.pf_project(g.ctx, C.byref(pp._c()), float(dt), C.byref(cfg), C.byref(st)), g.ctx,
            "pf_project")
    return st


def spG2P3D_tp(g: SparseMacGrid3D, ps, saved: SparseMacGrid3D, aL, aG):
    g.upload(ps)
    L.check(g.lib.pf_g2p(g.ctx, saved.ctx if saved is not None else None, float(aL), float(aG)), g.ctx,
            "pf_g2p")
    g.download(ps, pos=False, vel=True)


def spAdvect3D_tp(ps, g: SparseMacGrid3D, dt, stats: ParticleEscapeStats3D | None = None, advectionOrder=2,
                  escapeBuffer: ParticleEscapeBuffer3D | None = None):
    g.upload(ps)
    cs = L.ClampStats()
    n = len(ps.pos)
    esc = np.zeros((max(n, 1), 8), np.float64) if escapeBuffer is not None else None
    nesc = C.c_size_t()
    rc = g.lib.pf_advect(g.ctx, float(dt), int(advectionOrder), C.byref(cs),
                         esc.ctypes.data if esc is not None else None, C.byref(nesc))
    L.check(rc, g.ctx, "pf_advect")
    g.download(ps, pos=True, vel=False)
    if stats is not None:
        (stats.clamped_liquid, stats.clamped_gas, stats.clamped_x_lo, stats.clamped_x_hi, stats.clamped_y_lo,
         stats.clamped_y_hi, stats.clamped_z_lo, stats.clamped_z_hi) = cs.as_tuple()
    if escapeBuffer is not None:
        for r in esc[: nesc.value]:
            escapeBuffer.records.append({"type": int(r[0]), "pos": r[1:4].copy(), "vel": r[4:7].copy(),
                                         "volume": float(r[7])})
    return cs


# ---------------------------------------------------------------------------
# device-resident step (SparseSim3DTP)
# ---------------------------------------------------------------------------

def diagnoseSparseInterface3D(g: SparseMacGrid3D, pp: PhaseParams) -> L.InterfaceStats:
    """diagnoseSparseInterface3D (src/driver/interface_diagnostics3d.cpp:363-379) on the device."""
    st = L.InterfaceStats()
    L.check(g.lib.pf_interface_diagnostics(g.ctx, C.byref(pp._c()), C.byref(st)), g.ctx, "pf_interface_diagnostics")
    return st


def defaultRenderCacheCamera3D(nx, ny, nz, dx) -> L.RenderCamera:
    """defaultRenderCacheCamera3D (src/driver/render_cache3d.h:47-61)."""
    cam = L.RenderCamera()
    L.check(L.load().pf_default_render_camera(int(nx), int(ny), int(nz), float(dx), C.byref(cam)), None,
            "pf_default_render_camera")
    return cam


def writeSparseRenderCache3D(sim, path, frame, time, camera=None) -> int:
    """writeSparseRenderCache3D (src/driver/render_cache3d.h:551-600): one JSONL
    frame of the simulation's grid and particles, phase cells compacted on the
    device.  Returns the bytes written; raises on an empty path or invalid
    metadata, as the reference does."""
    if not str(path):
        raise RuntimeError("render cache path is empty")
    g = sim.grid
    nbytes = C.c_longlong(0)
    cam = C.byref(camera) if camera is not None else None
    L.check(g.lib.pf_write_render_cache(g.ctx, str(path).encode(), int(frame), float(time),
                                        float(sim.effective_dt_last), C.byref(sim.phase._c()), float(sim.Vp), cam,
                                        C.byref(nbytes)), g.ctx, "pf_write_render_cache")
    return int(nbytes.value)


@dataclass
class RenderCacheManifestFrame3D:
    """RenderCacheManifestFrame3D (src/driver/render_cache3d.h:39-45)."""
    frame: int = 0
    step: int = 0
    time: float = 0.0
    path: str = ""
    bytes: int = 0


def writeRenderCacheManifest3D(path, simKind, nx, ny, nz, dx, frames):
    """writeRenderCacheManifest3D (src/driver/render_cache3d.h:711-755): the
    JSON manifest of a frame sequence, written by the library's host code
    (pf_write_render_manifest; no device needed).  Raises on the reference's
    invalid arguments."""
    lib = L.load()
    keep = [str(f.path).encode() for f in frames]
    arr = (L.RenderManifestFrame * max(1, len(frames)))(
        *[L.RenderManifestFrame(int(f.frame), int(f.step), float(f.time), p, int(f.bytes)) for f, p in zip(frames, keep)])
    rc = lib.pf_write_render_manifest(str(path).encode(), str(simKind).encode(), int(nx), int(ny), int(nz), float(dx),
                                      arr, len(frames))
    if rc:
        raise ValueError("invalid render cache manifest metadata or unwritable path")


def applySparseSurfaceTension3D(g: SparseMacGrid3D, pp: PhaseParams, dt, strength, maxDeltaSpeed,
                                curvatureSmoothingRadius) -> L.SurfaceStats:
    """applySparseSurfaceTension3D (src/driver/interface_diagnostics3d.cpp:405-447) on the device."""
    st = L.SurfaceStats()
    L.check(g.lib.pf_surface_tension(g.ctx, C.byref(pp._c()), float(dt), float(strength), float(maxDeltaSpeed),
                                     int(curvatureSmoothingRadius), C.byref(st)), g.ctx, "pf_surface_tension")
    return st


# ---------------------------------------------------------------------------
# particle adaptivity (src/driver/particle_adaptivity3d.h), on the device; the
# grid supplies the cell domain (ParticleCellDomain3D) and holds the particles
# for the call
# ---------------------------------------------------------------------------

def applyNarrowBandAir(particles, grid: SparseMacGrid3D, enabled=True, radius=2) -> L.BandStats:
    """pa3d::applyNarrowBandAir (src/driver/particle_adaptivity3d.h:111-166)."""
    st = L.BandStats()
    if not enabled:
        return st
    grid.upload(particles)
    L.check(grid.lib.pf_narrow_band_air(grid.ctx, int(radius), C.byref(st)), grid.ctx, "pf_narrow_band_air")
    grid.take_particles(particles)
    return st


def applyTypedParticleCoarsening(particles, grid: SparseMacGrid3D, enabled=True, particleType=1,
                                 particlesPerCellTarget=4, seed=0x9e3779b9) -> L.CoarsenStats:
    """pa3d::applyTypedParticleCoarsening (src/driver/particle_adaptivity3d.h:168-248)."""
    st = L.CoarsenStats()
    if not enabled:
        return st
    grid.upload(particles)
    rc = grid.lib.pf_coarsen_particles(grid.ctx, int(particleType), int(particlesPerCellTarget),
                                       int(seed) & 0xffffffff, C.byref(st))
    L.check(rc, grid.ctx, "pf_coarsen_particles")
    grid.take_particles(particles)
    return st


def applyGasParticleCoarsening(particles, grid: SparseMacGrid3D, enabled=True, particlesPerCellTarget=4,
                               seed=0x9e3779b9) -> L.CoarsenStats:
    """pa3d::applyGasParticleCoarsening (src/driver/particle_adaptivity3d.h:250-262)."""
    return applyTypedParticleCoarsening(particles, grid, enabled, 1, particlesPerCellTarget, seed)


def applyLiquidParticleRefill(particles, grid: SparseMacGrid3D, enabled=True, particlesPerCellTarget=4,
                              seed=0x6a09e667, interfaceOnly=False, interfaceRadius=1,
                              maxAddedPerStep=0) -> L.RefillStats:
    """pa3d::applyLiquidParticleRefill (src/driver/particle_adaptivity3d.h:264-374).  The grid's
    max_particles must hold the particles after the refill (PfError PF_ERR_CAPACITY otherwise)."""
    st = L.RefillStats()
    if not enabled:
        return st
    grid.upload(particles)
    rc = grid.lib.pf_refill_liquid(grid.ctx, int(particlesPerCellTarget), int(seed) & 0xffffffff,
                                   int(bool(interfaceOnly)), int(interfaceRadius), int(maxAddedPerStep),
                                   C.byref(st))
    L.check(rc, grid.ctx, "pf_refill_liquid")
    grid.take_particles(particles)
    return st


# SparseSim3DTP's secondary-particle totals and the per-step statistic each accumulates
_SECONDARY_TOTALS = {
    "secondary_droplets_advected": "advected_droplets", "secondary_bubbles_advected": "advected_bubbles",
    "secondary_droplets_reabsorbed": "reabsorbed_droplets", "secondary_bubbles_reabsorbed": "reabsorbed_bubbles",
    "secondary_droplets_expired": "expired_droplets", "secondary_bubbles_expired": "expired_bubbles",
    "secondary_droplets_dragged": "dragged_droplets", "secondary_bubbles_dragged": "dragged_bubbles",
    "secondary_droplets_reabsorbed_to_primary": "reabsorbed_droplets_to_primary",
    "secondary_bubbles_reabsorbed_to_primary": "reabsorbed_bubbles_to_primary",
    "secondary_droplet_volume_reabsorbed": "reabsorbed_droplet_volume",
    "secondary_bubble_volume_reabsorbed": "reabsorbed_bubble_volume",
    "secondary_droplet_volume_expired": "expired_droplet_volume",
    "secondary_bubble_volume_expired": "expired_bubble_volume",
    "secondary_droplet_volume_reabsorbed_to_primary": "reabsorbed_droplet_volume_to_primary",
    "secondary_bubble_volume_reabsorbed_to_primary": "reabsorbed_bubble_volume_to_primary",
    "secondary_spray_emitted_droplets": "spray_emitted_droplets",
    "secondary_spray_emitted_bubbles": "spray_emitted_bubbles",
    "secondary_spray_emitted_droplet_volume": "spray_emitted_droplet_volume",
    "secondary_spray_emitted_bubble_volume": "spray_emitted_bubble_volume",
    "escaped_droplets_added": None, "escaped_bubbles_added": None,
    "escaped_droplet_volume_added": None, "escaped_bubble_volume_added": None,
}


class SparseSim3DTP:
    """SparseSim3DTP with particles resident on the GPU; step() runs
    markCells, P2G, saved copy, gravity, walls, projection, G2P and
    advection in the reference's order (src/driver/sparse_sim3d_tp.cpp:854-884).
    Defaults follow src/driver/sparse_sim3d_tp.h:12-28."""

    def __init__(self, nx, ny, nz, dx, max_particles=1 << 20, device=0):
        self.grid = SparseMacGrid3D(nx, ny, nz, dx, max_particles=max_particles, device=device)
        self.phase = PhaseParams()
        self.dt, self.gravity, self.Vp = 0.02, -9.81, 1.0
        self.alpha_liquid = self.alpha_gas = 0.95
        self.advection_order = 2
        self.cg_iters, self.cg_tol = 600, 1e-7
        self.c_div_last = 0.0
        self.solver = SolverConfig()
        self.n = 0
        self.last_stats = None
        # particle adaptivity switches (src/driver/sparse_sim3d_tp.h:29-66), all off by default
        self.narrow_band_air, self.narrow_band_air_radius = False, 2
        self.gas_particle_coarsening, self.gas_particles_per_cell_target = False, 4
        self.gas_particle_coarsening_seed = 0x9e3779b9
        self.liquid_particle_coarsening, self.liquid_particles_per_cell_target = False, 4
        self.liquid_particle_coarsening_seed = 0x7f4a7c15
        self.liquid_particle_refill, self.liquid_refill_particles_per_cell_target = False, 4
        self.liquid_particle_refill_seed = 0x6a09e667
        self.liquid_particle_refill_interface_only = False
        self.liquid_particle_refill_interface_radius = 1
        self.liquid_particle_refill_max_added_per_step = 0
        self.adaptivity_last = L.AdaptStats()
        self.interface_diagnostics_last = L.InterfaceStats()
        # surface tension (src/driver/sparse_sim3d_tp.h:156-159), off by default
        self.surface_tension, self.surface_tension_strength = False, 0.02
        self.surface_tension_max_delta_speed, self.surface_tension_curvature_smoothing_radius = 0.25, 0
        self.surface_tension_stats_last = L.SurfaceStats()
        # adaptive timestep and volume correction (src/driver/sparse_sim3d_tp.h:13-26), off by default
        self.adaptive_timestep, self.adaptive_cfl, self.adaptive_min_dt = False, 0.5, 1e-5
        self.c_div_volume_correction, self.c_div_strength, self.liquid_volume_target = False, 1.0, 0.0
        self.effective_dt_last, self.max_particle_speed_last, self.cfl_limit_dt_last = self.dt, 0.0, self.dt
        self.adaptive_timestep_limited_last = 0
        self.liquid_volume_current_last = self.liquid_volume_error_last = 0.0
        # secondary particles (src/driver/sparse_sim3d_tp.h:82-137), off by default
        self.escaped_particle_branching = False
        self.secondary_particle_lifecycle = False
        self.secondary_droplet_lifetime_steps = self.secondary_bubble_lifetime_steps = 48
        self.secondary_velocity_damping, self.secondary_reabsorb_margin_cells = 0.98, 1.0
        self.secondary_droplet_gravity_scale, self.secondary_bubble_buoyancy_scale = 1.0, 0.25
        self.secondary_droplet_drag = self.secondary_bubble_drag = 0.0
        self.secondary_reabsorb_to_primary = False
        self.secondary_spray_emission, self.secondary_spray_particles_per_step = False, 0
        self.secondary_spray_droplet_fraction = 0.9
        self.secondary_spray_droplet_volume, self.secondary_spray_bubble_volume = 0.55, 0.45
        self.secondary_spray_interface_gate, self.secondary_spray_min_interface_cells = False, 1
        self.secondary_spray_min_interface_grad_max = 1e-5
        self.secondary_spray_min_interface_curvature_abs_max = 0.0
        self.secondary_spray_impact_candidates = False
        self.secondary_spray_impact_region_fraction = 0.55
        self.secondary_spray_impact_downward_speed_min = 1.0
        self.secondary_spray_impact_foam_fraction = 0.3
        self.secondary_stats_last = L.SecondaryStats()
        self.secondary_spray_emission_step_index = 0
        self.secondary_totals = {k: 0 for k in _SECONDARY_TOTALS}
        self._secondary_configured = False

    def set_particles(self, pos, vel, type, volume):
        """Upload FP32 (n,3) pos/vel, uint8 type, FP32 volume (host or device pointers via numpy)."""
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        typ = np.ascontiguousarray(type, np.uint8)
        vol = np.ascontiguousarray(volume, np.float32)
        n = len(pos)
        self.grid._ensure_capacity(n)
        rc = self.grid.lib.pf_upload_particles(self.grid.ctx, n, pos.ctypes.data, vel.ctypes.data,
                                               typ.ctypes.data, vol.ctypes.data)
        L.check(rc, self.grid.ctx, "pf_upload_particles")
        self.n = n

    def seed_scene(self, scene, seed=0):
        """Seed the resident particle set on the device with a benchmark scene
        ("rayleigh_taylor", "bubble_tank" or "dam_break", pf_seed_scene): the
        particles the scenes module's generator of that name gives for this
        grid and seed.
        Returns the particle count."""
        kind = {"rayleigh_taylor": L.PF_SCENE_RAYLEIGH_TAYLOR, "bubble_tank": L.PF_SCENE_BUBBLE_TANK,
                "dam_break": L.PF_SCENE_DAM_BREAK}[scene]
        n = C.c_size_t()
        L.check(self.grid.lib.pf_seed_scene(self.grid.ctx, kind, int(seed), C.byref(n)), self.grid.ctx, "pf_seed_scene")
        self.n = int(n.value)
        return self.n

    def get_particles(self):
        n = self.n = int(self.grid.lib.pf_num_particles(self.grid.ctx))
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        typ = np.empty(n, np.uint8)
        vol = np.empty(n, np.float32)
        rc = self.grid.lib.pf_download_particles(self.grid.ctx, pos.ctypes.data, vel.ctypes.data, typ.ctypes.data,
                                                 vol.ctypes.data)
        L.check(rc, self.grid.ctx, "pf_download_particles")
        return pos, vel, typ, vol

    def adapt_cfg(self):
        return L.AdaptCfg(
            narrow_band_air=int(self.narrow_band_air), narrow_band_radius=int(self.narrow_band_air_radius),
            gas_coarsening=int(self.gas_particle_coarsening),
            gas_per_cell_target=int(self.gas_particles_per_cell_target),
            gas_seed=int(self.gas_particle_coarsening_seed) & 0xffffffff,
            liquid_coarsening=int(self.liquid_particle_coarsening),
            liquid_per_cell_target=int(self.liquid_particles_per_cell_target),
            liquid_seed=int(self.liquid_particle_coarsening_seed) & 0xffffffff,
            liquid_refill=int(self.liquid_particle_refill),
            refill_per_cell_target=int(self.liquid_refill_particles_per_cell_target),
            refill_seed=int(self.liquid_particle_refill_seed) & 0xffffffff,
            refill_interface_only=int(self.liquid_particle_refill_interface_only),
            refill_interface_radius=int(self.liquid_particle_refill_interface_radius),
            refill_max_added=int(self.liquid_particle_refill_max_added_per_step))

    def _adaptivity_on(self):
        return (self.narrow_band_air or self.gas_particle_coarsening or self.liquid_particle_coarsening
                or self.liquid_particle_refill)

    def applyParticleAdaptivity(self):
        """SparseSim3DTP::applyParticleAdaptivity (src/driver/sparse_sim3d_tp.cpp:843-848) on the resident
        particles: narrow band, gas coarsening, liquid coarsening, liquid refill, each when switched on."""
        a, out = self.adapt_cfg(), L.AdaptStats()
        ctx, lib = self.grid.ctx, self.grid.lib
        if a.narrow_band_air:
            L.check(lib.pf_narrow_band_air(ctx, a.narrow_band_radius, C.byref(out.band)), ctx, "pf_narrow_band_air")
        if a.gas_coarsening:
            L.check(lib.pf_coarsen_particles(ctx, 1, a.gas_per_cell_target, a.gas_seed, C.byref(out.gas)), ctx,
                    "pf_coarsen_particles")
        if a.liquid_coarsening:
            L.check(lib.pf_coarsen_particles(ctx, 0, a.liquid_per_cell_target, a.liquid_seed, C.byref(out.liquid)),
                    ctx, "pf_coarsen_particles")
        if a.liquid_refill:
            L.check(lib.pf_refill_liquid(ctx, a.refill_per_cell_target, a.refill_seed, a.refill_interface_only,
                                         a.refill_interface_radius, a.refill_max_added, C.byref(out.refill)), ctx,
                    "pf_refill_liquid")
        self.adaptivity_last = out
        self.n = int(lib.pf_num_particles(ctx))
        return out

    def secondary_cfg(self) -> L.SecondaryCfg:
        return L.SecondaryCfg(
            int(self.escaped_particle_branching), int(self.secondary_particle_lifecycle),
            int(self.secondary_droplet_lifetime_steps), int(self.secondary_bubble_lifetime_steps),
            float(self.secondary_velocity_damping), float(self.secondary_reabsorb_margin_cells),
            float(self.secondary_droplet_gravity_scale), float(self.secondary_bubble_buoyancy_scale),
            float(self.secondary_droplet_drag), float(self.secondary_bubble_drag),
            int(self.secondary_reabsorb_to_primary), int(self.secondary_spray_emission),
            int(self.secondary_spray_particles_per_step), float(self.secondary_spray_droplet_fraction),
            float(self.secondary_spray_droplet_volume), float(self.secondary_spray_bubble_volume),
            int(self.secondary_spray_interface_gate), int(self.secondary_spray_min_interface_cells),
            float(self.secondary_spray_min_interface_grad_max),
            float(self.secondary_spray_min_interface_curvature_abs_max),
            int(self.secondary_spray_impact_candidates), float(self.secondary_spray_impact_region_fraction),
            float(self.secondary_spray_impact_downward_speed_min), float(self.secondary_spray_impact_foam_fraction))

    def _secondary_on(self):
        return self.escaped_particle_branching or self.secondary_particle_lifecycle or self.secondary_spray_emission

    def secondary_set(self, which):
        """The droplet (0) or bubble (1) set: FP64 positions and velocities (n, 3),
        volumes and ages (escaped_droplets / escaped_droplet_ages of the reference)."""
        ctx, lib = self.grid.ctx, self.grid.lib
        n = C.c_size_t()
        L.check(lib.pf_secondary_count(ctx, int(which), C.byref(n)), ctx, "pf_secondary_count")
        n = int(n.value)
        pos, vel = np.zeros((n, 3)), np.zeros((n, 3))
        vol, age = np.zeros(n), np.zeros(n, np.int32)
        if n:
            L.check(lib.pf_get_secondary(ctx, int(which), pos.ctypes.data, vel.ctypes.data, vol.ctypes.data,
                                         age.ctypes.data), ctx, "pf_get_secondary")
        return pos, vel, vol, age

    def set_secondary_set(self, which, pos, vel, vol, age):
        ctx, lib = self.grid.ctx, self.grid.lib
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float64).reshape(-1, 3)
        vol = np.ascontiguousarray(vol, np.float64).reshape(-1)
        age = np.ascontiguousarray(age, np.int32).reshape(-1)
        if not (len(pos) == len(vel) == len(vol) == len(age)):
            raise ValueError("secondary set arrays differ in length")
        L.check(lib.pf_set_secondary_particles(ctx, int(which), len(pos), pos.ctypes.data, vel.ctypes.data,
                                               vol.ctypes.data, age.ctypes.data), ctx, "pf_set_secondary_particles")

    @property
    def escaped_droplets(self):
        return self.secondary_set(0)

    @property
    def escaped_bubbles(self):
        return self.secondary_set(1)

    def _secondary_after_step(self):
        """The reference's *_last and *_total bookkeeping of the secondary
        particles (src/driver/sparse_sim3d_tp.cpp:192-337), from the step's statistics."""
        ctx, lib = self.grid.ctx, self.grid.lib
        st = L.SecondaryStats()
        L.check(lib.pf_get_secondary_stats(ctx, C.byref(st)), ctx, "pf_get_secondary_stats")
        self.secondary_stats_last = st
        self.secondary_spray_emission_step_index = st.spray_step_index
        t = self.secondary_totals
        for key, field in _SECONDARY_TOTALS.items():
            if key.startswith("escaped_"):
                continue
            t[key] += getattr(st, field)
        # storeEscapedParticles adds the escaped particles, emitSecondarySpray the seeds
        t["escaped_droplets_added"] += st.escaped_droplets_added - st.spray_emitted_droplets
        t["escaped_bubbles_added"] += st.escaped_bubbles_added - st.spray_emitted_bubbles
        if self.escaped_particle_branching:
            t["escaped_droplet_volume_added"] += st.escape_droplet_volume
            t["escaped_bubble_volume_added"] += st.escape_bubble_volume
        t["escaped_droplets_added"] += st.spray_emitted_droplets
        t["escaped_bubbles_added"] += st.spray_emitted_bubbles
        t["escaped_droplet_volume_added"] += st.spray_emitted_droplet_volume
        t["escaped_bubble_volume_added"] += st.spray_emitted_bubble_volume

    def step_cfg(self):
        solve = self.solver._c(self.cg_iters, self.cg_tol, self.c_div_last)
        return L.StepCfg(self.dt, self.gravity, self.Vp, self.alpha_liquid, self.alpha_gas, self.phase._c(), solve,
                         int(self.advection_order))

    def step(self):
        cfg = self.step_cfg()
        st = L.StepStats()
        ctx, lib = self.grid.ctx, self.grid.lib
        # the step starts with applyParticleAdaptivity (src/driver/sparse_sim3d_tp.cpp:854-856)
        if self._adaptivity_on():
            ac = self.adapt_cfg()
            L.check(lib.pf_set_adaptivity(ctx, C.byref(ac)), ctx, "pf_set_adaptivity")
        else:
            L.check(lib.pf_set_adaptivity(ctx, None), ctx, "pf_set_adaptivity")
        ctl = L.StepControls(int(self.adaptive_timestep), float(self.adaptive_cfl), float(self.adaptive_min_dt),
                             int(self.c_div_volume_correction), float(self.c_div_strength),
                             float(self.liquid_volume_target))
        L.check(lib.pf_set_step_controls(ctx, C.byref(ctl)), ctx, "pf_set_step_controls")
        L.check(lib.pf_set_surface_tension(ctx, float(self.surface_tension_strength) if self.surface_tension else 0.0,
                                           float(self.surface_tension_max_delta_speed),
                                           int(self.surface_tension_curvature_smoothing_radius)), ctx,
                "pf_set_surface_tension")
        if self._secondary_on():
            sc = self.secondary_cfg()
            L.check(lib.pf_set_secondary(ctx, C.byref(sc)), ctx, "pf_set_secondary")
            self._secondary_configured = True
        elif self._secondary_configured:
            L.check(lib.pf_set_secondary(ctx, None), ctx, "pf_set_secondary")
        L.check(lib.pf_step(ctx, C.byref(cfg), C.byref(st)), ctx, "pf_step")
        if self._secondary_configured:
            self._secondary_after_step()
        L.check(lib.pf_get_surface_stats(ctx, C.byref(self.surface_tension_stats_last)), ctx, "pf_get_surface_stats")
        cs = L.StepControlStats()
        L.check(lib.pf_get_step_control_stats(ctx, C.byref(cs)), ctx, "pf_get_step_control_stats")
        self.effective_dt_last, self.max_particle_speed_last = cs.effective_dt, cs.max_particle_speed
        self.cfl_limit_dt_last, self.adaptive_timestep_limited_last = cs.cfl_limit_dt, cs.limited
        self.liquid_volume_current_last, self.liquid_volume_error_last = cs.liquid_volume_current, cs.liquid_volume_error
        if self.c_div_volume_correction:
            self.c_div_last = cs.c_div
        if self._adaptivity_on():
            L.check(lib.pf_get_adaptivity_stats(ctx, C.byref(self.adaptivity_last)), ctx, "pf_get_adaptivity_stats")
        L.check(lib.pf_get_interface_stats(ctx, C.byref(self.interface_diagnostics_last)), ctx,
                "pf_get_interface_stats")
        self.n = int(lib.pf_num_particles(ctx))
        self.last_stats = st
        return st
