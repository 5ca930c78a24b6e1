"""The reference's 2-level multires simulation (MRSim3DTP,
src/driver/multires_sim3d_tp.h:10-191) with particles and grid on the GPU.

``MRSim3DTP.step()`` runs pf_mr_step: updateDynamicRefinement, markCells,
mrP2G3D_tp, the saved copy, gravity, walls, projectMR3D (Jacobi PCG with
adaptive restart and optional flexible beta), mrG2P3D_tp and mrAdvect3D_tp
(src/driver/multires_sim3d_tp.cpp:671-733).  Settings and defaults follow
src/driver/multires_sim3d_tp.h:15-67; the coarse-correction, coarse
preconditioner, relaxation, particle adaptivity, surface tension and
secondary-particle options of MRSim3DTP are not part of this step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .sparse import PhaseParams, SparseMacGrid3D, calibrateRhoTilde0

FACE_NAMES = ("u", "v", "w", "mu", "mv", "mw", "saved_u", "saved_v", "saved_w")


def face_shape(nx, ny, nz, axis):
    """(Z, Y, X) of the fine face lattice of one axis."""
    return (nz + (axis == 2), ny + (axis == 1), nx + (axis == 0))


def valid_faces(levels, nx, ny, nz, axis):
    """The fine face patches on a leaf cell's boundary (the face list of
    MRMacGrid3D, src/grid/multires_mac_grid3d.h:123-163) for a layout given
    as one byte per level-1 block: the position along the axis is even, the
    domain's far side, or beside a fine cell of a refined block."""
    Z, Y, X = face_shape(nx, ny, nz, axis)
    fine = np.repeat(np.repeat(np.repeat(np.asarray(levels, bool), 8, 0), 8, 1), 8, 2)[:nz, :ny, :nx]
    n = (nx, ny, nz)[axis]
    ax = 2 - axis
    pos = np.arange((X, Y, Z)[axis])
    shape = [1, 1, 1]
    shape[ax] = -1
    pos = pos.reshape(shape)
    ok = np.broadcast_to((pos % 2 == 0) | (pos == n), (Z, Y, X)).copy()
    pad = [(0, 0)] * 3
    pad[ax] = (1, 0)
    before = np.pad(fine, pad)  # cell pos-1 refined
    pad[ax] = (0, 1)
    after = np.pad(fine, pad)   # cell pos refined
    return ok | before | after


def interface_levels(liquid, radius=3):
    """A layout refined around a free surface: one byte per level-1 block
    (8^3 fine cells), 1 when both liquid cells and empty interior cells lie
    within the block widened by `radius` cells.  `liquid` is a (nz, ny, nx)
    bool array of liquid cells; the domain's boundary layer counts as
    neither.  The layout goes to MRSim3DTP.set_levels."""
    liquid = np.asarray(liquid, bool)
    nz, ny, nx = liquid.shape
    interior = np.zeros_like(liquid)
    interior[1:-1, 1:-1, 1:-1] = True
    out = []
    for mask in (liquid & interior, ~liquid & interior):
        s = np.zeros((nz + 1, ny + 1, nx + 1), np.int64)
        s[1:, 1:, 1:] = mask.cumsum(0).cumsum(1).cumsum(2)
        MX, MY, MZ = (nx + 7) // 8, (ny + 7) // 8, (nz + 7) // 8
        lo = [np.clip(np.arange(m) * 8 - radius, 0, n) for m, n in ((MZ, nz), (MY, ny), (MX, nx))]
        hi = [np.clip(np.arange(m) * 8 + 8 + radius, 0, n) for m, n in ((MZ, nz), (MY, ny), (MX, nx))]
        z0, y0, x0 = np.ix_(*lo)
        z1, y1, x1 = np.ix_(*hi)
        tot = (s[z1, y1, x1] - s[z0, y1, x1] - s[z1, y0, x1] - s[z1, y1, x0] + s[z0, y0, x1] + s[z0, y1, x0]
               + s[z1, y0, x0] - s[z0, y0, x0])
        out.append(tot > 0)
    return (out[0] & out[1]).astype(np.uint8)


class MRSim3DTP:
    def __init__(self, nx, ny, nz, dx, max_particles=1 << 20, device=0):
        self.grid = SparseMacGrid3D(nx, ny, nz, dx, max_particles=max_particles, device=device)
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(dx)
        self.phase = PhaseParams()
        self.dt, self.gravity, self.Vp = 0.02, -9.81, 1.0
        self.alpha_liquid = self.alpha_gas = 0.95
        self.advection_order = 2
        self.c_div_last = 0.0
        self.cg_iters, self.cg_tol, self.cg_rel_tol = 160, 1e-7, 1e-6
        self.cg_jacobi_preconditioner = True
        self.cg_flexible_beta = False
        self.cg_adaptive_restart, self.cg_restart_growth = True, 10.0
        self.dynamic_refinement = True
        self.dynamic_particle_padding, self.dynamic_gas_padding = 1, 2
        self.dynamic_hysteresis_cells, self.dynamic_max_fine_leaves = 1, 0
        self.dynamic_last_fine_leaves = 0
        self.dynamic_budget_limited = False
        self.dynamic_retained_box_valid = False
        self.last_pressure_stats = L.MRStepStats()
        self.particle_boundary_clamped_liquid_last = self.particle_boundary_clamped_gas_last = 0
        self.particle_boundary_clamped_liquid_total = self.particle_boundary_clamped_gas_total = 0
        self.n = 0

    @property
    def ctx(self):
        return self.grid.ctx

    @property
    def lib(self):
        return self.grid.lib

    def close(self):
        self.grid.close()

    # ---- particles ------------------------------------------------------
    def set_particles(self, pos, vel, type, volume=None):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        n = len(pos)
        vel = np.ascontiguousarray(vel, np.float32).reshape(n, 3)
        typ = np.ascontiguousarray(type, np.uint8).reshape(n)
        vol = np.ascontiguousarray(np.ones(n) if volume is None else volume, np.float32).reshape(n)
        self.grid._ensure_capacity(n)
        L.check(self.lib.pf_upload_particles(self.ctx, n, pos.ctypes.data, vel.ctypes.data, typ.ctypes.data,
                                             vol.ctypes.data), self.ctx, "pf_upload_particles")
        self.n = n

    def seed_scene(self, scene, seed=0):
        """Seed the particle set on the device (pf_seed_scene): "dam_break",
        "bubble_tank" or "rayleigh_taylor", the particles of the scenes
        module's generator of that name.  Returns the count."""
        kind = {"rayleigh_taylor": L.PF_SCENE_RAYLEIGH_TAYLOR, "bubble_tank": L.PF_SCENE_BUBBLE_TANK,
                "dam_break": L.PF_SCENE_DAM_BREAK}[scene]
        n = C.c_size_t()
        L.check(self.lib.pf_seed_scene(self.ctx, kind, int(seed), C.byref(n)), self.ctx, "pf_seed_scene")
        self.n = int(n.value)
        return self.n

    def get_particles(self):
        n = self.n
        pos, vel = np.empty((n, 3), np.float32), np.empty((n, 3), np.float32)
        typ, vol = np.empty(n, np.uint8), np.empty(n, np.float32)
        L.check(self.lib.pf_download_particles(self.ctx, pos.ctypes.data, vel.ctypes.data, typ.ctypes.data,
                                               vol.ctypes.data), self.ctx, "pf_download_particles")
        return pos, vel, typ, vol

    # ---- layout ---------------------------------------------------------
    def set_layout(self, boxes):
        """setCoarseEverywhere(1) and refineFineCellBox of each (x0, y0, z0,
        x1, y1, z1) box of fine cells."""
        arr = (L.MRBox * max(1, len(boxes)))(*[L.MRBox(*map(int, b)) for b in boxes])
        L.check(self.lib.pf_mr_set_layout(self.ctx, arr, len(boxes)), self.ctx, "pf_mr_set_layout")

    def set_levels(self, refined):
        r = np.ascontiguousarray(refined, np.uint8)
        L.check(self.lib.pf_mr_set_levels(self.ctx, r.ctypes.data), self.ctx, "pf_mr_set_levels")

    def levels(self):
        """One byte per level-1 block, (MZ, MY, MX), 1 where refined."""
        dims = (C.c_int * 3)()
        L.check(self.lib.pf_mr_get_levels(self.ctx, None, dims), self.ctx, "pf_mr_get_levels")
        out = np.zeros((dims[2], dims[1], dims[0]), np.uint8)
        L.check(self.lib.pf_mr_get_levels(self.ctx, out.ctypes.data, None), self.ctx, "pf_mr_get_levels")
        return out

    def _dynamic(self):
        d = L.MRDynamic(int(self.dynamic_refinement), int(self.dynamic_particle_padding), int(self.dynamic_gas_padding),
                        int(self.dynamic_hysteresis_cells), int(self.dynamic_max_fine_leaves))
        L.check(self.lib.pf_mr_set_dynamic(self.ctx, C.byref(d)), self.ctx, "pf_mr_set_dynamic")

    def updateDynamicRefinement(self):
        """src/driver/multires_sim3d_tp.cpp:577-669; returns the retained box
        state (valid, x0, y0, z0, x1, y1, z1, budget_limited)."""
        self._dynamic()
        st = (C.c_int * 8)()
        L.check(self.lib.pf_mr_update_refinement(self.ctx, st), self.ctx, "pf_mr_update_refinement")
        self.dynamic_retained_box_valid = bool(st[0])
        self.dynamic_budget_limited = bool(st[7])
        self.dynamic_last_fine_leaves = self.fine_leaf_blocks()
        return tuple(st)

    def fine_leaf_blocks(self):
        """layout.countLevel(0): level-0 blocks intersecting the domain."""
        lv = self.levels()
        n = 0
        for bz, by, bx in zip(*np.nonzero(lv)):
            for c in range(8):
                if ((2 * bx + (c & 1)) * 4 < self.nx and (2 * by + ((c >> 1) & 1)) * 4 < self.ny
                        and (2 * bz + (c >> 2)) * 4 < self.nz):
                    n += 1
        return n

    def initBubbleTankInterfaceBand(self):
        """src/driver/multires_sim3d_tp.cpp:457-503: calibrate rho_tilde_0,
        the refined lower band and bubble box (refineBubbleStaticBand,
        :229-242), eight particles per cell of water below ny / 2 with a gas
        sphere, then the dynamic refinement when it is on."""
        self.phase.rho_tilde_0 = calibrateRhoTilde0(self.phase, self.Vp, self.grid)
        L.check(self.lib.pf_mr_reset_refinement(self.ctx), self.ctx, "pf_mr_reset_refinement")
        nx, ny, nz = self.nx, self.ny, self.nz
        wl = ny // 2
        band = (0, 0, 0, nx, min(ny, wl + 2), nz)
        box = (max(0, nx // 2 - nx // 4), max(0, wl // 4), max(0, nz // 2 - nz // 4),
               min(nx, nx // 2 + nx // 4), min(ny, wl), min(nz, nz // 2 + nz // 4))
        self.set_layout([band, box])
        cx, cy, cz = nx * 0.5, wl * 0.375, nz * 0.5
        r = max(1.25, min(nx, nz) * 0.1875)
        k, j, i = np.meshgrid(np.arange(1, nz - 1), np.arange(1, wl), np.arange(1, nx - 1), indexing="ij")
        k, j, i = k.ravel(), j.ravel(), i.ravel()
        gas = ((i + 0.5) - cx) ** 2 + ((j + 0.5) - cy) ** 2 + ((k + 0.5) - cz) ** 2 < r * r
        s = np.arange(8)
        pos = np.empty((len(i), 8, 3))
        pos[:, :, 0] = (i[:, None] + 0.25 + 0.5 * (s & 1)) * self.dx
        pos[:, :, 1] = (j[:, None] + 0.25 + 0.5 * ((s >> 1) & 1)) * self.dx
        pos[:, :, 2] = (k[:, None] + 0.25 + 0.5 * ((s >> 2) & 1)) * self.dx
        typ = np.repeat(gas.astype(np.uint8), 8)
        self.set_particles(pos.reshape(-1, 3), np.zeros((len(typ), 3)), typ)
        if self.dynamic_refinement:
            self.updateDynamicRefinement()

    # ---- the step ---------------------------------------------------------
    def step_cfg(self):
        return L.MRStepCfg(self.dt, self.gravity, self.Vp, self.alpha_liquid, self.alpha_gas, self.phase._c(),
                           int(self.advection_order), int(self.cg_iters), float(self.cg_tol), float(self.cg_rel_tol),
                           int(self.cg_jacobi_preconditioner), int(self.cg_flexible_beta),
                           int(self.cg_adaptive_restart), float(self.cg_restart_growth), float(self.c_div_last))

    def step(self):
        self._dynamic()
        st = L.MRStepStats()
        L.check(self.lib.pf_mr_step(self.ctx, C.byref(self.step_cfg()), C.byref(st)), self.ctx, "pf_mr_step")
        self.last_pressure_stats = st
        self.dynamic_last_fine_leaves = st.fine_leaves
        self.particle_boundary_clamped_liquid_last = st.clamp.clamped_liquid
        self.particle_boundary_clamped_gas_last = st.clamp.clamped_gas
        self.particle_boundary_clamped_liquid_total += st.clamp.clamped_liquid
        self.particle_boundary_clamped_gas_total += st.clamp.clamped_gas
        return st

    def p2g(self):
        """mrP2G3D_tp alone on the current layout."""
        L.check(self.lib.pf_mr_p2g(self.ctx, C.byref(self.phase._c()), float(self.Vp)), self.ctx, "pf_mr_p2g")

    # ---- views ------------------------------------------------------------
    def face(self, f):
        out = np.zeros(face_shape(self.nx, self.ny, self.nz, f % 3), np.float32)
        L.check(self.lib.pf_mr_get_face(self.ctx, int(f), out.ctypes.data), self.ctx, "pf_mr_get_face")
        return out

    def cells(self):
        """(marker, pressure) per fine cell, (nz, ny, nx)."""
        mk = np.zeros((self.nz, self.ny, self.nx), np.uint8)
        p = np.zeros((self.nz, self.ny, self.nx), np.float32)
        L.check(self.lib.pf_mr_get_cells(self.ctx, mk.ctypes.data, p.ctypes.data), self.ctx, "pf_mr_get_cells")
        return mk, p

    def activePressureCellCount(self):
        """grid.p.leafCells().size(): every leaf cell intersecting the domain."""
        lv = self.levels().astype(bool)
        fine = np.repeat(np.repeat(np.repeat(lv, 8, 0), 8, 1), 8, 2)[: self.nz, : self.ny, : self.nx]
        n_fine = int(fine.sum())
        coarse = np.repeat(np.repeat(np.repeat(~lv, 4, 0), 4, 1), 4, 2)
        cz, cy, cx = np.nonzero(coarse)
        inside = (2 * cx < self.nx) & (2 * cy < self.ny) & (2 * cz < self.nz)
        return n_fine + int(inside.sum())

    def _face_count(self, axis):
        return int(valid_faces(self.levels(), self.nx, self.ny, self.nz, axis).sum())

    def uFaceCount(self):
        return self._face_count(0)

    def vFaceCount(self):
        return self._face_count(1)

    def wFaceCount(self):
        return self._face_count(2)
