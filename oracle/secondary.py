"""Secondary particles on the CPU -- TEST INFRASTRUCTURE ONLY.

The oracle's restatement (``pf_oracle_sec.c``) of the reference's
secondary-particle bookkeeping (src/driver/secondary_particles3d.h:9-467) and
``SparseSim3DTP::step()`` composed from the oracle's passes with the escape
branching, the lifecycle and the spray emission at the reference's places
(src/driver/sparse_sim3d_tp.cpp:854-884, 192-337); and the same settings and
read-backs for the compiled reference's own ``SparseSim3DTP``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import ClampStats, InterfaceStats, Oracle, Particles, ReferenceGrid, _ip, oracle_lib, ref_lib


class _Set(C.Structure):
    _fields_ = [("n", C.c_size_t), ("cap", C.c_size_t), ("pos", C.POINTER(C.c_double)),
                ("vel", C.POINTER(C.c_double)), ("vol", C.POINTER(C.c_double)), ("age", C.POINTER(C.c_int))]


class _Domain(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("ox", C.c_double),
                ("oy", C.c_double), ("oz", C.c_double)]


class _LifeCfg(C.Structure):
    _fields_ = [("enabled", C.c_int), ("droplet_lifetime_steps", C.c_int), ("bubble_lifetime_steps", C.c_int),
                ("velocity_damping", C.c_double), ("reabsorb_margin_cells", C.c_double), ("gravity", C.c_double),
                ("droplet_gravity_scale", C.c_double), ("bubble_buoyancy_scale", C.c_double),
                ("droplet_drag", C.c_double), ("bubble_drag", C.c_double), ("particle_volume_scale", C.c_double)]


class LifeStats(C.Structure):
    """SecondaryParticleLifecycleStats3D (src/driver/secondary_particles3d.h:33-54)."""
    _fields_ = [(n, C.c_int) for n in ("enabled", "finite", "advected_droplets", "advected_bubbles",
                                        "reabsorbed_droplets", "reabsorbed_bubbles", "expired_droplets",
                                        "expired_bubbles", "dragged_droplets", "dragged_bubbles",
                                        "reabsorbed_droplets_to_primary", "reabsorbed_bubbles_to_primary")] + \
               [(n, C.c_double) for n in ("current_droplet_volume", "current_bubble_volume",
                                           "reabsorbed_droplet_volume", "reabsorbed_bubble_volume",
                                           "expired_droplet_volume", "expired_bubble_volume",
                                           "reabsorbed_droplet_volume_to_primary",
                                           "reabsorbed_bubble_volume_to_primary")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class _SprayCfg(C.Structure):
    _fields_ = [("enabled", C.c_int), ("requested_particles", C.c_int), ("droplet_fraction", C.c_double),
                ("droplet_volume", C.c_double), ("bubble_volume", C.c_double),
                ("particle_volume_scale", C.c_double), ("interface_gate", C.c_int), ("interface_cells", C.c_int),
                ("interface_grad_max", C.c_double), ("interface_curvature_abs_max", C.c_double),
                ("min_interface_cells", C.c_int), ("min_interface_grad_max", C.c_double),
                ("min_interface_curvature_abs_max", C.c_double), ("impact_splash_candidates", C.c_int),
                ("impact_region_fraction", C.c_double), ("impact_downward_speed_min", C.c_double),
                ("impact_foam_fraction", C.c_double)]


class SprayStats(C.Structure):
    """SecondarySprayEmissionStats3D (src/driver/secondary_particles3d.h:76-93)."""
    _fields_ = [(n, C.c_int) for n in ("enabled", "finite", "requested_particles", "effective_requested_particles",
                                        "interface_gate_enabled", "interface_gate_passed", "interface_cells",
                                        "candidate_liquid_particles", "impact_candidate_liquid_particles",
                                        "foam_ready_droplets", "emitted_droplets", "emitted_bubbles")] + \
               [(n, C.c_double) for n in ("interface_grad_max", "interface_curvature_abs_max",
                                           "emitted_droplet_volume", "emitted_bubble_volume")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


@dataclass
class SecondarySettings:
    """SparseSim3DTP's secondary-particle settings and their defaults
    (src/driver/sparse_sim3d_tp.h:82-137)."""
    escaped_particle_branching: bool = False
    secondary_particle_lifecycle: bool = False
    secondary_droplet_lifetime_steps: int = 48
    secondary_bubble_lifetime_steps: int = 48
    secondary_velocity_damping: float = 0.98
    secondary_reabsorb_margin_cells: float = 1.0
    secondary_droplet_gravity_scale: float = 1.0
    secondary_bubble_buoyancy_scale: float = 0.25
    secondary_droplet_drag: float = 0.0
    secondary_bubble_drag: float = 0.0
    secondary_reabsorb_to_primary: bool = False
    secondary_spray_emission: bool = False
    secondary_spray_particles_per_step: int = 0
    secondary_spray_droplet_fraction: float = 0.9
    secondary_spray_droplet_volume: float = 0.55
    secondary_spray_bubble_volume: float = 0.45
    secondary_spray_interface_gate: bool = False
    secondary_spray_min_interface_cells: int = 1
    secondary_spray_min_interface_grad_max: float = 1e-5
    secondary_spray_min_interface_curvature_abs_max: float = 0.0
    secondary_spray_impact_candidates: bool = False
    secondary_spray_impact_region_fraction: float = 0.55
    secondary_spray_impact_downward_speed_min: float = 1.0
    secondary_spray_impact_foam_fraction: float = 0.3

    def int_vector(self):
        return np.array([self.escaped_particle_branching, self.secondary_particle_lifecycle,
                         self.secondary_droplet_lifetime_steps, self.secondary_bubble_lifetime_steps,
                         self.secondary_reabsorb_to_primary, self.secondary_spray_emission,
                         self.secondary_spray_particles_per_step, self.secondary_spray_interface_gate,
                         self.secondary_spray_min_interface_cells, self.secondary_spray_impact_candidates],
                        np.int32)

    def double_vector(self):
        return np.array([self.secondary_velocity_damping, self.secondary_reabsorb_margin_cells,
                         self.secondary_droplet_gravity_scale, self.secondary_bubble_buoyancy_scale,
                         self.secondary_droplet_drag, self.secondary_bubble_drag,
                         self.secondary_spray_droplet_fraction, self.secondary_spray_droplet_volume,
                         self.secondary_spray_bubble_volume, self.secondary_spray_min_interface_grad_max,
                         self.secondary_spray_min_interface_curvature_abs_max,
                         self.secondary_spray_impact_region_fraction,
                         self.secondary_spray_impact_downward_speed_min,
                         self.secondary_spray_impact_foam_fraction], np.float64)


@dataclass
class SecSet:
    """One secondary set (droplets or bubbles): positions, velocities, volumes, ages."""
    pos: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    vel: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    vol: np.ndarray = field(default_factory=lambda: np.zeros(0))
    age: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    def __len__(self):
        return len(self.vol)

    def append(self, pos, vel, vol, age):
        self.pos = np.vstack([self.pos, np.asarray(pos, np.float64).reshape(-1, 3)])
        self.vel = np.vstack([self.vel, np.asarray(vel, np.float64).reshape(-1, 3)])
        self.vol = np.concatenate([self.vol, np.asarray(vol, np.float64).reshape(-1)])
        self.age = np.concatenate([self.age, np.asarray(age, np.int32).reshape(-1)])

    def _c(self, extra):
        cap = len(self) + extra
        self._bufs = [np.zeros((cap, 3)), np.zeros((cap, 3)), np.zeros(cap), np.zeros(cap, np.int32)]
        n = len(self)
        self._bufs[0][:n], self._bufs[1][:n], self._bufs[2][:n], self._bufs[3][:n] = \
            self.pos, self.vel, self.vol, self.age
        dp = C.POINTER(C.c_double)
        return _Set(n, cap, self._bufs[0].ctypes.data_as(dp), self._bufs[1].ctypes.data_as(dp),
                    self._bufs[2].ctypes.data_as(dp), self._bufs[3].ctypes.data_as(C.POINTER(C.c_int)))

    def _from_c(self, s):
        n = s.n
        self.pos, self.vel = self._bufs[0][:n].copy(), self._bufs[1][:n].copy()
        self.vol, self.age = self._bufs[2][:n].copy(), self._bufs[3][:n].copy()


def _typed():
    lib = oracle_lib()
    if getattr(lib, "_sec_typed", False):
        return lib
    lib.pfo_sec_advance.argtypes = [C.POINTER(_Domain), C.POINTER(_LifeCfg), C.c_double, C.POINTER(_Set),
                                    C.POINTER(_Set), C.POINTER(_Set), C.POINTER(_Set), C.POINTER(LifeStats)]
    lib.pfo_spray_emit.argtypes = [C.c_size_t, np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                                   np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                                   np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"),
                                   np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.POINTER(_SprayCfg),
                                   C.c_int, C.POINTER(_Set), C.POINTER(_Set), C.POINTER(SprayStats)]
    lib._sec_typed = True
    return lib


@dataclass
class SecondaryState:
    """The secondary sets and the per-step statistics of a simulation."""
    droplets: SecSet = field(default_factory=SecSet)
    bubbles: SecSet = field(default_factory=SecSet)
    spray_step_index: int = 0
    lifecycle: LifeStats = field(default_factory=LifeStats)
    spray: SprayStats = field(default_factory=SprayStats)
    added: tuple = (0, 0, 0.0, 0.0)  # droplets, bubbles added last step and their volumes


def advance(state: SecondaryState, domain, s: SecondarySettings, gravity, Vp, dt):
    """advanceSecondaryLifecycle: returns the (droplet, bubble) sets reabsorbed
    to the primary particles (empty when that option is off)."""
    lib = _typed()
    cfg = _LifeCfg(int(s.secondary_particle_lifecycle), s.secondary_droplet_lifetime_steps,
                   s.secondary_bubble_lifetime_steps, s.secondary_velocity_damping, s.secondary_reabsorb_margin_cells,
                   gravity, s.secondary_droplet_gravity_scale, s.secondary_bubble_buoyancy_scale,
                   s.secondary_droplet_drag, s.secondary_bubble_drag, Vp)
    d = _Domain(*domain)
    rd, rb = SecSet(), SecSet()
    cd, cb = state.droplets._c(0), state.bubbles._c(0)
    crd, crb = rd._c(len(state.droplets)), rb._c(len(state.bubbles))
    st = LifeStats()
    rd_p = C.byref(crd) if s.secondary_reabsorb_to_primary else None
    rb_p = C.byref(crb) if s.secondary_reabsorb_to_primary else None
    if lib.pfo_sec_advance(C.byref(d), C.byref(cfg), float(dt), C.byref(cd), C.byref(cb), rd_p, rb_p, C.byref(st)):
        raise RuntimeError("pfo_sec_advance failed")
    state.droplets._from_c(cd)
    state.bubbles._from_c(cb)
    rd._from_c(crd)
    rb._from_c(crb)
    state.lifecycle = st
    return rd, rb


def spray(state: SecondaryState, ps: Particles, s: SecondarySettings, Vp, iface: InterfaceStats):
    """emitSecondarySpray (src/driver/sparse_sim3d_tp.cpp:276-337)."""
    lib = _typed()
    cfg = _SprayCfg(int(s.secondary_spray_emission), s.secondary_spray_particles_per_step,
                    s.secondary_spray_droplet_fraction, s.secondary_spray_droplet_volume,
                    s.secondary_spray_bubble_volume, Vp, int(s.secondary_spray_interface_gate), iface.interface_cells,
                    iface.grad_max, iface.curvature_abs_max, s.secondary_spray_min_interface_cells,
                    s.secondary_spray_min_interface_grad_max, s.secondary_spray_min_interface_curvature_abs_max,
                    int(s.secondary_spray_impact_candidates), s.secondary_spray_impact_region_fraction,
                    s.secondary_spray_impact_downward_speed_min, s.secondary_spray_impact_foam_fraction)
    req = max(0, s.secondary_spray_particles_per_step)
    cd, cb = state.droplets._c(req), state.bubbles._c(req)
    st = SprayStats()
    if lib.pfo_spray_emit(len(ps), ps.pos, ps.vel, ps.type, ps.volume, C.byref(cfg), int(state.spray_step_index),
                          C.byref(cd), C.byref(cb), C.byref(st)):
        raise RuntimeError("pfo_spray_emit failed")
    state.droplets._from_c(cd)
    state.bubbles._from_c(cb)
    state.spray = st
    state.spray_step_index += 1


def oracle_step(o: Oracle, g, ps: Particles, pp, cfg: dict, s: SecondarySettings, state: SecondaryState):
    """SparseSim3DTP::step() (adaptivity and the adaptive timestep off) on the
    oracle's passes with the secondary-particle hooks at the reference's
    places; returns the solve and clamp statistics."""
    dt, Vp = cfg["dt"], cfg["Vp"]
    domain = (g.nx, g.ny, g.nz, g.dx, *g.origin)
    rd, rb = advance(state, domain, s, cfg["gravity"], Vp, dt)
    if s.secondary_reabsorb_to_primary:
        for part, t in ((rd, 0), (rb, 1)):
            for i in range(len(part)):
                ps.add(part.pos[i], part.vel[i], t, part.vol[i])
    o.mark_cells(g, ps)
    o.p2g(g, ps, pp, Vp)
    iface = o.interface_diagnostics(g, pp)
    saved = g.copy()
    o.apply_gravity(g, dt, cfg["gravity"])
    o.apply_wall_boundary(g)
    sst = o.project(g, pp, dt, cfg["cg_iters"], cfg["cg_tol"])
    o.g2p(g, ps, saved, cfg["alpha_l"], cfg["alpha_g"])
    if s.escaped_particle_branching:
        cst, rec = o.advect(ps, g, dt, cfg.get("advect_order", 2), escape=True)
    else:
        cst, rec = o.advect(ps, g, dt, cfg.get("advect_order", 2)), np.zeros((0, 8))
    # storeEscapedParticles (:192-218)
    nd = nb = 0
    vd = vb = 0.0
    for r in rec:
        if int(r[0]) == 0:
            state.droplets.append(r[1:4], r[4:7], r[7], 0)
            nd += 1
            vd += r[7] * Vp
        elif int(r[0]) == 1:
            state.bubbles.append(r[1:4], r[4:7], r[7], 0)
            nb += 1
            vb += r[7] * Vp
    spray(state, ps, s, Vp, iface)
    st = state.spray
    state.added = (nd + st.emitted_droplets, nb + st.emitted_bubbles, vd + st.emitted_droplet_volume,
                   vb + st.emitted_bubble_volume)
    return sst, cst


def reference_configure(g: ReferenceGrid, s: SecondarySettings):
    lib = ref_lib()
    _typed_ref(lib)
    lib.pfr_set_secondary(g.h, s.int_vector(), s.double_vector())


def _typed_ref(lib):
    if getattr(lib, "_sec_typed", False):
        return
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.pfr_set_secondary.argtypes = [C.c_void_p, _ip, dp]
    lib.pfr_secondary_count.restype = C.c_size_t
    lib.pfr_secondary_count.argtypes = [C.c_void_p, C.c_int]
    lib.pfr_get_secondary.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, _ip]
    lib.pfr_set_secondary_set.argtypes = [C.c_void_p, C.c_int, C.c_size_t, dp, dp, dp, _ip]
    lib.pfr_secondary_stats.argtypes = [C.c_void_p, _ip, dp]
    lib._sec_typed = True


def reference_sets(g: ReferenceGrid):
    lib = ref_lib()
    _typed_ref(lib)
    out = []
    for which in (0, 1):
        n = int(lib.pfr_secondary_count(g.h, which))
        s = SecSet(np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n, np.int32))
        if n:
            lib.pfr_get_secondary(g.h, which, s.pos, s.vel, s.vol, s.age)
        out.append(s)
    return out


def reference_stats(g: ReferenceGrid):
    """(lifecycle dict, spray dict, added tuple, spray step index)."""
    lib = ref_lib()
    _typed_ref(lib)
    iv, dv = np.zeros(30, np.int32), np.zeros(20, np.float64)
    lib.pfr_secondary_stats(g.h, iv, dv)
    life = LifeStats(*[int(v) for v in iv[:12]], *[float(v) for v in dv[:8]])
    spr = SprayStats(*[int(v) for v in iv[12:24]], *[float(v) for v in dv[8:12]])
    return life, spr, (int(iv[24]), int(iv[25]), float(dv[12]), float(dv[13])), int(iv[26])
