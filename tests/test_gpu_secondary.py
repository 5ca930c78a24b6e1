"""GPU secondary particles against the oracle (src/driver/secondary_particles3d.h:
9-467, src/driver/sparse_sim3d_tp.cpp:185-337), through the C ABI.

The oracle (oracle/pf_oracle_sec.c) is pinned bit for bit to the compiled
reference's SparseSim3DTP::step() with the secondary particles switched on
(tests/test_secondary_oracle.py).  The device keeps both sets in FP64 and
does the reference's arithmetic in its order, so on the same inputs:

* the lifecycle (pf_secondary_advance against pfo_sec_advance): both sets,
  their ages, the particles reabsorbed into the primary set (rounded to its
  FP32 storage) and every statistic are identical, step after step;
* the spray (pf_secondary_spray against pfo_spray_emit) on FP32-representable
  primary particles: the seeds, their ages and every statistic are identical,
  frame after frame;
* the step's escape branching: the sets pf_step fills equal the escape
  records of the same step taken pass by pass (pf_advect with records);
* the whole step: the lifecycle part of the first step is identical to the
  oracle's step from the same state, and the sets pf_step leaves are the
  survivors of the lifecycle (bit-identical to the oracle's lifecycle of the
  sets before the step), then the step's escaped particles, then its seeds.
"""
import ctypes as C
import types

import numpy as np
import pytest

import oracle as O
from oracle.secondary import SecondarySettings, SecondaryState, SecSet, advance, oracle_step, spray

pytestmark = pytest.mark.gpu

LIFE_FIELDS = {"enabled": "lifecycle_enabled", "finite": "lifecycle_finite",
               "current_droplet_volume": "lifecycle_droplet_volume",
               "current_bubble_volume": "lifecycle_bubble_volume"}
for _n in ("advected_droplets", "advected_bubbles", "reabsorbed_droplets", "reabsorbed_bubbles", "expired_droplets",
           "expired_bubbles", "dragged_droplets", "dragged_bubbles", "reabsorbed_droplets_to_primary",
           "reabsorbed_bubbles_to_primary", "reabsorbed_droplet_volume", "reabsorbed_bubble_volume",
           "expired_droplet_volume", "expired_bubble_volume", "reabsorbed_droplet_volume_to_primary",
           "reabsorbed_bubble_volume_to_primary"):
    LIFE_FIELDS[_n] = _n


def _sim(pf, n, settings: SecondarySettings, max_particles):
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=max_particles)
    for k, v in vars(settings).items():
        setattr(sim, k, v)
    ctx, lib = sim.grid.ctx, sim.grid.lib
    sc = sim.secondary_cfg()
    pf._lib.check(lib.pf_set_secondary(ctx, C.byref(sc)), ctx, "pf_set_secondary")
    return sim


def _stats(pf, sim):
    st = pf._lib.SecondaryStats()
    pf._lib.check(sim.grid.lib.pf_get_secondary_stats(sim.grid.ctx, C.byref(st)), sim.grid.ctx, "stats")
    return st


def _gpu_sets(sim):
    return [SecSet(*sim.secondary_set(w)) for w in (0, 1)]


def _same_set(a: SecSet, b: SecSet, what):
    assert len(a) == len(b), f"{what}: {len(a)} vs {len(b)} particles"
    for name in ("pos", "vel", "vol", "age"):
        x, y = getattr(a, name), getattr(b, name)
        assert np.array_equal(x, y, equal_nan=name != "age"), f"{what}: {name} differs"


def _random_set(rng, m, n, nonfinite):
    """Half the particles anywhere in the domain, half within a cell of a wall."""
    pos = rng.uniform(0.0, 1.0, (m, 3))
    near = rng.random(m) < 0.5
    axis = rng.integers(0, 3, m)
    side = rng.random(m) < 0.5
    pos[near, axis[near]] = np.where(side[near], rng.uniform(0.0, 1.5 / n, near.sum()),
                                     rng.uniform(1.0 - 1.5 / n, 1.0, near.sum()))
    vel = rng.normal(0.0, 0.6, (m, 3))
    vol = rng.uniform(0.5, 1.5, m)
    age = rng.integers(0, 5, m).astype(np.int32)
    for k, (a, b) in enumerate(nonfinite):
        (pos if a == "pos" else vel)[3 + 7 * k, b] = np.nan if k % 2 == 0 else np.inf
    return SecSet(pos, vel, vol, age)


@pytest.mark.parametrize("to_primary", [False, True])
def test_lifecycle_matches_oracle(pf, to_primary):
    n, Vp, gravity, dt = 16, 0.7, -9.81, 1 / 30
    rng = np.random.default_rng(11 + to_primary)
    s = SecondarySettings(secondary_particle_lifecycle=True, secondary_droplet_lifetime_steps=3,
                          secondary_bubble_lifetime_steps=-1, secondary_droplet_drag=2.0, secondary_bubble_drag=0.0,
                          secondary_reabsorb_to_primary=to_primary, secondary_reabsorb_margin_cells=0.5,
                          secondary_velocity_damping=0.97)
    state = SecondaryState(_random_set(rng, 900, n, [("pos", 1), ("vel", 0)]),
                           _random_set(rng, 700, n, [("vel", 2)]))
    prim = rng.uniform(0.1, 0.9, (500, 3)).astype(np.float32)
    sim = _sim(pf, n, s, max_particles=500 + 2000)
    sim.set_particles(prim, np.zeros_like(prim), np.zeros(500, np.uint8), np.ones(500, np.float32))
    for w, st in enumerate((state.droplets, state.bubbles)):
        sim.set_secondary_set(w, st.pos, st.vel, st.vol, st.age)
    ctx, lib = sim.grid.ctx, sim.grid.lib
    domain = (n, n, n, 1.0 / n, 0.0, 0.0, 0.0)
    n_prim, seen_reab, seen_expired, finite = 500, 0, 0, []
    for step in range(5):
        rd, rb = advance(state, domain, s, gravity, Vp, dt)
        pf._lib.check(lib.pf_secondary_advance(ctx, dt, gravity, Vp), ctx, "pf_secondary_advance")
        gd, gb = _gpu_sets(sim)
        _same_set(gd, state.droplets, f"step {step} droplets")
        _same_set(gb, state.bubbles, f"step {step} bubbles")
        st = _stats(pf, sim)
        for of, gf in LIFE_FIELDS.items():
            assert getattr(st, gf) == getattr(state.lifecycle, of), f"step {step}: {gf}"
        # reabsorbed droplets, then bubbles, appended to the primary set in FP32
        pos, vel, typ, vol = sim.get_particles()
        added = len(rd) + len(rb) if to_primary else 0
        assert len(pos) == n_prim + added
        if added:
            want_pos = np.vstack([rd.pos, rb.pos]).astype(np.float32)
            want_vel = np.vstack([rd.vel, rb.vel]).astype(np.float32)
            assert np.array_equal(pos[n_prim:], want_pos)
            assert np.array_equal(vel[n_prim:], want_vel)
            assert np.array_equal(vol[n_prim:], np.concatenate([rd.vol, rb.vol]).astype(np.float32))
            assert np.array_equal(typ[n_prim:], np.r_[np.zeros(len(rd)), np.ones(len(rb))].astype(np.uint8))
        n_prim += added
        seen_reab += st.reabsorbed_droplets + st.reabsorbed_bubbles
        seen_expired += st.expired_droplets + st.expired_bubbles
        finite.append(st.lifecycle_finite)
    assert seen_reab > 0 and seen_expired > 0
    assert finite[0] == 0 and all(finite[1:])  # the planted non-finite particles go in the first step
    sim.grid.close()


def _liquid_blob(rng, m):
    pos = np.c_[rng.uniform(0.1, 0.9, m), rng.uniform(0.05, 0.6, m), rng.uniform(0.1, 0.9, m)]
    vel = rng.normal(0.0, 0.8, (m, 3))
    typ = (rng.random(m) < 0.2).astype(np.uint8)
    return pos.astype(np.float32), vel.astype(np.float32), typ


@pytest.mark.parametrize("case", ["impact_foam", "gate_closed", "plain"])
def test_spray_matches_oracle(pf, case):
    n, Vp = 16, 0.9
    rng = np.random.default_rng({"impact_foam": 3, "gate_closed": 4, "plain": 5}[case])
    s = SecondarySettings(secondary_spray_emission=True, secondary_spray_particles_per_step=14,
                          secondary_spray_droplet_fraction=0.6)
    if case == "impact_foam":
        s.secondary_spray_impact_candidates = True
        s.secondary_spray_impact_downward_speed_min = 0.3
        s.secondary_spray_impact_foam_fraction = 0.5
    if case != "plain":
        s.secondary_spray_interface_gate = True
        s.secondary_spray_min_interface_cells = 10
    iface = types.SimpleNamespace(interface_cells=50 if case != "gate_closed" else 5, grad_max=3.5,
                                  curvature_abs_max=12.0)
    pos, vel, typ = _liquid_blob(rng, 6000)
    vel[17] = np.nan  # a liquid particle that is not finite
    typ[17] = 0
    m = len(pos)
    ps = O.Particles(pos.astype(np.float64), vel.astype(np.float64), typ, np.ones(m))
    sim = _sim(pf, n, s, max_particles=m)
    sim.set_particles(pos, vel, typ, np.ones(m, np.float32))
    state = SecondaryState()
    ctx, lib = sim.grid.ctx, sim.grid.lib
    gi = pf._lib.InterfaceStats(interface_cells=iface.interface_cells, grad_max=iface.grad_max,
                                curvature_abs_max=iface.curvature_abs_max)
    for frame in range(3):
        spray(state, ps, s, Vp, iface)
        pf._lib.check(lib.pf_secondary_spray(ctx, Vp, C.byref(gi)), ctx, "pf_secondary_spray")
        gd, gb = _gpu_sets(sim)
        _same_set(gd, state.droplets, f"frame {frame} droplets")
        _same_set(gb, state.bubbles, f"frame {frame} bubbles")
        st = _stats(pf, sim)
        for of, _ in state.spray._fields_:
            assert getattr(st, "spray_" + of) == getattr(state.spray, of), f"frame {frame}: {of}"
        assert st.spray_step_index == state.spray_step_index
    if case == "gate_closed":
        assert len(state.droplets) == 0 and not state.spray.interface_gate_passed
    else:
        assert len(state.droplets) == 3 * 8 and len(state.bubbles) == 3 * 6
        assert state.spray.finite == 0  # the non-finite liquid particle
    if case == "impact_foam":
        assert state.spray.impact_candidate_liquid_particles > 0
    sim.grid.close()


def _escape_scene(pf, n, seed):
    sc = pf.scenes.bubble_tank(n, seed=seed)
    rng = np.random.default_rng(seed)
    vel = rng.normal(0.0, 2.0, sc["vel"].shape).astype(np.float32)
    return sc, vel


def _configure(sim, pp, dt):
    sim.phase = pp
    sim.dt = dt
    sim.alpha_liquid, sim.alpha_gas = 0.97, 0.9
    sim.cg_iters, sim.cg_tol = 4000, 0.0


def test_step_escape_branching_equals_advect_records(pf):
    """pf_step with escape branching (the per-particle advection writes the
    clamp flags) against the same step pass by pass, pf_advect returning the
    escape records: the droplet and bubble sets hold exactly the records of
    their type, in particle order, and the primary particles are unchanged
    by the branching."""
    from gpu_helpers import phase_for

    L = pf._lib
    n = 32
    sc, vel = _escape_scene(pf, n, 21)
    pp = phase_for(sc, pf)
    a = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
    b = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
    for sim in (a, b):
        _configure(sim, pp, 1 / 8)
        sim.solver = pf.SolverConfig(rel_tol=1e-8)
        sim.set_particles(sc["pos"], vel, sc["type"], sc["volume"])
    a.escaped_particle_branching = True
    st = a.step()
    cfg = b.step_cfg()
    ctx, lib = b.grid.ctx, b.grid.lib
    L.check(lib.pf_grid_clear_all(ctx), ctx, "pf_grid_clear_all")
    L.check(lib.pf_mark_cells(ctx), ctx, "pf_mark_cells")
    L.check(lib.pf_p2g(ctx, C.byref(cfg.phase), cfg.Vp), ctx, "pf_p2g")
    L.check(lib.pf_save_velocity(ctx), ctx, "pf_save_velocity")
    L.check(lib.pf_apply_gravity(ctx, cfg.dt, cfg.gravity), ctx, "pf_apply_gravity")
    L.check(lib.pf_apply_wall_boundary(ctx), ctx, "pf_apply_wall_boundary")
    sst = L.SolveStats()
    L.check(lib.pf_project(ctx, C.byref(cfg.phase), cfg.dt, C.byref(cfg.solve), C.byref(sst)), ctx, "pf_project")
    L.check(lib.pf_g2p(ctx, None, cfg.alpha_l, cfg.alpha_g), ctx, "pf_g2p")
    cs = L.ClampStats()
    rec = np.zeros((len(sc["pos"]), 8))
    nrec = C.c_size_t()
    L.check(lib.pf_advect(ctx, cfg.dt, 2, C.byref(cs), rec.ctypes.data, C.byref(nrec)), ctx, "pf_advect")
    rec = rec[: nrec.value]
    pa, va, _, _ = a.get_particles()
    pb, vb, _, _ = b.get_particles()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert st.clamp.as_tuple() == cs.as_tuple()
    sets = _gpu_sets(a)
    stats = a.secondary_stats_last
    for t, got in enumerate(sets):
        r = rec[rec[:, 0] == t]
        assert len(r) > 0
        _same_set(got, SecSet(r[:, 1:4], r[:, 4:7], r[:, 7], np.zeros(len(r), np.int32)), f"type {t}")
        vol = 0.0
        for v in r[:, 7]:
            vol += v * 1.0
        assert getattr(stats, ("escaped_droplets_added", "escaped_bubbles_added")[t]) == len(r)
        assert getattr(stats, ("escaped_droplet_volume_added", "escaped_bubble_volume_added")[t]) == vol
    for sim in (a, b):
        sim.grid.close()


def _tank_scene(n, seed, speed):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(1, n - 1), np.arange(1, int(0.6 * n)), np.arange(1, n - 1), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(np.float64)
    sub = np.stack([0.25 + 0.5 * (np.arange(8) & 1), 0.25 + 0.5 * ((np.arange(8) >> 1) & 1),
                    0.25 + 0.5 * ((np.arange(8) >> 2) & 1)], 1)
    pos = ((cells[:, None, :] + sub[None] + rng.uniform(-0.2, 0.2, (len(cells), 8, 3))).reshape(-1, 3) / n)
    c = pos - np.array([0.5, 0.3, 0.5])
    typ = ((c * c).sum(1) < 0.15 ** 2).astype(np.uint8)
    vel = rng.normal(0.0, speed, pos.shape)
    vel[:, 1] += 0.5 * speed
    return pos.astype(np.float32), vel.astype(np.float32), typ


@pytest.mark.parametrize("case", ["lifecycle_reabsorb", "spray"])
def test_step_with_secondary_composes_as_the_reference(pf, case):
    n, dt, Vp = 16, 1 / 6, 1.0
    s = {"lifecycle_reabsorb": SecondarySettings(
        escaped_particle_branching=True, secondary_particle_lifecycle=True, secondary_droplet_lifetime_steps=3,
        secondary_bubble_lifetime_steps=4, secondary_droplet_drag=2.0, secondary_bubble_drag=0.5,
        secondary_reabsorb_to_primary=True, secondary_reabsorb_margin_cells=0.5),
        "spray": SecondarySettings(
        escaped_particle_branching=True, secondary_particle_lifecycle=True, secondary_spray_emission=True,
        secondary_spray_particles_per_step=14, secondary_spray_interface_gate=True,
        secondary_spray_impact_candidates=True, secondary_spray_impact_downward_speed_min=0.3,
        secondary_spray_impact_foam_fraction=0.5)}[case]
    pos, vel, typ = _tank_scene(n, 3, 1.5)
    m = len(pos)
    pp = pf.PhaseParams(1000.0, 1.0, 1.0, 1.0)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, Vp)
    sim = _sim(pf, n, s, max_particles=2 * m)
    _configure(sim, pp, dt)
    sim.alpha_liquid = sim.alpha_gas = 0.95
    sim.cg_iters, sim.cg_tol = 400, 1e-9
    sim.set_particles(pos, vel, typ, np.ones(m, np.float32))
    # identical starting sets on both sides
    rng = np.random.default_rng(8)
    start = SecondaryState(_random_set(rng, 300, n, []), _random_set(rng, 200, n, []))
    for w, st in enumerate((start.droplets, start.bubbles)):
        sim.set_secondary_set(w, st.pos, st.vel, st.vol, st.age)
    # the oracle's whole step from the same state: its lifecycle is identical
    ostate = SecondaryState(SecSet(start.droplets.pos.copy(), start.droplets.vel.copy(), start.droplets.vol.copy(),
                                   start.droplets.age.copy()),
                            SecSet(start.bubbles.pos.copy(), start.bubbles.vel.copy(), start.bubbles.vol.copy(),
                                   start.bubbles.age.copy()))
    opp = O.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0)
    ps = O.Particles(pos.astype(np.float64), vel.astype(np.float64), typ, np.ones(m))
    cfg = dict(dt=dt, gravity=-9.81, Vp=Vp, alpha_l=0.95, alpha_g=0.95, cg_iters=400, cg_tol=1e-9, advect_order=2)
    oracle_step(O.Oracle(), O.OracleGrid(n, n, n, 1.0 / n), ps, opp, cfg, s, ostate)
    domain = (n, n, n, 1.0 / n, 0.0, 0.0, 0.0)
    seen_esc = seen_seed = 0
    for step in range(4):
        before = SecondaryState(*_gpu_sets(sim))
        n_before = sim.n
        rd, rb = advance(before, domain, s, -9.81, Vp, dt)  # the oracle's lifecycle of the GPU's own sets
        sim.step()
        st = sim.secondary_stats_last
        for of, gf in LIFE_FIELDS.items():
            assert getattr(st, gf) == getattr(before.lifecycle, of), f"step {step}: {gf}"
        if step == 0:
            for of, gf in LIFE_FIELDS.items():
                assert getattr(st, gf) == getattr(ostate.lifecycle, of), f"first step against the oracle: {gf}"
        reab = len(rd) + len(rb) if s.secondary_reabsorb_to_primary else 0
        assert sim.n == n_before + reab
        for t, (got, life) in enumerate(zip(_gpu_sets(sim), (before.droplets, before.bubbles))):
            k = len(life)
            _same_set(SecSet(got.pos[:k], got.vel[:k], got.vol[:k], got.age[:k]), life, f"step {step} set {t}")
            emitted = (st.spray_emitted_droplets, st.spray_emitted_bubbles)[t]
            escaped = (st.escaped_droplets_added, st.escaped_bubbles_added)[t] - emitted
            assert len(got) == k + escaped + emitted
            esc = SecSet(got.pos[k:k + escaped], got.vel[k:k + escaped], got.vol[k:k + escaped],
                         got.age[k:k + escaped])
            assert np.all(esc.age == 0)
            # an escaped particle sits on the clamp bounds of at least one axis
            lo, hi = np.float32(0.5 / n), np.float32(1.0 - 0.5 / n)
            on = np.any((esc.pos == lo) | (esc.pos == hi), axis=1)
            assert np.all(on), f"step {step} set {t}: escaped particles off the bounds"
            seeds = got.vol[k + escaped:]
            assert np.all(seeds == (s.secondary_spray_droplet_volume, s.secondary_spray_bubble_volume)[t])
            vol = 0.0
            for v in got.vol:
                vol += v * Vp
            cur = (st.droplet_volume_current, st.bubble_volume_current)[t]
            assert cur == vol
            seen_esc += escaped
            seen_seed += emitted
        assert st.spray_step_index == step + 1
    assert seen_esc > 0
    if case == "spray":
        assert seen_seed > 0
    sim.grid.close()
