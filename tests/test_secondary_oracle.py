"""Secondary particles: the oracle's restatement (oracle/pf_oracle_sec.c,
composed into the sparse step by oracle/secondary.py) against the reference's
own SparseSim3DTP::step() with escape branching, the secondary lifecycle
(gravity, buoyancy, damping, drag, expiry, reabsorption into the primary set)
and spray emission (interface gate, impact candidates, foam-ready droplets)
switched on (src/driver/sparse_sim3d_tp.cpp:192-337, 854-884;
src/driver/secondary_particles3d.h:9-467).  Primary particles, both secondary
sets with their ages, and every statistic must agree bit for bit, step after
step."""
import numpy as np
import pytest

import oracle as O
from oracle.secondary import SecondarySettings, SecondaryState, oracle_step, reference_configure, \
    reference_sets, reference_stats

pytestmark = pytest.mark.skipif(not O.reference_available(), reason="compiled reference (oracle/_ref) not built")


def _scene(n, seed, speed):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(1, n - 1), np.arange(1, int(0.6 * n)), np.arange(1, n - 1), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(np.float64)
    s = np.arange(8)
    sub = np.stack([0.25 + 0.5 * (s & 1), 0.25 + 0.5 * ((s >> 1) & 1), 0.25 + 0.5 * ((s >> 2) & 1)], 1)
    pos = (cells[:, None, :] + sub[None] + rng.uniform(-0.2, 0.2, (len(cells), 8, 3))).reshape(-1, 3) / n
    c = pos - np.array([0.5, 0.3, 0.5])
    typ = ((c * c).sum(1) < 0.15 ** 2).astype(np.uint8)
    vel = rng.normal(0.0, speed, pos.shape)
    vel[:, 1] += 0.5 * speed
    return O.Particles(pos, vel, typ, np.ones(len(pos)))


SETTINGS = {
    "lifecycle_reabsorb": SecondarySettings(escaped_particle_branching=True, secondary_particle_lifecycle=True,
                                            secondary_droplet_lifetime_steps=3, secondary_bubble_lifetime_steps=4,
                                            secondary_droplet_drag=2.0, secondary_bubble_drag=0.5,
                                            secondary_reabsorb_to_primary=True, secondary_reabsorb_margin_cells=0.5),
    "spray": SecondarySettings(escaped_particle_branching=True, secondary_particle_lifecycle=True,
                               secondary_spray_emission=True, secondary_spray_particles_per_step=14,
                               secondary_spray_interface_gate=True, secondary_spray_impact_candidates=True,
                               secondary_spray_impact_downward_speed_min=0.3, secondary_spray_impact_foam_fraction=0.5),
    "spray_only": SecondarySettings(secondary_spray_emission=True, secondary_spray_particles_per_step=9,
                                    secondary_spray_droplet_fraction=0.6),
}


@pytest.mark.parametrize("case", sorted(SETTINGS))
def test_secondary_step_equals_reference(case):
    n, speed = 16, 1.5
    s = SETTINGS[case]
    pp = O.PhaseParams(1000.0, 1.0)
    pp.rho_tilde_0 = O.Oracle().calibrate_rho_tilde0(pp, 1.0)
    cfg = dict(dt=1 / 6, gravity=-9.81, Vp=1.0, alpha_l=0.95, alpha_g=0.95, cg_iters=400, cg_tol=1e-9,
               advect_order=2)
    ps_o = _scene(n, 3, speed)
    ps_r = ps_o.copy()
    o, R = O.Oracle(), O.Reference()
    og = O.OracleGrid(n, n, n, 1.0 / n)
    rg = O.ReferenceGrid(n, n, n, 1.0 / n)
    reference_configure(rg, s)
    state = SecondaryState()
    seen_sets = seen_reab = 0
    for step in range(5):
        oracle_step(o, og, ps_o, pp, cfg, s, state)
        R.step(rg, ps_r, pp, cfg)
        assert len(ps_o) == len(ps_r), f"step {step}: primary count"
        for a in ("pos", "vel", "type", "volume"):
            assert np.array_equal(getattr(ps_o, a), getattr(ps_r, a)), f"step {step}: primary {a}"
        rd, rb = reference_sets(rg)
        for mine, theirs, name in ((state.droplets, rd, "droplets"), (state.bubbles, rb, "bubbles")):
            assert len(mine) == len(theirs), f"step {step}: {name} count {len(mine)} vs {len(theirs)}"
            for a in ("pos", "vel", "vol", "age"):
                assert np.array_equal(getattr(mine, a), getattr(theirs, a)), f"step {step}: {name} {a}"
        life, spr, added, idx = reference_stats(rg)
        assert state.lifecycle.as_dict() == life.as_dict(), f"step {step}: lifecycle statistics"
        assert state.spray.as_dict() == spr.as_dict(), f"step {step}: spray statistics"
        assert state.added == added, f"step {step}: added"
        assert state.spray_step_index == idx
        seen_sets += len(state.droplets) + len(state.bubbles)
        seen_reab += life.reabsorbed_droplets_to_primary + life.reabsorbed_bubbles_to_primary
    assert seen_sets > 0, "no secondary particles in the scene"
    if case == "lifecycle_reabsorb":
        assert seen_reab > 0, "nothing reabsorbed"
    if case == "spray":
        assert state.spray.emitted_droplets > 0 and state.spray.interface_gate_passed
