"""GPU particle adaptivity against the oracle (src/driver/particle_adaptivity3d.h).

The oracle is pinned bit for bit to the compiled reference
(tests/test_adapt_oracle.py).  Inputs are FP32-representable, and the device
does the reference's FP64 arithmetic in the reference's order before it rounds
to its FP32 storage.  So the GPU result must equal the oracle's result rounded
to FP32, exactly: the particle count and order, types, positions, velocities,
volumes and every statistic.
"""
import numpy as np
import pytest

import oracle as O
from test_adapt_oracle import adapt_scene

pytestmark = pytest.mark.gpu


def _grid(pf, ps, n=10, extra=8):
    return pf.SparseMacGrid3D(n, n, n, 1.0 / n, max_particles=len(ps) * extra + 64)


def _to_pf(pf, ps):
    return pf.Particles3DTP(ps.pos.copy(), ps.vel.copy(), ps.type.copy(), ps.volume.copy())


def _equal_fp32(gpu, ora: O.Particles):
    assert len(gpu) == len(ora)
    assert np.array_equal(gpu.type, ora.type)
    for name in ("pos", "vel", "volume"):
        a = getattr(gpu, name).astype(np.float32)
        b = getattr(ora, name).astype(np.float32)
        assert np.array_equal(np.isnan(a), np.isnan(b)), name
        assert np.array_equal(np.nan_to_num(a), np.nan_to_num(b)), name


@pytest.mark.parametrize("radius,seed", [(0, 1), (1, 2), (2, 3), (3, 4)])
def test_narrow_band_air_matches_oracle(pf, radius, seed):
    ps = adapt_scene(seed, nonfinite=3)
    g = _grid(pf, ps)
    q = _to_pf(pf, ps)
    st = pf.applyNarrowBandAir(q, g, True, radius)
    so = O.Oracle().narrow_band_air(O.OracleGrid(10, 10, 10, 0.1), ps, radius)
    assert st.as_tuple() == so.as_tuple()
    _equal_fp32(q, ps)
    g.close()


def test_narrow_band_air_without_liquid(pf):
    ps = adapt_scene(5)
    ps.type[ps.type == 0] = 1
    g = _grid(pf, ps)
    q = _to_pf(pf, ps)
    st = pf.applyNarrowBandAir(q, g, True, 2)
    assert st.as_tuple() == (0, 0, 0, 0)
    _equal_fp32(q, ps)
    g.close()


@pytest.mark.parametrize("ptype,target,seed", [(1, 1, 11), (1, 2, 12), (1, 4, 13), (0, 3, 14), (0, 8, 15),
                                               (1, 0, 16)])
def test_coarsening_matches_oracle(pf, ptype, target, seed):
    ps = adapt_scene(seed, nonfinite=2)
    g = _grid(pf, ps)
    q = _to_pf(pf, ps)
    st = pf.applyTypedParticleCoarsening(q, g, True, ptype, target, 0x9e3779b9 ^ seed)
    so = O.Oracle().coarsen_particles(O.OracleGrid(10, 10, 10, 0.1), ps, ptype, target, 0x9e3779b9 ^ seed)
    assert st.as_tuple() == so.as_tuple()
    assert so.overfull_cells > 0
    _equal_fp32(q, ps)
    g.close()


@pytest.mark.parametrize("target,only,radius,budget,seed", [
    (4, False, 1, 0, 21), (8, False, 1, 0, 22), (11, False, 1, 0, 23),
    (6, True, 1, 0, 24), (6, True, 2, 0, 25), (6, False, 1, 37, 26), (1, False, 0, 0, 27), (5, True, 0, 1, 28),
])
def test_refill_matches_oracle(pf, target, only, radius, budget, seed):
    ps = adapt_scene(seed, npart=1500, nonfinite=2)
    g = _grid(pf, ps, extra=12)
    q = _to_pf(pf, ps)
    st = pf.applyLiquidParticleRefill(q, g, True, target, 0x6a09e667 + seed, only, radius, budget)
    so = O.Oracle().refill_liquid(O.OracleGrid(10, 10, 10, 0.1), ps, target, 0x6a09e667 + seed, only, radius,
                                  budget)
    assert st.as_tuple() == so.as_tuple()
    _equal_fp32(q, ps)
    g.close()


def test_refill_over_capacity_fails_and_changes_nothing(pf):
    ps = adapt_scene(30, npart=800)
    g = pf.SparseMacGrid3D(10, 10, 10, 0.1, max_particles=len(ps) + 5)
    q = _to_pf(pf, ps)
    g.upload(q)
    with pytest.raises(pf.PfError):
        st = pf.sparse.L.RefillStats()
        pf.sparse.L.check(g.lib.pf_refill_liquid(g.ctx, 8, 1, 0, 1, 0, pf.sparse.C.byref(st)), g.ctx, "refill")
    back = pf.Particles3DTP()
    g.take_particles(back)
    _equal_fp32(back, ps)
    g.close()


def test_step_applies_adaptivity_first(pf):
    """SparseSim3DTP::step() with every switch on: the adaptivity part of the
    step equals the oracle's sequence of the four functions."""
    n = 16
    sc = pf.scenes.rayleigh_taylor(n, seed=3)
    rng = np.random.default_rng(3)
    keep = rng.random(len(sc["pos"])) < 0.6  # thin the seeding so refill has work
    pos, vel = sc["pos"][keep], np.zeros_like(sc["pos"][keep])
    typ, vol = sc["type"][keep], sc["volume"][keep]
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=4 * len(pos))
    sim.phase = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    sim.phase.rho_tilde_0 = pf.calibrateRhoTilde0(sim.phase, 1.0)
    sim.dt = 1 / 240
    sim.solver = pf.SolverConfig(rel_tol=1e-6)
    sim.narrow_band_air = sim.gas_particle_coarsening = True
    sim.liquid_particle_coarsening = sim.liquid_particle_refill = True
    sim.gas_particles_per_cell_target, sim.liquid_particles_per_cell_target = 2, 6
    sim.liquid_refill_particles_per_cell_target = 5
    sim.narrow_band_air_radius = 1
    sim.set_particles(pos, vel, typ, vol)
    a = sim.applyParticleAdaptivity()
    ps = O.Particles(pos.astype(np.float64), vel.astype(np.float64), typ, vol.astype(np.float64))
    go = O.OracleGrid(n, n, n, 1.0 / n)
    o = O.Oracle()

    def fp32(st):
        # the device keeps FP32 particles between the calls
        for name in ("pos", "vel", "volume"):
            setattr(ps, name, getattr(ps, name).astype(np.float32).astype(np.float64))
        return st.as_tuple()

    assert a.band.as_tuple() == fp32(o.narrow_band_air(go, ps, 1))
    assert a.gas.as_tuple() == fp32(o.coarsen_particles(go, ps, 1, 2, 0x9e3779b9))
    assert a.liquid.as_tuple() == fp32(o.coarsen_particles(go, ps, 0, 6, 0x7f4a7c15))
    assert a.refill.as_tuple() == fp32(o.refill_liquid(go, ps, 5, 0x6a09e667, False, 1, 0))
    assert a.band.removed > 0 and a.gas.removed > 0 and a.refill.added > 0
    p2, v2, t2, w2 = sim.get_particles()
    assert len(p2) == len(ps) == sim.n
    assert np.array_equal(t2, ps.type)
    assert np.array_equal(p2, ps.pos.astype(np.float32))
    assert np.array_equal(w2, ps.volume.astype(np.float32))
    # and a whole step with the switches on runs and keeps the count it reports
    sim.step()
    assert sim.n == int(sim.grid.lib.pf_num_particles(sim.grid.ctx))
    assert np.all(np.isfinite(sim.get_particles()[0]))
