"""Particle adaptivity (src/driver/particle_adaptivity3d.h): the C restatement
against the compiled reference, bit for bit, on seeded particle sets.

Covers applyNarrowBandAir, applyTypedParticleCoarsening (gas and liquid) and
applyLiquidParticleRefill with its interface-only and budget options, plus the
edge cases the functions branch on: no liquid at all, particles outside the
grid or at non-finite positions, overfull cells, refill targets above the 8
sub-cell slots, and an exhausted budget.
"""
import numpy as np
import pytest

import oracle as O

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")


def adapt_scene(seed, n=10, npart=3000, outside=0.02, clusters=3, nonfinite=0):
    """Liquid below y = 0.45 and gas above, a few dense clusters, some
    particles outside the unit domain, FP32-representable values."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, (npart, 3))
    k = int(outside * npart)
    pos[:k] = rng.uniform(-0.08, 1.08, (k, 3))
    for c in range(clusters):
        centre = rng.uniform(0.1, 0.9, 3)
        m = 40
        pos[k + c * m:k + (c + 1) * m] = centre + rng.uniform(-0.03, 0.03, (m, 3))
    typ = (pos[:, 1] > 0.45).astype(np.uint8)
    typ[rng.random(npart) < 0.02] = 2  # a third type, left alone by every function
    vel = rng.normal(0, 0.5, (npart, 3))
    vol = rng.uniform(0.5, 1.5, npart)
    pos, vel, vol = (a.astype(np.float32).astype(np.float64) for a in (pos, vel, vol))
    if nonfinite:
        pos[-nonfinite:, 0] = np.nan
    return O.Particles(pos, vel, typ, vol)


def _same(a: O.Particles, b: O.Particles):
    assert len(a) == len(b)
    assert np.array_equal(a.type, b.type)
    for name in ("pos", "vel", "volume"):
        x, y = getattr(a, name), getattr(b, name)
        assert np.array_equal(np.isnan(x), np.isnan(y)), name
        assert np.array_equal(np.nan_to_num(x), np.nan_to_num(y)), name


def _both(n=10):
    dx = 1.0 / n
    return O.OracleGrid(n, n, n, dx), O.ReferenceGrid(n, n, n, dx)


@needs_ref
@pytest.mark.parametrize("radius,seed", [(0, 1), (1, 2), (2, 3), (3, 4)])
def test_narrow_band_air_matches_reference(radius, seed):
    go, gr = _both()
    ps = adapt_scene(seed, nonfinite=3)
    po, pr = ps.copy(), ps.copy()
    so = O.Oracle().narrow_band_air(go, po, radius)
    sr = O.Reference().narrow_band_air(gr, pr, radius)
    assert so.as_tuple() == sr.as_tuple()
    assert so.removed > 0
    _same(po, pr)


@needs_ref
def test_narrow_band_air_without_liquid_changes_nothing():
    go, gr = _both()
    ps = adapt_scene(5)
    ps.type[ps.type == 0] = 1
    po, pr = ps.copy(), ps.copy()
    so = O.Oracle().narrow_band_air(go, po, 2)
    sr = O.Reference().narrow_band_air(gr, pr, 2)
    assert so.as_tuple() == sr.as_tuple() == (0, 0, 0, 0)
    _same(po, ps)
    _same(pr, ps)


@needs_ref
@pytest.mark.parametrize("ptype,target,seed", [(1, 1, 11), (1, 2, 12), (1, 4, 13), (0, 3, 14), (0, 8, 15),
                                               (1, 0, 16)])
def test_coarsening_matches_reference(ptype, target, seed):
    go, gr = _both()
    ps = adapt_scene(seed, nonfinite=2)
    po, pr = ps.copy(), ps.copy()
    so = O.Oracle().coarsen_particles(go, po, ptype, target, 0x9e3779b9 ^ seed)
    sr = O.Reference().coarsen_particles(gr, pr, ptype, target, 0x9e3779b9 ^ seed)
    assert so.as_tuple() == sr.as_tuple()
    assert so.overfull_cells > 0
    _same(po, pr)


@needs_ref
@pytest.mark.parametrize("target,only,radius,budget,seed", [
    (4, False, 1, 0, 21), (8, False, 1, 0, 22), (11, False, 1, 0, 23),   # 11 > 8 slots: slots wrap
    (6, True, 1, 0, 24), (6, True, 2, 0, 25), (6, False, 1, 37, 26),     # interface-only, budget
    (1, False, 0, 0, 27), (5, True, 0, 1, 28),
])
def test_refill_matches_reference(target, only, radius, budget, seed):
    go, gr = _both()
    ps = adapt_scene(seed, npart=1500, nonfinite=2)
    po, pr = ps.copy(), ps.copy()
    so = O.Oracle().refill_liquid(go, po, target, 0x6a09e667 + seed, only, radius, budget)
    sr = O.Reference().refill_liquid(gr, pr, target, 0x6a09e667 + seed, only, radius, budget)
    assert so.as_tuple() == sr.as_tuple()
    if target > 1:
        assert so.added > 0
    if budget:
        assert so.budget_limited == 1 and so.added == budget
    _same(po, pr)


def test_scores_follow_the_hash():
    """particleScore / slotScore are deterministic, seed-dependent and spread."""
    o = O.Oracle()
    g = O.OracleGrid(8, 8, 8, 0.125)
    lib = o.lib
    x = np.array([0.3, 0.4, 0.55])
    a = lib.pfo_particle_score(g.h, x, 2, 3, 4, 7)
    assert a == lib.pfo_particle_score(g.h, x, 2, 3, 4, 7)
    assert a != lib.pfo_particle_score(g.h, x, 2, 3, 4, 8)
    s = {lib.pfo_slot_score(c, k, 1) for c in range(64) for k in range(8)}
    assert len(s) == 64 * 8
