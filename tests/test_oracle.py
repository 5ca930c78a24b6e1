"""CPU pinning of the oracle (the C restatement in oracle/pf_oracle.c).

1. Against the committed golden fixtures (outputs of the unmodified
   reference, tests/golden/make_golden.py): bit-for-bit.
2. Against the compiled reference itself (oracle/_ref) on fresh seeded
   scenes, when that library is present: bit-for-bit for P2G, projection,
   G2P, advection with escape records, and whole steps.
3. The reference's own inline known-answer tests, restated on the oracle
   (tests/test_sparse_transfer3d_tp.cpp, test_sparse_vc3d.cpp, test_pressure3d_vc.cpp,
   test_phasefield.cpp, test_block_color.cpp).
"""
import json
import math
import os

import numpy as np
import pytest

import oracle as O
import vc_cases
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")


def _particles(z):
    return O.Particles(z["pos"].astype(np.float64), z["vel"].astype(np.float64), z["type"],
                       z["volume"].astype(np.float64))


def _phase(arr):
    return O.PhaseParams(*[float(v) for v in arr])


def _assert_grid_equal(g, z, prefix="", fields=range(8)):
    for f in fields:
        name = O.FIELD_NAMES[f]
        d, a = g.get_field(f)
        assert np.array_equal(a, z[prefix + name + "_act4"]), f"{name}: activity differs"
        assert np.array_equal(d, z[prefix + name]), f"{name}: values differ"


# ---------------------------------------------------------------- golden

@pytest.mark.parametrize("fname", ["p2g_rt12.npz", "p2g_bubble16.npz"])
def test_oracle_p2g_matches_golden(fname):
    z = np.load(os.path.join(GOLDEN, fname))
    n = int(z["n"])
    g = O.OracleGrid(n, n, n, float(z["dx"]))
    O.Oracle().p2g(g, _particles(z), _phase(z["phase"]), 1.0)
    _assert_grid_equal(g, z, fields=range(6))


def test_oracle_steps_match_golden():
    z = np.load(os.path.join(GOLDEN, "step_rt12.npz"))
    n = int(z["n"])
    cfg = json.loads(str(z["cfg"]))
    cfg["cg_rel_tol"] = 0.0
    ps = _particles(z)
    g, s = O.OracleGrid(n, n, n, float(z["dx"])), O.OracleGrid(n, n, n, float(z["dx"]))
    for step in range(3):
        O.Oracle().step(g, s, ps, _phase(z["phase"]), cfg)
        assert np.array_equal(ps.pos, z[f"pos{step}"]), f"step {step} positions"
        assert np.array_equal(ps.vel, z[f"vel{step}"]), f"step {step} velocities"
    _assert_grid_equal(g, z, "last_")


def test_known_answers_match_golden():
    ka = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    o = O.Oracle()
    d = O.PhaseParams()
    assert o.phi_from_raw(d.rho_g, d) == ka["phi_rho_g"]
    assert o.phi_from_raw(d.rho_l, d) == ka["phi_rho_l"]
    assert o.calibrate_rho_tilde0(d, 1.0) == ka["calibrate_default"]
    assert o.calibrate_rho_tilde0(O.PhaseParams(1000.0, 1.0), 1.0) == ka["calibrate_1000_1"]
    g = O.OracleGrid(8, 8, 8, 1.0)
    one = O.Particles(np.array([[3.0, 2.5, 2.5]]), np.array([[4.0, 3.0, 2.0]]), np.array([0]), np.array([1.0]))
    o.p2g(g, one, d, 1.0)
    u, _ = g.get_field(O.U)
    mu, act = g.get_field(O.MU)
    assert float((u.astype(np.float64) * mu.astype(np.float64)).sum()) == ka["p2g_momentum_u"]
    assert int(act.sum()) == ka["p2g_mu_active_blocks"]


# ------------------------------------------------------ live reference

def _random_scene(n, seed, npart, air_fraction=0.0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    pos = rng.uniform(0.6 * dx, 1 - 0.6 * dx, (npart, 3)).astype(np.float32).astype(np.float64)
    if air_fraction:
        keep = pos[:, 1] < 1.0 - air_fraction
        pos = pos[keep]
    vel = rng.normal(0, 0.3, pos.shape)
    typ = (pos[:, 1] > 0.45).astype(np.uint8)
    vol = rng.uniform(0.5, 1.5, len(pos))
    return O.Particles(pos, vel, typ, vol)


@needs_ref
@pytest.mark.parametrize("seed,n,air", [(0, 8, 0.0), (1, 12, 0.3), (2, 10, 0.5)])
def test_oracle_equals_reference_per_call(seed, n, air):
    o, r = O.Oracle(), O.Reference()
    pp = O.PhaseParams(1000.0, 1.0)
    pp.rho_tilde_0 = r.calibrate_rho_tilde0(pp, 1.0)
    ps = _random_scene(n, seed, 40 * n ** 2, air)
    go, gr = O.OracleGrid(n, n, n, 1.0 / n), O.ReferenceGrid(n, n, n, 1.0 / n)
    o.p2g(go, ps, pp, 1.0)
    r.p2g(gr, ps, pp, 1.0)
    for f in range(6):
        a, b = go.get_field(f), gr.get_field(f)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[0], b[0]), O.FIELD_NAMES[f]
    # markers through the oracle, copied to the reference; then project both
    o.mark_cells(go, ps)
    o.apply_gravity(go, 1 / 240, -9.81)
    o.apply_wall_boundary(go)
    for f in range(8):
        gr.set_field(f, *go.get_field(f))
    so, sr = go.copy(), gr.copy()
    st = o.project(go, pp, 1 / 240, 600, 1e-9)
    r.project(gr, pp, 1 / 240, 600, 1e-9)
    for f in range(8):
        a, b = go.get_field(f), gr.get_field(f)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[0], b[0]), O.FIELD_NAMES[f]
    assert st.iterations > 0
    po, pr = ps.copy(), ps.copy()
    o.g2p(go, po, so, 0.95, 0.8)
    r.g2p(gr, pr, sr, 0.95, 0.8)
    assert np.array_equal(po.vel, pr.vel)
    for order in (2, 3):
        qo, qr = po.copy(), pr.copy()
        so_st, so_esc = o.advect(qo, go, 0.05, order, escape=True)
        sr_st, sr_esc = r.advect(qr, gr, 0.05, order, escape=True)
        assert np.array_equal(qo.pos, qr.pos)
        assert so_st.as_tuple() == sr_st.as_tuple()
        assert np.array_equal(so_esc, sr_esc)


@needs_ref
def test_oracle_equals_reference_full_steps():
    o, r = O.Oracle(), O.Reference()
    n = 10
    ps = _random_scene(n, 5, 30 * n ** 2, 0.3)
    pp = O.PhaseParams(1000.0, 1.0)
    pp.rho_tilde_0 = r.calibrate_rho_tilde0(pp, 1.0)
    cfg = dict(dt=1 / 120, gravity=-9.81, Vp=1.0, alpha_l=0.95, alpha_g=0.9, cg_iters=400, cg_tol=1e-8)
    po, pr = ps.copy(), ps.copy()
    go, so, gr = O.OracleGrid(n, n, n, 1.0 / n), O.OracleGrid(n, n, n, 1.0 / n), O.ReferenceGrid(n, n, n, 1.0 / n)
    for _ in range(4):
        o.step(go, so, po, pp, cfg)
        r.step(gr, pr, pp, cfg)
        assert np.array_equal(po.pos, pr.pos)
        assert np.array_equal(po.vel, pr.vel)
    for f in range(8):
        a, b = go.get_field(f), gr.get_field(f)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[0], b[0]), O.FIELD_NAMES[f]


@needs_ref
def test_reference_allocation_order_is_a_permutation_of_the_sorted_set():
    """The reference lists active blocks in first-touch order; the GPU returns
    them sorted.  The sets are what must agree."""
    r = O.Reference()
    n = 12
    ps = _random_scene(n, 3, 2000, 0.4)
    g = O.ReferenceGrid(n, n, n, 1.0 / n)
    r.p2g(g, ps, O.PhaseParams(), 1.0)
    order = g.allocation_order(O.U)
    assert sorted(order.tolist()) == g.active_blocks(O.U).tolist()


@needs_ref
@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_cell_list_equals_reference_collect(seed):
    """The oracle's fluid-cell list (pfo_collect_cells, the projection's
    enumeration) is the reference's collectCellsWithMarker, bit for bit, on
    markCells output and on a random marker field with holes."""
    n = 14
    o = O.Oracle()
    go = O.OracleGrid(n, n, n, 1.0 / n)
    o.mark_cells(go, _random_scene(n, seed, 3000, 0.3))
    rng = np.random.default_rng(seed)
    for mk in (go.cell_markers(), rng.choice([0, 1, 2], size=(n, n, n), p=[0.4, 0.5, 0.1])):
        a, b = O.OracleGrid(n, n, n, 1.0 / n), O.ReferenceGrid(n, n, n, 1.0 / n)
        a.set_cells(mk)
        b.set_cells(mk)
        ref = b.collect_cells(1)
        assert len(ref) > 0
        assert np.array_equal(a.fluid_cells(), ref)


# ------------------------------------------- reference tests, restated

def test_phase_field_curve():
    # tests/test_phasefield.cpp:4-13
    o = O.Oracle()
    pp = O.PhaseParams()
    assert o.phi_from_raw(pp.rho_g, pp) == pytest.approx(0.0)
    # doctest::Approx(1.0).epsilon(0.02): |a-b| < eps * (scale 1 + max(|a|,|b|))
    f = o.phi_from_raw(pp.rho_l, pp)
    assert abs(f - 1.0) < 0.02 * (1.0 + max(abs(f), 1.0))
    prev = -1.0
    for rt in np.arange(0.0, 1.0 + 1e-12, 0.05):
        f = o.phi_from_raw(rt, pp)
        assert prev - 1e-12 <= f and 0.0 <= f <= 1.0
        prev = f
    rmin = math.log(pp.rho_l / pp.rho_g) * pp.rho_g * pp.rho_tilde_0
    assert o.phi_from_raw(rmin * 0.99, pp) == pytest.approx(0.0)
    assert o.phi_from_raw(rmin * 1.01 + 0.05, pp) > 0.0


def test_p2g_momentum_and_sparsity():
    # tests/test_sparse_transfer3d_tp.cpp:11-29
    g = O.OracleGrid(8, 8, 8, 1.0)
    ps = O.Particles(np.array([[3.0, 2.5, 2.5]]), np.array([[4.0, 3.0, 2.0]]), np.array([0]), np.array([1.0]))
    O.Oracle().p2g(g, ps, O.PhaseParams(), 1.0)
    u, _ = g.get_field(O.U)
    mu, act = g.get_field(O.MU)
    assert float((u.astype(np.float64) * mu).sum()) == pytest.approx(4.0, rel=1e-6)
    assert 0 < act.sum() < act.size


def test_p2g_phase_separation():
    # tests/test_sparse_transfer3d_tp.cpp:31-58
    pos, typ = [], []
    for k in range(1, 7):
        for j in range(1, 7):
            for i in range(1, 7):
                for s in range(8):
                    pos.append((i + 0.25 + 0.5 * (s & 1), j + 0.25 + 0.5 * ((s >> 1) & 1), k + 0.25 + 0.5 * ((s >> 2) & 1)))
                    typ.append(0 if j < 4 else 1)
    ps = O.Particles(np.array(pos), None, np.array(typ), None)
    o = O.Oracle()
    pp = O.PhaseParams()
    pp.rho_tilde_0 = o.calibrate_rho_tilde0(pp, 1.0)
    g = O.OracleGrid(8, 8, 8, 1.0)
    o.p2g(g, ps, pp, 1.0)
    mu, _ = g.get_field(O.MU)
    assert o.phi_from_raw(float(mu[3, 2, 4]), pp) > 0.8
    assert o.phi_from_raw(float(mu[3, 5, 4]), pp) < 0.2


def test_g2p_phase_alpha():
    # tests/test_sparse_transfer3d_tp.cpp:60-78
    g, s = O.OracleGrid(8, 8, 8, 1.0), O.OracleGrid(8, 8, 8, 1.0)
    ug = np.zeros((8, 8, 9), np.float32)
    us = np.zeros((8, 8, 9), np.float32)
    ug[1:3, 1:3, 2:4] = 5.0
    us[1:3, 1:3, 2:4] = 2.0
    act = np.zeros(g.bdims(O.U)[::-1], np.uint8)
    act[0, 0, 0] = 1
    g.set_field(O.U, ug, act)
    s.set_field(O.U, us, act)
    ps = O.Particles(np.array([[2.0, 2.0, 2.0]] * 2), np.array([[10.0, 0, 0]] * 2), np.array([0, 1]), None)
    O.Oracle().g2p(g, ps, s, 1.0, 0.0)
    assert ps.vel[0, 0] == pytest.approx(13.0)
    assert ps.vel[1, 0] == pytest.approx(5.0)


def test_advect_clamp_statistics():
    # tests/test_sparse_transfer3d_tp.cpp:123-161
    g = O.OracleGrid(8, 8, 8, 1.0)
    g.set_field(O.U, np.full((8, 8, 9), 10.0, np.float32), np.ones(g.bdims(O.U)[::-1], np.uint8))
    g.set_field(O.V, np.full((8, 9, 8), -10.0, np.float32), np.ones(g.bdims(O.V)[::-1], np.uint8))
    ps = O.Particles(np.array([[7.45, 4.0, 4.0], [4.0, 0.55, 4.0]]), None, np.array([0, 1]), None)
    st, esc = O.Oracle().advect(ps, g, 0.1, 2, escape=True)
    assert ps.pos[0, 0] == pytest.approx(7.5, rel=1e-12)
    assert ps.pos[1, 1] == pytest.approx(0.5, rel=1e-12)
    assert (st.clamped_liquid, st.clamped_gas, st.x_hi, st.y_lo) == (1, 1, 1, 1)
    assert len(esc) == 2 and esc[0, 0] == 0 and esc[1, 0] == 1
    assert esc[0, 1] == pytest.approx(7.5) and esc[1, 2] == pytest.approx(0.5) and esc[0, 7] == 1.0


def test_advect_rk3_linear_field():
    # tests/test_sparse_transfer3d_tp.cpp:163-180
    g = O.OracleGrid(8, 8, 8, 1.0)
    u = np.broadcast_to(np.arange(9, dtype=np.float32), (8, 8, 9)).copy()
    g.set_field(O.U, u, np.ones(g.bdims(O.U)[::-1], np.uint8))
    ps = O.Particles(np.array([[2.0, 4.0, 4.0]]), None, np.array([0]), None)
    O.Oracle().advect(ps, g, 0.1, 3)
    assert ps.pos[0, 0] == pytest.approx(2.0 + 0.1 / 6.0 * (2.0 + 4.0 * 2.1 + 2.22), rel=1e-6)


def _box(with_u):
    g = O.OracleGrid(8, 8, 8, 1.0)
    mk = np.zeros((8, 8, 8))
    mk[[0, -1], :, :] = 2
    mk[:, [0, -1], :] = 2
    mk[:, :, [0, -1]] = 2
    mk[2:6, 2:6, 2:6] = 1
    g.set_cells(mk)
    full = {f: np.ones(g.bdims(f)[::-1], np.uint8) for f in range(8)}
    mu = np.zeros((8, 8, 9), np.float32); mu[2:6, 2:6, 2:7] = 1
    mv = np.zeros((8, 9, 8), np.float32); mv[2:6, 2:6, 2:6] = 1
    mw = np.zeros((9, 8, 8), np.float32); mw[2:7, 2:6, 2:6] = 1
    g.set_field(O.MU, mu, full[O.MU]); g.set_field(O.MV, mv, full[O.MV]); g.set_field(O.MW, mw, full[O.MW])
    if with_u:
        u = np.zeros((8, 8, 9), np.float32)
        for i in range(2, 7):
            u[2:6, 2:6, i] = i
        g.set_field(O.U, u, full[O.U])
    return g


def _divergence(g):
    u, _ = g.get_field(O.U)
    v, _ = g.get_field(O.V)
    w, _ = g.get_field(O.W)
    u, v, w = (a.astype(np.float64) for a in (u, v, w))
    return (u[2:6, 2:6, 3:7] - u[2:6, 2:6, 2:6]) + (v[2:6, 3:7, 2:6] - v[2:6, 2:6, 2:6]) + \
        (w[3:7, 2:6, 2:6] - w[2:6, 2:6, 2:6])


def test_vc_projection_divergence_and_pressure_blocks():
    # tests/test_sparse_vc3d.cpp:8-54
    g = _box(True)
    O.Oracle().project(g, O.PhaseParams(), 1.0, 1000, 1e-9)
    assert np.max(np.abs(_divergence(g))) < 1e-4
    assert len(g.active_blocks(O.P)) == 8


def test_vc_projection_target_cdiv():
    # tests/test_sparse_vc3d.cpp:56-100
    g = _box(False)
    O.Oracle().project(g, O.PhaseParams(), 1.0, 1000, 1e-9, c_div=0.125)
    assert _divergence(g).mean() == pytest.approx(0.125, rel=1e-4)


def test_vc_beta_one_box_removes_divergence():
    # tests/test_pressure3d_vc.cpp:5-16
    g = O.OracleGrid(8, 8, 8, 1.0)
    dt = vc_cases.beta_one_box(g)
    st = O.Oracle().project(g, O.PhaseParams(*vc_cases.PHASE), dt, 1000, 1e-10)
    assert st.converged
    assert vc_cases.fluid_divergence(g) < 1e-5


def test_vc_hydrostatic_two_phase_bounded():
    # tests/test_pressure3d_vc.cpp:17-32
    g = O.OracleGrid(6, 16, 6, 1.0)
    dt = vc_cases.hydrostatic_two_phase(g)
    st = O.Oracle().project(g, O.PhaseParams(*vc_cases.PHASE), dt, 2000, 1e-10)
    assert st.converged and st.pin_cell >= 0
    assert vc_cases.interior_max_v(g) < 0.6


def test_relative_tolerance_rule_and_stats():
    """Relative stop max|r| < rel*max|r0| (multires_pressure3d.cpp:858-863)."""
    g = _box(True)
    st = O.Oracle().project(g, O.PhaseParams(), 1.0, 1000, 0.0, rel_tol=1e-6)
    assert st.converged and st.res_final < 1e-6 * st.res0
    assert st.tol_effective == pytest.approx(1e-6 * st.res0)


def test_block_colouring_separates_neighbours():
    # tests/test_block_color.cpp:19-31 -- colour8 of the 4^3 block lattice
    nbx, nby, nbz = 4, 3, 2
    col = lambda bx, by, bz: (bx & 1) + 2 * (by & 1) + 4 * (bz & 1)
    counts = np.zeros(8, int)
    for bz in range(nbz):
        for by in range(nby):
            for bx in range(nbx):
                c = col(bx, by, bz)
                counts[c] += 1
                for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                    q = (bx + d[0], by + d[1], bz + d[2])
                    if 0 <= q[0] < nbx and 0 <= q[1] < nby and 0 <= q[2] < nbz:
                        assert col(*q) != c
    assert counts.sum() == nbx * nby * nbz
