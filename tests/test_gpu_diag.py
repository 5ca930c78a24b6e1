"""GPU interface diagnostics against the oracle (diagnoseSparseInterface3D,
src/driver/interface_diagnostics3d.cpp:363-379), which is pinned to the
compiled reference in tests/test_diag_oracle.py.

Every per-cell value (phi, gradient, curvature) rounds as the reference's, so
the counts, the finite and candidate flags, and the minima and maxima must be
equal.  The three means are sums over the fluid cells in another order than
the reference's ascending one: within 1e-12 relative."""
import numpy as np
import pytest

import oracle as O
from gpu_helpers import scene_particles
from test_diag_oracle import stepped_pair

pytestmark = pytest.mark.gpu

EXACT = ("sample_cells", "interface_cells", "finite", "surface_tension_candidate", "phi_min", "phi_max", "grad_max",
         "curvature_abs_max")
MEANS = ("phi_mean", "grad_mean", "curvature_abs_mean")


def _check(gs, os_):
    for f in EXACT:
        assert getattr(gs, f) == getattr(os_, f), f
    for f in MEANS:
        a, b = getattr(gs, f), getattr(os_, f)
        assert abs(a - b) <= 1e-12 * max(abs(b), 1e-300), (f, a, b)


@pytest.mark.parametrize("n,seed,air", [(8, 1, 0.0), (12, 2, 0.3), (16, 3, 0.5), (24, 7, 0.2)])
def test_interface_diagnostics_match_oracle(pf, n, seed, air):
    go, _, pp = stepped_pair(n, seed, air)
    g = pf.SparseMacGrid3D(n, n, n, 1.0 / n)
    for f in range(8):
        g.set_field(f, *go.get_field(f))
    gs = pf.diagnoseSparseInterface3D(g, pf.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0))
    os_ = O.Oracle().interface_diagnostics(go, pp)
    assert os_.interface_cells > 0
    _check(gs, os_)
    g.close()


def test_step_records_diagnostics_after_p2g(pf):
    """pf_step computes the diagnostics right after P2G, as the reference's step does."""
    n = 16
    sc = pf.scenes.rayleigh_taylor(n, seed=2)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0)
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
    sim.phase, sim.dt = pp, 1 / 240
    sim.solver = pf.SolverConfig(rel_tol=1e-6)
    sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
    sim.step()
    # the same markCells + P2G on the oracle
    ps = scene_particles(sc)
    go = O.OracleGrid(n, n, n, 1.0 / n)
    opp = O.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0)
    O.Oracle().mark_cells(go, ps)
    O.Oracle().p2g(go, ps, opp, 1.0)
    os_ = O.Oracle().interface_diagnostics(go, opp)
    got = sim.interface_diagnostics_last
    assert got.sample_cells == os_.sample_cells and got.interface_cells == os_.interface_cells
    assert got.finite == 1 and got.surface_tension_candidate == os_.surface_tension_candidate
    # P2G's FP32 accumulation order differs from the reference's: phi agrees to rounding
    for f in ("phi_min", "phi_max", "phi_mean", "grad_mean", "grad_max"):
        assert abs(getattr(got, f) - getattr(os_, f)) <= 1e-4 * max(abs(getattr(os_, f)), 1.0), f


@pytest.mark.parametrize("n,seed,air,strength,maxdv,radius", [
    (12, 2, 0.3, 0.07, 0.0, 0), (12, 3, 0.3, 0.07, 0.0, 1), (16, 4, 0.5, 0.2, 0.05, 2), (24, 5, 0.0, 1.0, 0.0, 3),
    (10, 6, 0.2, 0.0, 0.0, 1),
])
def test_surface_tension_matches_oracle(pf, n, seed, air, strength, maxdv, radius):
    """applySparseSurfaceTension3D: face velocities equal the oracle's bit for
    bit; counts, flags and maxima exact, means within 1e-12."""
    go, _, pp = stepped_pair(n, seed, air)
    g = pf.SparseMacGrid3D(n, n, n, 1.0 / n)
    for f in range(8):
        g.set_field(f, *go.get_field(f))
    dt = 1 / 120
    gs = pf.applySparseSurfaceTension3D(g, pf.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0), dt,
                                        strength, maxdv, radius)
    os_ = O.Oracle().surface_tension(go, pp, dt, strength, maxdv, radius)
    for f in ("enabled", "applied_cells", "finite", "curvature_smoothing_radius", "capillary_stable", "strength",
              "max_delta_speed_limit", "max_delta_speed", "raw_curvature_abs_max", "smoothed_curvature_abs_max",
              "capillary_dt_limit"):
        assert getattr(gs, f) == getattr(os_, f), f
    for f in ("mean_delta_speed", "raw_curvature_abs_mean", "smoothed_curvature_abs_mean"):
        a, b = getattr(gs, f), getattr(os_, f)
        assert abs(a - b) <= 1e-12 * max(abs(b), 1e-300), f
    for f in range(8):
        a, b = g.get_field(f), go.get_field(f)
        assert np.array_equal(a[1], b[1]), f"field {f}: activity"
        assert np.array_equal(a[0], b[0]), f"field {f}: values"
    if strength > 0:
        assert os_.applied_cells > 0
    g.close()
