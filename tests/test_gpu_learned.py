"""GPU tests of the LEARNED pressure mode.

* The network's forward pass, loss, parameter gradient and Adam step through
  the C ABI (pf_learned_eval / pf_learned_adam) against the FP64 CPU
  restatement in oracle/coarse_net.py with the same BF16 operand rounding.
* The two-level flexible PCG: the exact coarse correction cuts iterations,
  Jacobi-only flexible PCG matches plain PCG, and every variant lands on the
  plain FP64 solution.
* Training on pairs harvested from exact two-level solves, then the ablation:
  the trained network against the same solver without it.
* The fallback: a network that yields non-finite corrections is rejected by
  the r.z guard, switched off after the rejection streak, and the solve
  still converges to the plain solution.
"""
import numpy as np
import pytest

from oracle import coarse_net as cn

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def small(pf):
    g = pf.SparseMacGrid3D(16, 16, 16, 1.0 / 16, max_particles=1)
    net = pf.LearnedCoarseSolver(g)
    net.init(seed=7)
    yield g, net
    g.close()


DIMS = (7, 5, 6)  # odd sizes exercise the ragged pooling / upsampling edges


def _system(seed, B=3, dims=DIMS):
    cop = cn.random_system(dims, seed=seed, contrast=1000.0)
    rng = np.random.default_rng(seed + 100)
    nt = int(np.prod(dims))
    rc = (rng.normal(0, 1, (B, nt, 2)) * cn.live_mask(cop)[None]).astype(np.float32)
    tgt = cn.exact_correction(cop, dims, rc).astype(np.float32)
    return cop, rc, tgt


@pytest.mark.parametrize("dims,B", [(DIMS, 3), (DIMS, 1), ((9, 9, 9), 1), ((13, 9, 6), 1)])
def test_forward_matches_cpu(small, dims, B):
    """Batches of residuals and the solver's single residual, on odd lattices."""
    _, net = small
    cop, rc, _ = _system(1, B=B, dims=dims)
    params = cn.unflatten(net.params())
    e_gpu = net.eval(dims, cop, rc)
    e_cpu = cn.coarse_correction(params, cop, dims, rc, round_bf16=True)
    assert np.all(np.isfinite(e_gpu))
    assert rel_l2(e_gpu, e_cpu) < 2e-3
    # dead unknowns get no correction
    live = cn.live_mask(cop)
    assert np.all(e_gpu[:, ~live] == 0.0)


@pytest.mark.parametrize("dims", [DIMS, (17, 3, 3)])  # 4 and 5 levels of G (the last weight shared)
def test_loss_and_gradient_match_cpu(small, dims):
    _, net = small
    cop, rc, tgt = _system(2, dims=dims)
    params = cn.unflatten(net.params())
    e_gpu, loss_gpu, grad_gpu = net.eval(dims, cop, rc, tgt)
    loss_cpu, grads_cpu, e_cpu = cn.loss_and_grad(params, cop, dims, rc, tgt, round_bf16=True)
    assert abs(loss_gpu - loss_cpu) <= 2e-3 * abs(loss_cpu)
    assert rel_l2(e_gpu, e_cpu) < 2e-3
    g_cpu = cn.flatten(grads_cpu)
    # per tensor: weights and biases of every layer
    names = [layer[0] for layer in cn.LAYERS] + [layer[0] for layer in cn.G_LAYERS]
    o = 0
    for q, s in enumerate(cn.param_shapes()):
        n = int(np.prod(s))
        err = rel_l2(grad_gpu[o:o + n], g_cpu[o:o + n])
        assert err < 2e-2, (names[q // 2], "W" if q % 2 == 0 else "b", err)
        o += n


def test_correction_is_linear_and_symmetric_up_to_bf16(small):
    """e = S G^T G S r: linear and symmetric in r up to the BF16 rounding of
    the convolution operands, and positive."""
    _, net = small
    cop, rc, _ = _system(3, B=2)
    e = net.eval(DIMS, cop, np.concatenate([rc, (2.0 * rc[:1] - 3.0 * rc[1:])], axis=0))
    lin = e[2] - (2.0 * e[0] - 3.0 * e[1])
    assert np.linalg.norm(lin) < 2e-2 * np.linalg.norm(e[2])
    s12, s21 = float(np.sum(rc[0] * e[1])), float(np.sum(rc[1] * e[0]))
    assert abs(s12 - s21) < 2e-2 * max(abs(s12), abs(s21))
    assert float(np.sum(rc[0] * e[0])) > 0 and float(np.sum(rc[1] * e[1])) > 0


def test_adam_matches_cpu(pf):
    g = pf.SparseMacGrid3D(16, 16, 16, 1.0 / 16, max_particles=1)
    try:
        net = pf.LearnedCoarseSolver(g)
        net.init(seed=3)
        p0 = cn.unflatten(net.params())
        rng = np.random.default_rng(5)
        m = [np.zeros_like(p) for p in p0]
        v = [np.zeros_like(p) for p in p0]
        p = p0
        for step in (1, 2, 3):
            grad = rng.normal(0, 1e-2, cn.num_params()).astype(np.float32)
            net.adam(grad, lr=1e-3)
            p = cn.adam(p, cn.unflatten(grad.astype(np.float64)), m, v, step, 1e-3)
        got = net.params()
        assert rel_l2(got, cn.flatten(p)) < 1e-6
        assert np.max(np.abs(got - cn.flatten(p))) < 1e-6
    finally:
        g.close()


def test_load_rejects_bad_parameter_vectors(small, pf):
    _, net = small
    with pytest.raises(pf.PfError):
        net.load(np.zeros(cn.num_params() - 1, np.float32))
    bad = np.zeros(cn.num_params(), np.float32)
    bad[10] = np.nan
    with pytest.raises(pf.PfError):
        net.load(bad)


# ---------------------------------------------------------------------------
# the solver


def _pressure_system(pf, n, seed, g=None):
    """The ellipsoid pressure system of `seed` on grid g (a new n^3 grid if
    None); returns the grid and a solve(cfg) that resets the velocities."""
    sc = pf.scenes.ellipsoid_pressure(n, seed=seed)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    if g is None:
        g = pf.SparseMacGrid3D(n, n, n, sc["dx"], max_particles=1)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0, grid=g)
    f = pf.scenes.pressure_grid_fields(sc, pp.rho_tilde_0)
    names = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")
    full = {k: np.ones(g.bdims(i)[::-1], np.uint8) for i, k in enumerate(names)}
    for k in ("mu", "mv", "mw", "mk"):
        g.set_field(names.index(k), f[k], full[k])

    def solve(cfg, max_iter=20000):
        for k in ("u", "v", "w"):
            g.set_field(names.index(k), f[k], full[k])
        st = pf.spProjectStepVC3D(g, pp, 1.0 / 240.0, max_iter, 0.0, solver=cfg)
        p, _ = g.get_field(pf.PF_P)
        return st, p.astype(np.float64)

    return g, solve


@pytest.fixture(scope="module")
def trained(pf):
    """A network trained on pairs harvested from exact two-level solves of
    three seeded 64^3 systems (seeds 1-3); seed 0 is kept for evaluation."""
    L = pf.PF_SOLVER_LEARNED
    g = None
    net = None
    for seed in (1, 2, 3):
        g, solve = _pressure_system(pf, 64, seed=seed, g=g)
        if net is None:
            net = pf.LearnedCoarseSolver(g)
            net.init(seed=11)
            net.harvest(True, stride=2, max_per_system=200, capacity_floats=1 << 24)
        st, _ = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_EXACT_COARSE))
        assert st.converged
    net.harvest(False)
    systems, pairs = net.dataset()
    assert systems == 3 and pairs >= 3 * 150
    losses = net.train(steps=1200, batch=8, lr=1e-3, seed=1)
    out = {"losses": losses, "params": net.params(), "dataset": (systems, pairs)}
    g.close()
    return out


def test_two_level_solvers_agree_with_plain(pf):
    L = pf.PF_SOLVER_LEARNED
    g, solve = _pressure_system(pf, 64, seed=0)
    try:
        st_p, p_plain = solve(pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6))
        st_j, p_j = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI))
        st_e, p_e = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_EXACT_COARSE))
        for st in (st_p, st_j, st_e):
            assert st.converged and st.res_final <= 1e-6 * st.res0
        scale = np.abs(p_plain).max()
        assert np.abs(p_j - p_plain).max() < 1e-5 * scale
        assert np.abs(p_e - p_plain).max() < 1e-5 * scale
        # flexible Jacobi-PCG is plain PCG up to rounding; the exact coarse term cuts iterations 3x or more
        assert abs(st_j.iterations - st_p.iterations) <= 0.05 * st_p.iterations
        assert st_e.iterations * 3 <= st_j.iterations
        assert st_e.precond_applied > 0
    finally:
        g.close()


def test_training_reduces_the_loss(trained):
    ls = trained["losses"]
    assert np.all(np.isfinite(ls))
    assert ls[-50:].mean() < 0.5 * ls[:20].mean()


def test_learned_preconditioner_ablation(pf, trained):
    """Trained network vs the same flexible PCG without it (Jacobi), on a
    system it was not trained on; both must reach the plain solution."""
    L = pf.PF_SOLVER_LEARNED
    g, solve = _pressure_system(pf, 64, seed=0)
    try:
        net = pf.LearnedCoarseSolver(g)
        net.load(trained["params"])
        st_p, p_plain = solve(pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6))
        st_j, _ = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI))
        st_n, p_n = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK))
        assert st_n.converged and st_n.res_final <= 1e-6 * st_n.res0
        # two solves that both meet max|r| <= 1e-6 max|r0| differ by the
        # conditioning times that residual, not by 1e-6
        assert np.abs(p_n - p_plain).max() < 2e-4 * np.abs(p_plain).max()
        assert st_n.precond_applied > 0
        assert st_n.iterations < 0.85 * st_j.iterations, (st_n.iterations, st_j.iterations)
    finally:
        g.close()


def test_fallback_on_a_network_that_overflows(pf):
    L = pf.PF_SOLVER_LEARNED
    g, solve = _pressure_system(pf, 32, seed=4)
    try:
        net = pf.LearnedCoarseSolver(g)
        net.load(np.full(cn.num_params(), 1e30, np.float32))  # finite weights, non-finite activations
        st_p, p_plain = solve(pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6))
        st_j, _ = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI))
        st_n, p_n = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK))
        assert st_n.converged
        assert st_n.precond_applied == 0
        assert st_n.precond_rejected == 8  # the streak that switches the coarse term off
        assert abs(st_n.iterations - st_j.iterations) <= 0.05 * st_j.iterations + 2
        assert np.abs(p_n - p_plain).max() < 1e-5 * np.abs(p_plain).max()
    finally:
        g.close()


def test_network_mode_without_weights_is_an_error(pf):
    g, solve = _pressure_system(pf, 32, seed=5)
    try:
        with pytest.raises(pf.PfError):
            solve(pf.SolverConfig(mode=pf.PF_SOLVER_LEARNED, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK))
    finally:
        g.close()


def test_merge_dataset_across_grid_sizes(pf):
    """Pairs harvested on two grids of different size train in one context."""
    L = pf.PF_SOLVER_LEARNED
    g1, solve1 = _pressure_system(pf, 32, seed=6)
    g2, solve2 = _pressure_system(pf, 48, seed=7)
    try:
        n1, n2 = pf.LearnedCoarseSolver(g1), pf.LearnedCoarseSolver(g2)
        n1.init(seed=1)
        n2.load(n1.params())
        for net, solve in ((n1, solve1), (n2, solve2)):
            net.harvest(True, stride=1, max_per_system=20, capacity_floats=1 << 22)
            st, _ = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_EXACT_COARSE))
            assert st.converged
            net.harvest(False)
        s1, p1 = n1.dataset()
        s2, p2 = n2.dataset()
        assert s1 == 1 and s2 == 1 and p1 > 0 and p2 > 0
        n1.merge_dataset(n2)
        assert n1.dataset() == (s1 + s2, p1 + p2)
        losses = n1.train(steps=20, batch=4, lr=1e-3, seed=3)
        assert np.all(np.isfinite(losses))
    finally:
        g1.close()
        g2.close()


def test_shipped_weights_ablation_128(pf):
    """The shipped weights on a 128^3 system none of the training systems
    was: at most 0.6x the iterations of the same flexible PCG without the
    network, same plain solution."""
    L = pf.PF_SOLVER_LEARNED
    g, solve = _pressure_system(pf, 128, seed=0)
    try:
        net = pf.LearnedCoarseSolver(g)
        net.load_default()
        st_p, p_plain = solve(pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6))
        st_j, _ = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI))
        st_n, p_n = solve(pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK))
        assert st_n.converged and st_n.res_final <= 1e-6 * st_n.res0
        assert st_n.precond_rejected == 0
        assert np.abs(p_n - p_plain).max() < 2e-4 * np.abs(p_plain).max()
        assert st_n.iterations < 0.6 * st_j.iterations, (st_n.iterations, st_j.iterations)
    finally:
        g.close()


@pytest.mark.parametrize("name", ["mixed_fp32", "mixed_bf16", "mixed_bf16_dir", "learned_mixed"])
def test_inner_outer_solvers_reach_the_fp64_tolerance(pf, name):
    """The reduced-precision solvers at 1000:1: FP64 flexible CG on the exact
    operator, preconditioned by an inner solve in FP32 (Jacobi-PCG with FP32
    or BF16 couplings and directions, or the learned flexible PCG).  Each
    reaches the 1e-6 relative FP64 residual and the plain solution, where
    FP32 iterative refinement stalls at this condition number."""
    g, solve = _pressure_system(pf, 64, seed=0)
    try:
        cfg = {
            "mixed_fp32": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6),
            "mixed_bf16": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6, bf16_storage=1),
            "mixed_bf16_dir": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6, bf16_storage=2),
            "learned_mixed": pf.SolverConfig(mode=pf.PF_SOLVER_LEARNED, rel_tol=1e-6,
                                             precond=pf.PF_PRECOND_NETWORK, inner_fp32=True),
        }[name]
        if name == "learned_mixed":
            pf.LearnedCoarseSolver(g).load_default()
        st_p, p_plain = solve(pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6))
        st, p = solve(cfg, max_iter=60000)
        assert st.converged and st.res_final <= 1e-6 * st.res0, (st.iterations, st.res_final / st.res0)
        assert st.refinements > 0  # outer FP64 iterations
        assert np.abs(p - p_plain).max() < 2e-4 * np.abs(p_plain).max()
    finally:
        g.close()


def test_solutions_against_the_fp64_oracle(pf):
    """Every solver mode's pressure on a 48^3 ellipsoid system at 1000:1 (the
    network with its shipped weights) against the CPU FP64 oracle's
    (oracle/pf_oracle.c, Jacobi-PCG to a 1e-10 relative residual).  The
    single-level FP64 Krylov solves on the exact operator (PLAIN, and the
    flexible PCG with or without the network) land within 1e-6 of the
    pressure scale.  The inner-outer solvers stop at the same 1e-6 relative
    FP64 residual along another Krylov path, and at 1000:1 that residual
    bounds the error only to about 1e-5."""
    import oracle as O

    n = 48
    sc = pf.scenes.ellipsoid_pressure(n, seed=0)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    names = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")
    g, solve = _pressure_system(pf, n, seed=0)
    try:
        pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0, grid=g)
        f = pf.scenes.pressure_grid_fields(sc, pp.rho_tilde_0)
        go = O.OracleGrid(n, n, n, sc["dx"])
        for k in ("u", "v", "w", "mu", "mv", "mw", "mk"):
            i = names.index(k)
            go.set_field(i, f[k], np.ones(go.bdims(i)[::-1], np.uint8))
        st_o = O.Oracle().project(go, O.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0), 1.0 / 240.0,
                                  200000, 0.0, rel_tol=1e-10)
        assert st_o.converged
        p_o, _ = go.get_field(O.P)
        p_o = p_o.astype(np.float64)
        scale = np.abs(p_o).max()
        pf.LearnedCoarseSolver(g).load_default()
        L = pf.PF_SOLVER_LEARNED
        modes = {
            "plain": (pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6), 1e-6),
            "learned": (pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK), 1e-6),
            "flex_jacobi": (pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI), 1e-6),
            "mixed_fp32": (pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6), 1e-5),
            "learned_mixed": (pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK, inner_fp32=True),
                              1e-5),
            "mixed_bf16": (pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6, bf16_storage=1), 1e-5),
        }
        errs = {}
        for name, (cfg, tol) in modes.items():
            st, p = solve(cfg, max_iter=60000)
            assert st.converged and st.res_final <= 1e-6 * st.res0, name
            errs[name] = float(np.abs(p - p_o).max() / scale)
        print("error against the FP64 oracle:", errs)
        for name, (_, tol) in modes.items():
            assert errs[name] <= tol, (name, errs)
    finally:
        g.close()
