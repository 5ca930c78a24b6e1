"""CPU checks of the FP64 restatement of the learned coarse solve
(oracle/coarse_net.py): its hand-written backward pass against central
finite differences, and the structure of its seeded coarse systems."""
import numpy as np
import pytest

from oracle import coarse_net as cn


def test_coarse_operator_is_symmetric_positive_definite():
    dims = (4, 3, 3)
    cop = cn.random_system(dims, seed=3)
    live = cn.live_mask(cop).ravel()
    A = cn.dense_matrix(cop, dims)[np.ix_(live, live)]
    assert np.allclose(A, A.T, rtol=0, atol=1e-9 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0


@pytest.mark.parametrize("dims", [(5, 4, 3), (17, 3, 3)])  # 4 G levels; 5 (the last G weight shared)
def test_backward_matches_finite_differences(dims):
    cop = cn.random_system(dims, seed=1, contrast=30.0)
    rng = np.random.default_rng(2)
    params = [rng.normal(0, np.sqrt(2 / (27 * s[1])), s) if len(s) == 3 else rng.normal(0, 0.1, s)
              for s in cn.param_shapes()]
    rc = rng.normal(0, 1, (2, int(np.prod(dims)), 2)) * cn.live_mask(cop)[None]
    target = cn.exact_correction(cop, dims, rc)
    loss, grads, _ = cn.loss_and_grad(params, cop, dims, rc, target)
    assert np.isfinite(loss) and loss > 0
    flat, g = cn.flatten(params), cn.flatten(grads)
    # a sample of weights from every layer plus biases
    idx = []
    o = 0
    for s in cn.param_shapes():
        n = int(np.prod(s))
        idx += list(o + rng.choice(n, min(n, 3), replace=False))
        o += n
    h = 1e-6
    errs = []
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += h
        fm[i] -= h
        fd = (cn.loss_and_grad(cn.unflatten(fp), cop, dims, rc, target)[0]
              - cn.loss_and_grad(cn.unflatten(fm), cop, dims, rc, target)[0]) / (2 * h)
        # entries far below the gradient's scale are dominated by FD rounding
        if abs(fd) + abs(g[i]) > 1e-5 * np.abs(g).max():
            errs.append(abs(fd - g[i]) / (abs(fd) + abs(g[i])))
    assert len(errs) > 10
    assert max(errs) < 1e-4, max(errs)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38, 1e-40], np.float64)
    r = cn.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie -> even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5
    # every result is representable in 8 mantissa bits
    f = r.astype(np.float32).view(np.uint32)
    assert np.all(f & 0xFFFF == 0)


def test_learned_correction_is_linear_symmetric_positive():
    """e(r) = S G^T G S r: linear in r, symmetric, positive semi-definite --
    the property that keeps PCG's convergence theory with the learned term."""
    dims = (5, 4, 3)
    cop = cn.random_system(dims, seed=4)
    rng = np.random.default_rng(9)
    params = [rng.normal(0, 0.3, s) for s in cn.param_shapes()]
    nt = int(np.prod(dims))
    r1, r2 = rng.normal(0, 1, (2, 1, nt, 2)) * cn.live_mask(cop)[None]
    e1 = cn.coarse_correction(params, cop, dims, r1)
    e2 = cn.coarse_correction(params, cop, dims, r2)
    e12 = cn.coarse_correction(params, cop, dims, 2.0 * r1 - 3.0 * r2)
    assert np.allclose(e12, 2.0 * e1 - 3.0 * e2, rtol=1e-10, atol=1e-12 * np.abs(e12).max())
    assert abs(np.sum(r1 * e2) - np.sum(r2 * e1)) <= 1e-10 * np.abs(np.sum(r1 * e2))
    assert np.sum(r1 * e1) >= 0 and np.sum(r2 * e2) >= 0
