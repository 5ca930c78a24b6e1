"""GPU tile pool and projection restating the reference's grid tests.

* tests/test_sparse_grid3d.cpp (SparseBlockGrid3D<4>): allocation, access
  and sparsity of 4^3 blocks, clearing and reactivation, a 7-point Laplacian
  over an active region, and iteration over the active blocks.  The GPU pool
  is checked through the cell-centred pressure field of the SparseMacGrid3D
  mirror (one activity byte per 4^3 block, bid = bx + nbx*(by + nby*bz)).
  A dense write stands in for the reference's ref() calls: every nonzero node
  written activates its block.
* tests/test_sparse_pressure3d.cpp: a compact fluid box inside solid walls
  with linear face velocities, projected with beta = 1.  The result must be
  divergence-free, and its pressure must match the oracle's.
"""
import numpy as np
import pytest

import oracle as O
from gpu_helpers import rel_err, to_oracle_phase

pytestmark = pytest.mark.gpu


def test_allocate_access_sparsity(pf):
    # tests/test_sparse_grid3d.cpp:6-26
    g = pf.SparseMacGrid3D(17, 10, 9, 1.0)
    P = pf.PF_P
    assert tuple(g.bdims(P)) == (5, 3, 3)
    assert g.activeBlockCount(P) == 0
    d = np.zeros((9, 10, 17), np.float32)
    assert g.get_field(P)[0][3, 5, 10] == 0.0
    d[3, 5, 10] = 3.5
    g.set_values(P, d)
    assert g.get_field(P)[0][3, 5, 10] == 3.5
    assert g.activeBlockCount(P) == 1
    d[2, 6, 11] = 1.0  # same block
    g.set_values(P, d)
    assert g.activeBlockCount(P) == 1
    d[8, 9, 16] = 2.0
    g.set_values(P, d)
    assert g.activeBlockCount(P) == 2
    ids = set(g.active_blocks(P).tolist())
    assert 2 + 5 * (1 + 3 * 0) in ids
    assert 4 + 5 * (2 + 3 * 2) in ids
    assert 0 not in ids
    g.close()


def test_clear_and_reactivate(pf):
    # tests/test_sparse_grid3d.cpp:28-49; pooled tiles are kept and reused
    g = pf.SparseMacGrid3D(16, 16, 16, 1.0)
    P = pf.PF_P
    d = np.zeros((16, 16, 16), np.float32)
    d[1, 3, 2] = 1.0
    d[9, 8, 12] = 2.0
    g.set_values(P, d)
    assert g.activeBlockCount(P) == 2
    tiles = g.active_tiles()
    g.clear_field(P)
    assert g.activeBlockCount(P) == 0
    assert g.active_tiles() == tiles
    assert g.get_field(P)[0][1, 3, 2] == 0.0
    d2 = np.zeros_like(d)
    d2[9, 8, 12] = 7.0
    g.set_values(P, d2)
    assert g.activeBlockCount(P) == 1
    assert g.active_tiles() == tiles
    out = g.get_field(P)[0]
    assert out[9, 8, 12] == 7.0 and out[1, 3, 2] == 0.0
    g.close()


def test_seven_point_laplacian_matches_dense(pf):
    # tests/test_sparse_grid3d.cpp:51-76
    n = 16
    g = pf.SparseMacGrid3D(n, n, n, 1.0)
    P = pf.PF_P
    uni = np.zeros((n, n, n), np.float32)
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    box = (i >= 4) & (i < 12) & (j >= 4) & (j < 12) & (k >= 4) & (k < 12)
    uni[box] = (i * i + 2 * j + 3 * k)[box].astype(np.float32)
    g.set_values(P, uni)
    sp = g.get_field(P)[0]

    def lap(a):
        c = a[5:11, 5:11, 5:11].astype(np.float64)
        return (a[5:11, 5:11, 6:12] + a[5:11, 5:11, 4:10] + a[5:11, 6:12, 5:11] + a[5:11, 4:10, 5:11] +
                a[6:12, 5:11, 5:11] + a[4:10, 5:11, 5:11]).astype(np.float64) - 6 * c

    assert np.max(np.abs(lap(uni) - lap(sp))) < 1e-5
    assert g.activeBlockCount(P) == 8
    g.close()


def test_active_block_iteration_covers_written_cells(pf):
    # tests/test_sparse_grid3d.cpp:78-89
    g = pf.SparseMacGrid3D(16, 16, 16, 1.0)
    P = pf.PF_P
    d = np.zeros((16, 16, 16), np.float32)
    d[3, 3, 3] = 1.0
    d[9, 10, 12] = 2.0
    g.set_values(P, d)
    out = g.get_field(P)[0]
    nbx, nby, _ = g.bdims(P)
    seen = 0
    for b in g.active_blocks(P).tolist():
        bx, by, bz = b % nbx, (b // nbx) % nby, b // (nbx * nby)
        seen += int(np.count_nonzero(out[4 * bz:4 * bz + 4, 4 * by:4 * by + 4, 4 * bx:4 * bx + 4]))
    assert seen == 2
    g.close()


def test_compact_fluid_box_projection(pf):
    # tests/test_sparse_pressure3d.cpp:9-82, with beta = 1 (equal phase densities)
    n = 8
    g = pf.SparseMacGrid3D(n, n, n, 1.0)
    mk = np.zeros((n, n, n), np.float32)
    mk[[0, -1], :, :] = 2
    mk[:, [0, -1], :] = 2
    mk[:, :, [0, -1]] = 2
    mk[2:6, 2:6, 2:6] = 1
    g.set_cells(mk)
    u = np.zeros((n, n, n + 1), np.float32)
    v = np.zeros((n, n + 1, n), np.float32)
    w = np.zeros((n + 1, n, n), np.float32)
    mu, mv, mw = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
    for k in range(2, 6):
        for j in range(2, 6):
            for i in range(2, 7):
                u[k, j, i] = 0.7 * i + 0.1 * j - 0.2 * k
                mu[k, j, i] = 1.0
            for i in range(2, 6):
                v[k, j, i] = -0.3 * i + 0.5 * j + 0.15 * k
                mv[k, j, i] = 1.0
                mv[k, j + 1, i] = 1.0
    for k in range(2, 7):
        for j in range(2, 6):
            for i in range(2, 6):
                w[k, j, i] = 0.2 * i - 0.4 * j + 0.6 * k
                mw[k, j, i] = 1.0
    for f, a in ((pf.PF_U, u), (pf.PF_V, v), (pf.PF_W, w), (pf.PF_MU, mu), (pf.PF_MV, mv), (pf.PF_MW, mw)):
        g.set_values(f, a)
    pp = pf.PhaseParams(1.0, 1.0, 1.0, 1.0)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0)
    go = O.OracleGrid(n, n, n, 1.0)
    for f in range(8):
        go.set_field(f, *g.get_field(f))
    st = pf.spProjectStepVC3D(g, pp, 1.0, 1000, 1e-10)
    O.Oracle().project(go, to_oracle_phase(pp), 1.0, 1000, 1e-10)
    assert st.converged
    assert g.activeBlockCount(pf.PF_P) == 8
    gu, gv, gw = (g.get_field(f)[0].astype(np.float64) for f in (pf.PF_U, pf.PF_V, pf.PF_W))
    div = (gu[2:6, 2:6, 3:7] - gu[2:6, 2:6, 2:6]) + (gv[2:6, 3:7, 2:6] - gv[2:6, 2:6, 2:6]) + \
          (gw[3:7, 2:6, 2:6] - gw[2:6, 2:6, 2:6])
    assert np.max(np.abs(div)) < 1e-5
    p, po = g.get_field(pf.PF_P)[0], go.get_field(O.P)[0]
    assert rel_err(p, po) < 1e-5
    g.close()
