"""Grid set-ups of tests/test_pressure3d_vc.cpp restated on the sparse grid.

The reference's dense VC cases give beta per face directly.  On the sparse
path beta comes from the face raw mass through Eq. 7, so a face that should
carry beta = 1 gets a raw mass of 2 (phi clamps to 1, rho = rho_l = 1) and a
face that should carry beta = 100 keeps raw mass 0 (phi = 0, rho = rho_g =
0.01).  The builders fill any grid with set_field(f, dense, act) and
bdims(f): the oracle's and the GPU's alike.  Field ids: u v w mu mv mw p mk.
"""
import numpy as np

U, V, W, MU, MV, MW, P, MK = range(8)
LIQUID_RAW = 2.0
PHASE = (1.0, 0.01, 1.0, 1.0)  # rho_l, rho_g, alpha_phi, rho_tilde_0


def set_values(g, f, a):
    """Dense (Z,Y,X) write; every nonzero node activates its 4^3 block."""
    a = np.asarray(a, np.float32)
    act = np.zeros(g.bdims(f)[::-1], np.uint8)
    kk, jj, ii = np.nonzero(a)
    act[kk // 4, jj // 4, ii // 4] = 1
    g.set_field(f, a, act)


def walls(nx, ny, nz):
    mk = np.zeros((nz, ny, nx), np.float32)
    mk[[0, -1], :, :] = 2
    mk[:, [0, -1], :] = 2
    mk[:, :, [0, -1]] = 2
    return mk


def beta_one_box(g):
    """tests/test_pressure3d_vc.cpp:5-16: 8^3, fluid 2..5 in air inside solid
    walls, beta = 1 on every face, u = i on every u face.  Returns dt."""
    n = 8
    mk = walls(n, n, n)
    mk[2:6, 2:6, 2:6] = 1
    set_values(g, MK, mk)
    for f, shape in ((MU, (n, n, n + 1)), (MV, (n, n + 1, n)), (MW, (n + 1, n, n))):
        set_values(g, f, np.full(shape, LIQUID_RAW, np.float32))
    u = np.broadcast_to(np.arange(n + 1, dtype=np.float32), (n, n, n + 1))
    set_values(g, U, u)
    return 1.0


def hydrostatic_two_phase(g):
    """tests/test_pressure3d_vc.cpp:17-32: 6x16x6 all fluid inside solid
    walls, beta = 1 below row 8 and 100 from row 8 up, v += dt*g on every v
    face of rows 1..15.  Returns dt."""
    nx, ny, nz = 6, 16, 6
    mk = walls(nx, ny, nz)
    mk[1:5, 1:15, 1:5] = 1
    set_values(g, MK, mk)
    for f, shape in ((MU, (nz, ny, nx + 1)), (MV, (nz, ny + 1, nx)), (MW, (nz + 1, ny, nx))):
        m = np.zeros(shape, np.float32)
        m[:, :8, :] = LIQUID_RAW
        set_values(g, f, m)
    dt = 0.1
    v = np.zeros((nz, ny + 1, nx), np.float32)
    v[:, 1:ny, :] = np.float32(dt * -9.81)
    set_values(g, V, v)
    return dt


def fluid_divergence(g):
    """Max |div u| over the fluid cells (marker 1)."""
    u, v, w = (g.get_field(f)[0].astype(np.float64) for f in (U, V, W))
    d = (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:, :, :] - w[:-1, :, :])
    mk = g.get_field(MK)[0]
    return float(np.max(np.abs(d[mk == 1])))


def interior_max_v(g):
    """The reference's bound: max |v| over i,k in 1..n-2 and j in 2..ny-2."""
    v = g.get_field(V)[0].astype(np.float64)
    nz, nyp, nx = v.shape
    return float(np.max(np.abs(v[1:nz - 1, 2:nyp - 2, 1:nx - 1])))
