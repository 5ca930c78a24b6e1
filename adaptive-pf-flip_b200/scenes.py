"""Seeded synthetic scenes for the solver-step workloads.

The reference seeds deterministic 2x2x2 sub-cell centres
(seedCell, src/driver/sparse_sim3d_tp.cpp:12-20) and perturbs its
Rayleigh-Taylor interface by a cell index (:739-754).  The workloads here
keep its cell layout (interior cells 1..n-2, eight particles per cell, one
per 2x2x2 sub-cell) but jitter each particle uniformly inside its sub-cell
with a counter-based generator, so a scene is a pure function of
(seed, cell, sub-cell, axis) and any prefix or subset can be rebuilt
identically.  Positions/velocities are FP32; the same arrays feed the GPU and
(converted exactly to FP64) the CPU oracle.
"""
from __future__ import annotations

import math

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014), vectorised on uint64."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, key: np.ndarray, stream: int) -> np.ndarray:
    """U[0,1) doubles from (seed, key, stream) with 53 random bits."""
    with np.errstate(over="ignore"):
        x = (np.uint64(seed) * np.uint64(0x632BE59BD9B4E019)) ^ (key.astype(np.uint64) * np.uint64(8)
                                                                  + np.uint64(stream))
    return (splitmix64(x) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal01(seed: int, key: np.ndarray, stream: int) -> np.ndarray:
    """N(0,1) by Box-Muller on two counter-based uniforms."""
    u1 = uniform01(seed, key, 2 * stream)
    u2 = uniform01(seed, key, 2 * stream + 1)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


def _seed_cells(ii, jj, kk, n, dx, seed, jitter=True):
    """Eight particles per listed cell, one per sub-cell; returns (N,3) float64
    positions and the per-particle key (cell linear index * 8 + sub-cell)."""
    ii = np.asarray(ii, np.int64)
    jj = np.asarray(jj, np.int64)
    kk = np.asarray(kk, np.int64)
    cell = ii + n[0] * (jj + n[1] * kk)
    s = np.arange(8, dtype=np.int64)
    key = (cell[:, None] * 8 + s[None, :]).reshape(-1)
    sx = (s & 1)[None, :]
    sy = ((s >> 1) & 1)[None, :]
    sz = ((s >> 2) & 1)[None, :]
    if jitter:
        ux = uniform01(seed, key, 0).reshape(-1, 8)
        uy = uniform01(seed, key, 1).reshape(-1, 8)
        uz = uniform01(seed, key, 2).reshape(-1, 8)
    else:
        ux = uy = uz = np.full((len(cell), 8), 0.5)
    x = (ii[:, None] + 0.5 * sx + 0.5 * ux) * dx
    y = (jj[:, None] + 0.5 * sy + 0.5 * uy) * dx
    z = (kk[:, None] + 0.5 * sz + 0.5 * uz) * dx
    pos = np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], axis=1)
    return pos, key


def _interior(n):
    k, j, i = np.meshgrid(np.arange(1, n[2] - 1), np.arange(1, n[1] - 1), np.arange(1, n[0] - 1), indexing="ij")
    return i.reshape(-1), j.reshape(-1), k.reshape(-1)


def rayleigh_taylor(n=48, seed=0, amp=0.05, rho_heavy=1000.0, rho_light=1.0, jitter=True):
    """Sparse two-phase Rayleigh-Taylor: n^3 cells, dx = 1/n, heavy fluid
    (type 0, rho_l) above y = 0.5 + amp*cos(2 pi x)cos(2 pi z), light fluid
    (type 1, rho_g) below, zero velocity.  n=48 gives 46^3*8 = 778,688 particles."""
    dims = (n, n, n)
    dx = 1.0 / n
    i, j, k = _interior(dims)
    pos, key = _seed_cells(i, j, k, dims, dx, seed, jitter)
    pos = pos.astype(np.float32)
    p64 = pos.astype(np.float64)
    iface = 0.5 + amp * np.cos(2 * math.pi * p64[:, 0]) * np.cos(2 * math.pi * p64[:, 2])
    typ = np.where(p64[:, 1] > iface, 0, 1).astype(np.uint8)
    vel = np.zeros_like(pos)
    vol = np.ones(len(pos), np.float32)
    return dict(name=f"rayleigh_taylor_{n}", nx=n, ny=n, nz=n, dx=dx, pos=pos, vel=vel, type=typ, volume=vol,
                rho_l=rho_heavy, rho_g=rho_light)


def bubble_tank(n=128, seed=0, level=0.7, center=(0.5, 0.3, 0.5), radius=0.15, sigma=0.1, rho_water=1000.0,
                rho_air=1.0):
    """Bubble tank: water fills cells whose centre is below y = level (j in
    1..), an air bubble (type 1) of the given radius sits inside it, the
    headspace stays empty; velocities N(0, sigma^2) per component."""
    dims = (n, n, n)
    dx = 1.0 / n
    jmax = int(math.floor(level * n - 0.5 - 1e-12))  # last j with centre < level
    jmax = min(jmax, n - 2)
    k, j, i = np.meshgrid(np.arange(1, n - 1), np.arange(1, jmax + 1), np.arange(1, n - 1), indexing="ij")
    pos, key = _seed_cells(i.reshape(-1), j.reshape(-1), k.reshape(-1), dims, dx, seed)
    pos = pos.astype(np.float32)
    p64 = pos.astype(np.float64)
    c = np.asarray(center)
    gas = ((p64 - c) ** 2).sum(axis=1) < radius * radius
    typ = np.where(gas, 1, 0).astype(np.uint8)
    vel = np.stack([normal01(seed + 1, key, a) for a in range(3)], axis=1) * sigma
    vol = np.ones(len(pos), np.float32)
    return dict(name=f"bubble_tank_{n}", nx=n, ny=n, nz=n, dx=dx, pos=pos, vel=vel.astype(np.float32), type=typ,
                volume=vol, rho_l=rho_water, rho_g=rho_air)


def _last_centre_below(frac, n):
    """Largest index whose cell centre (c + 0.5) / n lies below frac."""
    return min(int(math.floor(frac * n - 0.5 - 1e-12)), n - 2)


def dam_break_cells(n, column=(0.4, 0.6), pool=0.15):
    """The liquid cells of the dam break, in seeding order: the column
    (interior cells whose centre has x < column[0] and y < column[1]), then the
    pool beside it (x beyond the column, y < pool), each x fastest, then y,
    then z.  Returns (i, j, k) index arrays."""
    ic, cj, pj = _last_centre_below(column[0], n), _last_centre_below(column[1], n), _last_centre_below(pool, n)
    k, j, i = np.meshgrid(np.arange(1, n - 1), np.arange(1, cj + 1), np.arange(1, ic + 1), indexing="ij")
    k2, j2, i2 = np.meshgrid(np.arange(1, n - 1), np.arange(1, pj + 1), np.arange(ic + 1, n - 1), indexing="ij")
    return (np.concatenate([i.reshape(-1), i2.reshape(-1)]), np.concatenate([j.reshape(-1), j2.reshape(-1)]),
            np.concatenate([k.reshape(-1), k2.reshape(-1)]))


def dam_break(n=128, seed=0, column=(0.4, 0.6), pool=0.15, rho_water=1000.0, rho_air=1.0):
    """Dam break: a water column (x < 0.4, y < 0.6) beside a pool 0.15 deep,
    eight particles per water cell (type 0) at rest, the air above empty."""
    dims = (n, n, n)
    dx = 1.0 / n
    i, j, k = dam_break_cells(n, column, pool)
    pos, _ = _seed_cells(i, j, k, dims, dx, seed)
    pos = pos.astype(np.float32)
    typ = np.zeros(len(pos), np.uint8)
    vel = np.zeros_like(pos)
    vol = np.ones(len(pos), np.float32)
    return dict(name=f"dam_break_{n}", nx=n, ny=n, nz=n, dx=dx, pos=pos, vel=vel, type=typ, volume=vol,
                rho_l=rho_water, rho_g=rho_air)


def ellipsoid_pressure(n=256, seed=0, n_ellipsoids=64, semi=(0.02, 0.08), kmax=8, rho_background=1000.0,
                       rho_bubble=1.0):
    """Pressure-only system on an n^3 grid: every interior cell fluid, solid
    walls.  beta = 1/rho per face with rho = rho_bubble inside any of the
    random ellipsoids (centres U(0,1)^3, semi-axes U[semi]) and rho_background
    elsewhere; ``air_u/v/w`` flag the bubble faces.  The velocity is a
    band-limited random field -- Fourier modes with |k| <= kmax, N(0,1) real
    and imaginary amplitudes -- sampled exactly on the faces by an inverse FFT
    with half-cell phase shifts; wall-normal faces (index 0, 1, n-1, n) are
    zeroed.  Returns dense per-field arrays shaped (Z,Y,X)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, (n_ellipsoids, 3))
    axes = rng.uniform(semi[0], semi[1], (n_ellipsoids, 3))
    dx = 1.0 / n
    out = dict(name=f"ellipsoid_pressure_{n}", nx=n, ny=n, nz=n, dx=dx, rho_l=rho_background, rho_g=rho_bubble,
               centres=centres, axes=axes)
    kf = np.fft.fftfreq(n, d=1.0 / n)  # integer wave numbers
    KZ, KY, KX = np.meshgrid(kf, kf, kf, indexing="ij")
    band = (KX ** 2 + KY ** 2 + KZ ** 2) <= kmax * kmax
    band[0, 0, 0] = False
    nb = int(band.sum())
    for a, name in enumerate(("u", "v", "w")):
        dims = [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)][a]
        coef = np.zeros((n, n, n), np.complex128)
        coef[band] = rng.normal(0.0, 1.0, nb) + 1j * rng.normal(0.0, 1.0, nb)
        # face centre of (i,j,k): axis a at index, the others at index + 1/2
        shift = [0.5, 0.5, 0.5]
        shift[a] = 0.0
        coef *= np.exp(2j * math.pi * (KX * shift[0] + KY * shift[1] + KZ * shift[2]) / n)
        field = np.real(np.fft.ifftn(coef)) * (n ** 3) / math.sqrt(max(nb, 1))
        # periodic extension to the extra face layer along the face axis
        field = np.concatenate([field, np.take(field, [0], axis=2 - a)], axis=2 - a).astype(np.float32)
        assert field.shape == dims[::-1]
        idx = np.arange(dims[a])
        wall = (idx <= 1) | (idx >= n - 1)
        sl = [slice(None)] * 3
        sl[2 - a] = wall
        field[tuple(sl)] = 0.0
        out[name] = field
        # bubble faces: test each ellipsoid only inside its bounding box
        air = np.zeros(dims[::-1], bool)
        for cc, ax in zip(centres, axes):
            lo = [int(max(0, math.floor((cc[b] - ax[b]) / dx) - 1)) for b in range(3)]
            hi = [int(min(dims[b] - 1, math.ceil((cc[b] + ax[b]) / dx) + 1)) for b in range(3)]
            if any(hi[b] < lo[b] for b in range(3)):
                continue
            kk, jj, ii = np.meshgrid(np.arange(lo[2], hi[2] + 1), np.arange(lo[1], hi[1] + 1),
                                     np.arange(lo[0], hi[0] + 1), indexing="ij")
            pc = [ii * dx, jj * dx, kk * dx]
            pc = [pc[b] + (0.0 if b == a else 0.5 * dx) for b in range(3)]
            m = sum(((pc[b] - cc[b]) / ax[b]) ** 2 for b in range(3)) < 1.0
            air[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] |= m
        out["air_" + name] = air
    return out


def pressure_grid_fields(sc, rho_tilde_0, face_mass_liquid=None):
    """Grid fields encoding an ellipsoid_pressure scene for spProjectStepVC3D:
    markers (walls 2, interior 1), face raw masses (0 on bubble faces, a mass
    that saturates phi = 1 elsewhere) and the face velocities."""
    n = sc["nx"]
    rho_l, rho_g = sc["rho_l"], sc["rho_g"]
    rmin = math.log(rho_l / rho_g) * rho_g * rho_tilde_0
    m_liq = face_mass_liquid or 2.0 * (rmin + rho_tilde_0 * rho_l)
    mk = np.ones((n, n, n), np.float32)
    mk[0, :, :] = mk[-1, :, :] = 2
    mk[:, 0, :] = mk[:, -1, :] = 2
    mk[:, :, 0] = mk[:, :, -1] = 2
    f = dict(mk=mk)
    for name, mname in (("u", "mu"), ("v", "mv"), ("w", "mw")):
        f[name] = sc[name]
        f[mname] = np.where(sc["air_" + name], 0.0, m_liq).astype(np.float32)
    return f
