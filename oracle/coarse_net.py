"""FP64 CPU restatement of the learned coarse solve -- TEST INFRASTRUCTURE ONLY.

The learned preconditioner does not exist in adaptive-pf-flip; this module
restates, from the mathematics, what the CUDA code in
``adaptive-pf-flip_b200/csrc/pf_learned.cu`` computes, so tests can check the
GPU forward pass, its gradients and its Adam step:

* the two-class coarse operator on the tile lattice (17 floats per tile:
  diagonals d0 d1, in-tile coupling e, the 2x2 couplings to the -x, -y, -z
  neighbour tile, the aggregate sizes n0 n1) and its product A_c x;
* the input features of A_c and the 4-level gate U-Net (3x3x3 convolutions,
  ReLU, 2x2x2 average pooling, nearest upsampling with skip concatenation);
* the learned coarse correction e = S G^T G S r_c: S = diag(d_c)^-1/2, G the
  gated multilevel operator h_0 = g_0 C_0 S r, h_l = g_l C_min(l,3) P h_{l-1};
* the energy-norm loss (e - e*)^T A_c (e - e*) / (e*^T r_c) and its gradient
  by reverse-mode differentiation written out by hand;
* Adam.

``bf16=True`` rounds the operands of every convolution (inputs after the
ReLU gate, weights) to bfloat16 the way the tensor-core kernels do, so GPU and
CPU see the same products; sums stay FP64 here (FP32 on the GPU).
"""
from __future__ import annotations

import numpy as np

STRIDE = 17
KD, KE, KX, KY, KZ, KN = 0, 2, 3, 7, 11, 15
N_FEATURES = 19
IN_CHANNELS = 32

# (name, C_in, C_out, relu); the level of each layer is implied by the U-Net
LAYERS = [
    ("enc0a", 32, 16, True), ("enc0b", 16, 16, True),
    ("enc1a", 16, 32, True), ("enc1b", 32, 32, True),
    ("enc2a", 32, 64, True), ("enc2b", 64, 64, True),
    ("enc3a", 64, 64, True), ("enc3b", 64, 64, True),
    ("dec2", 128, 64, True), ("dec1", 96, 32, True), ("dec0", 48, 16, True),
    ("out", 16, 16, False),
]
# the linear operator G: (name, C_in, C_out), one per level, no bias (the
# bias slots exist in the parameter vector and stay zero)
G_LAYERS = [("g0", 2, 16), ("g1", 16, 16), ("g2", 16, 16), ("g3", 16, 16)]


def param_shapes():
    out = []
    for _, ci, co, _ in LAYERS:
        out.append((27, ci, co))
        out.append((co,))
    for _, ci, co in G_LAYERS:
        out.append((27, ci, co))
        out.append((co,))
    return out


def num_params():
    return sum(int(np.prod(s)) for s in param_shapes())


def unflatten(flat):
    flat = np.asarray(flat, np.float64)
    out, o = [], 0
    for s in param_shapes():
        n = int(np.prod(s))
        out.append(flat[o:o + n].reshape(s))
        o += n
    assert o == flat.size
    return out


def flatten(parts):
    return np.concatenate([np.asarray(p, np.float64).ravel() for p in parts])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), kept as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


# ---------------------------------------------------------------------------
# coarse operator


def coarse_apply(cop, dims, x):
    """y = A_c x; cop (nt, 17), x (..., nt, 2) with tile index t = i + X (j + Y k)."""
    X, Y, Z = dims
    nt = X * Y * Z
    c = np.asarray(cop, np.float64).reshape(nt, STRIDE)
    xs = np.asarray(x, np.float64).reshape(-1, nt, 2)
    y = np.empty_like(xs)
    for a in (0, 1):
        y[:, :, a] = c[:, KD + a] * xs[:, :, a] - c[:, KE] * xs[:, :, 1 - a]
    t = np.arange(nt)
    ti, tj, tk = t % X, (t // X) % Y, t // (X * Y)
    for base, step, has in ((KX, 1, ti > 0), (KY, X, tj > 0), (KZ, X * Y, tk > 0)):
        tt = t[has]
        uu = tt - step  # unique, so fancy-index updates do not collide
        for a in (0, 1):
            for b in (0, 1):
                w = c[tt, base + 2 * a + b]  # between (t, a) and (t - e, b)
                y[:, tt, a] -= w * xs[:, uu, b]
                y[:, uu, b] -= w * xs[:, tt, a]
    return y.reshape(np.shape(x))


def live_mask(cop):
    c = np.asarray(cop, np.float64)
    return np.stack([(c[:, KN + a] > 0) & (c[:, KD + a] > 0) for a in (0, 1)], axis=-1)


def d_ref(cop):
    """Largest diagonal of a class-0 (heavy-phase) aggregate, else of any."""
    c = np.asarray(cop, np.float64)
    live = live_mask(c)
    d0 = c[:, KD][live[:, 0]]
    if d0.size:
        return float(d0.max())
    d1 = c[:, KD + 1][live[:, 1]]
    return float(d1.max()) if d1.size else 0.0


# ---------------------------------------------------------------------------
# features and the network


def features(cop, dims, rc):
    """Input channels (B, nt, 32) and the per-sample scale s = max|rc| over live unknowns."""
    X, Y, Z = dims
    c = np.asarray(cop, np.float64)
    nt = X * Y * Z
    live = live_mask(c)
    dref = d_ref(c)
    rc = np.asarray(rc, np.float64).reshape(-1, nt, 2)
    B = rc.shape[0]
    s = np.array([np.abs(np.where(live, rc[b], 0.0)).max(initial=0.0) for b in range(B)])
    F = np.zeros((B, nt, IN_CHANNELS))
    inv_s = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    for a in (0, 1):
        F[:, :, a] = np.where(live[:, a], rc[:, :, a], 0.0) * inv_s[:, None]
        F[:, :, 2 + a] = live[:, a]
        with np.errstate(divide="ignore"):
            lg = np.log(np.where(live[:, a], c[:, KD + a], 1.0) / (dref if dref > 0 else 1.0)) / np.log(1e4)
        F[:, :, 4 + a] = np.where(live[:, a], lg, 0.0)
    both = live[:, 0] & live[:, 1]
    F[:, :, 6] = np.where(both, c[:, KE] / np.sqrt(np.where(both, c[:, KD] * c[:, KD + 1], 1.0)), 0.0)
    t = np.arange(nt)
    ti, tj, tk = t % X, (t // X) % Y, t // (X * Y)
    for q, (base, step, has) in enumerate(((KX, 1, ti > 0), (KY, X, tj > 0), (KZ, X * Y, tk > 0))):
        u = np.where(has, t - step, 0)
        for a in (0, 1):
            for b in (0, 1):
                ok = has & live[:, a] & live[u, b]
                den = np.sqrt(np.where(ok, c[:, KD + a] * c[u, KD + b], 1.0))
                F[:, :, 7 + 4 * q + 2 * a + b] = np.where(ok, c[:, base + 2 * a + b] / den, 0.0)
    return F, s, dref


def level_dims(dims, count=4):
    out = [tuple(dims)]
    for _ in range(count - 1):
        out.append(tuple((d + 1) // 2 for d in out[-1]))
    return out


MAX_LEVELS = 8


def g_levels(dims):
    """Levels of G: halve until every extent is <= 2 (at least 4, at most 8)."""
    n, d = 1, tuple(dims)
    while max(d) > 2 and n < MAX_LEVELS:
        d = tuple((v + 1) // 2 for v in d)
        n += 1
    return max(4, n)


TAPS = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def _shift(x5, dx, dy, dz):
    """out[p] = x[p + (dx, dy, dz)] with zeros outside; x5 shaped (B, Z, Y, X, C)."""
    out = np.zeros_like(x5)
    B, Z, Y, X, C = x5.shape

    def rng(d, n):  # target p in [max(0,-d), n-max(0,d)), source p + d
        return slice(max(0, -d), n - max(0, d)), slice(max(0, d), n + min(0, d))

    tz, sz = rng(dz, Z)
    ty, sy = rng(dy, Y)
    tx, sx = rng(dx, X)
    out[:, tz, ty, tx] = x5[:, sz, sy, sx]
    return out


def conv(x, dims, W, b, relu, round_bf16):
    """x (B, n, Ci) -> (B, n, Co): y[p] = b + sum_tap x[p + tap] W[tap]."""
    X, Y, Z = dims
    B, n, Ci = x.shape
    x5 = x.reshape(B, Z, Y, X, Ci)
    Wr = bf16(W) if round_bf16 else W
    xr = bf16(x5) if round_bf16 else x5
    y = np.zeros((B, Z, Y, X, W.shape[2]))
    for k, (dx, dy, dz) in enumerate(TAPS):
        y += _shift(xr, dx, dy, dz) @ Wr[k]
    y = y + b
    if relu:
        y = np.maximum(y, 0.0)
    return y.reshape(B, n, -1)


def conv_backward(x, dims, W, dz, round_bf16):
    """Gradients of y = conv(x) given dz = dL/d(pre-activation): (dx, dW, db)."""
    X, Y, Z = dims
    B, n, Ci = x.shape
    Co = W.shape[2]
    x5 = x.reshape(B, Z, Y, X, Ci)
    d5 = dz.reshape(B, Z, Y, X, Co)
    Wr = bf16(W) if round_bf16 else W
    xr = bf16(x5) if round_bf16 else x5
    dr = bf16(d5) if round_bf16 else d5
    dW = np.zeros_like(W)
    dx = np.zeros((B, Z, Y, X, Ci))
    for k, (sx, sy, sz) in enumerate(TAPS):
        xs = _shift(xr, sx, sy, sz)                       # x[p + tap]
        dW[k] = np.einsum("bzyxi,bzyxo->io", xs, dr)
        dx += _shift(dr, -sx, -sy, -sz) @ Wr[k].T         # dz[p - tap] W[tap]^T
    db = d5.sum(axis=(0, 1, 2, 3))  # the bias gradient sums the unrounded dz
    return dx.reshape(B, n, Ci), dW, db


def pool(x, dims):
    X, Y, Z = dims
    B, n, C = x.shape
    X2, Y2, Z2 = (X + 1) // 2, (Y + 1) // 2, (Z + 1) // 2
    x5 = np.zeros((B, 2 * Z2, 2 * Y2, 2 * X2, C))
    x5[:, :Z, :Y, :X] = x.reshape(B, Z, Y, X, C)
    y = x5.reshape(B, Z2, 2, Y2, 2, X2, 2, C).sum(axis=(2, 4, 6)) / 8.0
    return y.reshape(B, -1, C)


def pool_backward(dy, dims):
    X, Y, Z = dims
    B, _, C = dy.shape
    X2, Y2, Z2 = (X + 1) // 2, (Y + 1) // 2, (Z + 1) // 2
    d5 = dy.reshape(B, Z2, 1, Y2, 1, X2, 1, C) / 8.0
    full = np.broadcast_to(d5, (B, Z2, 2, Y2, 2, X2, 2, C)).reshape(B, 2 * Z2, 2 * Y2, 2 * X2, C)
    return full[:, :Z, :Y, :X].reshape(B, -1, C).copy()


def upsample(x, dims_coarse, dims_fine):
    X, Y, Z = dims_fine
    Xc, Yc, Zc = dims_coarse
    B, _, C = x.shape
    x5 = x.reshape(B, Zc, Yc, Xc, C)
    k, j, i = np.arange(Z) // 2, np.arange(Y) // 2, np.arange(X) // 2
    return x5[:, k][:, :, j][:, :, :, i].reshape(B, -1, C)


def upsample_backward(dy, dims_coarse, dims_fine):
    X, Y, Z = dims_fine
    Xc, Yc, Zc = dims_coarse
    B, _, C = dy.shape
    out = np.zeros((B, Zc, Yc, Xc, C))
    d5 = dy.reshape(B, Z, Y, X, C)
    k, j, i = np.arange(Z) // 2, np.arange(Y) // 2, np.arange(X) // 2
    np.add.at(out, (slice(None), k[:, None, None], j[None, :, None], i[None, None, :]), d5)
    return out.reshape(B, -1, C)


def forward(params, F, dims, round_bf16=False, keep=False):
    """U-Net forward; returns the output (B, n0, 2) and, with keep, the tape."""
    P = params
    D = level_dims(dims)
    t = {}
    L = {name: (P[2 * q], P[2 * q + 1], relu) for q, (name, _, _, relu) in enumerate(LAYERS)}

    def run(name, x, lvl):
        W, b, relu = L[name]
        y = conv(x, D[lvl], W, b, relu, round_bf16)
        t[name] = (x, lvl, y)
        return y

    a0 = run("enc0a", F, 0)
    s0 = run("enc0b", a0, 0)
    a1 = run("enc1a", pool(s0, D[0]), 1)
    s1 = run("enc1b", a1, 1)
    a2 = run("enc2a", pool(s1, D[1]), 2)
    s2 = run("enc2b", a2, 2)
    a3 = run("enc3a", pool(s2, D[2]), 3)
    b3 = run("enc3b", a3, 3)
    u2 = run("dec2", np.concatenate([upsample(b3, D[3], D[2]), s2], axis=-1), 2)
    u1 = run("dec1", np.concatenate([upsample(u2, D[2], D[1]), s1], axis=-1), 1)
    u0 = run("dec0", np.concatenate([upsample(u1, D[1], D[0]), s0], axis=-1), 0)
    o = run("out", u0, 0)
    return (o, t) if keep else o


def backward(params, tape, dims, do, round_bf16=False):
    """Gradients of every parameter given dL/do (B, n0, 2); same order as params."""
    D = level_dims(dims)
    grads = {}
    idx = {name: q for q, (name, _, _, _) in enumerate(LAYERS)}

    def back(name, dy):
        x, lvl, y = tape[name]
        W = params[2 * idx[name]]
        relu = LAYERS[idx[name]][3]
        dz = dy * (y > 0) if relu else dy
        dx, dW, db = conv_backward(x, D[lvl], W, dz, round_bf16)
        grads[name] = (dW, db)
        return dx

    du0 = back("out", do)
    dc0 = back("dec0", du0)
    du1 = upsample_backward(dc0[..., :32], D[1], D[0])
    ds0 = dc0[..., 32:].copy()
    dc1 = back("dec1", du1)
    du2 = upsample_backward(dc1[..., :64], D[2], D[1])
    ds1 = dc1[..., 64:].copy()
    dc2 = back("dec2", du2)
    db3 = upsample_backward(dc2[..., :64], D[3], D[2])
    ds2 = dc2[..., 64:].copy()
    da3 = back("enc3b", db3)
    dq3 = back("enc3a", da3)
    ds2 += pool_backward(dq3, D[2])
    da2 = back("enc2b", ds2)
    dq2 = back("enc2a", da2)
    ds1 += pool_backward(dq2, D[1])
    da1 = back("enc1b", ds1)
    dq1 = back("enc1a", da1)
    ds0 += pool_backward(dq1, D[0])
    da0 = back("enc0b", ds0)
    back("enc0a", da0)
    out = []
    for name, _, _, _ in LAYERS:
        out.extend(grads[name])
    return out


# ---------------------------------------------------------------------------
# the preconditioner: e = S G^T G S rc, G linear in rc, gated by the U-Net


def convT(x, dims, W, round_bf16):
    """Adjoint of conv without bias: out[p] = sum_tap x[p - tap] W[tap]^T."""
    X, Y, Z = dims
    B, n, Co = x.shape
    x5 = x.reshape(B, Z, Y, X, Co)
    xr = bf16(x5) if round_bf16 else x5
    Wr = bf16(W) if round_bf16 else W
    out = np.zeros((B, Z, Y, X, W.shape[1]))
    for k, (sx, sy, sz) in enumerate(TAPS):
        out += _shift(xr, -sx, -sy, -sz) @ Wr[k].T
    return out.reshape(B, n, -1)


def wgrad(x, dims, dy, round_bf16):
    """dW[tap] = sum_p x[p + tap] (outer) dy[p]."""
    X, Y, Z = dims
    B, n, Ci = x.shape
    x5 = x.reshape(B, Z, Y, X, Ci)
    d5 = dy.reshape(B, Z, Y, X, -1)
    xr = bf16(x5) if round_bf16 else x5
    dr = bf16(d5) if round_bf16 else d5
    return np.stack([np.einsum("bzyxi,bzyxo->io", _shift(xr, *tap), dr) for tap in TAPS])


def inv_sqrt_diag(cop):
    c = np.asarray(cop, np.float64)
    live = live_mask(c)
    d = np.stack([c[:, KD], c[:, KD + 1]], axis=-1)
    return np.where(live, 1.0 / np.sqrt(np.where(live, d, 1.0)), 0.0)


def gates(params, cop, dims, round_bf16=False, keep=False):
    """Per-level gates gamma_l (1, n_l, 16) of every G level, from the operator alone."""
    F, _, _ = features(cop, dims, np.zeros((1, int(np.prod(dims)), 2)))
    D = level_dims(dims, g_levels(dims))
    g0, tape = forward(params, F, dims, round_bf16, keep=True)
    gs = [g0]
    for l in range(len(D) - 1):
        gs.append(pool(gs[-1], D[l]))
    return (gs, tape) if keep else gs


def _gW(params):
    base = 2 * len(LAYERS)
    return [params[base + 2 * q] for q in range(len(G_LAYERS))]


def apply_gtg(params, gs, cop, dims, rc, round_bf16=False, keep=False):
    """e = S G^T G S rc, G r = (h_0 .. h_{L-1}), h_0 = gamma_0 C_0 S r,
    h_l = gamma_l C_min(l,3) P h_{l-1}; L = g_levels(dims)."""
    NL = g_levels(dims)
    D = level_dims(dims, NL)
    Wg = _gW(params)
    W = [Wg[min(l, 3)] for l in range(NL)]
    S = inv_sqrt_diag(cop)[None]
    x0 = S * np.asarray(rc, np.float64)
    a, h, q, b, t = [None] * NL, [None] * NL, [None] * NL, [None] * NL, [None] * NL
    for l in range(NL):
        xin = x0 if l == 0 else pool(h[l - 1], D[l - 1])
        q[l] = xin
        a[l] = conv(xin, D[l], W[l], 0.0, False, round_bf16)
        h[l] = gs[l] * a[l]
    b[NL - 1] = h[NL - 1]
    t[NL - 1] = gs[NL - 1] * h[NL - 1]
    for l in range(NL - 1, 0, -1):
        b[l - 1] = h[l - 1] + pool_backward(convT(t[l], D[l], W[l], round_bf16), D[l - 1])
        t[l - 1] = gs[l - 1] * b[l - 1]
    e = S * convT(t[0], D[0], W[0], round_bf16)
    if not keep:
        return e
    return e, dict(S=S, a=a, h=h, q=q, b=b, t=t)


def apply_gtg_backward(params, gs, dims, tape, de, round_bf16=False):
    """Gradients of <de, e> w.r.t. the four G weights (the last shared by the
    deeper levels) and the gate gamma_0 (deeper gates are its poolings)."""
    NL = g_levels(dims)
    D = level_dims(dims, NL)
    Wg = _gW(params)
    W = [Wg[min(l, 3)] for l in range(NL)]
    S = tape["S"]
    a, h, q, b, t = tape["a"], tape["h"], tape["q"], tape["b"], tape["t"]
    gW = [np.zeros_like(w) for w in Wg]
    dg = [np.zeros_like(g) for g in gs]
    dh = [None] * NL
    # transposed half, fine to coarse
    dv = S * de
    for l in range(NL):
        if l > 0:
            dv = pool(dh[l - 1], D[l - 1])
        dt = conv(dv, D[l], W[l], 0.0, False, round_bf16)
        gW[min(l, 3)] += wgrad(dv, D[l], t[l], round_bf16)
        dg[l] += (dt * b[l]).sum(axis=0, keepdims=True)
        dh[l] = gs[l] * dt
    # forward half, coarse to fine
    for l in range(NL - 1, -1, -1):
        da = gs[l] * dh[l]
        dg[l] += (a[l] * dh[l]).sum(axis=0, keepdims=True)
        gW[min(l, 3)] += wgrad(q[l], D[l], da, round_bf16)
        if l > 0:
            dh[l - 1] += pool_backward(convT(da, D[l], W[l], round_bf16), D[l - 1])
    # gamma_{l+1} = P gamma_l
    for l in range(NL - 2, -1, -1):
        dg[l] += pool_backward(dg[l + 1], D[l])
    return gW, dg[0]


def coarse_correction(params, cop, dims, rc, round_bf16=False):
    """The learned approximation of A_c^-1 rc (live unknowns)."""
    gs = gates(params, cop, dims, round_bf16)
    return apply_gtg(params, gs, cop, dims, rc, round_bf16)


def loss_and_grad(params, cop, dims, rc, target, round_bf16=False):
    """Mean over the batch of (e - e*)^T A_c (e - e*) / (e*^T rc), its gradient, and e."""
    nt = int(np.prod(dims))
    rc = np.asarray(rc, np.float64).reshape(-1, nt, 2)
    target = np.asarray(target, np.float64).reshape(-1, nt, 2)
    B = rc.shape[0]
    live = live_mask(cop)
    gs, utape = gates(params, cop, dims, round_bf16, keep=True)
    e, tape = apply_gtg(params, gs, cop, dims, rc, round_bf16, keep=True)
    v = np.where(live[None], e - target, 0.0)
    Av = coarse_apply(cop, dims, v)
    den = np.einsum("btc,btc->b", np.where(live[None], target, 0.0), np.where(live[None], rc, 0.0))
    num = np.einsum("btc,btc->b", v, Av)
    ok = den > 0
    loss = float(np.sum(np.where(ok, num / np.where(ok, den, 1.0), 0.0)) / B)
    de = np.where(ok[:, None, None] & live[None], 2.0 * Av / np.where(ok, den, 1.0)[:, None, None], 0.0) / B
    gW, dg0 = apply_gtg_backward(params, gs, dims, tape, de, round_bf16)
    grads = backward(params, utape, dims, dg0, round_bf16)
    for w in gW:
        grads.extend([w, np.zeros(w.shape[2])])
    return loss, grads, e


def adam(params, grads, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    out = []
    for q, (p, g) in enumerate(zip(params, grads)):
        m[q] = b1 * m[q] + (1 - b1) * g
        v[q] = b2 * v[q] + (1 - b2) * g * g
        mh = m[q] / (1 - b1 ** step)
        vh = v[q] / (1 - b2 ** step)
        out.append(p - lr * mh / (np.sqrt(vh) + eps))
    return out


# ---------------------------------------------------------------------------
# seeded coarse systems for tests


def random_system(dims, seed, contrast=1000.0, dead_fraction=0.1):
    """A two-class coarse operator with the structure of a Galerkin product:
    non-negative couplings, diagonal = row sum of couplings + a positive
    Dirichlet part, class-1 aggregates `contrast` times stiffer, some
    aggregates empty.  Returns cop (nt, 17) float32."""
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    nt = X * Y * Z
    cop = np.zeros((nt, STRIDE))
    n = rng.integers(1, 400, (nt, 2)).astype(np.float64)
    n[rng.uniform(size=(nt, 2)) < dead_fraction] = 0
    cop[:, KN:KN + 2] = n
    live = n > 0
    strength = np.where(np.arange(2) == 1, contrast, 1.0)
    t = np.arange(nt)
    ti, tj, tk = t % X, (t // X) % Y, t // (X * Y)
    for base, step, has in ((KX, 1, ti > 0), (KY, X, tj > 0), (KZ, X * Y, tk > 0)):
        u = np.where(has, t - step, 0)
        for a in (0, 1):
            for b in (0, 1):
                w = rng.uniform(0.5, 1.5, nt) * np.sqrt(strength[a] * strength[b]) * (1.0 if a == b else 0.02)
                cop[:, base + 2 * a + b] = np.where(has & live[:, a] & live[u, b], w, 0.0)
    cop[:, KE] = np.where(live[:, 0] & live[:, 1], rng.uniform(0.5, 1.5, nt) * 0.02 * np.sqrt(contrast), 0.0)
    rowsum = -coarse_apply(cop, dims, np.ones((1, nt, 2)))[0]  # = -(sum of couplings) with zero diagonal
    dirichlet = rng.uniform(0.01, 0.1, (nt, 2)) * strength
    cop[:, KD:KD + 2] = np.where(live, rowsum + dirichlet, 0.0)
    return cop.astype(np.float32)


def dense_matrix(cop, dims):
    nt = int(np.prod(dims))
    eye = np.eye(2 * nt).reshape(2 * nt, nt, 2)
    return coarse_apply(np.asarray(cop, np.float64), dims, eye).reshape(2 * nt, 2 * nt)


def exact_correction(cop, dims, rc):
    """A_c^-1 rc restricted to live unknowns (dead ones stay 0)."""
    nt = int(np.prod(dims))
    live = live_mask(cop).ravel()
    A = dense_matrix(cop, dims)[np.ix_(live, live)]
    rc = np.asarray(rc, np.float64).reshape(-1, 2 * nt)
    out = np.zeros_like(rc)
    out[:, live] = np.linalg.solve(A, rc[:, live].T).T
    return out.reshape(-1, nt, 2)
