"""Render-cache export (src/driver/render_cache3d.h:551-600) on the GPU.

1. Byte for byte against the reference's own writer (writeSparseRenderCache3D,
   compiled into oracle/_ref): the reference runs its own markCells on the
   same particles -- its marker blocks then sit in their first-touch order,
   the order it lists phase cells in -- and is given the GPU's face fields and
   particles (and, in one case, the same secondary droplet and bubble sets,
   with ages and speeds across every render channel); both files must be
   identical, the liquid-volume sum included.
2. Against a restatement of the writer's selection and number format
   (sparsePhaseCells, :497-526, and writeParticleSection, :541-560), on a grid
   imported from the oracle.
3. The metadata checks and the empty-grid sections.
"""
import ctypes as C
import json
import re

import numpy as np
import pytest

import oracle as O
from gpu_helpers import phase_for, scene_particles, to_oracle_phase

pytestmark = pytest.mark.gpu


def _state(pf, n, seed):
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    go = O.OracleGrid(n, n, n, 1.0 / n)
    o = O.Oracle()
    o.mark_cells(go, ps)
    o.p2g(go, ps, to_oracle_phase(pp), 1.0)
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(ps))
    sim.phase, sim.Vp, sim.effective_dt_last = pp, 1.0, 1 / 240
    sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
    for f in range(8):
        sim.grid.set_field(f, *go.get_field(f))
    return sim, go, ps, pp


def _split(path):
    lines = open(path).read().splitlines()
    cells = [ln for ln in lines if ln.startswith('{"section":"phase_cell"')]
    rest = [ln for ln in lines if not ln.startswith('{"section":"phase_cell"')]
    return rest, cells


def _g(x):
    return "%.17g" % x


def _expected_cells(go, pp):
    o = O.Oracle()
    opp = to_oracle_phase(pp)
    nx, ny, nz = go.nx, go.ny, go.nz
    mk, act = go.get_field(O.FIELD_NAMES.index("mk"))
    mu, mv, mw = (go.get_field(O.FIELD_NAMES.index(f))[0] for f in ("mu", "mv", "mw"))
    phi = lambda raw: o.phi_from_raw(float(raw), opp)
    dv = go.dx * go.dx * go.dx  # cellVolume (render_cache3d.h:520)
    out = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                if not act[k // 4, j // 4, i // 4]:
                    continue
                m = int(mk[k, j, i] + np.float32(0.5))
                s = 0.0
                for raw in (mu[k, j, i], mu[k, j, i + 1], mv[k, j, i], mv[k, j + 1, i], mw[k, j, i], mw[k + 1, j, i]):
                    s += phi(raw)
                p = s / 6.0
                if m == 0 and p <= 1e-8:
                    continue
                out.append('{"section":"phase_cell","i":%d,"j":%d,"k":%d,"level":0,"marker":%d,"phi":%s,'
                           '"liquid_volume":%s}' % (i, j, k, m, _g(p), _g(p * dv)))
    return out


def _expected_particles(ps, Vp):
    out = []
    for p in range(len(ps)):
        liq = ps.type[p] == 0
        x, v = ps.pos[p], ps.vel[p]
        out.append('{"section":"particle","kind":"primary","render_channel":"%s","index":%d,"phase":"%s",'
                   '"position":[%s,%s,%s],"velocity":[%s,%s,%s],"volume":%s}'
                   % ("water" if liq else "air", p, "liquid" if liq else "gas", _g(x[0]), _g(x[1]), _g(x[2]),
                      _g(v[0]), _g(v[1]), _g(v[2]), _g(ps.volume[p] * Vp)))
    return out


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference (oracle/_ref) not built")
def _secondary_sets(rng, n):
    out = []
    for m in (140, 60):
        pos = rng.uniform(0.5 / n, 1.0 - 0.5 / n, (m, 3))
        vel = rng.normal(0.0, 0.6, (m, 3))
        vol = rng.uniform(0.3, 1.2, m)
        age = rng.integers(-1, 8, m).astype(np.int32)  # ages <= 1 and >= 4, and a negative one
        pos[5] = [np.nan, 0.5, 0.5]  # left out of the secondary bounds
        out.append((pos, vel, vol, age))
    return out


@pytest.mark.parametrize("scene,n,seed,secondary", [("rayleigh_taylor", 16, 3, False), ("bubble_tank", 20, 5, False),
                                                    ("bubble_tank", 20, 7, True)])
def test_render_cache_equals_reference_writer(pf, tmp_path, scene, n, seed, secondary):
    sc = getattr(pf.scenes, scene)(n, seed=seed)
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    opp = to_oracle_phase(pp)
    dt, frame, time = 1 / 240, 4, 0.5
    # GPU: markCells and P2G of the scene
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(ps))
    sim.phase, sim.Vp, sim.effective_dt_last = pp, 1.0, dt
    sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
    lib = pf.load()
    pf._lib.check(lib.pf_mark_cells(sim.grid.ctx), sim.grid.ctx, "pf_mark_cells")
    pf._lib.check(lib.pf_p2g(sim.grid.ctx, C.byref(pp._c()), 1.0), sim.grid.ctx, "pf_p2g")
    # reference: its own step marks the cells of the same particles (marker
    # blocks in first-touch order); then the GPU's fields and particles
    rg = O.ReferenceGrid(n, n, n, 1.0 / n)
    O.Reference().step(rg, ps.copy(), opp, dict(dt=dt, gravity=-9.81, Vp=1.0, alpha_l=0.95, alpha_g=0.95,
                                                cg_iters=50, cg_tol=1e-7))
    dg, ag = sim.grid.get_field(pf.PF_MK)
    dr, ar = rg.get_field(O.MK)
    assert np.array_equal(dg, dr) and np.array_equal(ag, ar)
    for f in range(7):
        rg.set_field(f, *sim.grid.get_field(f))
    pos, vel, typ, vol = sim.get_particles()
    rg._put(O.Particles(pos.astype(np.float64), vel.astype(np.float64), typ, vol.astype(np.float64)))
    if secondary:
        from oracle.secondary import _typed_ref
        _typed_ref(rg.lib)
        for w, (sp, sv, svol, sage) in enumerate(_secondary_sets(np.random.default_rng(seed), n)):
            sim.set_secondary_set(w, sp, sv, svol, sage)
            rg.lib.pfr_set_secondary_set(rg.h, w, len(sp), sp, sv, svol, sage)
    cam = pf.defaultRenderCacheCamera3D(n, n, n, 1.0 / n)
    a, b = tmp_path / "gpu.jsonl", tmp_path / "ref.jsonl"
    pf.writeSparseRenderCache3D(sim, a, frame, time, cam)
    rg.write_render_cache(b, frame, time, dt, opp, 1.0,
                          list(cam.position) + list(cam.target) + list(cam.up) +
                          [cam.fov_degrees, cam.near_clip, cam.far_clip, cam.focal_length_mm])
    ta, tb = a.read_text(), b.read_text()
    la, lb = ta.splitlines(), tb.splitlines()
    assert len(la) == len(lb)
    bad = [(i, x, y) for i, (x, y) in enumerate(zip(la, lb)) if x != y]
    assert not bad, bad[:3]
    assert ta == tb
    if secondary:
        # (the planted NaN position makes its line non-JSON, as the reference writes it)
        channels = {re.search(r'"render_channel":"(\w+)"', ln).group(1) for ln in la
                    if '"kind":"secondary_droplet","render' in ln}
        assert channels == {"droplet", "spray", "foam"}
    sim.grid.close()


@pytest.mark.parametrize("n,seed", [(16, 3), (12, 5)])
def test_render_cache_matches_restated_writer(pf, tmp_path, n, seed):
    sim, go, ps, pp = _state(pf, n, seed)
    a = tmp_path / "gpu.jsonl"
    nbytes = pf.writeSparseRenderCache3D(sim, a, 7, 0.125)
    assert nbytes == a.stat().st_size
    rest, cells = _split(a)
    exp = _expected_cells(go, pp)
    assert len(cells) == len(exp) > 0
    # the set and the number format (the order is checked against the
    # reference's writer above)
    assert sorted(cells) == sorted(exp)
    parts = [ln for ln in rest if ln.startswith('{"section":"particle",')]
    assert parts == _expected_particles(ps, 1.0)
    sec = {json.loads(ln)["section"]: json.loads(ln) for ln in rest if not ln.startswith('{"section":"particle"')}
    head = sec["header"]
    assert head["sim_kind"] == "sparse3d_tp" and head["dims"] == [n, n, n] and head["frame"] == 7
    assert head["dt"] == 1 / 240 and head["shutter_close"] == 0.125 + 1 / 240
    wv = sec["water_volume"]
    assert wv["phase_field_cells"] == len(exp)
    assert wv["primary_liquid_count"] == int(np.sum(ps.type == 0))
    assert wv["primary_gas_count"] == int(np.sum(ps.type == 1))
    vol = sum(json.loads(c)["liquid_volume"] for c in exp)
    assert wv["phase_field_liquid_volume"] == pytest.approx(vol, rel=1e-12)
    cm = sec["cinematic_metadata"]
    assert cm["water_bounds_valid"] is True and cm["secondary_bounds_valid"] is False
    assert cm["secondary_bounds_min"] == [0.0, 0.0, 0.0]
    assert sec["phase_field"]["count"] == len(exp)
    cam = sec["camera"]
    assert cam["target"] == [0.5, 0.5, 0.5] and cam["up"] == [0.0, 1.0, 0.0]


def test_render_cache_rejects_bad_metadata(pf, tmp_path):
    sim = pf.SparseSim3DTP(8, 8, 8, 0.125, max_particles=16)
    with pytest.raises(Exception):
        pf.writeSparseRenderCache3D(sim, "", 0, 0.0)
    cam = pf.defaultRenderCacheCamera3D(8, 8, 8, 0.125)
    assert list(cam.target) == [0.5, 0.5, 0.5] and cam.near_clip == 0.05 * 0.125
    cam.far_clip = cam.near_clip / 2
    with pytest.raises(Exception):
        pf.writeSparseRenderCache3D(sim, tmp_path / "x.jsonl", 0, 0.0, cam)
    sim.effective_dt_last = float("nan")
    with pytest.raises(Exception):
        pf.writeSparseRenderCache3D(sim, tmp_path / "y.jsonl", 0, 0.0)
    # an empty grid writes the header sections and empty particle sets
    sim.effective_dt_last = 0.01
    pf.writeSparseRenderCache3D(sim, tmp_path / "z.jsonl", 1, 0.0)
    sections = [json.loads(ln)["section"] for ln in open(tmp_path / "z.jsonl")]
    assert sections[:6] == ["header", "camera", "water_volume", "secondary_channels", "cinematic_metadata",
                            "phase_field"]
