"""Parity at the benchmark configurations' own sizes, reproducibility, and
the projection's cell enumeration against the reference's.

* Rayleigh-Taylor at 48^3, density ratio 1000:1 (778,688 particles, dt 1/240,
  PCG to 1e-6 relative): ten whole steps on the GPU beside two oracle runs
  made at the same time on the host -- the oracle as the reference computes
  (FP64 particle state) and the same oracle with its particle state rounded
  to FP32 after every step, which is the storage this library keeps.  The
  second run measures what FP32 particle storage alone costs against the
  reference; that floor bounds the GPU's drift.
* Bubble tank at 128^3 (11.3M particles): one P2G against the oracle, the
  4^3 activity of all six face fields bit-exact and the fields within 1e-5.
* Reproducibility: P2G accumulates in a fixed order, so repeated P2G calls
  and repeated whole steps on the same particles are bit-identical.
* collectCellsWithMarker (src/driver/sparse_ops3d_common.h:65-85): the
  sorted fluid-cell list equals the compiled reference's.
"""
import threading

import numpy as np
import pytest

import oracle as O
from gpu_helpers import FIELDS, compare_grids, phase_for, rel_err, scene_particles, to_oracle_phase

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _oracle_run(n, ps, pp, cfg, steps, fp32_state, out):
    """Oracle steps; after each one the grid's fields and the particles."""
    o = O.Oracle()
    g, s = O.OracleGrid(n, n, n, 1.0 / n), O.OracleGrid(n, n, n, 1.0 / n)
    ps = ps.copy()
    for _ in range(steps):
        o.step(g, s, ps, pp, cfg)
        if fp32_state:
            ps.pos = ps.pos.astype(np.float32).astype(np.float64)
            ps.vel = ps.vel.astype(np.float32).astype(np.float64)
        out.append(([g.get_field(f) for f in range(8)], ps.pos.copy(), ps.vel.copy()))


def test_rayleigh_taylor_48_ten_steps(pf):
    n, steps = 48, 10
    sc = pf.scenes.rayleigh_taylor(n, seed=0)
    assert len(sc["pos"]) == 778688
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    opp = to_oracle_phase(pp)
    cfg = dict(dt=1 / 240, gravity=-9.81, Vp=1.0, alpha_l=0.95, alpha_g=0.95, cg_iters=20000, cg_tol=0.0,
               cg_rel_tol=1e-6)
    runs = {"fp64": [], "fp32": []}
    threads = [threading.Thread(target=_oracle_run, args=(n, ps, opp, cfg, steps, k == "fp32", runs[k]))
               for k in runs]
    for t in threads:
        t.start()
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(ps))
    sim.phase = pp
    sim.dt = 1 / 240
    sim.alpha_liquid = sim.alpha_gas = 0.95
    sim.cg_iters, sim.cg_tol = 20000, 0.0
    sim.solver = pf.SolverConfig(rel_tol=1e-6)
    sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
    gpu = []
    for _ in range(steps):
        st = sim.step()
        assert st.solve.converged
        pos, vel, _, _ = sim.get_particles()
        gpu.append(([sim.grid.get_field(f) for f in range(8)], pos.astype(np.float64), vel.astype(np.float64)))
    for t in threads:
        t.join()
    worst_gpu, worst_floor, failures = {}, {}, []
    print("\nstep  field: GPU vs reference arithmetic | FP32-state oracle vs reference arithmetic")
    for s in range(steps):
        (fg, pg, vg), (f64, p64, v64), (f32, _, v32) = gpu[s], runs["fp64"][s], runs["fp32"][s]
        row = []
        for f, name in enumerate(FIELDS[:7]):
            if not np.array_equal(fg[f][1], f64[f][1]):
                failures.append(f"step {s} {name}: 4^3 activity differs")
            e, e0 = rel_err(fg[f][0], f64[f][0]), rel_err(f32[f][0], f64[f][0])
            worst_gpu[name] = max(worst_gpu.get(name, 0.0), e)
            worst_floor[name] = max(worst_floor.get(name, 0.0), e0)
            row.append(f"{name} {e:.1e}|{e0:.1e}")
        ev, ev0 = rel_err(vg, v64), rel_err(v32, v64)
        worst_gpu["vel"] = max(worst_gpu.get("vel", 0.0), ev)
        worst_floor["vel"] = max(worst_floor.get("vel", 0.0), ev0)
        dpos = float(np.max(np.abs(pg - p64))) * n
        if dpos >= 1e-3:
            failures.append(f"step {s}: positions differ by {dpos} cells")
        print(f"{s:4d}  " + "  ".join(row) + f"  vel {ev:.1e}|{ev0:.1e}  pos {dpos:.1e} cells")
    print("worst over 10 steps (GPU | FP32-state floor):",
          {k: f"{worst_gpu[k]:.1e}|{worst_floor[k]:.1e}" for k in worst_gpu})
    # the first step starts from identical FP32-representable inputs
    (fg, _, vg), (f64, _, v64) = gpu[0], runs["fp64"][0]
    for f, name in enumerate(FIELDS[:7]):
        if rel_err(fg[f][0], f64[f][0]) >= 1e-5:
            failures.append(f"first step, {name}: {rel_err(fg[f][0], f64[f][0]):.2e}")
    if rel_err(vg, v64) >= 1e-5:
        failures.append(f"first step, particle velocities: {rel_err(vg, v64):.2e}")
    # after it, the drift is bounded by the FP32-storage floor's order of magnitude
    for k in worst_gpu:
        if worst_gpu[k] > max(1e-5, 4.0 * worst_floor[k]):
            failures.append(f"{k}: GPU drift {worst_gpu[k]:.2e} against FP32-storage floor {worst_floor[k]:.2e}")
    assert not failures, "; ".join(failures)


def test_p2g_bubble_tank_128_matches_oracle(pf):
    n = 128
    sc = pf.scenes.bubble_tank(n, seed=0)
    assert len(sc["pos"]) == 11303712
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    g = pf.SparseMacGrid3D(n, n, n, 1.0 / n, max_particles=len(ps))
    pf.spP2G3D_tp(g, ps, pp, 1.0)
    go = O.OracleGrid(n, n, n, 1.0 / n)
    O.Oracle().p2g(go, ps, to_oracle_phase(pp), 1.0)
    for name, (err, nact) in compare_grids(g, go, range(6)).items():
        assert nact == 0, f"{name}: {nact} 4^3 activity flags differ"
        assert err < 1e-5, f"{name}: relative error {err}"
    # the headspace (y >= 0.7) stays unallocated: no active block above the
    # water's reach (top particle cell j = 89, kernel reach two nodes)
    _, act = g.get_field(pf.PF_MV)
    by = np.nonzero(act.any(axis=(0, 2)))[0]
    assert by.max() * 4 <= 89 + 3
    g.close()


def _shuffled_rt(pf, n, seed):
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(sc["pos"]))
    for k in ("pos", "type", "volume"):
        sc[k] = np.ascontiguousarray(sc[k][perm])
    sc["vel"] = rng.normal(0, 0.3, sc["pos"].shape).astype(np.float32)
    return sc


def test_p2g_is_bit_reproducible(pf):
    """Two contexts and repeated calls on one context give identical bits.
    The particles are shuffled, so a cell's particles arrive at the binning
    in scattered order and the in-cell sort is exercised; one cell is packed
    with 40 particles to take the cooperative sort of large cells."""
    n = 32
    sc = _shuffled_rt(pf, n, seed=5)
    dense = np.tile(np.array([[0.51, 0.52, 0.53]], np.float32), (40, 1))
    dense += np.linspace(0, 0.01 / n, 40, dtype=np.float32)[:, None]
    sc["pos"] = np.concatenate([sc["pos"], dense])
    sc["vel"] = np.concatenate([sc["vel"], np.ones((40, 3), np.float32)])
    sc["type"] = np.concatenate([sc["type"], np.zeros(40, np.uint8)])
    sc["volume"] = np.concatenate([sc["volume"], np.ones(40, np.float32)])
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    runs = []
    g1 = pf.SparseMacGrid3D(n, n, n, 1.0 / n, max_particles=len(ps))
    g2 = pf.SparseMacGrid3D(n, n, n, 1.0 / n, max_particles=len(ps))
    for g in (g1, g2, g1):
        pf.spP2G3D_tp(g, ps, pp, 1.0)
        runs.append([g.get_field(f) for f in range(6)])
    for r in runs[1:]:
        for f in range(6):
            assert np.array_equal(_bits(r[f][0]), _bits(runs[0][f][0])), f"{FIELDS[f]} differs between runs"
            assert np.array_equal(r[f][1], runs[0][f][1])
    # and still the oracle's P2G to the usual tolerance
    go = O.OracleGrid(n, n, n, 1.0 / n)
    O.Oracle().p2g(go, ps, to_oracle_phase(pp), 1.0)
    for name, (err, nact) in compare_grids(g1, go, range(6)).items():
        assert nact == 0 and err < 1e-5, f"{name}: {err} {nact}"
    g1.close()
    g2.close()


def test_step_is_bit_reproducible(pf):
    n = 32
    sc = _shuffled_rt(pf, n, seed=6)
    pp = phase_for(sc, pf)
    out = []
    for _ in range(2):
        sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
        sim.phase = pp
        sim.dt = 1 / 240
        sim.cg_iters, sim.cg_tol = 4000, 0.0
        sim.solver = pf.SolverConfig(rel_tol=1e-8)
        sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
        its = [sim.step().solve.iterations for _ in range(3)]
        pos, vel, _, _ = sim.get_particles()
        out.append((its, pos, vel, sim.grid.get_field(pf.PF_P)[0]))
        sim.grid.close()
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(_bits(a), _bits(b))


@pytest.mark.parametrize("order", [2, 3])
def test_step_tiled_advection_equals_separate_passes(pf, order):
    """pf_step's last pass (G2P and RK2/RK3 advection fused over the P2G tile
    bins, the stages sampled from a staged box) against the same step taken
    pass by pass through the C ABI, where pf_g2p and pf_advect sample the
    grid per particle: positions, velocities and clamp counts bit-identical.
    Velocities of N(0, 2^2) at dt 1/8 move midpoints by several cells, so
    both the box and its fallback outside the box are exercised, and the
    walls clamp particles."""
    import ctypes as C

    L = pf._lib
    n = 32
    sc = pf.scenes.bubble_tank(n, seed=12)
    rng = np.random.default_rng(5)
    vel = rng.normal(0.0, 2.0, sc["vel"].shape).astype(np.float32)
    pp = phase_for(sc, pf)
    sims = []
    for _ in range(2):
        sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
        sim.phase = pp
        sim.dt = 1 / 8
        sim.advection_order = order
        sim.alpha_liquid, sim.alpha_gas = 0.97, 0.9
        sim.cg_iters, sim.cg_tol = 4000, 0.0
        sim.solver = pf.SolverConfig(rel_tol=1e-8)
        sim.set_particles(sc["pos"], vel, sc["type"], sc["volume"])
        sims.append(sim)
    a, b = sims
    st = a.step()
    cfg = b.step_cfg()
    ctx, lib = b.grid.ctx, b.grid.lib
    L.check(lib.pf_grid_clear_all(ctx), ctx, "pf_grid_clear_all")
    L.check(lib.pf_mark_cells(ctx), ctx, "pf_mark_cells")
    L.check(lib.pf_p2g(ctx, C.byref(cfg.phase), cfg.Vp), ctx, "pf_p2g")
    L.check(lib.pf_save_velocity(ctx), ctx, "pf_save_velocity")
    L.check(lib.pf_apply_gravity(ctx, cfg.dt, cfg.gravity), ctx, "pf_apply_gravity")
    L.check(lib.pf_apply_wall_boundary(ctx), ctx, "pf_apply_wall_boundary")
    sst = L.SolveStats()
    L.check(lib.pf_project(ctx, C.byref(cfg.phase), cfg.dt, C.byref(cfg.solve), C.byref(sst)), ctx, "pf_project")
    L.check(lib.pf_g2p(ctx, None, cfg.alpha_l, cfg.alpha_g), ctx, "pf_g2p")
    cs = L.ClampStats()
    L.check(lib.pf_advect(ctx, cfg.dt, order, C.byref(cs), None, None), ctx, "pf_advect")
    assert sst.iterations == st.solve.iterations
    pa, va, _, _ = a.get_particles()
    pb, vb, _, _ = b.get_particles()
    assert np.array_equal(_bits(va), _bits(vb))
    assert np.array_equal(_bits(pa), _bits(pb))
    assert st.clamp.as_tuple() == cs.as_tuple()
    assert st.clamp.clamped_liquid + st.clamp.clamped_gas > 0
    for sim in sims:
        sim.grid.close()


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("case", ["bubble", "rt", "random"])
def test_active_cells_match_reference_collect(pf, case):
    """pf_active_cells against the reference's collectCellsWithMarker on the
    same marker field: walls, fluid, empty headspace, and a random field with
    holes and isolated fluid cells."""
    n = 24
    if case == "random":
        rng = np.random.default_rng(3)
        mk = rng.choice([0, 1, 2], size=(n, n, n), p=[0.4, 0.5, 0.1]).astype(np.int32)
    else:
        sc = pf.scenes.bubble_tank(n, seed=1) if case == "bubble" else pf.scenes.rayleigh_taylor(n, seed=1)
        go = O.OracleGrid(n, n, n, 1.0 / n)
        O.Oracle().mark_cells(go, scene_particles(sc))
        mk = go.cell_markers()
    g = pf.SparseMacGrid3D(n, n, n, 1.0 / n)
    g.set_cells(mk)
    rg = O.ReferenceGrid(n, n, n, 1.0 / n)
    rg.set_cells(mk)
    ref = rg.collect_cells(1)
    assert len(ref) > 0
    assert np.array_equal(g.fluid_cells(), ref)
    g.close()


@pytest.mark.parametrize("scene,n,seed", [("rayleigh_taylor", 24, 0), ("rayleigh_taylor", 40, 3),
                                          ("bubble_tank", 32, 0), ("bubble_tank", 48, 5), ("dam_break", 32, 2),
                                          ("dam_break", 45, 7)])
def test_device_scene_equals_host_generator(pf, scene, n, seed):
    """pf_seed_scene against scenes.py: positions and types identical, volumes
    1, bubble-tank velocities within one FP32 ulp (Box-Muller on the device's
    libm)."""
    sc = getattr(pf.scenes, scene)(n, seed=seed)
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
    assert sim.seed_scene(scene, seed) == len(sc["pos"])
    pos, vel, typ, vol = sim.get_particles()
    assert np.array_equal(_bits(pos), _bits(sc["pos"]))
    assert np.array_equal(typ, sc["type"])
    assert np.all(vol == 1.0)
    ulp = np.spacing(np.abs(sc["vel"]).astype(np.float32))
    assert np.all(np.abs(vel - sc["vel"]) <= ulp)
    sim.grid.close()
