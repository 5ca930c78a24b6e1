"""Generate the golden fixtures in this directory from the UNMODIFIED reference.

The reference's sparse 3D two-phase sources are compiled by oracle/Makefile
into oracle/_ref/libpfref.so (this needs the reference source tree, so run it
where that tree exists):

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores its seeded inputs and the reference's outputs, so the
tests can pin the C restatement (and the GPU path) without the reference.
The reference ships no golden vectors of its own; its tests hold inline known
answers, which known_answers.json records as the reference computes them.
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def load_pkg():
    d = os.path.join(ROOT, "adaptive-pf-flip_b200")
    spec = importlib.util.spec_from_file_location("adaptive_pf_flip_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["adaptive_pf_flip_b200"] = m
    spec.loader.exec_module(m)
    return m


def grid_arrays(g, prefix=""):
    out = {}
    for f, name in enumerate(O.FIELD_NAMES):
        d, a = g.get_field(f)
        out[prefix + name] = d
        out[prefix + name + "_act4"] = a
    return out


def scene_inputs(sc, vel_sigma, seed):
    rng = np.random.default_rng(seed)
    vel = rng.normal(0, vel_sigma, sc["pos"].shape).astype(np.float32) if vel_sigma else sc["vel"]
    return dict(pos=sc["pos"].astype(np.float32), vel=vel.astype(np.float32), type=sc["type"].astype(np.uint8),
                volume=sc["volume"].astype(np.float32))


def particles(inp):
    return O.Particles(inp["pos"].astype(np.float64), inp["vel"].astype(np.float64), inp["type"],
                       inp["volume"].astype(np.float64))


def main():
    pf = load_pkg()
    ref = O.Reference()

    # 1. P2G on a jittered Rayleigh-Taylor scene with random velocities
    n = 12
    sc = pf.scenes.rayleigh_taylor(n, seed=21)
    inp = scene_inputs(sc, 0.3, 21)
    pp = O.PhaseParams(1000.0, 1.0)
    pp.rho_tilde_0 = ref.calibrate_rho_tilde0(pp, 1.0)
    g = O.ReferenceGrid(n, n, n, 1.0 / n)
    ref.p2g(g, particles(inp), pp, 1.0)
    np.savez_compressed(os.path.join(HERE, "p2g_rt12.npz"), n=n, dx=1.0 / n, phase=pp.as_array(), **inp,
                        **grid_arrays(g))

    # 2. three full reference steps (SparseSim3DTP::step), 1000:1, dt = 1/240
    ps = particles(inp)
    gs = O.ReferenceGrid(n, n, n, 1.0 / n)
    cfg = dict(dt=1 / 240, gravity=-9.81, Vp=1.0, alpha_l=0.95, alpha_g=0.95, cg_iters=600, cg_tol=1e-7,
               advect_order=2)
    out = {}
    for s in range(3):
        ref.step(gs, ps, pp, cfg)
        out[f"pos{s}"] = ps.pos.copy()
        out[f"vel{s}"] = ps.vel.copy()
    out.update(grid_arrays(gs, "last_"))
    np.savez_compressed(os.path.join(HERE, "step_rt12.npz"), n=n, dx=1.0 / n, phase=pp.as_array(),
                        cfg=json.dumps(cfg), **inp, **out)

    # 3. bubble-tank P2G (sparse headspace) at 16^3
    n = 16
    sc = pf.scenes.bubble_tank(n, seed=4)
    inp = scene_inputs(sc, 0, 4)
    pp2 = O.PhaseParams(1000.0, 1.0)
    pp2.rho_tilde_0 = ref.calibrate_rho_tilde0(pp2, 1.0)
    g = O.ReferenceGrid(n, n, n, 1.0 / n)
    ref.p2g(g, particles(inp), pp2, 1.0)
    np.savez_compressed(os.path.join(HERE, "p2g_bubble16.npz"), n=n, dx=1.0 / n, phase=pp2.as_array(), **inp,
                        **grid_arrays(g))

    # 4. known answers of the reference's own tests, as the reference computes them
    ka = {}
    d = O.PhaseParams()
    ka["phi_rho_g"] = ref.phi_from_raw(d.rho_g, d)
    ka["phi_rho_l"] = ref.phi_from_raw(d.rho_l, d)
    ka["calibrate_default"] = ref.calibrate_rho_tilde0(d, 1.0)
    ka["calibrate_1000_1"] = ref.calibrate_rho_tilde0(O.PhaseParams(1000.0, 1.0), 1.0)
    g = O.ReferenceGrid(8, 8, 8, 1.0)
    one = O.Particles(np.array([[3.0, 2.5, 2.5]]), np.array([[4.0, 3.0, 2.0]]), np.array([0]), np.array([1.0]))
    ref.p2g(g, one, d, 1.0)
    u, _ = g.get_field(O.U)
    mu, act = g.get_field(O.MU)
    ka["p2g_momentum_u"] = float((u.astype(np.float64) * mu.astype(np.float64)).sum())
    ka["p2g_mu_active_blocks"] = int(act.sum())
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1, sort_keys=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
