"""Train the learned coarse solve of the LEARNED pressure mode and save its
parameter vector (the file the package loads by default).

Training pairs (r_c, A_c^-1 r_c) are harvested on the GPU from exact
two-level solves (PF_PRECOND_EXACT_COARSE) of seeded pressure systems
(seed 0 of every scene is left for evaluation):

* 64 air ellipsoids in water at 1000:1 with a band-limited divergence
  (scenes.ellipsoid_pressure) at 64^3, 128^3 and 256^3;
* the pressure systems of whole solver steps: Rayleigh-Taylor at 48^3,
  128^3 and 256^3 (heavy over light, walls only) and the bubble tank at
  128^3 (air bubble in water under an open headspace), one to six
  consecutive steps each.

Each grid harvests on its own context; the pairs are then merged into one
context and trained with one optimiser (Adam with gradient-norm clipping,
32000 steps of batch 8).

    python adaptive-pf-flip_b200/train_coarse_net.py [--out PATH] [--steps N]
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "weights", "coarse_net.npy")
NAMES = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")


def _package():
    name = "adaptive_pf_flip_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pressure_system(pf, n, seed, grid=None):
    """Load the seeded ellipsoid pressure system into `grid` (new n^3 grid if
    None); returns (grid, solve) where solve(cfg, max_iter) resets u/v/w and
    projects."""
    sc = pf.scenes.ellipsoid_pressure(n, seed=seed)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    g = grid or pf.SparseMacGrid3D(n, n, n, sc["dx"], max_particles=1)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0, grid=g)
    f = pf.scenes.pressure_grid_fields(sc, pp.rho_tilde_0)
    full = {k: np.ones(g.bdims(i)[::-1], np.uint8) for i, k in enumerate(NAMES)}
    for k in ("mu", "mv", "mw", "mk"):
        g.set_field(NAMES.index(k), f[k], full[k])

    def solve(cfg, max_iter=20000):
        for k in ("u", "v", "w"):
            g.set_field(NAMES.index(k), f[k], full[k])
        st = pf.spProjectStepVC3D(g, pp, 1.0 / 240.0, max_iter, 0.0, solver=cfg)
        p, _ = g.get_field(pf.PF_P)
        return st, p.astype(np.float64)

    return g, solve


def step_systems(pf, scene, n, seed, steps, solve_cfg, harvest_on):
    """Run `steps` whole solver steps of a seeded scene with the given solver
    (the harvest is switched on by `harvest_on(grid)` after the first, plain,
    step so that every harvested system has a developed velocity field);
    returns (sim, iterations per harvested step)."""
    sc = pf.scenes.rayleigh_taylor(n, seed=seed) if scene == "rt" else pf.scenes.bubble_tank(n, seed=seed)
    sim = pf.SparseSim3DTP(n, n, n, sc["dx"], max_particles=len(sc["pos"]))
    sim.phase = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    sim.phase.rho_tilde_0 = pf.calibrateRhoTilde0(sim.phase, 1.0, grid=sim.grid)
    sim.dt = 1.0 / 240.0
    if scene == "bubble":
        sim.alpha_liquid = sim.alpha_gas = 0.97
    sim.cg_iters, sim.cg_tol = 20000, 0.0
    sim.solver = pf.SolverConfig(rel_tol=1e-6)
    sim.set_particles(sc["pos"], sc["vel"], sc["type"], sc["volume"])
    del sc
    sim.step()
    harvest_on(sim.grid)
    sim.solver = solve_cfg
    return sim, [sim.step().solve.iterations for _ in range(steps)]


# (scene, n, seed, steps): ellipsoid systems are solved once; step scenes
# harvest from `steps` consecutive steps
PLAN = (("ellipsoid", 64, 1, 1), ("ellipsoid", 64, 2, 1), ("ellipsoid", 64, 3, 1), ("ellipsoid", 128, 1, 1),
        ("ellipsoid", 128, 2, 1), ("ellipsoid", 256, 1, 1), ("rt", 48, 1, 6), ("rt", 128, 1, 3),
        ("bubble", 128, 1, 3), ("bubble", 128, 2, 2), ("rt", 256, 1, 1), ("rt", 128, 2, 3))


def train(plan=PLAN, steps=32000, batch=8, seed=11, log=print):
    pf = _package()
    nets, grids, params = {}, {}, None
    exact = pf.SolverConfig(mode=pf.PF_SOLVER_LEARNED, rel_tol=1e-6, precond=pf.PF_PRECOND_EXACT_COARSE)
    t0 = time.time()

    def start(key, g):
        nonlocal params
        net = pf.LearnedCoarseSolver(g)
        if params is None:
            net.init(seed)
            params = net.params()
        else:
            net.load(params)
        net.harvest(True, stride=2, max_per_system=200, capacity_floats=1 << 27)
        nets[key] = net

    for scene, n, s, k in plan:
        if scene == "ellipsoid":
            g, solve = pressure_system(pf, n, s, grids.get(("ellipsoid", n)))
            if ("ellipsoid", n) not in nets:
                grids[("ellipsoid", n)] = g
                start(("ellipsoid", n), g)
            st, _ = solve(exact)
            its = [st.iterations]
        else:
            key = (scene, n, s)
            sim, its = step_systems(pf, scene, n, s, k, exact, lambda g: start(key, g))
            grids[key] = sim.grid
        log(f"harvest {scene} n={n} seed={s}: exact two-level iterations {its}, {time.time() - t0:.1f} s")
    for net in nets.values():
        net.harvest(False)
    # one optimiser over every system: gather the pairs in the context of the largest lattice
    trainer = nets[("ellipsoid", max(n for sc_, n, _, _ in plan if sc_ == "ellipsoid"))]
    for key, net in nets.items():
        if net is not trainer:
            trainer.merge_dataset(net)
    systems, pairs = trainer.dataset()
    log(f"training set: {systems} systems, {pairs} pairs")
    phases = ((int(steps * 0.7), 1e-3), (steps - int(steps * 0.7), 3e-4))
    for q, (k, lr) in enumerate(phases):
        losses = trainer.train(steps=k, batch=batch, lr=lr, seed=seed + q)
        for a in range(0, k, max(1, k // 6)):
            log(f"steps {a}-{a + max(1, k // 6)} at lr {lr:g}: loss {losses[a:a + max(1, k // 6)].mean():.4f}")
    params = trainer.params()
    for g in grids.values():
        g.close()
    return params


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--steps", type=int, default=32000)
    args = ap.parse_args()
    params = train(steps=args.steps)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.save(args.out, params.astype(np.float32))
    print(f"saved {params.size} parameters to {args.out}")


if __name__ == "__main__":
    main()
