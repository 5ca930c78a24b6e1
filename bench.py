#!/usr/bin/env python
"""Solver-step benchmark for the B200 backend (one JSON line on rank 0).

Default workload (transfer stress): bubble tank on a 128^3 grid, 8^3-cell
tiles, water below y = 0.7 with an air bubble of radius 0.15 at
(0.5, 0.3, 0.5), 8 jittered particles per cell (11,303,712 particles),
velocities N(0, 0.1^2); one step = P2G (u, v, w and face raw mass, the phi
input) + saved copy + G2P with FLIP ratio 0.97, device-resident.

  value       step particles/s with inputs resident on the device, CUDA events
              on the library's stream around K steps (max over ranks)
  e2e         the same through the public C ABI from pinned host buffers:
              every step uploads the particles (29 B each) and reads back the
              updated velocities (12 B each); both copies are asynchronous,
              so they overlap the neighbouring steps' device work
  roofline    the dominant kernel's algorithmic bytes per launch / its mean
              device time (per-stage CUDA events), against the measured HBM
              copy bandwidth
  cpu_baseline the reference's own C++ P2G + G2P (compiled from its sources
              into oracle/_ref) on a bounded slab of the same scene

--impl reference times that reference CPU path alone (rank 0; other ranks
exit).  Multi-GPU runs are independent replicas (weak scaling): the solver
step is single-GPU by design.
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "adaptive-pf-flip_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_pkg():
    name = "adaptive_pf_flip_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


METRIC = "step particles/s (P2G + G2P transfer step, bubble tank 128^3)"
UNIT = "particles/s"
# algorithmic bytes (FP32 SoA particles: pos 12, vel 12, type 1, volume 4)
P2G_BYTES_PER_PARTICLE = 29
P2G_BYTES_PER_FACE = 8       # momentum->velocity + raw mass written once per active face node
G2P_BYTES_PER_PARTICLE = 37  # read pos+vel+type, write vel
G2P_BYTES_PER_FACE = 8       # current + saved face velocity read once
# warp instructions k_splat issues per particle (ncu, profiles/k_splat_bubble128.md): the
# splat's issue roofline is this count over 148 SMs x 4 schedulers at the SM clock
SPLAT_WARP_INST_PER_PARTICLE = 42.1
# Algorithmic bytes per unknown and iteration of the pressure solvers: the
# arrays each pass reads or writes once (FP64 8 B, FP32 4 B, BF16 2 B, the
# kind / coarse-class bytes 1 B); a neighbour's value is an L1/L2 hit and is
# not counted again.
PCG_BYTES = {
    "plain": 139,            # k_spmv_plain_tab 49 (p, 3 couplings, diagonal, kind, Ap), k_update_plain 57, k_direction_plain 33
    "flex64": 141,           # k_fx_spmv 49, k_fx_update 58, k_fx_dir 34 (the learned coarse path is not HBM-bound)
    "inner_fp32": 71,        # k_mixed_spmv 25, k_mixed_update 29, k_mixed_direction 17
    "inner_bf16": 65,        # the same with BF16 couplings
    "inner_bf16_dir": 57,    # BF16 couplings and search direction
    "inner_learned32": 73,   # FP32 k_fx_spmv 25, k_fx_update 30, k_fx_dir 18
    "outer": 165,            # per outer FCG(1) iteration: k_oc_beta 13, k_oc_dir 21, k_oc_spmv 57, k_oc_update 49, inner start 25
}


def pcg_bytes(pf, cfg, st):
    """Algorithmic bytes per unknown of one solve (PCG_BYTES x iterations)."""
    if cfg.mode == pf.PF_SOLVER_PLAIN:
        return PCG_BYTES["plain"] * st.iterations
    if cfg.mode == pf.PF_SOLVER_LEARNED and not cfg.inner_fp32:
        return PCG_BYTES["flex64"] * st.iterations
    if cfg.mode == pf.PF_SOLVER_LEARNED:
        inner = PCG_BYTES["inner_learned32"]
    else:
        inner = PCG_BYTES[{0: "inner_fp32", 1: "inner_bf16"}.get(int(cfg.bf16_storage), "inner_bf16_dir")]
    return inner * st.iterations + PCG_BYTES["outer"] * st.refinements


def pcg_roofline(pf, cfg, st, peak):
    """Achieved bytes/s of a solve's fine-level passes against the HBM peak."""
    b = pcg_bytes(pf, cfg, st) * st.n_cells
    gbs = b / max(st.solve_ms / 1000.0, 1e-12) / 1e9
    return {"bytes_per_unknown": pcg_bytes(pf, cfg, st), "achieved_gbs": gbs, "frac": gbs / peak}


def issue_roofline(n_particles, splat_ms, sm_mhz, sms=148, schedulers=4):
    """k_splat against its warp-instruction issue rate at the sampled SM clock."""
    inst = SPLAT_WARP_INST_PER_PARTICLE * n_particles
    bound_ms = inst / (sms * schedulers * sm_mhz * 1e6) * 1000.0
    return {"kernel": "k_splat (P2G)", "warp_inst_per_launch": inst, "issue_bound_ms": bound_ms,
            "mean_launch_ms": splat_ms, "frac": bound_ms / max(splat_ms, 1e-12), "sm_mhz": sm_mhz,
            "source": "warp instructions per particle from ncu (profiles/k_splat_bubble128.md)"}


def host_info():
    """The host's CPUs as this process sees them."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        affinity = len(os.sched_getaffinity(0))
    except AttributeError:
        affinity = os.cpu_count()
    return {"cpu_model": model, "online_cpus": os.cpu_count(), "affinity_cpus": affinity}


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local, dist


def reduce_max(dist, value, local):
    """The largest of every rank's value (the job's time is its slowest replica's)."""
    if dist is None:
        return value
    import torch
    device = "cpu" if dist.get_backend() == "gloo" else f"cuda:{local}"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, steps, world, ms_max):
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return units_per_rank * steps * world / (ms_max / 1000.0)


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

class TransferStep:
    """P2G + saved copy + G2P on one libpfgpu context."""

    def __init__(self, pf, sc, device, alpha=0.97):
        import torch
        self.pf, self.L = pf, pf._lib
        self.lib = pf.load()
        self.n = len(sc["pos"])
        nx = sc["nx"]
        self.g = pf.SparseMacGrid3D(nx, sc["ny"], sc["nz"], sc["dx"], max_particles=self.n, device=device)
        self.ctx = self.g.ctx
        pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
        pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0, grid=self.g)
        self.phase = pp._c()
        self.alpha = alpha
        # pinned host copies of the inputs (for the end-to-end leg)
        self.h_pos = torch.from_numpy(np.ascontiguousarray(sc["pos"], np.float32)).pin_memory()
        self.h_vel = torch.from_numpy(np.ascontiguousarray(sc["vel"], np.float32)).pin_memory()
        self.h_type = torch.from_numpy(np.ascontiguousarray(sc["type"], np.uint8)).pin_memory()
        self.h_vol = torch.from_numpy(np.ascontiguousarray(sc["volume"], np.float32)).pin_memory()
        self.h_out = torch.empty((self.n, 3), dtype=torch.float32).pin_memory()
        self.stream = torch.cuda.ExternalStream(self.lib.pf_stream(self.ctx), device=f"cuda:{device}")
        self.upload()

    def upload(self):
        rc = self.lib.pf_upload_particles(self.ctx, self.n, self.h_pos.data_ptr(), self.h_vel.data_ptr(),
                                          self.h_type.data_ptr(), self.h_vol.data_ptr())
        self.L.check(rc, self.ctx, "pf_upload_particles")

    def upload_async(self):
        """The step's inputs from pinned host memory into the second particle
        set; the copy overlaps the work already queued (the previous step)."""
        rc = self.lib.pf_upload_particles_async(self.ctx, self.n, self.h_pos.data_ptr(), self.h_vel.data_ptr(),
                                                self.h_type.data_ptr(), self.h_vol.data_ptr())
        self.L.check(rc, self.ctx, "pf_upload_particles_async")

    def download_vel(self):
        """The step's result to pinned host memory; the copy overlaps the next
        step's upload (the timed region joins it before its end event)."""
        rc = self.lib.pf_download_particles_async(self.ctx, None, self.h_out.data_ptr(), None, None)
        self.L.check(rc, self.ctx, "pf_download_particles_async")

    def join_downloads(self):
        self.L.check(self.lib.pf_join_downloads(self.ctx), self.ctx, "pf_join_downloads")

    def step(self):
        L, lib, ctx = self.L, self.lib, self.ctx
        L.check(lib.pf_p2g(ctx, C.byref(self.phase), 1.0), ctx, "pf_p2g")
        L.check(lib.pf_save_velocity(ctx), ctx, "pf_save_velocity")
        L.check(lib.pf_g2p(ctx, None, self.alpha, self.alpha), ctx, "pf_g2p")

    def active_faces(self):
        n = 0
        for f in (self.pf.PF_MU, self.pf.PF_MV, self.pf.PF_MW):
            m, _ = self.g.get_field(f)
            n += int((m > 0).sum())
        return n


def time_steps(ts, steps, warmup, dist, local, e2e=False):
    import torch
    for _ in range(warmup):
        if e2e:
            ts.upload_async()
        ts.step()
        if e2e:
            ts.download_vel()
    if e2e:
        ts.lib.pf_sync(ts.ctx)
    torch.cuda.synchronize(local)
    barrier(dist)
    torch.cuda.synchronize(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ts.lib.pf_launch_count(ts.ctx)
    ev0.record(ts.stream)
    for _ in range(steps):
        if e2e:
            ts.upload_async()
        ts.step()
        if e2e:
            ts.download_vel()
    if e2e:
        ts.join_downloads()
    ev1.record(ts.stream)
    ev1.synchronize()
    torch.cuda.synchronize(local)
    launches = ts.lib.pf_launch_count(ts.ctx) - launches0
    barrier(dist)
    ms = ev0.elapsed_time(ev1)
    return reduce_max(dist, ms, local), launches


def cpu_reference_sample(sc, slab_cells, steps, warmup=0, alpha=0.97):
    """Reference P2G + saved copy + G2P (oracle/_ref, the unmodified sources)
    on the particles of the first `slab_cells` x-columns of the scene."""
    import oracle as O
    n = sc["nx"]
    x = sc["pos"][:, 0].astype(np.float64)
    sel = x < slab_cells * sc["dx"]
    ps = O.Particles(sc["pos"][sel].astype(np.float64), sc["vel"][sel].astype(np.float64), sc["type"][sel],
                     sc["volume"][sel].astype(np.float64))
    ref = O.Reference()
    pp = O.PhaseParams(sc["rho_l"], sc["rho_g"])
    pp.rho_tilde_0 = ref.calibrate_rho_tilde0(pp, 1.0)
    g = O.ReferenceGrid(n, n, n, sc["dx"])
    saved = O.ReferenceGrid(n, n, n, sc["dx"])
    lib = g.lib
    g._put(ps)
    arr = pp.as_array()
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        lib.pfr_p2g(g.h, arr, 1.0)
        lib.pfr_copy_grid(saved.h, g.h)
        lib.pfr_g2p(g.h, saved.h, alpha, alpha)
        t1 = time.perf_counter()
        if it >= warmup:
            times.append(t1 - t0)
    return len(ps), times


def pcg_modes(pf, names):
    """Solver configurations of the pressure-only block, by name."""
    L = pf.PF_SOLVER_LEARNED
    table = {
        "plain_fp64": pf.SolverConfig(mode=pf.PF_SOLVER_PLAIN, rel_tol=1e-6),
        "mixed_fp32": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6),
        "mixed_bf16": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6, bf16_storage=1),
        "mixed_bf16_dir": pf.SolverConfig(mode=pf.PF_SOLVER_MIXED, rel_tol=1e-6, bf16_storage=2),
        # the learned two-level preconditioner and its net-free ablation
        "learned": pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK),
        "flex_jacobi": pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_JACOBI),
        # FP64 flexible CG preconditioned by the learned flexible PCG in FP32
        "learned_mixed": pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK, inner_fp32=True),
        # the same two-level solver with an exact coarse solve: the bound a perfect network reaches
        "exact_coarse": pf.SolverConfig(mode=L, rel_tol=1e-6, precond=pf.PF_PRECOND_EXACT_COARSE),
    }
    table["learned_fp32"] = table["learned_mixed"]
    # "name#k" repeats a mode (a second solve on the same context: allocations done);
    # "name@M:ETA" sets an inner-outer mode's inner cap and relative reduction
    out = []
    for name in names:
        base = name.split("#")[0]
        cfg = dataclasses.replace(table[base.split("@")[0]])
        if "@" in base:
            m, eta = base.split("@")[1].split(":")
            cfg.inner_max_iter, cfg.inner_rel_tol = int(m), float(eta)
        out.append((name, cfg))
    return out


def load_weights(pf, grid, path=None):
    """Load the shipped network weights (or the file at `path`) into a grid's context."""
    net = pf.LearnedCoarseSolver(grid)
    if path:
        net.load_file(path)
        return os.path.relpath(os.path.abspath(path), ROOT)
    return net.load_default()


def oracle_pressure(sc, f, pp, n, dt, rel_tol=1e-10):
    """The CPU FP64 oracle's pressure of the same system (oracle/pf_oracle.c,
    Jacobi-PCG to rel_tol), and its wall time."""
    import oracle as O
    names = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")
    go = O.OracleGrid(n, n, n, sc["dx"])
    for k in ("u", "v", "w", "mu", "mv", "mw", "mk"):
        i = names.index(k)
        go.set_field(i, f[k], np.ones(go.bdims(i)[::-1], np.uint8))
    t0 = time.perf_counter()
    st = O.Oracle().project(go, O.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0), dt, 200000, 0.0,
                            rel_tol=rel_tol)
    wall = time.perf_counter() - t0
    p, _ = go.get_field(O.P)
    return p.astype(np.float64), {"rel_tol": rel_tol, "iterations": st.iterations, "converged": bool(st.converged),
                                  "cpu_s": wall, "cores": 1}


def run_pcg(pf, n, modes, max_iter=20000, seed=0, weights_path=None, fp64_oracle=False):
    """Pressure-only system (n^3, every interior cell fluid, 64 air ellipsoids
    in water at 1000:1, band-limited RHS): device time to a 1e-6 relative
    FP64 residual per solver mode, and each mode's pressure against the
    PLAIN FP64 solve (the first mode) and, with fp64_oracle, against the CPU
    FP64 oracle solved to 1e-10."""
    sc = pf.scenes.ellipsoid_pressure(n, seed=seed)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    g = pf.SparseMacGrid3D(n, n, n, sc["dx"], max_particles=1)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0, grid=g)
    f = pf.scenes.pressure_grid_fields(sc, pp.rho_tilde_0)
    peak, _ = measured_hbm()
    p_oracle, oracle_note = None, None
    if fp64_oracle:
        p_oracle, oracle_note = oracle_pressure(sc, f, pp, n, 1.0 / 240.0)
    full = {k: np.ones(g.bdims(i)[::-1], np.uint8) for i, k in enumerate(("u", "v", "w", "mu", "mv", "mw", "p", "mk"))}
    for k in ("mu", "mv", "mw", "mk"):
        g.set_field(("u", "v", "w", "mu", "mv", "mw", "p", "mk").index(k), f[k], full[k])
    weights = None
    if any(cfg.mode == pf.PF_SOLVER_LEARNED and cfg.precond == pf.PF_PRECOND_NETWORK for _, cfg in modes):
        weights = load_weights(pf, g, weights_path)
    out, p_plain = {}, None
    lib = pf.load()
    for name, cfg in modes:
        for k in ("u", "v", "w"):
            g.set_field(("u", "v", "w").index(k), f[k], full[k])
        lib.pf_set_timing(g.ctx, 1)
        st = pf.spProjectStepVC3D(g, pp, 1.0 / 240.0, max_iter, 0.0, solver=cfg)
        tm = pf._lib.Timing()
        lib.pf_get_timing(g.ctx, C.byref(tm), 1)
        lib.pf_set_timing(g.ctx, 0)
        p, _ = g.get_field(pf.PF_P)
        rec = {"ms_to_1e-6": st.solve_ms, "iterations": st.iterations, "refinements": st.refinements,
               "converged": bool(st.converged), "rel_residual": st.res_final / max(st.res0, 1e-300),
               "setup_ms": tm.as_dict()["precond_setup"][0], "roofline": pcg_roofline(pf, cfg, st, peak)}
        if cfg.mode == pf.PF_SOLVER_LEARNED:
            rec["coarse_accepted"] = st.precond_applied
            rec["coarse_rejected"] = st.precond_rejected
            if cfg.precond == pf.PF_PRECOND_NETWORK:
                rec["weights"] = weights
        if p_plain is None:
            p_plain = p.astype(np.float64)
        else:
            rec["p_rel_diff_vs_plain"] = float(np.abs(p - p_plain).max() / max(np.abs(p_plain).max(), 1e-300))
        if p_oracle is not None:
            rec["err_vs_fp64_oracle"] = float(np.abs(p - p_oracle).max() / max(np.abs(p_oracle).max(), 1e-300))
        out[name] = rec
    base = out[modes[0][0]]["ms_to_1e-6"]
    for name in out:
        out[name]["speedup_vs_plain"] = base / max(out[name]["ms_to_1e-6"], 1e-9)
    res = {"workload": f"ellipsoid_pressure_{n}: {(n - 2) ** 3} unknowns, 64 air ellipsoids, 1000:1, "
                       "band-limited RHS |k|<=8", "peak_gbs": peak, "modes": out}
    if oracle_note:
        res["fp64_oracle"] = oracle_note
    return res


STEP_SCENES = {"rt": "rayleigh_taylor", "bubble": "bubble_tank"}


def seeded_sim(pf, name, n, seed=0, max_iter=20000):
    """A solver on the scene of a whole-step system, seeded on the device
    (pf_seed_scene: the particles scenes.py gives, without the host-side
    generation): Rayleigh-Taylor (heavy over light, 1000:1, walls only) or
    the bubble tank (air bubble in water, open headspace)."""
    if name not in STEP_SCENES:
        raise ValueError(f"unknown step scene {name!r} (rt, bubble)")
    dx = 1.0 / n
    sim = pf.SparseSim3DTP(n, n, n, dx, max_particles=8 * (n - 2) ** 3)
    sim.phase = pf.PhaseParams(1000.0, 1.0)
    sim.phase.rho_tilde_0 = pf.calibrateRhoTilde0(sim.phase, 1.0, grid=sim.grid)
    sim.dt = 1.0 / 240.0
    if name == "bubble":
        sim.alpha_liquid = sim.alpha_gas = 0.97
    sim.cg_iters, sim.cg_tol = max_iter, 0.0
    sim.solver = pf.SolverConfig(rel_tol=1e-6)
    sim.seed_scene(STEP_SCENES[name], seed)
    return sim


def run_step_pcg(pf, name, n, modes, pre_steps=1, max_iter=20000, seed=0, weights_path=None):
    """Pressure systems of real solver steps: the scene runs `pre_steps` plain
    steps, then every solver mode runs one whole step (markCells .. advect)
    from that same particle snapshot, once untimed and once timed.  Reports each solve's device time to a
    1e-6 relative FP64 residual, iterations, the coarse-correction fallback
    rate and the pressure against the PLAIN solve (the first mode)."""
    sim = seeded_sim(pf, name, n, seed, max_iter)
    np_ = sim.n
    peak, _ = measured_hbm()
    for _ in range(pre_steps):
        sim.step()
    snap = sim.get_particles()
    weights = None
    if any(cfg.mode == pf.PF_SOLVER_LEARNED and cfg.precond == pf.PF_PRECOND_NETWORK for _, cfg in modes):
        weights = load_weights(pf, sim.grid, weights_path)
    out, p_plain = {}, None
    lib = pf.load()
    for mname, cfg in modes:
        sim.solver = cfg
        # one untimed step from the snapshot first: the first solve of a mode
        # on a grid also allocates its working memory (neighbour table, pool
        # growth), which a running simulation pays once
        sim.set_particles(*snap)
        sim.step()
        sim.set_particles(*snap)
        lib.pf_set_timing(sim.grid.ctx, 1)
        st = sim.step().solve
        tm = pf._lib.Timing()
        lib.pf_get_timing(sim.grid.ctx, C.byref(tm), 1)
        lib.pf_set_timing(sim.grid.ctx, 0)
        p, _ = sim.grid.get_field(pf.PF_P)
        stages = tm.as_dict()
        rec = {"ms_to_1e-6": st.solve_ms, "iterations": st.iterations, "refinements": st.refinements,
               "converged": bool(st.converged), "rel_residual": st.res_final / max(st.res0, 1e-300),
               "setup_ms": stages["precond_setup"][0], "roofline": pcg_roofline(pf, cfg, st, peak)}
        if cfg.mode == pf.PF_SOLVER_LEARNED:
            tot = st.precond_applied + st.precond_rejected
            rec["coarse_accepted"] = st.precond_applied
            rec["coarse_rejected"] = st.precond_rejected
            rec["fallback_rate"] = st.precond_rejected / tot if tot else 0.0
            if cfg.precond == pf.PF_PRECOND_NETWORK:
                rec["weights"] = weights
        if p_plain is None:
            p_plain = p.astype(np.float64)
        else:
            rec["p_rel_diff_vs_plain"] = float(np.abs(p - p_plain).max() / max(np.abs(p_plain).max(), 1e-300))
        out[mname] = rec
    base = out[modes[0][0]]["ms_to_1e-6"]
    for mname in out:
        out[mname]["speedup_vs_plain"] = base / max(out[mname]["ms_to_1e-6"], 1e-9)
    sim.grid.close()
    return {"workload": f"{name}_{n} step pressure system after {pre_steps} plain step(s): {np_} particles, "
                        f"1000:1, dt 1/240; each mode's step run once untimed, then timed from the same particles",
            "unknowns": int(st.n_cells), "modes": out}


def run_full_step(pf, n=48, steps=20, seed=0, solvers=("plain",), warmup=3):
    """Whole solver step (markCells .. advection) on the Rayleigh-Taylor scene
    at 1000:1, pressure to 1e-6 relative; device-timed particles/s for each
    pressure solver ("plain": PLAIN PCG, "learned": the learned two-level
    preconditioner with the shipped weights), every solver from the same
    initial particles."""
    import torch
    out = {}
    for solver in solvers:
        sim = seeded_sim(pf, "rt", n, seed)
        if solver == "learned":
            pf.LearnedCoarseSolver(sim.grid).load_default()
            sim.solver = pf.SolverConfig(mode=pf.PF_SOLVER_LEARNED, rel_tol=1e-6, precond=pf.PF_PRECOND_NETWORK)
        out["workload"] = (f"rayleigh_taylor_{n}: {sim.n} particles, 1000:1, dt 1/240, pressure to 1e-6, "
                           f"{warmup} warm-up + {steps} timed steps")
        npart = sim.n
        stream = torch.cuda.ExternalStream(pf.load().pf_stream(sim.grid.ctx))
        for _ in range(warmup):
            sim.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        iters, rejected = 0, 0
        e0.record(stream)
        for _ in range(steps):
            st = sim.step().solve
            iters += st.iterations
            rejected += st.precond_rejected
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        rec = {"particles_per_s": npart * steps / (ms / 1000.0), "ms_per_step": ms / steps,
               "pcg_iterations_per_step": iters / steps}
        if solver == "learned":
            rec["coarse_rejected"] = rejected
        # where a step's time goes: per-stage device times (CUDA events on the
        # context stream) over two more steps, outside the timed region
        lib = pf.load()
        lib.pf_set_timing(sim.grid.ctx, 1)
        tm = pf._lib.Timing()
        lib.pf_get_timing(sim.grid.ctx, C.byref(tm), 1)
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(2):
            sim.step()
        e3.record(stream)
        e3.synchronize()
        lib.pf_get_timing(sim.grid.ctx, C.byref(tm), 1)
        lib.pf_set_timing(sim.grid.ctx, 0)
        step_ms = e2.elapsed_time(e3) / 2
        stages = {k: v[0] / 2 for k, v in tm.as_dict().items() if v[1]}
        rec["stages_ms_per_step"] = stages
        rec["g2p_advect_share"] = stages.get("g2p", 0.0) / step_ms
        out[solver] = rec
        sim.grid.close()
    if "plain" in out and "learned" in out:
        out["learned_speedup"] = out["plain"]["ms_per_step"] / out["learned"]["ms_per_step"]
    return out


def mr_dam_break_layout(pf, n):
    """The multires dam break's layout at n^3 fine cells: level-1 blocks
    refined where water and empty cells lie within 3 cells of each other."""
    i, j, k = pf.scenes.dam_break_cells(n)
    liquid = np.zeros((n, n, n), bool)
    liquid[k, j, i] = True
    return pf.multires.interface_levels(liquid, 3)


def run_multires_step(pf, n=256, steps=5, warmup=2, cpu_n=48, cpu=True, seed=0):
    """The 2-level multires step (pf_mr_step, the reference's MRSim3DTP::step)
    on the dam break at n^3 fine cells: a water column beside a pool, eight
    particles per water cell, 1000:1, dt 1/480, a static layout refined where
    water and empty cells lie within 3 cells of each other, the reference's
    default pressure solve (Jacobi PCG with adaptive restart, 160 iterations,
    tolerance max(1e-7, 1e-6 max|r0|)).  Device-timed particles/s and the
    stage times; beside it the reference's own MRSim3DTP::step on the same
    scene and layout rule at cpu_n^3 on one host core."""
    import torch
    sim = pf.MRSim3DTP(n, n, n, 1.0 / n, max_particles=8 * n ** 3 // 2)
    sim.phase = pf.PhaseParams(1000.0, 1.0)
    sim.phase.rho_tilde_0 = pf.calibrateRhoTilde0(sim.phase, 1.0, sim.grid)
    sim.dt = 1.0 / 480.0
    sim.dynamic_refinement = False
    npart = sim.seed_scene("dam_break", seed)
    levels = mr_dam_break_layout(pf, n)
    sim.set_levels(levels)
    lib = pf.load()
    stream = torch.cuda.ExternalStream(lib.pf_stream(sim.ctx))
    for _ in range(warmup):
        sim.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters, conv, cells = 0, 0, 0
    e0.record(stream)
    for _ in range(steps):
        st = sim.step()
        iters += st.iterations
        conv += st.converged
        cells = st.active_cells
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # stage times over two more steps, outside the timed region
    lib.pf_set_timing(sim.ctx, 1)
    tm = pf._lib.Timing()
    lib.pf_get_timing(sim.ctx, C.byref(tm), 1)
    for _ in range(2):
        last = sim.step()
    lib.pf_get_timing(sim.ctx, C.byref(tm), 1)
    lib.pf_set_timing(sim.ctx, 0)
    stages = {k: v[0] / 2 for k, v in tm.as_dict().items() if v[1]}
    fine_blocks = int(levels.sum())
    out = {"workload": f"dam_break_{n} multires: {npart} particles, 2 levels ({fine_blocks} of {levels.size} "
                       f"8^3 blocks fine), 1000:1, dt 1/480, MRSim3DTP default PCG, {warmup} warm-up + {steps} "
                       f"timed steps",
           "particles_per_s": npart / (ms / 1000.0), "ms_per_step": ms, "unknowns": cells,
           "pcg_iterations_per_step": iters / steps, "converged_steps": conv,
           "final_relative_residual": last.final_residual / max(last.initial_residual, 1e-300),
           "stages_ms_per_step": stages}
    sim.close()
    if cpu:
        from oracle.multires import MRSettings, ReferenceMR
        import oracle as O
        sc = pf.scenes.dam_break(cpu_n, seed=seed)
        ph = O.PhaseParams(1000.0, 1.0)
        ph.rho_tilde_0 = O.Oracle().calibrate_rho_tilde0(ph, 1.0)
        r = ReferenceMR(cpu_n, cpu_n, cpu_n, 1.0 / cpu_n,
                        MRSettings(dt=1.0 / 480.0, phase=ph, dynamic_refinement=False))
        lv = mr_dam_break_layout(pf, cpu_n)
        r.set_layout([(8 * bx, 8 * by, 8 * bz, 8 * bx + 8, 8 * by + 8, 8 * bz + 8)
                      for bz, by, bx in zip(*np.nonzero(lv))])
        r.set_particles(sc["pos"].astype(np.float64), sc["vel"].astype(np.float64), sc["type"])
        r.step()  # warm-up
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            r.step()
            times.append(time.perf_counter() - t0)
        mean = sum(times) / len(times)
        out["cpu_reference"] = {"particles_per_s": len(sc["pos"]) / mean, "s_per_step": mean, "cores": 1,
                                "sample": f"the reference's MRSim3DTP::step on the dam break at {cpu_n}^3 "
                                          f"({len(sc['pos'])} particles, same layout rule), 1 warm-up + 2 timed "
                                          f"steps"}
        out["speedup_vs_cpu_reference"] = out["particles_per_s"] / out["cpu_reference"]["particles_per_s"]
    return out


def run_pressure_cpu(pf, n=48, seed=0):
    """The reference's own projection (spProjectStepVC3D from oracle/_ref, the
    unmodified sources; single-threaded) on the pressure system of the first
    Rayleigh-Taylor step at n^3 (1000:1, dt 1/240: markCells, P2G, gravity
    and walls by the oracle), timed on the host beside the GPU's PLAIN and
    learned solves of the same system.  The reference stops on an absolute
    max-norm tolerance, set to 1e-6 max|r0| of this system: the relative rule
    the GPU solves use."""
    import oracle as O
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    opp = O.PhaseParams(sc["rho_l"], sc["rho_g"])
    opp.rho_tilde_0 = pp.rho_tilde_0 = O.Oracle().calibrate_rho_tilde0(opp, 1.0)
    ps = O.Particles(sc["pos"].astype(np.float64), sc["vel"].astype(np.float64), sc["type"],
                     sc["volume"].astype(np.float64))
    o = O.Oracle()
    go = O.OracleGrid(n, n, n, sc["dx"])
    o.mark_cells(go, ps)
    o.p2g(go, ps, opp, 1.0)
    o.apply_gravity(go, 1.0 / 240.0, -9.81)
    o.apply_wall_boundary(go)
    fields = [go.get_field(f) for f in range(8)]
    out = {"workload": f"rayleigh_taylor_{n} first-step pressure system: 1000:1, dt 1/240, to 1e-6 relative"}
    g = pf.SparseMacGrid3D(n, n, n, sc["dx"], max_particles=1)
    gpu_p = {}
    for name, cfg in (("plain", pf.SolverConfig(rel_tol=1e-6)),
                      ("learned", pf.SolverConfig(mode=pf.PF_SOLVER_LEARNED, rel_tol=1e-6,
                                                  precond=pf.PF_PRECOND_NETWORK))):
        if name == "learned":
            load_weights(pf, g)
        for f in range(8):
            g.set_field(f, *fields[f])
        st = pf.spProjectStepVC3D(g, pp, 1.0 / 240.0, 20000, 0.0, solver=cfg)
        gpu_p[name] = g.get_field(pf.PF_P)[0].astype(np.float64)
        out[f"gpu_{name}"] = {"ms": st.solve_ms, "iterations": st.iterations, "converged": bool(st.converged)}
        res0 = st.res0
    g.close()
    rg = O.ReferenceGrid(n, n, n, sc["dx"])
    for f in range(8):
        rg.set_field(f, *fields[f])
    t0 = time.perf_counter()
    O.Reference().project(rg, opp, 1.0 / 240.0, 20000, 1e-6 * res0)
    ref_ms = 1000.0 * (time.perf_counter() - t0)
    p_ref = rg.get_field(O.P)[0].astype(np.float64)
    scale = max(np.abs(p_ref).max(), 1e-300)
    out["reference"] = {"ms": ref_ms, "cores": 1, "abs_tol": 1e-6 * res0, "kind": "reference"}
    for name in gpu_p:
        out[f"gpu_{name}"]["speedup_vs_reference"] = ref_ms / max(out[f"gpu_{name}"]["ms"], 1e-9)
        out[f"gpu_{name}"]["p_rel_diff_vs_reference"] = float(np.abs(gpu_p[name] - p_ref).max() / scale)
    return out


def run_adapt(pf, n=128, seed=0, reps=5, cpu=True):
    """Particle adaptivity (src/driver/particle_adaptivity3d.h) on the
    Rayleigh-Taylor scene: each operation on the full particle set, device time
    (CUDA events on the library stream) per call over `reps` calls, each call on
    a freshly uploaded copy (upload untimed).  The reference's own pa3d
    functions (oracle/_ref, single-threaded) run once on the same particles.
    Operations: narrow band r = 2, gas coarsening to 4, liquid coarsening to 4,
    liquid refill to 10 per cell (every liquid cell gains two)."""
    import torch
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    npart = len(sc["pos"])
    L = pf._lib
    ops = [
        ("narrow_band_air", L.BandStats, lambda lib, h, st: lib.pf_narrow_band_air(h, 2, C.byref(st)),
         lambda lib, h, out: lib.pfr_narrow_band_air(h, 2, out), 4),
        ("gas_coarsening", L.CoarsenStats,
         lambda lib, h, st: lib.pf_coarsen_particles(h, 1, 4, 0x9e3779b9, C.byref(st)),
         lambda lib, h, out: lib.pfr_coarsen_particles(h, 1, 4, 0x9e3779b9, out), 5),
        ("liquid_coarsening", L.CoarsenStats,
         lambda lib, h, st: lib.pf_coarsen_particles(h, 0, 4, 0x7f4a7c15, C.byref(st)),
         lambda lib, h, out: lib.pfr_coarsen_particles(h, 0, 4, 0x7f4a7c15, out), 5),
        ("liquid_refill", L.RefillStats,
         lambda lib, h, st: lib.pf_refill_liquid(h, 10, 0x6a09e667, 0, 1, 0, C.byref(st)),
         lambda lib, h, out: lib.pfr_refill_liquid(h, 10, 0x6a09e667, 0, 1, 0, out), 7),
    ]
    g = pf.SparseMacGrid3D(n, n, n, sc["dx"], max_particles=int(npart * 1.3))
    lib = g.lib
    stream = torch.cuda.ExternalStream(lib.pf_stream(g.ctx))
    arrays = [np.ascontiguousarray(sc[k], dt) for k, dt in (("pos", np.float32), ("vel", np.float32),
                                                             ("type", np.uint8), ("volume", np.float32))]
    out = {"workload": f"rayleigh_taylor_{n}: {npart} particles, each operation on the full set, "
                       f"{reps} device-timed calls", "unit": "particles/s", "ops": {}}
    for name, Stats, call, _, _ in ops:
        ms = []
        st = Stats()
        for _ in range(reps + 1):  # the first call allocates the scratch: untimed
            L.check(lib.pf_upload_particles(g.ctx, npart, *[a.ctypes.data for a in arrays]), g.ctx, "upload")
            lib.pf_sync(g.ctx)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.check(call(lib, g.ctx, st), g.ctx, name)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = statistics.median(ms[1:])
        out["ops"][name] = {"gpu_ms": t, "particles_per_s": npart / (t / 1000.0), "stats": list(st.as_tuple())}
    g.close()
    if cpu:
        import oracle as O
        ps = O.Particles(sc["pos"].astype(np.float64), sc["vel"].astype(np.float64), sc["type"],
                         sc["volume"].astype(np.float64))
        rg = O.ReferenceGrid(n, n, n, sc["dx"])
        for name, _, _, rcall, nst in ops:
            rg._put(ps)
            res = np.zeros(nst, np.int32)
            t0 = time.perf_counter()
            rcall(rg.lib, rg.h, res)
            t1 = time.perf_counter()
            rec = out["ops"][name]
            rec["cpu_reference_ms"] = 1000.0 * (t1 - t0)
            rec["speedup_vs_reference"] = rec["cpu_reference_ms"] / rec["gpu_ms"]
            rec["reference_stats_equal"] = [int(v) for v in res] == rec["stats"]
        out["cpu_cores"] = 1
        out["host"] = host_info()
    return out


# solvers of the whole-step pressure systems: PLAIN, the learned two-level
# preconditioner, and the same with an exact coarse solve (the bound a perfect
# network reaches)
STEP_MODES = ["plain_fp64", "learned", "exact_coarse"]


def run_ours(args, rank, world, local, dist):
    import torch
    pf = load_pkg()
    torch.cuda.set_device(local)
    sc = pf.scenes.bubble_tank(args.n, seed=args.seed + rank, level=args.bubble_level)
    ts = TransferStep(pf, sc, local)
    n = ts.n
    # device-resident timing with per-stage events
    for _ in range(args.warmup):
        ts.step()
    torch.cuda.synchronize(local)
    ts.lib.pf_set_timing(ts.ctx, 1)
    tm = pf._lib.Timing()
    ts.lib.pf_get_timing(ts.ctx, C.byref(tm), 1)
    with ClockSampler(local) as clk:
        ms, launches = time_steps(ts, args.steps, 0, dist, local)
        ts.lib.pf_get_timing(ts.ctx, C.byref(tm), 1)
        stages = tm.as_dict()
        ts.lib.pf_set_timing(ts.ctx, 0)
        # end-to-end from pinned host buffers
        ms_e2e, _ = time_steps(ts, args.steps, max(1, args.warmup // 2), dist, local, e2e=True)
    n_faces = ts.active_faces()
    clk_mhz = clk.summary()["sm_mhz"] or 1965.0

    value = whole_job_rate(n, args.steps, world, ms)
    e2e_value = whole_job_rate(n, args.steps, world, ms_e2e)
    peak, peak_kind = measured_hbm()
    # dominant kernel of the step by device time
    splat_ms = stages["splat"][0] / max(stages["splat"][1], 1)
    g2p_ms = stages["g2p"][0] / max(stages["g2p"][1], 1)
    if splat_ms >= g2p_ms:
        kname, kms = "k_splat (P2G)", splat_ms
        kbytes = P2G_BYTES_PER_PARTICLE * n + P2G_BYTES_PER_FACE * n_faces
    else:
        kname, kms = "k_g2p (G2P)", g2p_ms
        kbytes = G2P_BYTES_PER_PARTICLE * n + G2P_BYTES_PER_FACE * n_faces
    achieved = kbytes / (kms / 1000.0) / 1e9
    # DRAM bytes per launch of the roofline kernel from an ncu capture
    # (profiles/traffic.json), valid for the 128^3 workload it was scaled to
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and args.n == 128:
        try:
            with open(tpath) as f:
                rec = json.load(f)
            if rec.get("kernel") == kname.split()[0] and rec.get("scaled_to_particles") == n:
                traffic = rec["bytes_per_launch"]
        except (OSError, ValueError, KeyError):
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded bubble tank scene)",
        "config": {"workload": f"bubble_tank_{args.n} transfer stress: P2G(u,v,w,raw mass)+G2P, FLIP 0.97"
                               + ("" if args.bubble_level == 0.7 else f", water level {args.bubble_level}"),
                   "grid": [args.n] * 3, "tile": 8, "particles_per_gpu": n, "global_particles": n * world,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (particle SoA %.0f MB per GPU)" % (n * 29 / 1e6)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * 29, "d2h_bytes_per_step": n * 12},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": kbytes, "mean_launch_ms": kms},
        # the splat's true bound: warp-instruction issue (HBM bytes are a few percent of the peak)
        "issue_roofline": issue_roofline(n, splat_ms, clk_mhz),
        "stages_ms_per_step": {k: v[0] / max(args.steps, 1) for k, v in stages.items() if v[1]},
        "gpu_launches": int(launches) * world,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_extras:
        line["pcg"] = run_pcg(pf, args.pcg_n, pcg_modes(pf, args.pcg_modes.split(",")), max_iter=args.pcg_max_iter)
        line["pcg_fp64_oracle"] = run_pcg(pf, 64, pcg_modes(pf, args.pcg_modes.split(",")),
                                          max_iter=args.pcg_max_iter, fp64_oracle=True)
        line["step_pcg"] = [run_step_pcg(pf, name, int(sz), pcg_modes(pf, STEP_MODES), max_iter=args.pcg_max_iter)
                            for name, sz in (item.split(":") for item in args.step_pcg_default.split(","))]
        line["full_step"] = run_full_step(pf, n=args.full_step_n, steps=args.full_step_steps,
                                          solvers=("plain", "learned"))
        line["adaptivity"] = run_adapt(pf, n=args.adapt_n, cpu=not args.no_cpu_baseline)
        line["multires_step"] = run_multires_step(pf, n=args.mr_n, steps=args.mr_steps, cpu=not args.no_cpu_baseline)
        if not args.no_cpu_baseline:
            line["pressure_cpu_baseline"] = run_pressure_cpu(pf)
    if rank == 0 and not args.no_cpu_baseline:
        host = host_info()
        # the reference's P2G runs its 8 colour threads (runColor8), G2P one
        cores = min(8, host["affinity_cpus"] or 1)
        np_s, times = cpu_reference_sample(sc, slab_cells=args.cpu_slab, steps=args.cpu_steps, warmup=1)
        mean = sum(times) / len(times)
        line["cpu_baseline"] = {"value": np_s / mean, "unit": UNIT, "cores": cores, "kind": "reference",
                                "host": host,
                                "sample": f"reference spP2G3D_tp + saved copy + spG2P3D_tp on the {np_s} particles "
                                          f"of the first {args.cpu_slab} x-columns of the 128^3 scene, 1 warm-up "
                                          f"+ {len(times)} timed steps ({mean:.2f} s each); P2G on up to 8 colour "
                                          f"threads, G2P on one"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    pf = load_pkg()
    sc = pf.scenes.bubble_tank(args.n, seed=args.seed)
    np_s, times = cpu_reference_sample(sc, slab_cells=args.cpu_slab, steps=args.steps, warmup=args.warmup)
    total = sum(times)
    value = np_s * len(times) / total
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / len(times), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded bubble tank scene)", "impl": "reference",
        "config": {"workload": f"bubble_tank_{args.n} transfer stress: P2G(u,v,w,raw mass)+G2P, FLIP 0.97"
                               + ("" if args.bubble_level == 0.7 else f", water level {args.bubble_level}"),
                   "grid": [args.n] * 3, "sample_particles": np_s},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": min(8, host_info()["affinity_cpus"] or 1),
                         "kind": "reference", "host": host_info(),
                         "sample": f"{np_s} particles (first {args.cpu_slab} x-columns) per step; P2G on up to 8 "
                                   f"colour threads, G2P on one"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n", type=int, default=128, help="grid cells per axis (128 is the benchmarked workload)")
    ap.add_argument("--bubble-level", type=float, default=0.7,
                    help="water level of the transfer scene (0.7 is the benchmarked workload; lower levels give "
                         "smaller cases of the same kernels for profiling)")
    ap.add_argument("--cpu-slab", type=int, default=4, help="x-columns of the scene in the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the PCG, full-step and adaptivity blocks")
    ap.add_argument("--pcg-n", type=int, default=256, help="grid of the pressure-only block")
    ap.add_argument("--pcg-only", action="store_true", help="run only the pressure-only block")
    ap.add_argument("--pcg-max-iter", type=int, default=60000, help="iteration cap of the pressure blocks")
    ap.add_argument("--pcg-modes", default="plain_fp64,learned,flex_jacobi,mixed_fp32,mixed_bf16,learned_mixed",
                    help="solvers of the pressure-only block (plain_fp64 first): plain_fp64, learned, "
                         "flex_jacobi, exact_coarse, mixed_fp32, mixed_bf16, mixed_bf16_dir, learned_mixed "
                         "(name@M:ETA sets an inner-outer mode's inner cap and reduction)")
    ap.add_argument("--step-pcg-default", default="rt:256,bubble:128",
                    help="whole-step pressure systems of the default run (plain, learned, exact coarse)")
    ap.add_argument("--cpu-steps", type=int, default=2, help="timed steps of the CPU reference sample")
    ap.add_argument("--step-pcg", default="",
                    help="run only whole-step pressure systems, e.g. rt:256,bubble:128 (modes from --pcg-modes)")
    ap.add_argument("--step-pcg-pre", type=int, default=1, help="plain steps before the step-pressure snapshot")
    ap.add_argument("--weights", default="", help="network weights for the learned mode (default: shipped)")
    ap.add_argument("--full-step-n", type=int, default=256, help="grid of the full-step block (Rayleigh-Taylor)")
    ap.add_argument("--full-step-steps", type=int, default=5, help="timed steps of the full-step block")
    ap.add_argument("--full-step-only", action="store_true", help="run only the full-step block")
    ap.add_argument("--adapt-n", type=int, default=128, help="grid of the particle-adaptivity block")
    ap.add_argument("--adapt-only", action="store_true", help="run only the particle-adaptivity block")
    ap.add_argument("--mr-n", type=int, default=256, help="fine grid of the multires block (dam break)")
    ap.add_argument("--mr-steps", type=int, default=5, help="timed steps of the multires block")
    ap.add_argument("--mr-only", action="store_true", help="run only the multires block")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, rank, world)
        return
    if args.adapt_only:  # the particle-adaptivity block alone
        pf = load_pkg()
        print(json.dumps(run_adapt(pf, n=args.adapt_n, cpu=not args.no_cpu_baseline)), flush=True)
        return
    if args.mr_only:  # the multires block alone
        pf = load_pkg()
        print(json.dumps(run_multires_step(pf, n=args.mr_n, steps=args.mr_steps, cpu=not args.no_cpu_baseline)),
              flush=True)
        return
    if args.full_step_only:  # the full-step block alone
        pf = load_pkg()
        print(json.dumps(run_full_step(pf, n=args.full_step_n, steps=args.full_step_steps,
                                       solvers=("plain", "learned"))), flush=True)
        return
    if args.step_pcg:  # whole-step pressure systems alone
        pf = load_pkg()
        modes = pcg_modes(pf, args.pcg_modes.split(","))
        for item in args.step_pcg.split(","):
            name, n = item.split(":")
            print(json.dumps(run_step_pcg(pf, name, int(n), modes, pre_steps=args.step_pcg_pre,
                                          max_iter=args.pcg_max_iter, weights_path=args.weights or None)),
                  flush=True)
        return
    if args.pcg_only:  # the pressure-only block alone (profiling)
        pf = load_pkg()
        print(json.dumps(run_pcg(pf, args.pcg_n, pcg_modes(pf, args.pcg_modes.split(",")),
                                 max_iter=args.pcg_max_iter, weights_path=args.weights or None)), flush=True)
        return
    rank, world, local, dist = dist_setup(args.gpus)
    try:
        run_ours(args, rank, world, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
