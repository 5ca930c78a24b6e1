"""Helpers shared by the GPU parity tests: run the same seeded inputs through
libpfgpu and through the CPU oracle, and compare."""
import numpy as np

import oracle as O

FIELDS = ("u", "v", "w", "mu", "mv", "mw", "p", "mk")


def rel_err(a, b):
    """max|a-b| / max|b| (field-scale relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    d = float(np.max(np.abs(a - b))) if b.size else 0.0
    if scale == 0.0:
        return d
    return d / scale


def scene_particles(sc):
    """FP32 scene arrays -> oracle Particles (FP64, exact conversion)."""
    return O.Particles(sc["pos"].astype(np.float64), sc["vel"].astype(np.float64), sc["type"],
                       sc["volume"].astype(np.float64))


def phase_for(sc, pf, oracle_impl=None):
    pp = pf.PhaseParams(sc["rho_l"], sc["rho_g"], 1.0, 1.0)
    pp.rho_tilde_0 = pf.calibrateRhoTilde0(pp, 1.0)
    return pp


def to_oracle_phase(pp):
    return O.PhaseParams(pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0)


def compare_grids(g_gpu, g_cpu, fields=range(8)):
    """Per field: (relative value error, number of differing 4^3 activity flags)."""
    out = {}
    for f in fields:
        dg, ag = g_gpu.get_field(f)
        dc, ac = g_cpu.get_field(f)
        out[FIELDS[f]] = (rel_err(dg, dc), int((ag != ac).sum()))
    return out


def copy_grid_to_oracle(g_gpu, g_cpu, fields=range(8)):
    for f in fields:
        d, a = g_gpu.get_field(f)
        g_cpu.set_field(f, d, a)
