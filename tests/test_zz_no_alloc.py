"""pf_project_noalloc: the projection for callers that may not allocate.

Some hosts keep the whole device budget to themselves and hand out buffers from
their own allocator, or run loops that must never wait on cudaMalloc; they call
pf_project_noalloc with their own dense device buffers, and the library works
entirely inside a fixed array it carries (no allocation at all).  This file
checks, through the C ABI, that two calls in a row give the same pressure and
projected velocities as the pooled entry point pf_project on the same inputs,
that calls after the first leave the device's free memory unchanged, that a
call after a device reset (in a child process) still finds its array, and
that a grid beyond the array's capacity is refused.  It is collected last so a
run that stops at the first failure has already run every other test.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from gpu_helpers import phase_for, rel_err, scene_particles, to_oracle_phase

pytestmark = pytest.mark.gpu

TOL = 1e-5  # field-scale relative tolerance of the parity tests


def _dense_inputs(pf, n, seed):
    """Markers, face masses and face velocities of a Rayleigh-Taylor scene
    after markCells, P2G, gravity and walls (computed by the CPU oracle)."""
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    rng = np.random.default_rng(seed)
    sc["vel"] = rng.normal(0, 0.3, sc["pos"].shape).astype(np.float32)
    pp = phase_for(sc, pf)
    ps = scene_particles(sc)
    o = O.Oracle()
    go = O.OracleGrid(n, n, n, 1.0 / n)
    o.mark_cells(go, ps)
    o.p2g(go, ps, to_oracle_phase(pp), 1.0)
    o.apply_gravity(go, 1 / 240, -9.81)
    o.apply_wall_boundary(go)
    return {name: go.get_field(f)[0] for f, name in enumerate(O.FIELD_NAMES)}, pp


def _with_pf_project(pf, n, fields, pp, dt, iters, rel):
    g = pf.SparseMacGrid3D(n, n, n, 1.0 / n)
    for f, name in enumerate(O.FIELD_NAMES):
        g.set_field(f, fields[name], np.ones(g.bdims(f)[::-1], np.uint8))
    st = pf.spProjectStepVC3D(g, pp, dt, iters, 0.0, solver=pf.SolverConfig(rel_tol=rel))
    return {k: g.get_field(f)[0] for k, f in (("p", pf.PF_P), ("u", pf.PF_U), ("v", pf.PF_V), ("w", pf.PF_W))}, st


def _with_noalloc(pf, n, fields, pp, dt, iters, rel):
    import torch
    lib = pf.load()
    dev = {k: torch.from_numpy(np.ascontiguousarray(fields[k], np.float32)).cuda()
           for k in ("mk", "mu", "mv", "mw", "u", "v", "w")}
    p = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    st = pf._lib.SolveStats()
    torch.cuda.synchronize()
    rc = lib.pf_project_noalloc(n, n, n, 1.0 / n, dev["mk"].data_ptr(), dev["mu"].data_ptr(), dev["mv"].data_ptr(),
                                dev["mw"].data_ptr(), dev["u"].data_ptr(), dev["v"].data_ptr(), dev["w"].data_ptr(),
                                p.data_ptr(), C.byref(pp._c()), dt, iters, 0.0, rel, 0.0, C.byref(st), None)
    assert rc == 0, rc
    return {"p": p.cpu().numpy(), "u": dev["u"].cpu().numpy(), "v": dev["v"].cpu().numpy(),
            "w": dev["w"].cpu().numpy()}, st


def test_noalloc_projection_matches_pf_project_on_two_calls_in_a_row(pf):
    dt, iters, rel = 1 / 240, 3000, 1e-10
    for n, seed in ((24, 3), (32, 8)):  # two calls, different grids and data
        fields, pp = _dense_inputs(pf, n, seed)
        ref, st_ref = _with_pf_project(pf, n, fields, pp, dt, iters, rel)
        got, st = _with_noalloc(pf, n, fields, pp, dt, iters, rel)
        assert st.converged and st_ref.converged
        assert st.n_cells == st_ref.n_cells and st.pin_cell == st_ref.pin_cell
        assert abs(st.iterations - st_ref.iterations) <= 3
        for k in ("p", "u", "v", "w"):
            assert rel_err(got[k], ref[k]) < TOL, (n, k, rel_err(got[k], ref[k]))


def test_noalloc_refuses_grids_beyond_its_capacity(pf):
    import torch
    lib = pf.load()
    buf = torch.zeros(8, dtype=torch.float32, device="cuda")
    ptr = buf.data_ptr()
    st = pf._lib.SolveStats()
    rc = lib.pf_project_noalloc(40, 40, 40, 1.0 / 40, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr,
                                C.byref(pf.PhaseParams()._c()), 0.01, 10, 1e-7, 0.0, 0.0, C.byref(st), None)
    assert rc == pf._lib.PF_ERR_INVALID


def test_noalloc_calls_after_the_first_allocate_nothing(pf):
    """The first call in a context may load the library's module (and with it
    the fixed array); the calls after it must not change the device's free
    memory."""
    import torch
    n = 24
    fields, pp = _dense_inputs(pf, n, 5)
    lib = pf.load()
    dev = {k: torch.from_numpy(np.ascontiguousarray(fields[k], np.float32)).cuda()
           for k in ("mk", "mu", "mv", "mw", "u", "v", "w")}
    p = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    st = pf._lib.SolveStats()

    def call():
        rc = lib.pf_project_noalloc(n, n, n, 1.0 / n, dev["mk"].data_ptr(), dev["mu"].data_ptr(),
                                    dev["mv"].data_ptr(), dev["mw"].data_ptr(), dev["u"].data_ptr(),
                                    dev["v"].data_ptr(), dev["w"].data_ptr(), p.data_ptr(), C.byref(pp._c()),
                                    1 / 240, 500, 0.0, 1e-6, 0.0, C.byref(st), None)
        assert rc == 0, rc

    torch.cuda.synchronize()
    call()
    free = [torch.cuda.mem_get_info()[0]]
    for _ in range(2):
        call()
        free.append(torch.cuda.mem_get_info()[0])
    assert free[1] == free[0] and free[2] == free[0], free


_RESET_CHILD = r"""
import ctypes as C, importlib.util, os, sys
import numpy as np
root = sys.argv[1]
spec = importlib.util.spec_from_file_location("adaptive_pf_flip_b200", os.path.join(root, "adaptive-pf-flip_b200", "__init__.py"),
                                              submodule_search_locations=[os.path.join(root, "adaptive-pf-flip_b200")])
pf = importlib.util.module_from_spec(spec); sys.modules[spec.name] = pf; spec.loader.exec_module(pf)
lib = pf.load()
rt = C.CDLL("libcudart.so.12")
n = 16
mk = np.zeros((n, n, n), np.float32); mk[[0, -1], :, :] = 2; mk[:, [0, -1], :] = 2; mk[:, :, [0, -1]] = 2
mk[2:12, 2:10, 2:12] = 1
host = {"mk": mk, "mu": np.ones((n, n, n + 1), np.float32), "mv": np.ones((n, n + 1, n), np.float32),
        "mw": np.ones((n + 1, n, n), np.float32)}
rng = np.random.default_rng(0)
for k, shape in (("u", (n, n, n + 1)), ("v", (n, n + 1, n)), ("w", (n + 1, n, n))):
    host[k] = rng.normal(0, 1, shape).astype(np.float32)
host["p"] = np.zeros((n, n, n), np.float32)

def run():
    ptr = {}
    for k, a in host.items():
        d = C.c_void_p()
        assert rt.cudaMalloc(C.byref(d), C.c_size_t(a.nbytes)) == 0
        assert rt.cudaMemcpy(d, a.ctypes.data, C.c_size_t(a.nbytes), 1) == 0
        ptr[k] = d.value
    st = pf._lib.SolveStats()
    rc = lib.pf_project_noalloc(n, n, n, 1.0 / n, ptr["mk"], ptr["mu"], ptr["mv"], ptr["mw"], ptr["u"], ptr["v"],
                                ptr["w"], ptr["p"], C.byref(pf.PhaseParams()._c()), 0.01, 400, 0.0, 1e-8, 0.0,
                                C.byref(st), None)
    assert rc == 0 and st.converged, (rc, st.converged)
    out = {}
    for k in ("p", "u", "v", "w"):
        a = np.empty_like(host[k])
        assert rt.cudaMemcpy(a.ctypes.data, C.c_void_p(ptr[k]), C.c_size_t(a.nbytes), 2) == 0
        out[k] = a
    for d in ptr.values():
        rt.cudaFree(C.c_void_p(d))
    return out

a = run()
assert rt.cudaDeviceReset() == 0
b = run()
for k in a:
    assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
print("reset ok")
"""


def test_noalloc_finds_its_array_after_a_device_reset(pf):
    """A host that resets the device (or brings its own context) between two
    calls: the array's address is looked up in the live context on every call,
    so the second call runs and gives the first call's result bit for bit.
    Runs in a child process, whose context alone the reset ends."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _RESET_CHILD, root], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and "reset ok" in out.stdout, out.stdout + out.stderr
