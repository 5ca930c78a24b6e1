"""The learned coarse solve of the LEARNED pressure mode (libpfgpu's pf_learned_*).

The reference's sparse path has no learned solver; its flexible PCG with a
guarded, auto-disabling coarse preconditioner
(src/pressure/multires_pressure3d.cpp:1301-1447) is the pattern the LEARNED
mode follows.  A ``LearnedCoarseSolver`` is bound to one SparseMacGrid3D (one
device context): it initialises or loads the network, harvests training pairs
from EXACT_COARSE solves on that grid, trains on the device, and exposes the
network on caller-given coarse systems for tests.

    net = LearnedCoarseSolver(grid)
    net.init(seed=0)
    net.harvest(True)
    spProjectStepVC3D(grid, pp, dt, it, 0.0, solver=SolverConfig(mode=PF_SOLVER_LEARNED,
                                                                  precond=PF_PRECOND_EXACT_COARSE, rel_tol=1e-6))
    net.harvest(False)
    net.train(steps=400, batch=8, lr=1e-3)
    spProjectStepVC3D(grid, pp, dt, it, 0.0, solver=SolverConfig(mode=PF_SOLVER_LEARNED, rel_tol=1e-6))
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L

COP_STRIDE = 17
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "coarse_net.npy")


def num_params() -> int:
    return int(L.load().pf_learned_num_params())


class LearnedCoarseSolver:
    def __init__(self, grid):
        self.grid = grid
        self.lib = L.load()

    @property
    def ctx(self):
        return self.grid.ctx

    def _check(self, rc, what):
        L.check(rc, self.ctx, what)

    def init(self, seed: int = 0):
        self._check(self.lib.pf_learned_init(self.ctx, C.c_ulonglong(seed)), "pf_learned_init")

    def load(self, params):
        p = np.ascontiguousarray(params, np.float32).ravel()
        self._check(self.lib.pf_learned_load(self.ctx, p.ctypes.data, p.size), "pf_learned_load")

    def params(self) -> np.ndarray:
        out = np.empty(num_params(), np.float32)
        self._check(self.lib.pf_learned_params(self.ctx, out.ctypes.data, out.size), "pf_learned_params")
        return out

    def save(self, path):
        np.save(path, self.params())

    def load_file(self, path):
        self.load(np.load(path))

    def load_default(self) -> str:
        """Load the weights shipped with the package (written by
        train_coarse_net.py); returns their path."""
        if not os.path.exists(DEFAULT_WEIGHTS):
            raise FileNotFoundError(f"no trained weights at {DEFAULT_WEIGHTS}: run train_coarse_net.py")
        self.load_file(DEFAULT_WEIGHTS)
        return os.path.relpath(DEFAULT_WEIGHTS, os.path.dirname(os.path.dirname(DEFAULT_WEIGHTS)))

    def harvest(self, enable: bool, stride: int = 1, max_per_system: int = 64, capacity_floats: int = 1 << 26):
        self._check(self.lib.pf_learned_harvest(self.ctx, int(bool(enable)), int(stride), int(max_per_system),
                                                int(capacity_floats)), "pf_learned_harvest")

    def dataset(self):
        s, p = C.c_int(), C.c_int()
        self._check(self.lib.pf_learned_dataset(self.ctx, C.byref(s), C.byref(p)), "pf_learned_dataset")
        return s.value, p.value

    def clear_dataset(self):
        self._check(self.lib.pf_learned_clear_dataset(self.ctx), "pf_learned_clear_dataset")

    def merge_dataset(self, other: "LearnedCoarseSolver"):
        """Append the training pairs harvested on another grid (same device)."""
        self._check(self.lib.pf_learned_merge_dataset(self.ctx, other.ctx), "pf_learned_merge_dataset")

    def train(self, steps: int, batch: int = 8, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(int(steps), 1), np.float64)
        self._check(self.lib.pf_learned_train(self.ctx, int(steps), int(batch), float(lr), C.c_ulonglong(seed),
                                              losses.ctypes.data), "pf_learned_train")
        return losses[:steps]

    def eval(self, dims, cop, rc, target=None):
        """e = net(rc) on a coarse system (dims = (X, Y, Z)); with a target also (loss, grad)."""
        X, Y, Z = (int(v) for v in dims)
        nt = X * Y * Z
        cop = np.ascontiguousarray(cop, np.float32).reshape(nt, COP_STRIDE)
        rc = np.ascontiguousarray(rc, np.float32).reshape(-1, nt, 2)
        B = rc.shape[0]
        e = np.empty((B, nt, 2), np.float32)
        loss = C.c_double(0.0)
        if target is None:
            self._check(self.lib.pf_learned_eval(self.ctx, X, Y, Z, cop.ctypes.data, rc.ctypes.data, None, B,
                                                 e.ctypes.data, None, None), "pf_learned_eval")
            return e
        tg = np.ascontiguousarray(target, np.float32).reshape(B, nt, 2)
        grad = np.empty(num_params(), np.float32)
        self._check(self.lib.pf_learned_eval(self.ctx, X, Y, Z, cop.ctypes.data, rc.ctypes.data, tg.ctypes.data,
                                             B, e.ctypes.data, C.byref(loss), grad.ctypes.data), "pf_learned_eval")
        return e, loss.value, grad

    def adam(self, grad, lr: float):
        g = np.ascontiguousarray(grad, np.float32).ravel()
        self._check(self.lib.pf_learned_adam(self.ctx, g.ctypes.data, g.size, float(lr)), "pf_learned_adam")
