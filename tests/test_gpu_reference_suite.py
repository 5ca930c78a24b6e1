"""The reference's own doctest cases for this path, run against the GPU drop-in.

oracle/_ref/ref_tests_gpu is the reference's tests/test_sparse_transfer3d_tp.cpp,
tests/test_sparse_vc3d.cpp and tests/test_sparse_sim3d_tp.cpp compiled unmodified,
with adaptive-pf-flip_b200/shim/sparse_ops3d_tp_gpu.cpp in place of the
reference's src/driver/sparse_ops3d_tp.cpp, so spP2G3D_tp, spProjectStepVC3D,
spG2P3D_tp and spAdvect3D_tp (also inside SparseSim3DTP::step()) run on the GPU
through the C ABI.  adaptive-pf-flip_b200/shim/driver/particle_adaptivity3d.h
shadows the reference's header of that name, so the step's particle
adaptivity (the narrow-band, coarsening and refill cases of
test_sparse_sim3d_tp.cpp) runs on the GPU too.  The binary is built by `make -C oracle ref_tests` where the
reference tree exists and travels prebuilt.
"""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "ref_tests_gpu")


@pytest.mark.skipif(not os.path.exists(BIN), reason="oracle/_ref/ref_tests_gpu not built")
def test_reference_doctest_suite_passes_on_gpu_dropin():
    out = subprocess.run([BIN, "--no-colors"], capture_output=True, text=True, timeout=1200)
    tail = "\n".join((out.stdout + out.stderr).splitlines()[-25:])
    assert out.returncode == 0, tail
    assert "Status: SUCCESS" in out.stdout, tail
