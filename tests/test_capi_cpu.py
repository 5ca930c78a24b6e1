"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/pfgpu.h declares, and the ctypes mirrors of its structs have the
sizes and field offsets a C compiler gives them."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pfgpu.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"PFGPU_API\s+[\w\s\*]+?\b(pf_\w+)\s*\(", txt)))


def test_header_declares_the_mirrored_exports(pf):
    names = declared_functions()
    assert len(names) >= 30
    assert sorted(pf._lib.EXPORTS) == names


def test_library_exports_every_declared_symbol(pf):
    lib = pf.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", pf._lib.LIB_PATH], capture_output=True, text=True)
    exported = set(re.findall(r" T (pf_\w+)", out.stdout))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_c(pf, tmp_path):
    L = pf._lib
    structs = {"pf_grid_desc": L.GridDesc, "pf_phase": L.Phase, "pf_solve_cfg": L.SolveCfg,
               "pf_solve_stats": L.SolveStats, "pf_clamp_stats": L.ClampStats, "pf_step_cfg": L.StepCfg,
               "pf_step_stats": L.StepStats, "pf_timing": L.Timing, "pf_band_stats": L.BandStats,
               "pf_coarsen_stats": L.CoarsenStats, "pf_refill_stats": L.RefillStats, "pf_adapt_cfg": L.AdaptCfg,
               "pf_adapt_stats": L.AdaptStats, "pf_interface_stats": L.InterfaceStats,
               "pf_step_controls": L.StepControls, "pf_step_control_stats": L.StepControlStats,
               "pf_surface_stats": L.SurfaceStats, "pf_render_camera": L.RenderCamera,
               "pf_render_manifest_frame": L.RenderManifestFrame, "pf_mr_box": L.MRBox,
               "pf_mr_dynamic": L.MRDynamic, "pf_mr_step_cfg": L.MRStepCfg, "pf_mr_step_stats": L.MRStepStats,
               "pf_secondary_cfg": L.SecondaryCfg, "pf_secondary_stats": L.SecondaryStats}
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "pfgpu.h"', "int main(void){"]
    for cname, py in structs.items():
        src.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            src.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, py in structs.items():
        import ctypes
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_create_without_gpu_fails_loudly(pf):
    """No CPU fallback: without a usable device pf_create returns an error."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pf.PfError):
        pf.SparseMacGrid3D(8, 8, 8, 1.0)
