"""The render-cache manifest (writeRenderCacheManifest3D,
src/driver/render_cache3d.h:711-755) written by the library's host code
(pf_write_render_manifest, no device involved) against the reference's own
writer compiled into oracle/_ref: the files must be identical byte for byte,
including the string escaping and 17-digit numbers.  The first case is the
reference's own test (tests/test_render_cache3d.cpp:118-145)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O


def _reference_manifest(path, kind, n, dx, frames):
    lib = O.ref_lib()
    m = len(frames)
    paths = (C.c_char_p * max(1, m))(*[f.path.encode() for f in frames])
    rc = lib.pfr_write_render_manifest(str(path).encode(), kind.encode(), n[0], n[1], n[2], dx, m,
                                       np.array([f.frame for f in frames] or [0], np.int32),
                                       np.array([f.step for f in frames] or [0], np.int32),
                                       np.array([f.time for f in frames] or [0.0], np.float64), paths,
                                       np.array([f.bytes for f in frames] or [0], np.int64))
    return rc


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("case", ["reference_test", "escapes", "empty", "fractional"])
def test_manifest_equals_reference_writer(pf, tmp_path, case):
    F = pf.RenderCacheManifestFrame3D
    if case == "reference_test":
        kind, n, dx = "sparse3d_tp", (8, 12, 8), 1.0
        frames = [F(0, 3, 0.06, "cache_000.jsonl", 123), F(1, 5, 0.10, "nested\\cache_001.jsonl", 456)]
    elif case == "escapes":
        kind, n, dx = 'multi"res\t3d', (16, 24, 16), 1.0 / 16
        frames = [F(i, 2 * i, i / 480.0, f"dir/frame_{i}\n\x01\x1f\b\f\r.jsonl", 1000 * i + 7) for i in range(5)]
    elif case == "empty":
        kind, n, dx = "sparse3d_tp", (48, 48, 48), 1.0 / 48
        frames = []
    else:
        rng = np.random.default_rng(3)
        kind, n, dx = "sparse3d_tp", (33, 7, 129), 0.1
        frames = [F(i, i * 3, float(rng.uniform(0, 10)), f"f{i:04d}.jsonl", int(rng.integers(0, 1 << 40)))
                  for i in range(20)]
    ours, theirs = tmp_path / "ours.json", tmp_path / "ref.json"
    pf.writeRenderCacheManifest3D(ours, kind, *n, dx, frames)
    assert _reference_manifest(theirs, kind, n, dx, frames) == 0
    a, b = ours.read_bytes(), theirs.read_bytes()
    assert a == b
    if case == "reference_test":
        text = a.decode()
        for needle in ('"lsfs_cache3d_manifest_version":1', '"cache_schema_version":2', '"world_units":"cell"',
                       '"sim_kind":"sparse3d_tp"', '"dims":[8,12,8]', '"frame_bounds_max":[8,12,8]',
                       '"shutter_open"', '"path":"cache_000.jsonl"', '"step":3', '"bytes":456',
                       'nested\\\\cache_001.jsonl'):
            assert needle in text


@pytest.mark.parametrize("bad", ["path", "kind", "dims", "dx", "frame", "time", "bytes"])
def test_manifest_rejects_what_the_reference_rejects(pf, tmp_path, bad):
    F = pf.RenderCacheManifestFrame3D
    path, kind, n, dx = tmp_path / "m.json", "sparse3d_tp", [8, 8, 8], 1.0
    frames = [F(0, 1, 0.5, "a.jsonl", 10)]
    if bad == "path":
        path = ""
    elif bad == "kind":
        kind = ""
    elif bad == "dims":
        n[1] = 0
    elif bad == "dx":
        dx = float("nan")
    elif bad == "frame":
        frames = [F(-1, 1, 0.5, "a.jsonl", 10)]
    elif bad == "time":
        frames = [F(0, 1, float("inf"), "a.jsonl", 10)]
    else:
        frames = [F(0, 1, 0.5, "a.jsonl", -5)]
    with pytest.raises(ValueError):
        pf.writeRenderCacheManifest3D(path, kind, *n, dx, frames)
