"""The native library builds, loads without a GPU and exports every symbol
that include/*.h declares; host-side logic that needs no device."""
import ctypes
import os
import re

import numpy as np

import timbir_b200
from timbir_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("mbir4d.h", "timbir_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith("mbir_") or name == "reconstruct":
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = timbir_b200.load_library()
    names = declared_functions()
    assert "reconstruct" in names and "mbir_update_voxels_time_slices" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_library_is_sm100a():
    data = open(timbir_b200.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def test_reconstruct_rejects_bad_dimensions(tmp_path):
    # proj_rows must be even and >= 4 (src/MBIR_4D/XT_Engine.c:101-104); the
    # check runs before any device work.
    s = synth.ellipsoid_scan(32, 4, 16, seed=0)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rc = timbir_b200.reconstruct(s.projections[:, :3], s.weights[:, :3], s.proj_angles, s.proj_times,
                                     s.recon_times, 3, 32, 16, 1, 1.0, 16.0, 0.002, 1.0, 1e-3, 1e-3, 1.0, 0, 1,
                                     0.5, 4.0, debug_log=str(tmp_path / "log.txt"))
    finally:
        os.chdir(cwd)
    assert rc == -1
    assert "[ERROR]" in open(tmp_path / "log.txt").read()


def test_interlaced_schedule_is_a_permutation_per_rotation():
    a = synth.interlaced_angles(16, 1024, 128)
    steps = np.round(a / (np.pi / 128)).astype(int)
    for rot in range(8):
        block = steps[rot * 128:(rot + 1) * 128] - rot * 128
        assert sorted(block.tolist()) == list(range(128))


def test_synthetic_scan_layout():
    s = synth.ellipsoid_scan(32, 4, 24, seed=0)
    assert s.projections.shape == (24, 4, 32) and s.projections.dtype == np.float32
    assert s.weights.min() >= 1.0
    assert s.phantom.shape == (1, 4, 32, 32)
    assert abs(s.phantom.max() - 0.02) < 1e-6
