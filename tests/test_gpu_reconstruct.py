"""The drop-in reconstruct() end to end on the GPU, against a full run of the
reference's own driver (tests/golden/recon_small.npz, made by
tests/golden/make_golden.py: 32x32x4, 48 views, 2 resolution stages,
convg_thresh 0.005, cost evaluated each iteration).

Both runs stop on the convergence test, not at the exact MAP point, so the
final objects are compared by their MAP cost evaluated afresh in FP64 (within
5e-5 relative, a few of the last iterations' decrease) and by RMSE against the
reference's object (below 1e-3 of the phantom's 0.02 range).  The output
files and their sizes are the reference's (src/MBIR_4D/XT_IOMisc.c:238-271,
XT_ICD_update.c:1205-1221, XT_Engine.c:176).
"""
import os

import numpy as np
import pytest

import timbir_b200
from oracle.bind import Oracle
from timbir_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ARGS = dict(sig_s=0.002, sig_t=1.0, c_s=1e-3, c_t=1e-3, convg_thresh=0.005, remove_rings=0, quad_convex=1,
            huber_delta=0.5, huber_T=4.0)


def run_reconstruct(tmp_path, scan, args, env=None, restart=0):
    old = {}
    for k, v in (env or {}).items():
        old[k] = os.environ.get(k)
        os.environ[k] = v
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rc = timbir_b200.reconstruct(scan.projections, scan.weights, scan.proj_angles, scan.proj_times,
                                     scan.recon_times, scan.proj_rows, scan.proj_cols, scan.proj_num, scan.recon_num,
                                     scan.vox_wid, scan.rot_center, restart=restart,
                                     debug_log=str(tmp_path / "log.txt"), **args)
    finally:
        os.chdir(cwd)
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return rc


def fresh_cost(scan, x):
    o = Oracle(scan, blocks=2, f64=True, **ARGS)
    o.prepare(x)
    return o.cost()[0]


@pytest.mark.parametrize("schedule", ["sv", "reference"])
def test_reconstruct_matches_reference_run(tmp_path, schedule):
    g = np.load(os.path.join(GOLD, "recon_small.npz"))
    scan = synth.ellipsoid_scan(32, 4, 48, seed=11)
    env = {"TIMBIR_SCHEDULE": schedule}
    if schedule == "reference":
        env["TIMBIR_Z_BLOCK_THREADS"] = str(int(g["threads"]))
    assert run_reconstruct(tmp_path, scan, ARGS, env) == 0
    x = np.fromfile(tmp_path / "object_time_0.bin", np.float32).reshape(1, 4, 32, 32)
    ref = g["object"].reshape(1, 4, 32, 32)
    c, cr = fresh_cost(scan, x), fresh_cost(scan, ref)
    assert abs(c - cr) / cr < 5e-5
    assert float(np.sqrt(np.mean((x - ref) ** 2))) < 1e-3 * 0.02
    # the reference's output file set
    assert (tmp_path / "proj_offset.bin").stat().st_size == 32 * 4 * 4
    assert np.fromfile(tmp_path / "status.bin", np.int32)[0] == 1
    assert (tmp_path / "variance_estimate.bin").stat().st_size == 8
    assert np.fromfile(tmp_path / "variance_estimate.bin", np.float64)[0] == 1.0
    assert (tmp_path / "projs_runtime.bin").stat().st_size == 48 * 32 * 4 * 4
    assert (tmp_path / "weights_runtime.bin").stat().st_size == 48 * 32 * 4 * 4
    assert (tmp_path / "mag_update.bin").exists()


def test_reconstruct_4d_rings_and_zingers(tmp_path):
    s = synth.ellipsoid_scan(32, 4, 64, seed=5, zinger_frac=0.002, ring_sigma=0.02)
    s.proj_angles = synth.interlaced_angles(4, 64, 32)
    s.recon_times = np.array([0, 16, 32, 48, 64], np.float32)
    s.recon_num = 4
    args = dict(ARGS, convg_thresh=0.5, remove_rings=2, quad_convex=0, sig_t=0.01)
    assert run_reconstruct(tmp_path, s, args) == 0
    for f in range(4):
        x = np.fromfile(tmp_path / f"object_time_{f}.bin", np.float32)
        assert x.size == 4 * 32 * 32 and np.all(np.isfinite(x))
    d = np.fromfile(tmp_path / "proj_offset.bin", np.float32)
    assert d.size == 32 * 4 and np.any(d != 0)
    var = np.fromfile(tmp_path / "variance_estimate.bin", np.float64)[0]
    assert np.isfinite(var) and var > 0 and var != 1.0


def test_reconstruct_restart_resumes_at_recorded_stage(tmp_path):
    scan = synth.ellipsoid_scan(32, 4, 48, seed=11)
    assert run_reconstruct(tmp_path, scan, ARGS) == 0
    first = np.fromfile(tmp_path / "object_time_0.bin", np.float32)
    # rewind to "stage 0 finished": coarse object, status 0, then restart
    coarse = first.reshape(4, 32, 32)[::2, ::2, ::2]
    coarse.astype(np.float32).tofile(tmp_path / "object_time_0.bin")
    np.array([1], np.int32).tofile(tmp_path / "status.bin")
    assert run_reconstruct(tmp_path, scan, ARGS, restart=1) == 0
    again = np.fromfile(tmp_path / "object_time_0.bin", np.float32)
    assert again.size == first.size and np.all(np.isfinite(again))
    assert float(np.sqrt(np.mean((again - first) ** 2))) < 2e-3 * 0.02
