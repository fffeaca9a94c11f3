"""GPU tests of the device NHICD selection (mbir_nhicd.cu).

VSC_based_Voxel_Line_Select (XT_NHICD.c:164-216) keeps, per (frame,
z-block) plane, the voxel lines whose 5x5 Hamming-filtered update magnitude
exceeds the plane's (N - n_sel)-th smallest filtered value.  The device
finds that order statistic by radix select instead of the reference's
randomized quickselect; the value, and so the selected set, must be the same
(bit-exact index work):
  * against the oracle's selection (oracle/mbir_oracle.c, pinned to the
    reference) on the magnitude maps of real iterations, several scenarios;
  * against a numpy order statistic on synthetic maps with ties, all-zero
    planes and n_sel = 0;
and the super-voxel schedule with its device NHICD pass turned on (it is
off by default) still reaches the reference's MAP.
"""
import os

import numpy as np
import pytest

import scenarios
import timbir_b200
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["plain", "frames4", "blocks4", "rings2"])
def test_device_selection_matches_the_oracle(name):
    o = scenarios.make(name, Oracle)
    o.prepare()
    for it in (1, 2):
        o.iterate(it)
    o.vsc_select()  # selection from the current magnitude maps
    mag = o.magmap()  # [N_time][nblk][N_y][N_x]
    planes = o.N_time * o.nblk
    nsel = np.array([len(o.lines(0, f, b)[0]) // 10 for f in range(o.N_time) for b in range(o.nblk)], np.int32)
    sel, _ = timbir_b200.nhicd_select(mag.reshape(planes, o.N_y, o.N_x), nsel)
    total = 0
    for f in range(o.N_time):
        for b in range(o.nblk):
            xs, ys = o.lines(1, f, b)
            want = np.zeros((o.N_y, o.N_x), np.uint8)
            want[ys, xs] = 1
            np.testing.assert_array_equal(sel[f * o.nblk + b], want)
            total += len(xs)
    assert total > 0
    o.close()


def _numpy_selection(mag, nsel):
    """The reference's rule restated in numpy: float64 5x5 Hamming filter
    stored as float32, threshold = the (N - nsel)-th smallest, keep > it."""
    hw = np.array([[0.0064, 0.0432, 0.0800, 0.0432, 0.0064],
                   [0.0432, 0.2916, 0.5400, 0.2916, 0.0432],
                   [0.0800, 0.5400, 1.0000, 0.5400, 0.0800],
                   [0.0432, 0.2916, 0.5400, 0.2916, 0.0432],
                   [0.0064, 0.0432, 0.0800, 0.0432, 0.0064]])
    ny, nx = mag.shape
    f = np.zeros((ny, nx))
    for j in range(ny):
        for k in range(nx):
            acc = 0.0
            for p in range(-2, 3):
                for q in range(-2, 3):
                    if 0 <= j + p < ny and 0 <= k + q < nx:
                        acc += hw[p + 2, q + 2] * float(mag[j + p, k + q])
            f[j, k] = acc
    f = f.astype(np.float32)
    n = f.size
    th = np.sort(f.reshape(-1))[n - nsel - 1] if nsel > 0 else f.max()
    return (f > th).astype(np.uint8), th


def test_device_selection_edge_cases():
    rng = np.random.default_rng(3)
    ny, nx = 37, 53
    maps = [
        np.zeros((ny, nx), np.float32),                                    # all zero: nothing selected
        np.full((ny, nx), 0.25, np.float32),                               # constant: ties, edge effects only
        np.round(rng.random((ny, nx)) * 4).astype(np.float32) / 4,         # heavy ties
        (rng.random((ny, nx)) ** 3).astype(np.float32),                    # distinct values
        np.where(rng.random((ny, nx)) < 0.1, rng.random((ny, nx)), 0).astype(np.float32),  # sparse
    ]
    for nsel in (0, 1, 37, (ny * nx) // 10):
        sel, th = timbir_b200.nhicd_select(np.stack(maps), nsel)
        for p, m in enumerate(maps):
            want, wth = _numpy_selection(m, nsel)
            np.testing.assert_array_equal(sel[p], want, err_msg=f"plane {p}, n_sel {nsel}")
            assert th[p] == wth


def test_sv_schedule_with_device_nhicd_reaches_the_reference_map():
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    ref = float(g["ref_fresh_cost"])
    for frac in (0.1, 0.0):
        s = scenarios.make("plain", timbir_b200.Stage)
        s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL)
        s.set_sv_nhicd(frac)
        s.prepare()
        s.iterate(1)
        s.iterate(2)
        # one sweep launch per iteration, plus the NHICD pass from the second
        _, n_icd, _ = s.kernel_stats()
        assert n_icd == (3 if frac > 0 else 2)
        for it in range(3, 301):
            s.iterate(it)
        o = scenarios.make("plain", Oracle, f64=True)
        o.prepare(s.object())
        c = o.cost()[0]
        assert abs(c - ref) / ref < 1e-5, f"NHICD fraction {frac}"
        s.close()
        o.close()
