"""GPU tests of the super-voxel schedule.

The super-voxel schedule updates voxels in a different order than the
reference (many super-voxels at once, each from a private copy of its
error-sinogram band), so its trajectory is not the reference's; parity is
checked on the result:
  * the MAP it converges to: final cost within 1e-5 relative of the
    reference's converged cost, and image RMSE below 1e-3 of the phantom's
    dynamic range against the FP64 oracle (both from
    tests/golden/converged_plain.npz), costs evaluated afresh in FP64;
  * bookkeeping: the error sinogram it maintains by atomics stays equal to
    y - A x - d recomputed from scratch (float tolerance);
  * no A-matrix column ever leaves the staged band (the kernel flags it and
    the iteration call fails);
  * the A-matrix column cache holds the reference's columns (bin indices
    bit-exact, values to float rounding) and gives the same iterates as
    columns computed in the kernel;
  * detectors whose width is not a multiple of four columns (staged and
    committed element by element instead of by 16-byte words) reach the
    FP64 oracle's MAP as well.
"""
import os

import numpy as np
import pytest

import scenarios
import timbir_b200
from oracle.bind import Oracle
from timbir_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
SCALE = 0.02


def fresh_cost_fp64(name, x, offset=None):
    o = scenarios.make(name, Oracle, f64=True)
    o.prepare(x, offset)
    return o.cost()[0]


def run_to_flat(s, max_iters=2000, flat=1e-10):
    """Iterations from iteration 1 until the stage's cost changes by less than
    `flat` (relative) over five iterations."""
    hist = []
    for it in range(1, max_iters + 1):
        s.iterate(it)
        hist.append(s.cost()[0])
        if it > 10 and abs(hist[-6] - hist[-1]) <= flat * abs(hist[-1]):
            break
    return it


def sv_stage(name, side=0, acache=-1, wps=0):
    s = scenarios.make(name, timbir_b200.Stage)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, side, wps, acache)
    return s


@pytest.mark.parametrize("acache", [1, 0])
def test_sv_converges_to_reference_map(acache):
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    s = sv_stage("plain", acache=acache)
    assert (s.schedule_info()["column_cache_bytes"] > 0) == (acache == 1)
    s.prepare()
    run_to_flat(s)
    x = s.object()
    c = fresh_cost_fp64("plain", x)
    assert abs(c - float(g["ref_fresh_cost"])) / float(g["ref_fresh_cost"]) < 1e-5
    rmse = float(np.sqrt(np.mean((x - g["f64_object"]) ** 2)))
    assert rmse < 1e-3 * SCALE


@pytest.mark.parametrize("side", [4, 6, 8])
def test_sv_side_does_not_change_the_map(side):
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    s = sv_stage("plain", side)
    assert s.schedule_info()["sv_side"] == side
    s.prepare()
    run_to_flat(s)
    c = fresh_cost_fp64("plain", s.object())
    assert abs(c - float(g["ref_fresh_cost"])) / float(g["ref_fresh_cost"]) < 1e-5


@pytest.mark.parametrize("acache", [1, 0])
@pytest.mark.parametrize("name", ["plain", "rings2", "frames4", "coarse4", "blocks4"])
def test_sv_error_sinogram_stays_consistent(name, acache):
    s = sv_stage(name, acache=acache)
    s.prepare()
    for it in range(1, 11):
        s.iterate(it)
    e_run = s.errorsino()
    x, d = s.object(), s.offset()
    f = scenarios.make(name, timbir_b200.Stage)
    f.prepare(x, d)
    e_fresh = f.errorsino()
    scale = np.abs(e_fresh).max()
    assert np.abs(e_run - e_fresh).max() < 2e-5 * scale


@pytest.mark.parametrize("name", list(scenarios.SCENARIOS))
def test_sv_decreases_cost(name):
    s = sv_stage(name)
    s.prepare()
    c0 = s.cost()[0]
    for it in range(1, 6):
        s.iterate(it)
    c5 = s.cost()[0]
    assert np.isfinite(c5) and c5 < c0
    assert s.update_count() > 0


def test_sv_one_warp_per_slice_for_tall_groups():
    # 16 slices in one z-group: one warp per slice (two only up to 15)
    from timbir_b200 import synth
    scan = synth.ellipsoid_scan(32, 16, 48, seed=21)
    kw = dict(scenarios.BASE)
    s = timbir_b200.Stage(scan, blocks=2, **kw)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0)
    assert s.schedule_info()["z_group"] == 16
    s.prepare()
    c0 = s.cost()[0]
    for it in range(1, 11):
        s.iterate(it)
    assert s.cost()[0] < c0
    f = timbir_b200.Stage(scan, blocks=2, **kw)
    f.prepare(s.object(), s.offset())
    scale = np.abs(f.errorsino()).max()
    assert np.abs(s.errorsino() - f.errorsino()).max() < 2e-5 * scale


@pytest.mark.parametrize("wps", [1, 2, 4])
def test_sv_warps_per_slice_reach_the_same_map(wps):
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    s = scenarios.make("plain", timbir_b200.Stage)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0, wps)
    assert s.schedule_info()["warps_per_slice"] == wps
    s.prepare()
    run_to_flat(s)
    c = fresh_cost_fp64("plain", s.object())
    assert abs(c - float(g["ref_fresh_cost"])) / float(g["ref_fresh_cost"]) < 1e-5


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("name", ["plain", "coarse2", "coarse4", "frames4"])
def test_sv_column_cache_holds_the_reference_columns(name, mode):
    # bin indices bit-exact, values within float rounding (FP32 cache) or half
    # rounding (FP16 cache, full-resolution stages; coarse stages keep FP32)
    # of the reference's double quotient (calcAMatrixColumnforAngle), over a
    # sample of lines
    s = sv_stage(name, acache=mode)
    fp16 = s.schedule_info()["column_cache_values"] == "fp16"
    assert fp16 == (mode == 2 and not name.startswith("coarse"))
    rtol = 4.9e-4 if fp16 else 1e-6
    s.prepare()
    o = scenarios.make(name, Oracle)
    o.prepare()  # detector response
    ys, xs = np.nonzero(s.mask())
    pick = np.random.default_rng(3).choice(len(ys), size=min(24, len(ys)), replace=False)
    for q in pick:
        row, col = int(ys[q]), int(xs[q])
        j0, n, vals = s.acache_line(row, col)
        for view in range(s.N_p):
            idx, val = o.amatrix(row, col, view)
            assert n[view] == len(idx), (row, col, view)
            if len(idx):
                assert np.array_equal(idx, j0[view] + np.arange(n[view])), (row, col, view)
                # FP16: half rounding of the column's largest value (small
                # values are subnormal in FP16)
                atol = rtol * float(np.abs(val).max()) if fp16 else 0.0
                np.testing.assert_allclose(vals[view, :n[view]], val, rtol=rtol, atol=atol)


@pytest.mark.parametrize("name", ["plain", "coarse2", "frames4", "rings2"])
def test_sv_cached_and_computed_columns_give_the_same_iterates(name):
    # one CTA per launch: super-voxels run one after another, so the run is
    # deterministic and the two column sources must give identical iterates
    # (same warps per slice: the split of a slice's views fixes the order of
    # its sums)
    side = sv_stage(name, acache=0).schedule_info()["sv_side"]
    out = []
    for acache in (1, 0):
        s = sv_stage(name, side, acache, wps=2)
        s.set_sv_ctas(1)
        s.prepare()
        for it in range(1, 4):
            s.iterate(it)
        out.append((s.object(), s.errorsino()))
    (x1, e1), (x0, e0) = out
    assert np.array_equal(x1, x0), float(np.abs(x1 - x0).max())
    assert np.array_equal(e1, e0), float(np.abs(e1 - e0).max())


def test_sv_one_warp_per_slice_with_eight_views_per_lane():
    # 192 views and one warp per slice: each lane holds 6 views of a slice in
    # registers (the 8-views-per-lane variant); it must reach the same
    # minimum as two warps per slice, and keep its error sinogram consistent
    from timbir_b200 import synth
    scan = synth.ellipsoid_scan(32, 4, 192, seed=9)
    kw = dict(scenarios.BASE)
    costs = []
    for wps in (1, 2):
        s = timbir_b200.Stage(scan, blocks=2, **kw)
        s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0, wps)
        assert s.schedule_info()["warps_per_slice"] == wps
        s.prepare()
        for it in range(1, 201):
            s.iterate(it)
        o = Oracle(scan, blocks=2, f64=True, **kw)
        o.prepare(s.object(), s.offset())
        costs.append(o.cost()[0])
    assert abs(costs[0] - costs[1]) / abs(costs[1]) < 1e-6
    # bookkeeping over 10 iterations, as the other consistency tests
    s = timbir_b200.Stage(scan, blocks=2, **kw)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0, 1)
    s.prepare()
    for it in range(1, 11):
        s.iterate(it)
    f = timbir_b200.Stage(scan, blocks=2, **kw)
    f.prepare(s.object(), s.offset())
    scale = np.abs(f.errorsino()).max()
    assert np.abs(s.errorsino() - f.errorsino()).max() < 2e-5 * scale


def test_sv_full_size_slices_converge_with_the_automatic_grid():
    # 256 x 256 slices: super-voxels in flight on one sinogram each correct
    # the rays they share; with too many at once (48 of side 6 here) the
    # iteration diverges.  The automatic grid must keep the cost falling.
    from timbir_b200 import synth
    scan = synth.ellipsoid_scan(256, 8, 256, I0=1e4, seed=0)
    kw = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=0, quad_convex=1)
    s = timbir_b200.Stage(scan, blocks=8, **kw)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0)
    info = s.schedule_info()
    assert info["ctas"] <= info["inflight_per_group"]
    s.prepare(np.asarray(scan.phantom, np.float32) * 0.9)
    costs = [s.cost()[0]]
    for it in range(1, 11):
        s.iterate(it)
        costs.append(s.cost()[0])
    assert all(np.isfinite(costs))
    assert all(b < a for a, b in zip(costs, costs[1:])), costs


def test_sv_fp16_columns_reach_the_map_within_the_fp64_oracle_bar():
    # FP16 A values with FP32 accumulation: the iteration minimises the cost of
    # the rounded A matrix; its image must still lie within 1e-3 of the range
    # of the FP64-converged oracle, like the FP32 path's, and its exact-model
    # cost close to the reference's converged cost
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    out = {}
    for mode in (1, 2):
        s = sv_stage("plain", acache=mode)
        s.prepare()
        run_to_flat(s)
        x = s.object()
        rmse = float(np.sqrt(np.mean((x - g["f64_object"]) ** 2)))
        c = fresh_cost_fp64("plain", x)
        out[mode] = (rmse / SCALE, abs(c - float(g["ref_fresh_cost"])) / float(g["ref_fresh_cost"]))
    print("relative RMSE vs FP64 oracle and relative cost error: fp32 %.2e %.2e, fp16 %.2e %.2e"
          % (out[1] + out[2]))
    assert out[2][0] < 1e-3
    assert out[2][1] < 1e-4


def test_stability_guard_recovers_a_diverging_sweep():
    # 256 x 256 x 16 slices, 384 views, a random-ellipsoid phantom, from zero:
    # the automatic grid (148 super-voxels of side 9 in flight, over-relaxation
    # 0.94) over-corrects the shared rays and the MAP cost explodes in the
    # second iteration; with the guard the cost never rises (the iteration is
    # redone from the state before it with half as many in flight)
    from timbir_b200 import synth
    rng = np.random.default_rng(6000)
    I0 = float(np.exp(rng.uniform(np.log(2e3), np.log(5e4))))
    scan = synth.ellipsoid_scan_device(256, 16, 384, I0=I0, seed=6000)
    kw = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=0, quad_convex=1,
              huber_delta=0.5, huber_T=4.0, blocks=2)
    costs = {}
    for guard in (False, True):
        s = timbir_b200.Stage(scan, **kw)
        s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0, 0, 1)
        s.set_sv_guard(guard)
        s.prepare()
        c = [s.cost()[0]]
        for it in range(1, 7 if guard else 3):
            s.iterate(it)
            c.append(s.cost()[0])
        costs[guard] = (c, s.schedule_info()["stability_adjustments"])
        s.close()
    unguarded, _ = costs[False]
    guarded, adjustments = costs[True]
    assert unguarded[2] > unguarded[1]  # the unguarded sweep diverges
    assert adjustments >= 1
    assert all(np.isfinite(guarded)) and all(b <= a * (1 + 1e-6) for a, b in zip(guarded, guarded[1:]))


RAGGED_KW = dict(blocks=2, mult_xy=1, mult_z=1, **scenarios.BASE)
_ragged_map = {}


def ragged_map(cols):
    """(scan, converged FP64 oracle object, its cost) of a 4-slice, 48-view
    scan whose detector rows have `cols` columns."""
    if cols not in _ragged_map:
        scan = synth.ellipsoid_scan(cols, 4, 48, seed=11)
        o = Oracle(scan, f64=True, **RAGGED_KW)
        o.prepare()
        run_to_flat(o, flat=1e-12)
        _ragged_map[cols] = (scan, o.object(), o.cost()[0])
        o.close()
    return _ragged_map[cols]


@pytest.mark.parametrize("acache", [1, 0], ids=["cached", "computed"])
@pytest.mark.parametrize("cols", [30, 33])
def test_sv_ragged_detector_reaches_the_fp64_map(cols, acache):
    scan, ref, cref = ragged_map(cols)
    s = timbir_b200.Stage(scan, **RAGGED_KW)
    s.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL, 0, 0, acache)
    s.prepare()
    run_to_flat(s)
    x = s.object()
    s.close()
    o = Oracle(scan, f64=True, **RAGGED_KW)
    o.prepare(x)
    c = o.cost()[0]
    o.close()
    rmse = float(np.sqrt(np.mean((x.astype(np.float64) - ref) ** 2)))
    print(f"{cols} columns: fresh FP64 cost - oracle MAP cost = {(c - cref) / cref:.3g} relative, "
          f"RMSE / range = {rmse / SCALE:.3g}")
    assert abs(c - cref) / cref < 1e-5
    assert rmse < 1e-3 * SCALE
