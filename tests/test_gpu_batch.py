"""GPU tests of batched super-voxel ICD (many independent problems per
persistent launch, iterations replayed as CUDA graphs) and of the autotuner.

Batching changes which super-voxels run at the same time, not the
iteration each problem performs, so each problem must reach the same MAP as
when reconstructed alone:
  * the "plain" scenario inside a batch of three differently sized problems
    converges to the reference's converged cost (within 1e-5 relative, FP64
    cost evaluated afresh) and to the FP64 oracle's image (RMSE below 1e-3
    of the phantom's range), like the single-problem schedule;
  * the other problems reach the cost the single-problem schedule converges to;
  * each problem's error sinogram, maintained by atomics from many CTAs of
    several problems, stays equal to y - A x recomputed from scratch;
  * a problem whose convergence test passes is retired (its object no longer
    changes) while the others go on;
  * the autotuner leaves the stage's state as prepared and picks a
    configuration the batch runs;
  * problems whose detector rows are not a multiple of four columns wide
    reach the FP64 oracle's MAP inside a batch;
  * a problem whose stage asks for the NHICD pass gets it after each batched
    sweep and still reaches the reference's MAP.
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
SV = timbir_b200.Stage.SCHEDULE_SUPERVOXEL


def make_stage(n_xy, rows, views, seed, thresh=0.0, side=0, prepare=True):
    scan = synth.ellipsoid_scan(n_xy, rows, views, seed=seed)
    args = dict(scenarios.BASE, convg_thresh=thresh)
    s = timbir_b200.Stage(scan, blocks=2, **args)
    s.set_batch_schedule(side, 1, 1)
    if prepare:
        s.prepare()
    return s


def plain_stage(thresh=0.0):
    # the "plain" scenario (tests/scenarios.py) with its convergence test set
    return make_stage(32, 4, 48, seed=1, thresh=thresh)


def fresh_cost_fp64(scan, x, thresh=0.0):
    o = Oracle(scan, blocks=2, f64=True, **dict(scenarios.BASE, convg_thresh=thresh))
    o.prepare(x)
    return o.cost()[0]


def run_until_flat(step, costs, chunk=100, max_iters=3000, tol=1e-9):
    """Iterate `chunk` at a time until no cost moved by more than tol
    (relative) over a chunk; returns the final costs."""
    prev = costs()
    for _ in range(max_iters // chunk):
        step(chunk)
        cur = costs()
        if all(abs(a - b) <= tol * abs(b) for a, b in zip(prev, cur)):
            break
        prev = cur
    return cur


def test_batch_reaches_the_reference_map():
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    sizes = [(48, 6, 72, 11), (24, 2, 36, 12)]
    stages = [plain_stage()] + [make_stage(*z) for z in sizes]
    b = timbir_b200.Batch(stages)
    assert b.iterate(300, check_every=50) == 3  # convergence test off: all still iterating
    st = b.stats()
    assert list(st["iterations"]) == [300, 300, 300]
    assert all(st["updates"] > 0)
    x = stages[0].object()
    c = fresh_cost_fp64(stages[0].scan, x)
    assert abs(c - float(g["ref_fresh_cost"])) / float(g["ref_fresh_cost"]) < 1e-5
    rmse = float(np.sqrt(np.mean((x - g["f64_object"]) ** 2)))
    assert rmse < 1e-3 * SCALE
    # the other problems: the cost the single-problem schedule converges to
    # (both iterated until their costs stop moving)
    run_until_flat(lambda k: b.iterate(k, check_every=k), lambda: [s.cost()[0] for s in stages[1:]])
    b.close()
    for k, z in enumerate(sizes, start=1):
        alone = make_stage(*z)
        it = [0]

        def step(n):
            for _ in range(n):
                it[0] += 1
                alone.iterate(it[0])

        run_until_flat(step, lambda: [alone.cost()[0]])
        c_alone = fresh_cost_fp64(alone.scan, alone.object())
        c_batch = fresh_cost_fp64(stages[k].scan, stages[k].object())
        assert abs(c_batch - c_alone) / c_alone < 1e-5
        alone.close()
    for s in stages:
        s.close()


def test_batch_error_sinograms_stay_consistent():
    stages = [plain_stage(), make_stage(48, 6, 72, seed=11), make_stage(40, 4, 60, seed=13)]
    b = timbir_b200.Batch(stages)
    b.iterate(10)
    b.close()
    for s in stages:
        e_run = s.errorsino()
        f = timbir_b200.Stage(s.scan, blocks=2, **dict(scenarios.BASE, convg_thresh=0.0))
        f.prepare(s.object(), s.offset())
        e_fresh = f.errorsino()
        scale = np.abs(e_fresh).max()
        assert np.abs(e_run - e_fresh).max() < 2e-5 * scale
        f.close()
        s.close()


def test_batch_retires_converged_problems():
    quick = plain_stage(thresh=20.0)
    slow = make_stage(48, 6, 72, seed=11, thresh=0.0)
    b = timbir_b200.Batch([quick, slow])
    c0 = quick.cost()[0]
    assert b.iterate(20) == 1
    st = b.stats()
    assert st["converged"][0] == 1 and st["iterations"][0] < 20 and st["percent"][0] < 20.0
    assert st["converged"][1] == 0 and st["iterations"][1] == 20
    assert quick.cost()[0] < c0
    xq, xs = quick.object(), slow.object()
    b.iterate(3)
    st2 = b.stats()
    assert st2["iterations"][0] == st["iterations"][0] and st2["iterations"][1] == 23
    assert np.array_equal(quick.object(), xq)
    assert not np.array_equal(slow.object(), xs)
    b.close()
    quick.close()
    slow.close()


def test_batch_stops_when_every_problem_converged():
    stages = [plain_stage(thresh=20.0), make_stage(24, 2, 36, seed=12, thresh=20.0)]
    b = timbir_b200.Batch(stages)
    assert b.iterate(50) == 0
    st = b.stats()
    assert all(st["converged"] == 1) and all(st["iterations"] < 50)
    assert b.info()["replays"] == max(st["iterations"])
    b.close()


def test_batch_rejects_unsupported_stages():
    rings = scenarios.make("rings2", timbir_b200.Stage)
    rings.set_batch_schedule(0, 1, 1)
    rings.prepare()
    with pytest.raises(timbir_b200.MbirError, match="plain ICD"):
        timbir_b200.Batch([rings])
    nocache = make_stage(32, 4, 48, seed=1, prepare=False)
    nocache.set_batch_schedule(0, 1, 0)
    nocache.prepare()
    with pytest.raises(timbir_b200.MbirError, match="column cache"):
        timbir_b200.Batch([nocache])
    rings.close()
    nocache.close()


def test_autotune_restores_the_stage_and_runs_in_a_batch():
    s = make_stage(48, 8, 72, seed=14)
    x0, e0 = s.object(), s.errorsino()
    t = s.autotune()
    assert 4 <= t["sv_side"] <= 8 and t["warps_per_slice"] in (1, 2, 4)
    assert t["z_group"] * t["warps_per_slice"] <= 8 and t["ns_per_update"] > 0
    info = s.schedule_info()
    assert info["sv_side"] == t["sv_side"] and info["warps_per_slice"] == t["warps_per_slice"]
    assert np.array_equal(s.object(), x0) and np.array_equal(s.errorsino(), e0)
    c0 = s.cost()[0]
    b = timbir_b200.Batch([s])
    b.iterate(5)
    b.close()
    assert s.cost()[0] < c0
    s.close()


def test_batch_of_ragged_detectors_reaches_the_fp64_map():
    # detector rows of 30 and 33 columns: the band is staged and committed
    # element by element instead of by 16-byte words
    stages = [make_stage(cols, 4, 48, seed=11) for cols in (30, 33)]
    b = timbir_b200.Batch(stages)
    run_until_flat(lambda n: b.iterate(n, check_every=50), lambda: [s.cost()[0] for s in stages], tol=1e-10)
    for s in stages:
        x = s.object()
        o = Oracle(s.scan, blocks=2, f64=True, **dict(scenarios.BASE, convg_thresh=0.0))
        o.prepare()
        hist = []
        for it in range(1, 3000):
            o.iterate(it)
            hist.append(o.cost()[0])
            if it > 10 and abs(hist[-6] - hist[-1]) <= 1e-12 * abs(hist[-1]):
                break
        ref, cref = o.object(), hist[-1]
        o.close()
        c = fresh_cost_fp64(s.scan, x)
        rmse = float(np.sqrt(np.mean((x.astype(np.float64) - ref) ** 2)))
        print(f"{s.scan.projections.shape[2]} columns in a batch: fresh FP64 cost - oracle MAP cost = "
              f"{(c - cref) / cref:.3g} relative, RMSE / range = {rmse / SCALE:.3g}")
        assert abs(c - cref) / cref < 1e-5
        assert rmse < 1e-3 * SCALE
    b.close()


def test_batch_with_device_nhicd_reaches_the_reference_map():
    # a problem whose stage asks for the NHICD pass gets it after every
    # batched sweep from its second iteration (its stage's own selection and
    # launch); the other problem of the batch does not, and both still reach
    # the MAP: the plain scenario the reference's converged cost and the FP64
    # oracle's image, as without the pass
    g = np.load(os.path.join(GOLD, "converged_plain.npz"))
    ref = float(g["ref_fresh_cost"])
    plain = make_stage(32, 4, 48, seed=1, prepare=False)
    plain.set_sv_nhicd(0.1)
    plain.prepare()
    other = make_stage(48, 6, 72, seed=11)
    b = timbir_b200.Batch([plain, other])
    assert b.iterate(300, check_every=50) == 2
    assert plain.kernel_stats()[1] == 299  # one NHICD launch per batched iteration from the second
    assert other.kernel_stats()[1] == 0
    st = b.stats()
    assert list(st["iterations"]) == [300, 300]
    assert plain.update_count() > st["updates"][0]  # the sweeps' updates and the passes'
    assert other.update_count() == st["updates"][1]
    b.close()
    x = plain.object()
    c = fresh_cost_fp64(plain.scan, x)
    assert abs(c - ref) / ref < 1e-5
    rmse = float(np.sqrt(np.mean((x - g["f64_object"]) ** 2)))
    assert rmse < 1e-3 * SCALE
    plain.close()
    other.close()
