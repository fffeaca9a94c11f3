"""Parity of the default super-voxel schedule at the benchmark sizes.

The super-voxel schedule's trajectory differs from the reference's, so parity
is checked on the MAP estimate it converges to, at the full sizes the
benchmark runs (fixtures from tests/golden/make_converged_full.py: the
reference library iterated to a flat cost, then the FP64 oracle from there):

  * 3-D workload (256x256x8, 256 views, I0 1e4, quadratic data term): the
    fresh FP64 cost (FP64 oracle, error sinogram recomputed from the object)
    within 1e-5 relative of C*, the converged cost of the reference / FP64
    oracle, and image RMSE against the FP64 oracle's converged image below
    1e-3 of its range -- with FP32 and with FP16 A-matrix values;
  * convex 4-D workload (16 frames of 256x256x16, 1024 interlaced views,
    zingers and rings in the data, quadratic data term, no ring correction:
    the reference's zero-mean ring-offset iteration creeps too slowly to fix
    a C* at this size): the GPU's fresh cost (error sinogram recomputed from
    the object, FP64 sums) within 1e-5 relative of C*, and RMSE at
    262,144 seeded voxel positions against the FP64 oracle below 1e-3 of
    the range -- with FP32 and with FP16 A-matrix values.

Each test first checks that it regenerated the fixture's scan (SHA-256 of the
projections and weights).  The schedule is the default one: automatic
super-voxel side, z-group, over-relaxation and grid.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

import timbir_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
from oracle.bind import Oracle  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def fixture(name):
    path = os.path.join(GOLD, f"converged_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated")
    return np.load(path)


class _Args:
    sv_side = 0
    warps_per_slice = 0
    zgroup = 0

    def __init__(self, acache):
        self.acache = acache


def converge(w, scan, start, acache, max_iters=400, flat=1e-9):
    """Default super-voxel schedule from `start` until the cost is flat
    (relative change below `flat` over five iterations); returns the stage."""
    st = bench.workload_stage(w, scan, 1, _Args(acache))
    st.prepare(start, bench.zero_offsets(scan) if w.prior["remove_rings"] else None)
    hist = []
    for it in range(1, max_iters + 1):
        st.iterate(it)
        hist.append(st.cost()[0])
        if it > 10 and abs(hist[-6] - hist[-1]) <= flat * abs(hist[-1]):
            break
    return st, it


@pytest.mark.parametrize("acache", [-1, 2], ids=["fp32_a", "fp16_a"])
def test_3d_workload_reaches_the_reference_map(acache):
    g = fixture("3d")
    w = bench.W3D
    scan = w.scan(0)
    assert digest(scan.projections) == str(g["proj_sha256"]) and digest(scan.weights) == str(g["weight_sha256"])
    _, fine = w.warm_start(scan)
    st, iters = converge(w, scan, fine, acache)
    assert (st.schedule_info()["column_cache_values"] == "fp16") == (acache == 2)
    x = st.object()
    st.close()
    o = Oracle(scan, **w.prior, blocks=int(g["blocks"]), f64=True)
    o.prepare(x)
    c = o.cost()[0]
    o.close()
    cstar, rng = float(g["cstar"]), float(g["value_range"])
    rel = (c - cstar) / cstar
    rmse = float(np.sqrt(np.mean((x.astype(np.float64) - g["f64_object"]) ** 2))) / rng
    print(f"3-D {'FP16' if acache == 2 else 'FP32'} A: {iters} iterations, fresh FP64 cost - C* = {rel:.3g} relative, "
          f"RMSE / range vs FP64 oracle = {rmse:.3g}")
    assert abs(rel) < 1e-5
    assert rmse < 1e-3


@pytest.mark.parametrize("acache", [-1, 2], ids=["fp32_a", "fp16_a"])
def test_convex_4d_workload_reaches_the_reference_map(acache):
    g = fixture("4dc")
    w = bench.W4DC
    scan = w.scan(0)
    assert digest(scan.projections) == str(g["proj_sha256"]) and digest(scan.weights) == str(g["weight_sha256"])
    _, fine = w.warm_start(scan)
    st, iters = converge(w, scan, fine, acache, max_iters=1500)
    assert (st.schedule_info()["column_cache_values"] == "fp16") == (acache == 2)
    x, d = st.object(), st.offset()
    st.close()
    # fresh cost: a new stage's error sinogram y - A x - d from the object and
    # offsets (FP32 forward projection), its cost summed in FP64
    f = bench.workload_stage(w, scan, 1, _Args(-1))
    f.prepare(x, d)
    c = f.cost()[0]
    f.close()
    cstar, rng = float(g["cstar"]), float(g["value_range"])
    rs = np.random.default_rng(int(g["sample_seed"]))
    pos = np.sort(rs.choice(x.size, int(g["sample_n"]), replace=False))
    rel = (c - cstar) / cstar
    rmse = float(np.sqrt(np.mean((x.reshape(-1)[pos].astype(np.float64) - g["f64_sample"]) ** 2))) / rng
    print(f"convex 4-D {'FP16' if acache == 2 else 'FP32'} A: {iters} iterations, fresh cost - C* = {rel:.3g} "
          f"relative, RMSE / range vs FP64 oracle (sampled) = {rmse:.3g}")
    assert abs(rel) < 1e-5
    assert rmse < 1e-3
