"""Converged MAP fixtures at the benchmark sizes.

For each workload the reference library itself (oracle/_ref, the reference's
own schedule: random line orders, HICD/NHICD sub-iterations, ring offsets) is
iterated from the benchmark's warm start until its MAP cost is flat, then the
FP64 oracle (oracle/_build/liboracle64.so) continues from the reference's
result until its cost is flat to FP64 precision.  Costs are evaluated afresh
in FP64 (the reference's running cost rides on an incrementally updated float
error sinogram and drifts by about 1e-5 relative).

  3d   bench.py's 3-D workload: 256x256x8, 256 views, I0 1e4, quadratic data
       term, no ring correction, 8 z-blocks (as XT_Main_ref schedules it on 8
       or more threads).  Stores, per reference iteration, the fresh FP64 cost
       of its object (so the reference's iterations to (1 + 1e-5) C* are
       known for its timed runs), C*, and the FP64 oracle's converged object.
  4dc  bench.py's 4-D workload (16 frames of 256x256x16, 1024 interlaced
       views, zingers and rings in the data) with the convex model: quadratic
       data term (quad_convex 1), no ring correction (with ring offsets the
       reference's image-offset iteration converges too slowly to fix a C*:
       on a 32x32x4 scene 1000 of its iterations still end 4e-4 above the
       joint minimum), 2 z-blocks.  The volume is 67 MB, so the fixture keeps
       the FP64 oracle's values at 262,144 seeded voxel positions and C*; the
       FP64 oracle (single-threaded) runs at most 8 iterations from the
       reference's result here.

Each fixture records SHA-256 digests of the scan's projections and weights, so
a test can check that it regenerated the same scan.  Run from the repository
root (needs the reference library built, ``make -C oracle ref``):

    python tests/golden/make_converged_full.py 3d
    python tests/golden/make_converged_full.py 4dc
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle.bind import Oracle, Reference  # noqa: E402

SAMPLE_SEED, SAMPLE_N = 12345, 262144


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def workload(name):
    if name == "3d":
        return bench.W3D, bench.W3D.prior, 8
    return bench.W4DC, bench.W4DC.prior, 2


def switches(prior):
    return bench.finest_stage_switches(prior)


def fresh_cost(scan, prior, blocks, x, d=None):
    o = Oracle(scan, **prior, blocks=blocks, f64=True)
    o.prepare(x, d)
    c = o.cost()[0]
    o.close()
    return c


def sample_positions(shape):
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(int(np.prod(shape)), SAMPLE_N, replace=False)).astype(np.int64)


def main(name):
    w, prior, blocks = workload(name)
    t0 = time.time()
    scan = w.scan(0)
    _, fine = w.warm_start(scan)
    print(f"[{name}] scan {time.time() - t0:.1f} s", flush=True)
    sw = switches(prior)

    # ---- the reference, to a flat cost ----
    R = Reference(scan, **prior, blocks=blocks, workdir=tempfile.mkdtemp())
    if sw:
        R.set_switches(**sw)
    zero_d = np.zeros((scan.proj_cols, scan.proj_rows), np.float32)
    R.prepare(fine, zero_d if prior["remove_rings"] else None)
    running, fresh = [], []
    track_fresh = name == "3d"
    max_iters = 300 if name == "3d" else 400
    for it in range(1, max_iters + 1):
        t = time.time()
        R.iterate(it)
        running.append(R.cost()[0])
        if track_fresh:
            fresh.append(fresh_cost(scan, prior, blocks, R.object()))
        c = fresh[-1] if track_fresh else running[-1]
        print(f"[{name}] reference iteration {it}: cost {c:.12g} ({time.time() - t:.1f} s)", flush=True)
        hist = fresh if track_fresh else running
        if it > 10 and abs(hist[-6] - hist[-1]) <= 1e-9 * abs(hist[-1]):
            break
    ref_iters = it
    x_ref, d_ref = R.object(), R.offset()
    ref_fresh = fresh[-1] if track_fresh else fresh_cost(scan, prior, blocks, x_ref, d_ref)
    R.close()
    print(f"[{name}] reference: {ref_iters} iterations, fresh FP64 cost {ref_fresh:.12g}", flush=True)

    # ---- the FP64 oracle, from the reference's result, to FP64 flatness ----
    O = Oracle(scan, **prior, blocks=blocks, f64=True)
    if sw:
        O.set_switches(**sw)
    O.prepare(x_ref, d_ref if prior["remove_rings"] else None)
    f64_costs = [O.cost()[0]]
    for it in range(1, (61 if name == "3d" else 9)):
        t = time.time()
        O.iterate(it)
        f64_costs.append(O.cost()[0])
        print(f"[{name}] FP64 oracle iteration {it}: cost {f64_costs[-1]:.15g} ({time.time() - t:.1f} s)",
              flush=True)
        if abs(f64_costs[-2] - f64_costs[-1]) <= 1e-13 * abs(f64_costs[-1]):
            break
    x64, d64 = O.object(), O.offset()
    O.close()
    f64_fresh = fresh_cost(scan, prior, blocks, x64, d64 if prior["remove_rings"] else None)
    cstar = min(ref_fresh, f64_fresh)
    out = dict(proj_sha256=digest(scan.projections), weight_sha256=digest(scan.weights),
               prior=str(sorted(prior.items())), blocks=blocks, ref_iterations=ref_iters,
               ref_running_costs=np.array(running), ref_fresh_cost=ref_fresh, f64_costs=np.array(f64_costs),
               f64_fresh_cost=f64_fresh, cstar=cstar, f64_offset=d64, ref_offset=d_ref,
               value_range=float(x64.max() - x64.min()))
    if track_fresh:
        fr = np.array(fresh)
        out["ref_fresh_costs"] = fr
        hit = np.flatnonzero(fr <= (1.0 + 1e-5) * cstar)
        out["ref_iterations_to_target"] = int(hit[0]) + 1 if len(hit) else -1
        out["f64_object"] = x64.astype(np.float32)
    else:
        pos = sample_positions(x64.shape)
        out["sample_seed"], out["sample_n"] = SAMPLE_SEED, SAMPLE_N
        out["f64_sample"] = x64.reshape(-1)[pos].astype(np.float32)
        out["ref_sample"] = x_ref.reshape(-1)[pos].astype(np.float32)
    path = os.path.join(HERE, f"converged_{name}.npz")
    np.savez_compressed(path, **out)
    rmse = float(np.sqrt(np.mean((x_ref.astype(np.float64) - x64) ** 2)))
    print(f"[{name}] C* {cstar:.12g}; reference vs FP64 oracle: cost rel {abs(ref_fresh - f64_fresh) / f64_fresh:.3g}, "
          f"RMSE / range {rmse / out['value_range']:.3g}; "
          f"{out.get('ref_iterations_to_target', '-')} reference iterations to (1 + 1e-5) C*; wrote {path} "
          f"({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    for n in sys.argv[1:] or ["3d", "4dc"]:
        main(n)
