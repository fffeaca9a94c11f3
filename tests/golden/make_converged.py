"""Converged MAP fixture for the super-voxel schedule's parity test.

Runs the "plain" scenario of tests/scenarios.py (32x32x4, 48 views, quadratic
data term, a single stage at full resolution) to convergence with
  * the reference library itself (oracle/_ref, float arrays), and
  * the FP64 oracle (oracle/_build/liboracle64.so),
300 reference-schedule iterations each, and stores the final MAP costs and
objects in converged_plain.npz.  Run from the repository root:

    python tests/golden/make_converged.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import scenarios  # noqa: E402
from oracle.bind import Oracle, Reference  # noqa: E402

ITERS = 300


def run(obj):
    obj.prepare()
    for it in range(1, ITERS + 1):
        obj.iterate(it)
    return obj.cost()[0], obj.object()


if __name__ == "__main__":
    ref_cost, ref_obj = run(scenarios.make("plain", Reference, workdir=tempfile.mkdtemp()))
    o64_cost, o64_obj = run(scenarios.make("plain", Oracle, f64=True))
    # the running costs ride on incrementally updated error sinograms (float
    # drift in the reference); evaluate both objects afresh in FP64
    def fresh_cost(x):
        o = scenarios.make("plain", Oracle, f64=True)
        o.prepare(x)
        return o.cost()[0]

    ref_fresh, o64_fresh = fresh_cost(ref_obj), fresh_cost(o64_obj)
    np.savez_compressed(os.path.join(HERE, "converged_plain.npz"), ref_cost=ref_cost, ref_object=ref_obj,
                        f64_cost=o64_cost, f64_object=o64_obj, ref_fresh_cost=ref_fresh,
                        f64_fresh_cost=o64_fresh, iterations=ITERS)
    print("running: reference", ref_cost, "fp64 oracle", o64_cost)
    print("fresh FP64 cost: reference object", ref_fresh, "fp64 object", o64_fresh,
          "rel", abs(ref_fresh - o64_fresh) / o64_fresh, "max|dx|", float(np.abs(ref_obj - o64_obj).max()))
