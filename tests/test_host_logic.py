"""CPU tests of host-side logic: the many-problem workload's seeded sizes,
the batched kernel's warp split, and the device (torch) scan generator
against the numpy one."""
import numpy as np

import timbir_b200
from timbir_b200 import synth


def test_batch_problem_specs_follow_the_workload_definition():
    a = synth.batch_problem_specs(64, 0)
    b = synth.batch_problem_specs(64, 0)
    assert a == b and len(a) == 64
    for k, sp in enumerate(a):
        assert sp["side"] in (128, 192, 256, 384, 512)
        assert sp["slices"] % 2 == 0 and 4 <= sp["slices"] <= 32
        assert sp["views"] == 3 * sp["side"] // 2
        assert 2e3 <= sp["I0"] <= 5e4 and sp["seed"] == k
    assert len({sp["side"] for sp in a}) == 5


def test_batch_split_fills_eight_warps_where_the_stack_allows():
    assert timbir_b200.batch_split(1, 8) == (1, 8)
    assert timbir_b200.batch_split(1, 32) == (1, 8)
    assert timbir_b200.batch_split(1, 4) == (2, 4)
    assert timbir_b200.batch_split(1, 2) == (4, 2)
    assert timbir_b200.batch_split(2, 16) == (2, 4)
    assert timbir_b200.batch_split(4, 22) == (4, 2)
    assert timbir_b200.batch_split(4, 1) == (4, 1)  # one slice: 4 warps at most


def test_device_scan_generator_matches_numpy():
    a = synth.ellipsoid_scan(32, 4, 48, seed=1)
    b = synth.ellipsoid_scan_device(32, 4, 48, seed=1, device="cpu")
    assert np.array_equal(a.projections, b.projections)
    assert np.array_equal(a.weights, b.weights)
    assert np.array_equal(a.proj_angles, b.proj_angles)
    assert b.phantom is None
