"""Pins the CPU oracle (oracle/mbir_oracle.c) to the reference.

* against the reference's own known-answer table for its generator
  (src/MBIR_4D/randlib.c:69-90), kept in tests/golden/park_miller_seed1.json;
* against golden fixtures that the reference library produced
  (tests/golden/make_golden.py): detector response, mask, initial error
  sinogram and cost, and the full state after ICD iterations 1 and 3 of the
  reference schedule, for every scenario of tests/scenarios.py.  Single-threaded
  float arithmetic in the same order as the reference, so the comparison is
  bit for bit; only the variance estimate, which the reference reduces with
  OpenMP, is compared to 1e-12;
* against the live reference build when it is present (oracle/_ref).
"""
import json
import os
import tempfile

import numpy as np
import pytest

import scenarios
from oracle.bind import Oracle, Reference

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_park_miller_known_answers(oracle_built):
    tab = json.load(open(os.path.join(GOLD, "park_miller_seed1.json")))
    o = scenarios.make("plain", Oracle)
    o.srandom2(tab["seed"])
    got = [round(o.random2() * 2147483647) for _ in range(20)]
    assert got == tab["values"]


def test_order_statistic_matches_sort(oracle_built):
    o = scenarios.make("plain", Oracle)
    rng = np.random.default_rng(0)
    for n in (1, 2, 7, 100, 1000):
        a = rng.random(n).astype(np.float32)
        a[rng.integers(0, n, n // 3)] = 0.0  # ties, as the zero update map has
        for i in sorted({1, n, (n + 1) // 2}):
            assert o.randomized_select(a, i) == np.sort(a)[i - 1]


@pytest.mark.parametrize("name", list(scenarios.SCENARIOS))
def test_oracle_matches_reference_golden(oracle_built, name):
    g = np.load(os.path.join(GOLD, f"stage_{name}.npz"))
    o = scenarios.make(name, Oracle)
    o.prepare()
    np.testing.assert_array_equal(o.hr(), g["hr"])
    np.testing.assert_array_equal(o.mask()[0], g["mask"])
    np.testing.assert_array_equal(o.errorsino(), g["e0"])
    assert o.cost()[0] == pytest.approx(float(g["cost0"]), rel=1e-12)
    for it in (1, 2, 3):
        conv = o.iterate(it)
        if it in (1, 3):
            np.testing.assert_array_equal(o.object(), g[f"obj{it}"])
            assert conv == int(g[f"conv{it}"])
            assert o.var_est() == pytest.approx(float(g[f"var{it}"]), rel=1e-12)
    np.testing.assert_array_equal(o.errorsino(), g["e3"])
    np.testing.assert_array_equal(o.offset(), g["offset3"])
    assert o.cost()[0] == pytest.approx(float(g["cost3"]), rel=1e-12)
    for kind, key in ((0, "hicd"), (1, "nhicd")):
        xs, ys = o.lines(kind, 0, 0)
        np.testing.assert_array_equal(xs, g[f"{key}_x3"])
        np.testing.assert_array_equal(ys, g[f"{key}_y3"])


@pytest.mark.parametrize("name", ["plain", "frames4"])
def test_oracle_matches_live_reference(oracle_built, reference_available, name):
    R = scenarios.make(name, Reference, workdir=tempfile.mkdtemp())
    o = scenarios.make(name, Oracle)
    np.testing.assert_array_equal(o.scalars(), R.scalars())
    for f in range(o.N_time):
        np.testing.assert_array_equal(o.view_map(f), R.view_map(f))
    R.prepare()
    o.prepare()
    for (row, col, view) in [(0, 0, 0), (3, 5, 7), (16, 16, 0), (31, 0, o.N_p - 1), (10, 20, 13)]:
        ri, rv = R.amatrix(row, col, view)
        oi, ov = o.amatrix(row, col, view)
        np.testing.assert_array_equal(oi, ri)
        np.testing.assert_array_equal(ov, rv)
    for it in (1, 2):
        assert o.iterate(it) == R.iterate(it)
        np.testing.assert_array_equal(o.object(), R.object())
        np.testing.assert_array_equal(o.errorsino(), R.errorsino())


def test_functional_substitution_matches_reference(oracle_built, reference_available):
    R = scenarios.make("frames4", Reference, workdir=tempfile.mkdtemp())
    o = scenarios.make("frames4", Oracle)
    rng = np.random.default_rng(3)
    for _ in range(50):
        sn = rng.normal(0.01, 0.005, 27)
        sf = (rng.random(27) < 0.8).astype(np.uint8)
        tn = rng.normal(0.01, 0.005, 2)
        tf = (rng.random(2) < 0.7).astype(np.uint8)
        V = float(sn[13]) if rng.random() < 0.2 else float(rng.normal(0.01, 0.005))
        sn[3] = V  # a zero difference exercises the rho''(0) branch
        th1, th2 = rng.normal(0, 10), abs(rng.normal(100, 10))
        assert o.functional_substitution(V, th1, th2, sn, sf, tn, tf) == \
            R.functional_substitution(V, th1, th2, sn, sf, tn, tf)
