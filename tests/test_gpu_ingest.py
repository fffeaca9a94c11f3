"""Data ingestion on the GPU (mbir_normalize_counts,
mbir_downsample_projections): against the reference's readers
(tests/golden/ingest.npz) and, at larger sizes and over rank splits, against
the oracle (oracle/ingest.py, itself pinned to the reference bit for bit).
Projections and weights are compared bit for bit, except that the APS
projections may differ by one float ulp where CUDA's double log and the host
library's round a double differently (counted: at most 1 in 1e4 samples)."""
import numpy as np
import pytest

from oracle import ingest as O
from timbir_b200 import ingest

pytestmark = pytest.mark.gpu

import os  # noqa: E402
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "ingest.npz"))
CASES = sorted({k.split("/")[0] for k in G.files if not k.startswith("views")})


def ulps(a, b):
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


def close_in_ulps(a, b):
    d = ulps(a, b)
    return d.max() <= 1 and np.count_nonzero(d) <= max(1, d.size // 10000)


@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_the_reference_readers(name):
    n, rows, cols, nw, nd, r0, pr, pc, ps, pn = [int(x) for x in G[f"{name}/params"]]
    P, W = ingest.normalize_counts(G[f"{name}/counts"], G[f"{name}/whites"], G[f"{name}/darks"], pr, pc, ps, pn, r0)
    assert np.array_equal(W, G[f"{name}/aps_weight"])
    assert close_in_ulps(P, G[f"{name}/aps_proj"])
    Ps, Ws = ingest.downsample_projections(G[f"{name}/std_in_proj"], G[f"{name}/std_in_weight"], pr, pc, ps, pn, r0)
    assert np.array_equal(Ps, G[f"{name}/std_proj"])
    assert np.array_equal(Ws, G[f"{name}/std_weight"])


def scan(seed, n=24, rows=64, cols=203, nw=7, nd=6):
    rng = np.random.default_rng(seed)
    counts = rng.integers(20, 30000, size=(n, rows, cols)).astype(np.uint16)
    whites = rng.integers(30000, 40000, size=(nw, rows, cols)).astype(np.uint16)
    darks = rng.integers(0, 100, size=(nd, rows, cols)).astype(np.uint16)
    return counts, whites, darks


def test_gpu_matches_the_oracle_and_splits_over_ranks():
    counts, whites, darks = scan(5)
    # 203 columns: 3 trimmed, ratio 4; 12 output rows = raw rows 2 .. 49; views 3 .. 21
    pr, pc, ps, pn, r0 = 12, 50, 3, 19, 2
    P, W = ingest.normalize_counts(counts, whites, darks, pr, pc, ps, pn, r0)
    Po, Wo = O.normalize_counts(counts, whites, darks, pr, pc, ps, pn, r0)
    assert np.array_equal(W, Wo)
    assert close_in_ulps(P, Po)
    parts = [ingest.normalize_counts(counts, whites, darks, pr, pc, ps, pn, r0, rank=r, ranks=3) for r in range(3)]
    assert np.array_equal(np.concatenate([p[0] for p in parts], axis=1), P)
    assert np.array_equal(np.concatenate([p[1] for p in parts], axis=1), W)


def test_dead_pixels_and_edge_cases():
    counts, whites, darks = scan(6, n=4, rows=8, cols=16)
    counts[0, :2, :2] = darks[1:-1, :2, :2].mean(axis=0).round().astype(np.uint16)  # counts at the dark level
    P, W = ingest.normalize_counts(counts, whites, darks, 8, 16)
    Po, Wo = O.normalize_counts(counts, whites, darks, 8, 16, 0, 4)
    assert np.array_equal(W, Wo)
    same = (P == Po) | (np.isnan(P) & np.isnan(Po)) | (np.isinf(P) & np.isinf(Po) & (np.sign(P) == np.sign(Po)))
    assert same.sum() >= P.size - max(1, P.size // 10000)
    # zero views
    P0, W0 = ingest.normalize_counts(counts, whites, darks, 8, 16, 0, 0)
    assert P0.shape == (0, 8, 16)
    with pytest.raises(RuntimeError):  # rows beyond the file
        ingest.normalize_counts(counts, whites, darks, 16, 16)
    with pytest.raises(RuntimeError):  # proj_rows not a multiple of the ranks
        ingest.normalize_counts(counts, whites, darks, 8, 16, ranks=3)
    with pytest.raises(RuntimeError):  # the bright stack needs 3 frames
        ingest.normalize_counts(counts, whites[:2], darks, 8, 16)
