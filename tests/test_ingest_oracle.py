"""The data-ingestion oracle (oracle/ingest.py) against the reference's own
readers and view generator (tests/golden/ingest.npz, made by
tests/golden/make_golden.py ingest from the reference's sources), bit for
bit; and the library's interlaced view generator (host code) against the
same fixtures."""
import numpy as np
import pytest

from oracle import ingest as O

G = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ingest.npz"))
CASES = sorted({k.split("/")[0] for k in G.files if not k.startswith("views")})
VIEWS = sorted({k.split("/")[0] for k in G.files if k.startswith("views")})


def params(name):
    return [int(x) for x in G[f"{name}/params"]]


@pytest.mark.parametrize("name", CASES)
def test_oracle_normalisation_matches_the_reference(name):
    n, rows, cols, nw, nd, r0, pr, pc, ps, pn = params(name)
    P, W = O.normalize_counts(G[f"{name}/counts"], G[f"{name}/whites"], G[f"{name}/darks"], pr, pc, ps, pn, r0)
    assert np.array_equal(P, G[f"{name}/aps_proj"])
    assert np.array_equal(W, G[f"{name}/aps_weight"])
    Ps, Ws = O.downsample_projections(G[f"{name}/std_in_proj"], G[f"{name}/std_in_weight"], pr, pc, ps, pn, r0)
    assert np.array_equal(Ps, G[f"{name}/std_proj"])
    assert np.array_equal(Ws, G[f"{name}/std_weight"])


@pytest.mark.parametrize("name", VIEWS)
def test_view_generators_match_the_reference(name):
    from timbir_b200 import ingest
    K, Nt, ps, npv, mat, rs = G[f"{name}/params"]
    for gen in (O.interlaced_views, ingest.interlaced_views):
        a, t, kept = gen(int(K), int(Nt), int(npv), int(ps), float(mat), float(rs))
        assert np.array_equal(a, G[f"{name}/angles"])
        assert np.array_equal(t, G[f"{name}/times"])
        assert kept == int(G[f"{name}/kept"])


def test_refused_ingestion_inputs_fail_before_any_device_work():
    # the readers' checks run on the host, before any CUDA call, so they hold
    # on a machine without a GPU too
    from timbir_b200 import ingest
    counts = np.zeros((4, 8, 16), np.uint16)
    stack = np.zeros((5, 8, 16), np.uint16)
    with pytest.raises(RuntimeError, match="rows"):  # 16 rows x ratio 1 > 8 in the file
        ingest.normalize_counts(counts, stack, stack, 16, 16)
    with pytest.raises(RuntimeError, match="ranks"):  # 8 rows over 3 ranks
        ingest.normalize_counts(counts, stack, stack, 8, 16, ranks=3)
    with pytest.raises(RuntimeError, match="columns"):  # more output columns than the file has
        ingest.normalize_counts(counts, stack, stack, 8, 32)
    with pytest.raises(RuntimeError, match="3 frames"):
        ingest.normalize_counts(counts, stack[:2], stack, 8, 16)
    with pytest.raises(RuntimeError, match="proj_start"):
        ingest.normalize_counts(counts, stack, stack, 8, 16, proj_start=2, proj_num=3)
    with pytest.raises(ValueError):
        ingest.interlaced_views(0, 16, 4)
