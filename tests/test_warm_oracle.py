"""CPU checks of the learned warm start's oracle (oracle/warm_net.py): its
hand-written backward pass against central differences of its own loss, and
BF16 rounding to nearest even."""
import numpy as np
import pytest

from oracle import warm_net as W


def random_params(rng):
    flat = np.zeros(W.param_count())
    off = 0
    for ci, co in W.LAYERS:
        flat[off:off + 27 * ci * co] = rng.normal(0, np.sqrt(2.0 / (27 * ci)), 27 * ci * co)
        off += 27 * ci * co
        flat[off:off + co] = rng.normal(0, 0.05, co)
        off += co
    return flat


@pytest.mark.parametrize("loss", ["plain", "weighted", "highpass"])
def test_oracle_gradients_match_finite_differences(loss):
    rng = np.random.default_rng(0)
    flat = random_params(rng)
    fbp = rng.random((1, 8, 16, 16)) * 0.02
    tgt = fbp + rng.normal(0, 0.002, fbp.shape)
    wts = rng.uniform(0.5, 4.0, fbp.shape) if loss != "plain" else None
    hp = (1.0, 2.0) if loss == "highpass" else None
    loss, g = W.grads_exact(flat, fbp, tgt, 50.0, weights=wts, highpass=hp)
    assert loss > 0
    # parameters with a gradient, from first, middle and last layers
    live = np.nonzero(np.abs(g) > 1e-6 * np.abs(g).max())[0]
    idx = np.concatenate([live[:3], live[len(live) // 2:len(live) // 2 + 3], live[-3:],
                          rng.choice(live, 6, replace=False)])
    # a small step keeps ReLU inputs near zero from changing sign
    fd = W.finite_difference(flat, fbp, tgt, 50.0, idx, h=1e-7, weights=wts, highpass=hp)
    assert np.allclose(g[idx], fd, rtol=1e-4, atol=1e-8 * np.abs(g).max())


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = W.bf16(x)
    # 1 + 2^-8 is half-way between 1 and 1 + 2^-7: ties to even (1)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0 and r[4] == -2.5
    assert abs(r[5] - 3.0e-3) / 3.0e-3 < 2 ** -8


def test_fbp_oracle_reconstructs_the_phantom():
    # the restatement is a reconstruction: within 6 % RMSE of the phantom's
    # range on the small scan, zero outside the reconstruction disc
    from oracle import fbp as F
    from timbir_b200 import synth
    scan = synth.ellipsoid_scan(32, 4, 48, seed=1)
    x = F.fbp(scan)
    assert x.shape == scan.phantom.shape
    assert np.sqrt(np.mean((x - scan.phantom) ** 2)) < 0.06 * 0.02
    k = np.arange(32) + 0.5 - 16
    outside = (k[None, :] ** 2 + k[:, None] ** 2) >= 16 ** 2
    assert np.all(x[..., outside] == 0)


def test_package_layer_table_matches_the_oracle():
    from timbir_b200 import warm
    assert [(ci, co) for ci, co, _ in warm.LAYERS] == W.LAYERS
    assert sum(27 * ci * co + co for ci, co, _ in warm.LAYERS) == W.param_count() == 1327824
