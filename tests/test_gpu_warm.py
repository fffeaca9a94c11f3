"""GPU tests of the learned warm start: the filtered backprojection and the
network's forward pass, parameter gradients and Adam step against the CPU
oracles (oracle/fbp.py, oracle/warm_net.py), and what a trained network
gains over the filtered backprojection as the start of ICD (a start closer
to the MAP image).

Tolerances: the network's tensor-core products take BF16 operands (the
oracle rounds the same operands to BF16) and accumulate in FP32 inside the
tensor cores, which is not IEEE round-to-nearest; every activation and
gradient is stored in BF16 (the residual output too, a relative rounding of
up to 2^-9 per value), and the skip additions, pooling and up-sampling act on
those BF16 values where the oracle keeps FP64 (measured: about 7e-3 relative
L2 at the output of the 15 layers).  Outputs and gradients are therefore
compared by relative L2 error, per layer, below 1e-2; the backward pass is
checked at the GPU's own layer outputs.
"""
import numpy as np
import pytest

import scenarios
import timbir_b200
from oracle import fbp as fbp_oracle
from oracle import warm_net as W
from timbir_b200 import synth
from timbir_b200 import warm

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def random_params(seed):
    rng = np.random.default_rng(seed)
    flat = np.zeros(W.param_count(), np.float32)
    off = 0
    for ci, co in W.LAYERS:
        flat[off:off + 27 * ci * co] = rng.normal(0, np.sqrt(2.0 / (27 * ci)), 27 * ci * co)
        off += 27 * ci * co
        flat[off:off + co] = rng.normal(0, 0.05, co)
        off += co
    return flat


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def inputs(seed, shape=(2, 8, 16, 16)):
    rng = np.random.default_rng(seed)
    fbp = (rng.random(shape) * 0.02).astype(np.float32)
    tgt = (fbp + rng.normal(0, 0.002, shape)).astype(np.float32)
    return fbp, tgt


def test_fbp_matches_the_oracle():
    scan = synth.ellipsoid_scan(32, 4, 48, seed=1)
    s = timbir_b200.Stage(scan, blocks=2, **scenarios.BASE)
    x = s.fbp()
    ref = fbp_oracle.fbp(scan)
    assert x.shape == ref.shape
    assert np.abs(x - ref).max() < 1e-4 * np.abs(ref).max()
    # and it is a reconstruction: within 10 % RMSE of the phantom's range
    assert np.sqrt(np.mean((x - scan.phantom) ** 2)) < 0.1 * 0.02
    s.close()


def test_network_forward_matches_the_oracle():
    net = warm.WarmNet(0)
    p = random_params(1)
    net.set_params(p)
    assert np.array_equal(net.params(), p)
    fbp, _ = inputs(2)
    out = net.forward(torch.from_numpy(fbp).cuda()).cpu().numpy()
    r_gpu = (out.astype(np.float64) - fbp) * warm.SCALE
    r_ref, A = W.forward(p, fbp, warm.SCALE)
    assert rel(r_gpu, r_ref) < 1e-2
    for k in range(15):
        assert rel(net.activation(k), A[k].reshape(-1)) < 1e-2, k
    net.close()


LEVEL = [0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0, 0]


def gpu_activations(net, shape):
    """The network's stored layer outputs, channels-last, by layer."""
    B, D, H, Wd = shape
    acts = {"x0": net.activation(-1).reshape(B, D, H, Wd, 16)}
    for k, (ci, co) in enumerate(W.LAYERS):
        lv = LEVEL[k]
        acts[k] = net.activation(k).reshape(B, D >> lv, H >> lv, Wd >> lv, co)
    return acts


@pytest.mark.parametrize("loss_kind", ["plain", "weighted", "highpass"])
def test_network_gradients_match_the_oracle(loss_kind):
    # the backward pass on its own: the oracle differentiates at the GPU's
    # own layer outputs (a forward difference near a ReLU's kink would
    # otherwise flip its mask on one side only); weighted: per-voxel loss
    # weights; highpass: weights and the residual's high frequencies
    net = warm.WarmNet(0)
    p = random_params(3)
    net.set_params(p)
    fbp, tgt = inputs(4)
    weighted = loss_kind != "plain"
    hp = (1.0, 2.0) if loss_kind == "highpass" else None
    wts = np.random.default_rng(5).uniform(0.5, 4.0, fbp.shape).astype(np.float32) if weighted else None
    net.set_loss_weights(torch.from_numpy(wts).cuda() if weighted else None)
    net.set_loss_highpass(*(hp or (0.0, 0.0)))
    loss = net.gradients(torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda())
    net.set_loss_weights(None)
    net.set_loss_highpass(0.0, 0.0)
    g = net.grads()
    trace = {}
    loss_ref, g_ref = W.loss_and_grads(p, fbp, tgt, warm.SCALE, trace, gpu_activations(net, fbp.shape), weights=wts,
                                       highpass=hp)
    assert abs(loss - loss_ref) < 1e-4 * loss_ref
    for k in range(15):  # each layer's output gradient (after its ReLU's mask)
        assert rel(net.activation(k, grad=True), trace[k].reshape(-1)) < 1e-2, k
    off = 0
    for k, (ci, co) in enumerate(W.LAYERS):
        nw = 27 * ci * co
        if np.linalg.norm(g_ref[off:off + nw]) > 0:
            assert rel(g[off:off + nw], g_ref[off:off + nw]) < 1e-2, k
        # a bias gradient is a sum of the layer's BF16 output gradient over the
        # voxels; under the high-pass loss the last layer's nearly cancels
        # (a high-pass has no mean), so it is also accepted within twice the
        # BF16 rounding of the terms it sums (per channel)
        a, b = g[off + nw:off + nw + co], g_ref[off + nw:off + nw + co]
        l1 = np.abs(trace[k]).reshape(-1, co).sum(axis=0)
        if np.linalg.norm(b) > 0:
            assert rel(a, b) < 1e-2 or np.all(np.abs(a - b) <= 2.0 ** -8 * l1), k
        off += nw + co
    net.close()


def test_adam_step_matches_the_oracle():
    net = warm.WarmNet(0)
    p = random_params(5)
    net.set_params(p)
    fbp, tgt = inputs(6)
    x, t = torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda()
    net.gradients(x, t)
    g1 = net.grads().astype(np.float64)
    net.adam_step(1e-3)
    net.gradients(x, t)
    g2 = net.grads().astype(np.float64)
    net.adam_step(5e-4)
    m = v = np.zeros_like(g1)
    q, m, v = W.adam(p.astype(np.float64), g1, m, v, 1, 1e-3)
    q, m, v = W.adam(q, g2, m, v, 2, 5e-4)
    assert np.abs(net.params() - q).max() < 1e-6
    net.close()


def test_training_reduces_the_loss():
    # a learnable map (the target is the input scaled by 0.8)
    fbp, _ = inputs(7, (4, 8, 16, 16))
    tgt = (0.8 * fbp).astype(np.float32)
    net = warm.WarmNet(1)
    x, t = torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda()
    losses = warm.train(net, x, t, steps=60, batch=2, patch=(8, 16, 16), lr=2e-3)
    assert np.mean(losses[-10:]) < 0.5 * np.mean(losses[:5])
    net.close()


def _scan_and_map(seed, n_xy=64, rows=16, views=96):
    """A seeded random-ellipsoid scan, its filtered backprojection and its MAP
    image (super-voxel schedule from the FBP to a flat cost)."""
    scan = synth.ellipsoid_scan(n_xy, rows, views, I0=1e4, seed=seed)
    prior = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=0, quad_convex=1)
    st = timbir_b200.Stage(scan, blocks=2, **prior)
    st.set_schedule(timbir_b200.Stage.SCHEDULE_SUPERVOXEL)
    fbp = st.fbp()
    st.prepare(fbp)
    hist = []
    for it in range(1, 800):
        st.iterate(it)
        hist.append(st.cost()[0])
        if it > 10 and abs(hist[-6] - hist[-1]) <= 1e-9 * abs(hist[-1]):
            break
    x, mask = st.object(), st.mask().astype(np.float32)
    st.close()
    return fbp, x, mask


def test_trained_network_starts_closer_to_the_map_than_fbp():
    # what the learned part gains: trained (hand-written forward, backward and
    # Adam kernels) on (FBP, converged MAP) pairs of eight seeded scans, the
    # network maps a held-out scan's FBP to a start image closer to that
    # scan's MAP image than the FBP itself (RMSE at most 0.7 of the FBP's)
    pairs = [_scan_and_map(300 + k) for k in range(8)]
    X = torch.from_numpy(np.concatenate([p[0] for p in pairs])).cuda()
    T = torch.from_numpy(np.concatenate([p[1] for p in pairs])).cuda()
    net = warm.WarmNet(seed=7)
    losses = warm.train(net, X, T, steps=400, batch=4, patch=(16, 32, 32), lr=1e-3, seed=3)
    assert np.mean(losses[-20:]) < np.mean(losses[:20])
    fbp, x_map, mask = _scan_and_map(999)
    start = warm.warm_start(net, fbp, mask, blend=None)  # the network's own output
    net.close()
    rmse = lambda a: float(np.sqrt(np.mean((a.astype(np.float64) - x_map) ** 2)))  # noqa: E731
    print(f"held-out scan: RMSE to the MAP image, FBP {rmse(fbp):.3g}, network {rmse(start):.3g}")
    assert rmse(start) < 0.7 * rmse(fbp)


@pytest.mark.parametrize("sig", [(1.0, 4.0), (0.0, 2.5), (2.0, 0.0)])
def test_lowpass_blend_matches_scipy(sig):
    # start + G (ref - start), G the Gaussian low-pass with scipy.ndimage's
    # truncation (4 sigma) and mirrored edges, per volume
    from scipy import ndimage
    rng = np.random.default_rng(9)
    ref = rng.random((2, 8, 40, 24)).astype(np.float32)
    start = rng.random((2, 8, 40, 24)).astype(np.float32)
    want = start.astype(np.float64) + ndimage.gaussian_filter((ref - start).astype(np.float64),
                                                              sigma=(0, sig[0], sig[1], sig[1]), mode="reflect")
    s = torch.from_numpy(start).cuda()
    warm.lowpass_blend(torch.from_numpy(ref).cuda(), s, *sig)
    got = s.cpu().numpy()
    assert np.abs(got - want).max() < 1e-5 * np.abs(want).max()
