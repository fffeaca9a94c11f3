"""GPU tests of the learned warm start: the filtered backprojection and the
network's forward pass, parameter gradients and Adam step against the CPU
oracles (oracle/fbp.py, oracle/warm_net.py), and what a trained network
gains over FBP-initialised ICD.

Tolerances: the network's tensor-core products take BF16 operands (the
oracle rounds the same operands to BF16) and accumulate in FP32 (the oracle
in FP64); an activation that lands within an FP32 rounding of a BF16
rounding boundary rounds differently on the two sides, so outputs and
gradients are compared by relative L2 error (< 5e-3), not bit for bit.
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
    r_ref, _ = W.forward(p, fbp, warm.SCALE)
    assert rel(r_gpu, r_ref) < 5e-3
    net.close()


def test_network_gradients_match_the_oracle():
    net = warm.WarmNet(0)
    p = random_params(3)
    net.set_params(p)
    fbp, tgt = inputs(4)
    loss = net.gradients(torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda())
    g = net.grads()
    loss_ref, g_ref = W.loss_and_grads(p, fbp, tgt, warm.SCALE)
    assert abs(loss - loss_ref) < 1e-3 * loss_ref
    off = 0
    for k, (ci, co) in enumerate(W.LAYERS):
        nw = 27 * ci * co
        gw, gw_ref = g[off:off + nw], g_ref[off:off + nw]
        gb, gb_ref = g[off + nw:off + nw + co], g_ref[off + nw:off + nw + co]
        off += nw + co
        if np.linalg.norm(gw_ref) > 0:
            assert rel(gw, gw_ref) < 5e-3, (k, rel(gw, gw_ref))
        if np.linalg.norm(gb_ref) > 0:
            assert rel(gb, gb_ref) < 5e-3, (k, rel(gb, gb_ref))
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
