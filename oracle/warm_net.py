"""CPU oracle of the learned warm-start network (test infrastructure only).

A numpy float64 restatement of the network in timbir_b200/csrc/warm_net.cu
(no reference counterpart: TIMBIR has no learned part): the same layers,
parameter layout and loss, with forward and backward passes written out by
hand.  The GPU rounds the two operands of every tensor-core product to BF16
(round to nearest even) and accumulates in FP32 inside the tensor cores; the
oracle rounds the same operands to BF16 and accumulates in FP64, so the two
differ by the tensor cores' accumulation error only.  ``finite_difference`` checks the oracle's own
gradients against its loss.

Activations are channels-last [B][D][H][W][C]; parameters are flat, per
layer the weights [27 taps][in][out] (tap = 9 (dz+1) + 3 (dy+1) + dx+1)
then the biases.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
          (128, 64), (64, 64), (64, 32), (32, 32), (32, 16), (16, 16), (16, 16)]
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def param_count() -> int:
    return sum(27 * ci * co + co for ci, co in LAYERS)


def bf16(a) -> np.ndarray:
    """Round to BF16 (nearest, ties to even) through the float32 bit pattern;
    returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(flat):
    out, off = [], 0
    for ci, co in LAYERS:
        w = np.asarray(flat[off:off + 27 * ci * co], np.float64).reshape(27, ci, co)
        off += 27 * ci * co
        b = np.asarray(flat[off:off + co], np.float64)
        off += co
        out.append((w, b))
    return out


def _shift(X, dz, dy, dx):
    """X[z + dz, y + dy, x + dx] with zeros outside."""
    P = np.pad(X, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    _, D, H, W, _ = X.shape
    return P[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]


def conv(X, w, b=None):
    """3x3x3 convolution, zero padding 1, BF16 operands, FP64 sums."""
    Xb, wb = bf16(X), bf16(w)
    Y = np.zeros(X.shape[:4] + (w.shape[2],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        Y += _shift(Xb, dz, dy, dx) @ wb[t]
    if b is not None:
        Y += b
    return Y


def conv_input_grad(dY, w):
    """Gradient of conv with respect to its input (BF16 dY and w)."""
    dYb, wb = bf16(dY), bf16(w)
    dX = np.zeros(dY.shape[:4] + (w.shape[1],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        dX += _shift(dYb, -dz, -dy, -dx) @ wb[t].T
    return dX


def conv_weight_grad(X, dY):
    """Gradients of conv with respect to its weights (BF16 X and dY) and bias."""
    Xb, dYb = bf16(X), bf16(dY)
    ci, co = X.shape[4], dY.shape[4]
    dw = np.zeros((27, ci, co))
    d2 = dYb.reshape(-1, co)
    for t, (dz, dy, dx) in enumerate(TAPS):
        dw[t] = _shift(Xb, dz, dy, dx).reshape(-1, ci).T @ d2
    return dw, dY.reshape(-1, co).sum(axis=0)


def pool(X):
    B, D, H, W, C = X.shape
    return X.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def pool_grad(dY):
    return np.repeat(np.repeat(np.repeat(dY, 2, 1), 2, 2), 2, 3) / 8.0


def up(X):
    return np.repeat(np.repeat(np.repeat(X, 2, 1), 2, 2), 2, 3)


def up_grad(dY):
    B, D, H, W, C = dY.shape
    return dY.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


def forward(flat, fbp, s):
    """Network output r (channel 0 of the last layer) and the activations."""
    P = unpack(flat)
    x0 = np.zeros(fbp.shape + (16,))
    x0[..., 0] = s * np.asarray(fbp, np.float64)
    A = {"x0": x0}
    relu = lambda z: np.maximum(z, 0.0)  # noqa: E731
    A[0] = relu(conv(x0, *P[0]))
    A[1] = relu(conv(A[0], *P[1]))
    A["p1"] = pool(A[1])
    A[2] = relu(conv(A["p1"], *P[2]))
    A[3] = relu(conv(A[2], *P[3]))
    A["p2"] = pool(A[3])
    A[4] = relu(conv(A["p2"], *P[4]))
    A[5] = relu(conv(A[4], *P[5]))
    A["p3"] = pool(A[5])
    A[6] = relu(conv(A["p3"], *P[6]))
    A[7] = relu(conv(A[6], *P[7]))
    A["u2"] = up(A[7])
    A[8] = relu(conv(A["u2"], *P[8]) + A[5])
    A[9] = relu(conv(A[8], *P[9]))
    A["u1"] = up(A[9])
    A[10] = relu(conv(A["u1"], *P[10]) + A[3])
    A[11] = relu(conv(A[10], *P[11]))
    A["u0"] = up(A[11])
    A[12] = relu(conv(A["u0"], *P[12]) + A[1])
    A[13] = relu(conv(A[12], *P[13]))
    A[14] = conv(A[13], *P[14])
    return A[14][..., 0], A


def predict(flat, fbp, s):
    """Warm start fbp + r / s."""
    r, _ = forward(flat, fbp, s)
    return np.asarray(fbp, np.float64) + r / s


def _lowpass_zero_edge(a, hp):
    """Gaussian low-pass of widths hp = (slices, voxels) of [B][D][H][W], zeros
    outside the volume, radius int(4 sigma + 0.5) (scipy.ndimage)."""
    from scipy import ndimage
    return ndimage.gaussian_filter(np.asarray(a, np.float64), sigma=(0, hp[0], hp[1], hp[1]), mode="constant",
                                   truncate=4.0)


def loss_and_grads(flat, fbp, target, s, trace=None, acts=None, weights=None, highpass=None):
    """Loss mean(w (s fbp + r - s target)^2) (w = the per-voxel weights, 1
    when None; with highpass = (sigma_z, sigma_xy) the residual is first
    high-passed, (I - G) d, G the zero-edge Gaussian low-pass) and its
    gradient with respect to
    the flat parameters; trace (a dict), when given, receives each layer's
    output gradient (after its ReLU's mask) under the layer's index.  acts,
    when given, are the layer outputs to differentiate at ({"x0": input,
    0..14: layer outputs}, channels-last), in place of the oracle's own
    forward pass (so that a backward pass can be checked on its own)."""
    P = unpack(flat)
    if acts is None:
        r, A = forward(flat, fbp, s)
    else:
        A = {k: np.asarray(v, np.float64) for k, v in acts.items()}
        A["p1"], A["p2"], A["p3"] = pool(A[1]), pool(A[3]), pool(A[5])
        A["u2"], A["u1"], A["u0"] = up(A[7]), up(A[9]), up(A[11])
        r = A[14][..., 0]
    d = s * np.asarray(fbp, np.float64) + r - s * np.asarray(target, np.float64)
    M = d.size
    wt = np.ones_like(d) if weights is None else np.asarray(weights, np.float64)
    dz14 = np.zeros(A[14].shape)
    if highpass:
        h = d - _lowpass_zero_edge(d, highpass)
        u = wt * h
        loss = float(np.mean(u * h))
        dz14[..., 0] = 2.0 * (u - _lowpass_zero_edge(u, highpass)) / M
    else:
        loss = float(np.mean(wt * d * d))
        dz14[..., 0] = 2.0 * wt * d / M
    grads = [None] * 15
    mask = lambda g, a: g * (a > 0)  # noqa: E731

    def layer(k, x, dz, need_dx=True):
        if trace is not None:
            trace[k] = dz
        grads[k] = conv_weight_grad(x, dz)
        return conv_input_grad(dz, P[k][0]) if need_dx else None

    dz = dz14
    d13 = mask(layer(14, A[13], dz), A[13])
    d12 = mask(layer(13, A[12], d13), A[12])
    du0 = layer(12, A["u0"], d12)
    d1 = d12.copy()  # skip into A1
    d11 = mask(up_grad(du0), A[11])
    d10 = mask(layer(11, A[10], d11), A[10])
    du1 = layer(10, A["u1"], d10)
    d3 = d10.copy()
    d9 = mask(up_grad(du1), A[9])
    d8 = mask(layer(9, A[8], d9), A[8])
    du2 = layer(8, A["u2"], d8)
    d5 = d8.copy()
    d7 = mask(up_grad(du2), A[7])
    d6 = mask(layer(7, A[6], d7), A[6])
    dp3 = layer(6, A["p3"], d6)
    d5 = mask(d5 + pool_grad(dp3), A[5])
    d4 = mask(layer(5, A[4], d5), A[4])
    dp2 = layer(4, A["p2"], d4)
    d3 = mask(d3 + pool_grad(dp2), A[3])
    d2 = mask(layer(3, A[2], d3), A[2])
    dp1 = layer(2, A["p1"], d2)
    d1 = mask(d1 + pool_grad(dp1), A[1])
    d0 = mask(layer(1, A[0], d1), A[0])
    layer(0, A["x0"], d0, need_dx=False)
    flat_g = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])
    return loss, flat_g


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba, 2015); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def loss_exact(flat, fbp, target, s, weights=None, highpass=None):
    """The loss without BF16 rounding (for finite differences of the
    oracle's own gradients, whose step would be lost in BF16)."""
    global bf16
    saved = bf16
    bf16 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    try:
        r, _ = forward(flat, fbp, s)
    finally:
        bf16 = saved
    d = s * np.asarray(fbp, np.float64) + r - s * np.asarray(target, np.float64)
    if highpass:
        d = d - _lowpass_zero_edge(d, highpass)
    wt = 1.0 if weights is None else np.asarray(weights, np.float64)
    return float(np.mean(wt * d * d))


def grads_exact(flat, fbp, target, s, weights=None, highpass=None):
    global bf16
    saved = bf16
    bf16 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    try:
        return loss_and_grads(flat, fbp, target, s, weights=weights, highpass=highpass)
    finally:
        bf16 = saved


def finite_difference(flat, fbp, target, s, idx, h=1e-6, weights=None, highpass=None):
    """Central differences of loss_exact at parameters idx."""
    out = []
    for i in idx:
        p1 = np.array(flat, np.float64)
        p2 = p1.copy()
        p1[i] += h
        p2[i] -= h
        out.append((loss_exact(p1, fbp, target, s, weights, highpass)
                    - loss_exact(p2, fbp, target, s, weights, highpass)) / (2 * h))
    return np.array(out)
