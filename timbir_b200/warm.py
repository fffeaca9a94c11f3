"""Learned warm start for ICD: the network of include/timbir_b200.h
(mbir_net_*), its training on (filtered backprojection, converged MBIR)
pairs that the plain method generates, and the warm start it gives.

The network maps a frame's filtered backprojection to a start image (whose
low frequencies are then taken back from the backprojection); ICD then runs
from it to its own convergence test, so the result is the MAP estimate
whatever the start (qGGMRF with 1 <= p <= 2 is convex) and FBP-initialised
ICD stays both the fallback and the yardstick.  Device memory comes from torch
(plumbing only); every kernel is the native library's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import MbirError, load_library

SCALE = 50.0  # attenuation per voxel ~0.02 -> order one inside the network
# (input channels, output channels, level) of the 15 convolutions, as in
# timbir_b200/csrc/warm_net.cu; level l works at 1 / 2^l of the input's sides
LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 3),
          (128, 128, 3), (128, 64, 2), (64, 64, 2), (64, 32, 1), (32, 32, 1), (32, 16, 0), (16, 16, 0),
          (16, 16, 0)]


def _lib():
    lib = load_library()
    if not getattr(lib, "_net_bound", False):
        i32, vp = C.c_int32, C.c_void_p
        lib.mbir_net_create.argtypes = [C.POINTER(vp), C.c_uint32]
        lib.mbir_net_free.argtypes = [vp]
        lib.mbir_net_last_error.restype = C.c_char_p
        lib.mbir_net_param_count.restype = C.c_int64
        for n in ("mbir_net_get_params", "mbir_net_set_params", "mbir_net_get_grads"):
            getattr(lib, n).argtypes = [vp, vp]
        lib.mbir_net_forward.argtypes = [vp, vp, vp, i32, i32, i32, i32, C.c_float, vp]
        lib.mbir_net_gradients.argtypes = [vp, vp, vp, i32, i32, i32, i32, C.c_float, C.POINTER(C.c_double), vp]
        lib.mbir_net_adam_step.argtypes = [vp, C.c_float, vp]
        lib.mbir_net_set_loss_weights.argtypes = [vp, vp]
        lib.mbir_net_set_loss_highpass.argtypes = [vp, C.c_float, C.c_float]
        lib.mbir_lowpass_blend.argtypes = [vp, vp, vp, i32, i32, i32, i32, C.c_float, C.c_float, vp]
        lib.mbir_net_get_activation.argtypes = [vp, i32, i32, vp, C.POINTER(C.c_int64)]
        lib._net_bound = True
    return lib


def _check(rc):
    if rc != 0:
        raise MbirError(_lib().mbir_net_last_error().decode(errors="replace"))


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class WarmNet:
    """The warm-start network on the current CUDA device."""

    def __init__(self, seed: int = 0):
        self.lib = _lib()
        h = C.c_void_p()
        _check(self.lib.mbir_net_create(C.byref(h), seed))
        self.h = h
        self.n = int(self.lib.mbir_net_param_count())

    def close(self):
        if self.h:
            self.lib.mbir_net_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        _check(self.lib.mbir_net_get_params(self.h, out.ctypes.data))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n
        _check(self.lib.mbir_net_set_params(self.h, p.ctypes.data))

    def grads(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        _check(self.lib.mbir_net_get_grads(self.h, out.ctypes.data))
        return out

    def activation(self, layer: int, grad: bool = False) -> np.ndarray:
        """Layer `layer`'s output (or its gradient) from the last call, flat."""
        n = C.c_int64()
        _check(self.lib.mbir_net_get_activation(self.h, layer, 1 if grad else 0, None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        _check(self.lib.mbir_net_get_activation(self.h, layer, 1 if grad else 0, out.ctypes.data, None))
        return out

    def forward(self, x, scale: float = SCALE):
        """x: CUDA float32 tensor [B][D][H][W] -> warm start of the same shape."""
        import torch
        x = x.contiguous()
        out = torch.empty_like(x)
        B, D, H, W = x.shape
        _check(self.lib.mbir_net_forward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), B, D, H, W,
                                         scale, _stream()))
        return out

    def gradients(self, x, t, scale: float = SCALE) -> float:
        """Parameter gradients of mean((s x + r - s t)^2); returns the loss."""
        x, t = x.contiguous(), t.contiguous()
        B, D, H, W = x.shape
        loss = C.c_double()
        _check(self.lib.mbir_net_gradients(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), B, D, H, W,
                                           scale, C.byref(loss), _stream()))
        return loss.value

    def set_loss_weights(self, w) -> None:
        """Per-voxel weights of the loss, mean(w (s x + r - s t)^2), for the
        following gradients() calls: a CUDA float32 tensor of the inputs'
        shape (kept referenced here), or None for unit weights."""
        self._loss_w = None if w is None else w.contiguous()
        _check(self.lib.mbir_net_set_loss_weights(
            self.h, None if self._loss_w is None else C.c_void_p(self._loss_w.data_ptr())))

    def set_loss_highpass(self, sigma_z: float = 0.0, sigma_xy: float = 0.0) -> None:
        """High-pass loss mean(w ((I - G) d)^2) for the following gradients()
        calls (G: Gaussian low-pass of widths sigma_z slices, sigma_xy voxels,
        zeros outside the patch); 0, 0 restores the plain loss."""
        _check(self.lib.mbir_net_set_loss_highpass(self.h, sigma_z, sigma_xy))

    def adam_step(self, lr: float) -> None:
        _check(self.lib.mbir_net_adam_step(self.h, lr, _stream()))


def train(net: WarmNet, inputs, targets, steps: int, batch: int = 4, patch=(16, 64, 64), lr: float = 1e-3,
          seed: int = 0, scale: float = SCALE, log_every: int = 0, weights=None, highpass=None):
    """Adam on random patches of the (input, target) volumes (CUDA tensors
    [N][D][H][W]), the loss weighted per voxel by the same patches of
    `weights` when given, and taken on the residual's high frequencies when
    `highpass` = (sigma_z, sigma_xy) is given; the learning rate decays by
    cosine to a tenth.  Returns the per-step losses."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    N, D, H, W = inputs.shape
    pd, ph, pw = (min(patch[0], D), min(patch[1], H), min(patch[2], W))
    losses = []
    xb = torch.empty((batch, pd, ph, pw), dtype=torch.float32, device=inputs.device)
    tb = torch.empty_like(xb)
    wb = torch.empty_like(xb) if weights is not None else None
    net.set_loss_weights(wb)
    net.set_loss_highpass(*(highpass or (0.0, 0.0)))
    for step in range(steps):
        for b in range(batch):
            n = int(torch.randint(N, (1,), generator=g))
            z = int(torch.randint(D - pd + 1, (1,), generator=g))
            y = int(torch.randint(H - ph + 1, (1,), generator=g))
            x = int(torch.randint(W - pw + 1, (1,), generator=g))
            xb[b] = inputs[n, z:z + pd, y:y + ph, x:x + pw]
            tb[b] = targets[n, z:z + pd, y:y + ph, x:x + pw]
            if wb is not None:
                wb[b] = weights[n, z:z + pd, y:y + ph, x:x + pw]
        losses.append(net.gradients(xb, tb, scale))
        cur = lr * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * step / max(steps, 1))))
        net.adam_step(cur)
        if log_every and (step + 1) % log_every == 0:
            print(f"step {step + 1} loss {np.mean(losses[-log_every:]):.5f}", flush=True)
    if wb is not None:
        net.set_loss_weights(None)
    if highpass:
        net.set_loss_highpass(0.0, 0.0)
    return losses


def lowpass_blend(ref, start, sigma_z: float, sigma_xy: float) -> None:
    """start += G (ref - start) in place (CUDA float32 tensors [N][D][H][W];
    G the Gaussian low-pass of widths sigma_z slices, sigma_xy voxels): the
    low frequencies of ref under the high frequencies of start."""
    import torch
    ref = ref.contiguous()
    assert start.is_contiguous() and ref.shape == start.shape
    N, D, H, W = start.shape
    scratch = torch.empty((2,) + tuple(start.shape), dtype=torch.float32, device=start.device)
    lib = _lib()
    _check(lib.mbir_lowpass_blend(C.c_void_p(ref.data_ptr()), C.c_void_p(start.data_ptr()),
                                  C.c_void_p(scratch.data_ptr()), N, D, H, W, sigma_z, sigma_xy, _stream()))


# widths of the low-pass under which warm_start keeps the FBP's frequencies
BLEND_SIGMA = (1.0, 4.0)


def warm_start(net: WarmNet, fbp: np.ndarray, mask: np.ndarray, scale: float = SCALE,
               blend=BLEND_SIGMA) -> np.ndarray:
    """Warm start [N_time][N_z][N_y][N_x] from the frames' filtered
    backprojections: the network per frame, its low frequencies replaced by
    the FBP's (Gaussian low-pass of widths blend = (slices, voxels); None:
    the network's output as it is), zero outside the reconstruction mask
    (ICD never updates those voxels)."""
    import torch
    x = torch.from_numpy(np.ascontiguousarray(fbp, np.float32)).cuda()
    out = net.forward(x, scale)
    if blend:
        lowpass_blend(x, out, float(blend[0]), float(blend[1]))
    return (out.cpu().numpy() * mask[None, None, :, :]).astype(np.float32)
