"""CPU oracle of the filtered backprojection (test infrastructure only): a
float64 numpy restatement of timbir_b200/csrc/mbir_fbp.cu -- the
band-limited Ram-Lak ramp filter (Kak and Slaney, Principles of
Computerized Tomographic Imaging, eq. 3.61) along each detector row of each
view, then per frame the backprojection pi / n_f sum_v q_v(x cos - y sin)
with linear interpolation, zero outside the reconstruction mask.  Geometry
as in the reference's A matrix (XT_AMatrix.c:62-68, XT_Init.c:517-540):
detector column j at R0 + (j + 0.5) vox_wid, R0 = -rot_center vox_wid; voxel
(j, k) at x = R0 + (k + 0.5) vox_wid, y = -N vox_wid / 2 + (j + 0.5) vox_wid;
mask x^2 + y^2 < (N vox_wid / 2)^2."""
from __future__ import annotations

import numpy as np


def ramp(p, dr):
    """p [..., N_r] -> dr * sum_k p[k] h[j - k]."""
    n = p.shape[-1]
    k = np.arange(-(n - 1), n)
    h = np.zeros(2 * n - 1)
    h[k == 0] = 1.0 / (4.0 * dr * dr)
    odd = (k % 2) != 0
    h[odd] = -1.0 / (np.pi ** 2 * k[odd].astype(np.float64) ** 2 * dr * dr)
    flat = p.reshape(-1, n).astype(np.float64)
    out = np.stack([np.convolve(r, h, mode="full")[n - 1:2 * n - 1] for r in flat])
    return dr * out.reshape(p.shape)


def fbp(scan):
    """[recon_num][rows][cols][cols] filtered backprojection of a synth.Scan
    (full resolution: one slice per detector row, voxel = detector column)."""
    n, dr = scan.proj_cols, float(scan.vox_wid)
    R0 = -scan.rot_center * dr
    q = ramp(np.asarray(scan.projections, np.float64), dr)  # [views][rows][cols]
    k = np.arange(n)
    x = R0 + (k + 0.5) * dr
    y = -n * dr / 2.0 + (k + 0.5) * dr
    X, Y = np.meshgrid(x, y)  # [j][k]
    mask = X * X + Y * Y < (n * dr / 2.0) ** 2
    out = np.zeros((scan.recon_num, scan.proj_rows, n, n))
    t = np.asarray(scan.proj_times, np.float64)
    rt = np.asarray(scan.recon_times, np.float64)
    for f in range(scan.recon_num):
        views = np.nonzero((t >= rt[f]) & (t < rt[f + 1]))[0]
        acc = np.zeros((scan.proj_rows, n, n))
        for v in views:
            th = np.float64(scan.proj_angles[v])
            r = X * np.cos(th) - Y * np.sin(th)
            tt = (r - R0) / dr - 0.5
            j0 = np.floor(tt).astype(int)
            w = tt - j0
            for row in range(scan.proj_rows):
                line = q[v, row]
                a = np.where((j0 >= 0) & (j0 < n), line[np.clip(j0, 0, n - 1)], 0.0)
                b = np.where((j0 + 1 >= 0) & (j0 + 1 < n), line[np.clip(j0 + 1, 0, n - 1)], 0.0)
                acc[row] += (1.0 - w) * a + w * b
        out[f] = np.pi / max(len(views), 1) * acc * mask[None]
    return out
