"""Seeded synthetic scans in TIMBIR's binary input layout.

The reference ships no projection data (its demo ``projections.bin`` /
``weights.bin`` are absent), so every workload here is generated:

* random-ellipsoid phantoms (a Shepp-Logan-like stack of ellipsoids with
  attenuation in [0, vmax]) with exact parallel-beam line integrals;
* a two-phase microstructure (thresholded smoothed Gaussian random field,
  coarsening between frames by a curvature-flow step) for 4-D scans;
* transmission counts ~ Poisson(I0 exp(-p)), optional zingers and ring offsets,
  weights = counts, projections = log(I0 / counts).

Geometry follows the reference: the detector column ``c`` has centre
``r = (c + 0.5 - rot_center) * vox_wid`` and a voxel at column ``k``, row ``j``
has centre ``x = (k + 0.5 - rot_center) * vox_wid``,
``y = (j + 0.5) * vox_wid - N * vox_wid / 2``; the view at angle ``theta``
integrates along lines with ``r = x cos(theta) - y sin(theta)``
(src/MBIR_4D/XT_AMatrix.c:62-68, XT_Init.c:517-540).  Detector rows are slices:
row ``t`` sits at ``z = (t + 0.5) * vox_wid - rows * vox_wid / 2``.

Input arrays use the layout ``reconstruct()`` takes: projections and weights
are ``[proj_num][proj_rows][proj_cols]`` float32 (columns fastest,
src/MBIR_4D/XT_Init.c:302).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class Scan:
    projections: np.ndarray  # [views][rows][cols] float32
    weights: np.ndarray  # [views][rows][cols] float32
    proj_angles: np.ndarray  # [views] float32, radians
    proj_times: np.ndarray  # [views] float32
    recon_times: np.ndarray  # [recon_num + 1] float32
    proj_rows: int
    proj_cols: int
    proj_num: int
    recon_num: int
    vox_wid: float
    rot_center: float
    phantom: np.ndarray | None = None  # [recon_num][rows][cols][cols] float32 (z, y, x)

    def write_bin(self, directory: str) -> None:
        """Write the file set read by the reference's bin_data driver
        (src/reconstruct/bin_data/XT_Main.c:115-138, XT_Main.h:33-37)."""
        os.makedirs(directory, exist_ok=True)
        self.projections.astype(np.float32).tofile(os.path.join(directory, "projections.bin"))
        self.weights.astype(np.float32).tofile(os.path.join(directory, "weights.bin"))
        self.proj_angles.astype(np.float32).tofile(os.path.join(directory, "proj_angles.bin"))
        self.proj_times.astype(np.float32).tofile(os.path.join(directory, "proj_times.bin"))
        self.recon_times.astype(np.float32).tofile(os.path.join(directory, "recon_times.bin"))


def random_ellipsoids(n: int, rng: np.random.Generator, vmax: float = 0.02) -> np.ndarray:
    """n ellipsoids in the unit cylinder: columns cx, cy, cz, a, b, c, phi, rho.

    The first one is a large outer body at vmax/2; the rest are smaller
    positive inclusions whose densities add (the scan rescales all densities
    so that the phantom's maximum is vmax)."""
    e = np.zeros((n, 8))
    e[0] = [0.0, 0.0, 0.0, 0.72, 0.9, 0.95, 0.0, 0.5 * vmax]
    for i in range(1, n):
        a, b = rng.uniform(0.08, 0.35, 2)
        r = rng.uniform(0.0, 0.55)
        th = rng.uniform(0, 2 * np.pi)
        e[i] = [
            r * np.cos(th) * 0.7,
            r * np.sin(th) * 0.85,
            rng.uniform(-0.4, 0.4),
            a,
            b,
            rng.uniform(0.3, 0.9),
            rng.uniform(0, np.pi),
            rng.uniform(0.1, 0.45) * vmax,
        ]
    return e


def ellipsoid_volume(ell: np.ndarray, n_xy: int, n_z: int, vox_wid: float, rot_center: float,
                     vmax: float) -> np.ndarray:
    """Voxelised phantom [n_z][n_xy][n_xy] sampled at voxel centres (for
    error statements; the sinogram itself uses exact line integrals of the
    same ellipsoid sum, so neither is clipped)."""
    half = n_xy * vox_wid / 2.0
    k = np.arange(n_xy)
    x = (k + 0.5 - rot_center) * vox_wid
    y = (k + 0.5) * vox_wid - half
    z = (np.arange(n_z) + 0.5) * vox_wid - n_z * vox_wid / 2.0
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    vol = np.zeros_like(X)
    scale_xy, scale_z = half, n_z * vox_wid / 2.0
    for cx, cy, cz, a, b, c, phi, rho in ell:
        xr = X / scale_xy - cx
        yr = Y / scale_xy - cy
        zr = Z / scale_z - cz
        u = xr * np.cos(phi) + yr * np.sin(phi)
        v = -xr * np.sin(phi) + yr * np.cos(phi)
        vol += rho * ((u / a) ** 2 + (v / b) ** 2 + (zr / c) ** 2 <= 1.0)
    return vol.astype(np.float32)


def ellipsoid_sinogram(ell: np.ndarray, angles: np.ndarray, cols: int, rows: int, vox_wid: float,
                       rot_center: float, n_xy: int, oversample: int = 4) -> np.ndarray:
    """Exact line integrals [views][rows][cols] of the (unclipped) ellipsoid sum.

    Each ellipsoid cross-section at height z is an ellipse; its projection at
    normal n = (cos t, -sin t) and offset s from the centre is
    2 a b / h^2 sqrt(h^2 - s^2), h^2 = a^2 (n.u)^2 + b^2 (n.v)^2.  The detector
    bin is averaged over `oversample` sub-positions."""
    half = n_xy * vox_wid / 2.0
    scale_z = rows * vox_wid / 2.0
    sub = (np.arange(oversample) + 0.5) / oversample - 0.5
    r = ((np.arange(cols)[:, None] + 0.5 + sub[None, :] - rot_center) * vox_wid).reshape(-1)
    z = (np.arange(rows) + 0.5) * vox_wid - scale_z
    th = angles.astype(np.float64)[:, None]
    nx, ny = np.cos(th), -np.sin(th)
    out = np.zeros((len(angles), rows, cols * oversample))
    for cx, cy, cz, a, b, c, phi, rho in ell:
        zz = (z / scale_z - cz) / c
        f = np.clip(1.0 - zz ** 2, 0.0, None)
        live = f > 0
        if not live.any():
            continue
        A = a * half * np.sqrt(f)  # [rows]
        B = b * half * np.sqrt(f)
        cxp = cx * half
        cyp = cy * half
        nu = nx * np.cos(phi) + ny * np.sin(phi)  # [views,1]
        nv = -nx * np.sin(phi) + ny * np.cos(phi)
        s0 = nx * cxp + ny * cyp  # [views,1]
        h2 = (A[None, :, None] ** 2) * (nu[:, :, None] ** 2) + (B[None, :, None] ** 2) * (nv[:, :, None] ** 2)
        s = r[None, None, :] - s0[:, :, None]
        with np.errstate(invalid="ignore", divide="ignore"):
            val = 2.0 * (A * B)[None, :, None] / h2 * np.sqrt(np.clip(h2 - s ** 2, 0.0, None))
        val[:, ~live, :] = 0.0
        out += rho * np.nan_to_num(val)
    return out.reshape(len(angles), rows, cols, oversample).mean(axis=3)


def counts_to_data(line_integrals: np.ndarray, I0: float, rng: np.random.Generator,
                   zinger_frac: float = 0.0, ring_sigma: float = 0.0):
    """Poisson transmission counts -> (projections, weights), both float32.

    Zingers multiply a fraction of the counts by 10 (bright outliers, so the
    log projection drops); rings add a per-(row, col) log-domain offset shared
    by all views."""
    lam = I0 * np.exp(-line_integrals)
    counts = rng.poisson(lam).astype(np.float64)
    if zinger_frac > 0:
        hit = rng.random(counts.shape) < zinger_frac
        counts[hit] *= 10.0
    counts = np.maximum(counts, 1.0)
    proj = np.log(I0 / counts)
    if ring_sigma > 0:
        proj = proj + rng.normal(0.0, ring_sigma, size=proj.shape[1:])[None, :, :]
    return proj.astype(np.float32), counts.astype(np.float32)


def ellipsoid_scan(n_xy: int = 64, rows: int = 4, views: int = 96, I0: float = 1e4,
                   n_ell: int = 10, seed: int = 0, vmax: float = 0.02, vox_wid: float = 1.0,
                   rot_center: float | None = None, zinger_frac: float = 0.0,
                   ring_sigma: float = 0.0) -> Scan:
    """3-D scan of a random-ellipsoid phantom, views uniform on [0, pi)."""
    rng = np.random.default_rng(seed)
    rc = n_xy / 2.0 if rot_center is None else rot_center
    ell = random_ellipsoids(n_ell, rng, vmax)
    peak = ellipsoid_volume(ell, n_xy, rows, vox_wid, rc, vmax).max()
    ell[:, 7] *= vmax / peak
    angles = (np.arange(views) * np.pi / views).astype(np.float32)
    li = ellipsoid_sinogram(ell, angles, n_xy, rows, vox_wid, rc, n_xy)
    proj, wts = counts_to_data(li, I0, rng, zinger_frac, ring_sigma)
    times = np.arange(views, dtype=np.float32)
    recon_times = np.array([0.0, float(views)], dtype=np.float32)
    vol = ellipsoid_volume(ell, n_xy, rows, vox_wid, rc, vmax)[None]
    return Scan(proj, wts, angles, times, recon_times, rows, n_xy, views, 1, vox_wid, rc, vol)


def _torch_line_integrals(ell: np.ndarray, angles: np.ndarray, cols: int, rows: int, vox_wid: float,
                          rot_center: float, n_xy: int, oversample: int, device: str) -> np.ndarray:
    """ellipsoid_sinogram's exact line integrals evaluated with torch (FP64)
    on `device`, a chunk of views at a time."""
    import torch
    half = n_xy * vox_wid / 2.0
    scale_z = rows * vox_wid / 2.0
    sub = (torch.arange(oversample, dtype=torch.float64, device=device) + 0.5) / oversample - 0.5
    r = ((torch.arange(cols, dtype=torch.float64, device=device)[:, None] + 0.5 + sub[None, :] - rot_center)
         * vox_wid).reshape(-1)
    z = (torch.arange(rows, dtype=torch.float64, device=device) + 0.5) * vox_wid - scale_z
    th_all = torch.as_tensor(angles.astype(np.float64), device=device)
    out = np.zeros((len(angles), rows, cols))
    chunk = max(1, int(2e7 // max(1, rows * cols * oversample)))
    for v0 in range(0, len(angles), chunk):
        th = th_all[v0:v0 + chunk, None]
        nx, ny = torch.cos(th), -torch.sin(th)
        acc = torch.zeros((th.shape[0], rows, cols * oversample), dtype=torch.float64, device=device)
        for cx, cy, cz, a, b, c, phi, rho in ell:
            zz = (z / scale_z - cz) / c
            f = torch.clamp(1.0 - zz ** 2, min=0.0)
            live = f > 0
            if not bool(live.any()):
                continue
            A = a * half * torch.sqrt(f)
            B = b * half * torch.sqrt(f)
            nu = nx * np.cos(phi) + ny * np.sin(phi)
            nv = -nx * np.sin(phi) + ny * np.cos(phi)
            s0 = nx * (cx * half) + ny * (cy * half)
            h2 = (A[None, :, None] ** 2) * (nu[:, :, None] ** 2) + (B[None, :, None] ** 2) * (nv[:, :, None] ** 2)
            s = r[None, None, :] - s0[:, :, None]
            val = 2.0 * (A * B)[None, :, None] / h2 * torch.sqrt(torch.clamp(h2 - s ** 2, min=0.0))
            val = torch.nan_to_num(val) * live[None, :, None]
            acc += rho * val
        out[v0:v0 + chunk] = acc.reshape(th.shape[0], rows, cols, oversample).mean(dim=3).cpu().numpy()
    return out


def _torch_volume_max(ell: np.ndarray, n_xy: int, n_z: int, vox_wid: float, rot_center: float,
                      device: str) -> float:
    """Maximum of ellipsoid_volume's voxelised phantom, evaluated with torch
    one slice at a time."""
    import torch
    half = n_xy * vox_wid / 2.0
    k = torch.arange(n_xy, dtype=torch.float64, device=device)
    x = (k + 0.5 - rot_center) * vox_wid
    y = (k + 0.5) * vox_wid - half
    Y, X = torch.meshgrid(y, x, indexing="ij")
    scale_z = n_z * vox_wid / 2.0
    best = 0.0
    for iz in range(n_z):
        zc = (iz + 0.5) * vox_wid - scale_z
        vol = torch.zeros_like(X)
        for cx, cy, cz, a, b, c, phi, rho in ell:
            xr = X / half - cx
            yr = Y / half - cy
            zr = zc / scale_z - cz
            u = xr * np.cos(phi) + yr * np.sin(phi)
            v = -xr * np.sin(phi) + yr * np.cos(phi)
            vol += rho * (((u / a) ** 2 + (v / b) ** 2 + (zr / c) ** 2) <= 1.0)
        best = max(best, float(vol.max()))
    return best


def ellipsoid_scan_device(n_xy: int, rows: int, views: int, I0: float = 1e4, n_ell: int = 10, seed: int = 0,
                          vmax: float = 0.02, device: str = "cuda") -> Scan:
    """ellipsoid_scan's scan (same seeded ellipsoids, exact line integrals,
    Poisson counts drawn on the host from the same generator) with the line
    integrals and the density normalisation evaluated by torch on `device`;
    no phantom volume is kept.  For the many-problem workloads, whose numpy
    evaluation would take minutes."""
    rng = np.random.default_rng(seed)
    rc = n_xy / 2.0
    ell = random_ellipsoids(n_ell, rng, vmax)
    ell[:, 7] *= vmax / _torch_volume_max(ell, n_xy, rows, 1.0, rc, device)
    angles = (np.arange(views) * np.pi / views).astype(np.float32)
    li = _torch_line_integrals(ell, angles, n_xy, rows, 1.0, rc, n_xy, 4, device)
    proj, wts = counts_to_data(li, I0, rng)
    times = np.arange(views, dtype=np.float32)
    recon_times = np.array([0.0, float(views)], dtype=np.float32)
    return Scan(proj, wts, angles, times, recon_times, rows, n_xy, views, 1, 1.0, rc, None)


def batch_problem_specs(n: int = 64, seed: int = 0, sides=(128, 192, 256, 384, 512)) -> list:
    """Seeded sizes of a many-problem workload: side drawn uniformly from
    `sides`, an even number of slices in [4, 32], views = 1.5 x side over
    180 degrees, I0 log-uniform in [2e3, 5e4]; problem k uses seed k."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        side = int(rng.choice(sides))
        out.append(dict(side=side, slices=2 * int(rng.integers(2, 17)), views=(3 * side) // 2,
                        I0=float(np.exp(rng.uniform(np.log(2e3), np.log(5e4)))), seed=k))
    return out


def interlaced_angles(K: int, n_views: int, views_per_rotation: int) -> np.ndarray:
    """Interlaced view schedule: each rotation of `views_per_rotation` views is
    split in K sub-frames whose angular offsets follow the bit-reversal of the
    sub-frame index (the TIMBIR acquisition scheme)."""
    bits = int(np.log2(K))
    rev = np.array([int(format(k, f"0{bits}b")[::-1], 2) for k in range(K)]) if bits > 0 else np.zeros(1, int)
    per_sub = views_per_rotation // K
    out = np.zeros(n_views)
    for v in range(n_views):
        rot, w = divmod(v, views_per_rotation)
        sub, m = divmod(w, per_sub)
        out[v] = rot * np.pi + (m * K + rev[sub]) * np.pi / views_per_rotation
    return out.astype(np.float32)


def moving_ellipsoid_scan(n_xy: int, rows: int, frames: int, views_per_rotation: int, K: int, rotations: int,
                          I0: float = 1e4, n_ell: int = 10, seed: int = 0, vmax: float = 0.02, drift: float = 0.05,
                          zinger_frac: float = 0.001, ring_sigma: float = 0.02, oversample: int = 2) -> Scan:
    """4-D scan of random ellipsoids whose inclusions drift in x-y over the
    scan (by up to `drift` of the half-width), interlaced views (K sub-frames
    per rotation of `views_per_rotation` views), `frames` frames of equal time.
    The object is static within a frame: a frame's views see the ellipsoids at
    the frame's mid time (the reconstruction's model).  Exact line integrals,
    Poisson counts at I0, zingers and ring offsets as in counts_to_data.  No
    phantom volume is kept (at this size it is not needed by the callers)."""
    rng = np.random.default_rng(seed)
    rc = n_xy / 2.0
    ell = random_ellipsoids(n_ell, rng, vmax)
    vel = rng.uniform(-drift, drift, size=(n_ell, 2))
    vel[0] = 0.0
    n_views = views_per_rotation * rotations
    angles = interlaced_angles(K, n_views, views_per_rotation)
    times = np.arange(n_views, dtype=np.float32)
    recon_times = np.linspace(0, n_views, frames + 1).astype(np.float32)
    li = np.zeros((n_views, rows, n_xy))
    per = n_views // frames
    for f in range(frames):
        e = ell.copy()
        e[:, 0:2] += vel * ((f + 0.5) / frames)
        sl = slice(f * per, (f + 1) * per)
        li[sl] = ellipsoid_sinogram(e, angles[sl], n_xy, rows, 1.0, rc, n_xy, oversample)
    proj, wts = counts_to_data(li, I0, rng, zinger_frac, ring_sigma)
    return Scan(proj, wts, angles, times, recon_times, rows, n_xy, n_views, frames, 1.0, rc, None)


def project_frames(frames: np.ndarray, angles: np.ndarray, recon_times: np.ndarray, proj_times: np.ndarray,
                   cols: int, vox_wid: float = 1.0, rot_center: float | None = None) -> np.ndarray:
    """Line integrals [views][rows][cols] of a voxelised 4-D object
    frames [N_time][rows][n_xy][n_xy] (z, y, x): each view sees the frame whose
    time interval [recon_times[t], recon_times[t+1]) holds its time.  Each
    voxel's mass goes to the two detector columns nearest its centre's
    projection r = x cos(theta) - y sin(theta), by linear interpolation
    (geometry as in the module docstring).  Float64 numpy on the CPU, so the
    data are the same on every machine; the reconstruction's own A matrix is
    not used."""
    import scipy.sparse as sp
    n_t, rows, n_xy, _ = frames.shape
    rc = n_xy / 2.0 if rot_center is None else rot_center
    live = np.flatnonzero(frames.reshape(n_t * rows, -1).any(axis=0))  # voxel lines ever non-zero
    yi, xi = np.divmod(live, n_xy)
    X = (xi + 0.5 - rc) * vox_wid
    Y = (yi + 0.5) * vox_wid - n_xy * vox_wid / 2.0
    col = np.arange(len(live))
    out = np.zeros((len(angles), rows, cols))
    dense = [frames[t].reshape(rows, -1)[:, live].T.astype(np.float64) for t in range(n_t)]  # [lines][rows]
    for v, th in enumerate(angles.astype(np.float64)):
        t = int(np.searchsorted(recon_times, proj_times[v], side="right")) - 1
        if t < 0 or t >= n_t:
            continue
        u = (X * np.cos(th) - Y * np.sin(th)) / vox_wid + rc - 0.5  # fractional detector column
        j0 = np.floor(u).astype(np.int64)
        f1 = u - j0
        ok0 = (j0 >= 0) & (j0 < cols)
        ok1 = (j0 + 1 >= 0) & (j0 + 1 < cols)
        M = sp.csr_matrix((np.concatenate([1.0 - f1[ok0], f1[ok1]]),
                           (np.concatenate([j0[ok0], j0[ok1] + 1]), np.concatenate([col[ok0], col[ok1]]))),
                          shape=(cols, len(live)))
        out[v] = (M @ dense[t]).T * vox_wid
    return out


def two_phase_frames(n_xy: int, n_z: int, frames: int, seed: int, vmax: float = 0.02,
                     smooth: float = 6.0, flow_steps: int = 3) -> np.ndarray:
    """[frames][n_z][n_xy][n_xy] two-phase microstructure: a smoothed Gaussian
    random field thresholded at 0, coarsened between frames by smoothing the
    signed field (a discrete curvature-flow step)."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((n_z, n_xy, n_xy))

    def blur(a, s):
        kz = np.fft.fftfreq(a.shape[0])[:, None, None]
        ky = np.fft.fftfreq(a.shape[1])[None, :, None]
        kx = np.fft.fftfreq(a.shape[2])[None, None, :]
        g = np.exp(-2 * (np.pi * s) ** 2 * (kx ** 2 + ky ** 2 + (kz ** 2) * 0.25))
        return np.real(np.fft.ifftn(np.fft.fftn(a) * g))

    f = blur(f, smooth)
    f /= f.std()
    half = n_xy / 2.0
    yy, xx = np.mgrid[0:n_xy, 0:n_xy]
    disc = ((xx + 0.5 - half) ** 2 + (yy + 0.5 - half) ** 2) < (0.45 * n_xy) ** 2
    out = np.zeros((frames, n_z, n_xy, n_xy), np.float32)
    for t in range(frames):
        out[t] = np.where((f > 0) & disc[None], vmax, 0.0)
        for _ in range(flow_steps):
            f = blur(np.tanh(2.0 * f), 1.0)
    return out
