"""Small seeded stage scenarios shared by the oracle pin, the golden fixtures
and the GPU parity tests.  Each scenario is one resolution stage driven for a
few ICD iterations with the reference schedule."""
from __future__ import annotations

import numpy as np

from timbir_b200 import synth


def _scan4d(seed=2):
    s = synth.ellipsoid_scan(32, 4, 64, seed=seed, zinger_frac=0.002, ring_sigma=0.02)
    s.proj_angles = synth.interlaced_angles(4, 64, 32)
    s.proj_times = np.arange(64, dtype=np.float32)
    s.recon_times = np.array([0, 16, 32, 48, 64], np.float32)
    s.recon_num = 4
    return s


BASE = dict(sig_s=0.002, sig_t=1.0, c_s=1e-3, c_t=1e-3, convg_thresh=0.1)

# name -> (scan factory, extra kwargs, stage switches, num_z_blocks, mult_xy, mult_z)
SCENARIOS = {
    "plain": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=1), {}, {}, 2, 1, 1),
    "rings1": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=3, ring_sigma=0.02),
               dict(remove_rings=1), dict(update_proj_offset=2), 2, 1, 1),
    "rings2": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=3, ring_sigma=0.02),
               dict(remove_rings=2), dict(update_proj_offset=2), 2, 1, 1),
    "rings3": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=3, ring_sigma=0.02),
               dict(remove_rings=3), dict(update_proj_offset=3), 2, 1, 1),
    # mode 3 with the rectangular-patch constraint windows built
    "rings3w": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=3, ring_sigma=0.02),
                dict(remove_rings=3), dict(update_proj_offset=3), 2, 1, 1),
    "zinger_var": (lambda: synth.ellipsoid_scan(32, 4, 48, seed=4, zinger_frac=0.003),
                   dict(remove_rings=2, quad_convex=0), dict(update_proj_offset=2, update_var=1, var_est=1.3),
                   2, 1, 1),
    "frames4": (_scan4d, dict(remove_rings=2, quad_convex=0, sig_t=0.01), dict(update_proj_offset=2, update_var=1),
                2, 1, 1),
    "blocks4": (lambda: synth.ellipsoid_scan(32, 8, 48, seed=5), {}, {}, 4, 1, 1),
    "coarse2": (lambda: synth.ellipsoid_scan(32, 8, 48, seed=6), {}, {}, 2, 2, 2),
    "coarse4": (lambda: synth.ellipsoid_scan(64, 8, 48, seed=6), dict(remove_rings=2), dict(update_proj_offset=3),
                2, 4, 2),
}


def make(name, cls, **extra):
    factory, kw, sw, blocks, mxy, mz = SCENARIOS[name]
    scan = factory()
    args = dict(BASE)
    args.update(kw)
    obj = cls(scan, blocks=blocks, mult_xy=mxy, mult_z=mz, **args, **extra)
    if sw:
        obj.set_switches(**sw)
    if name.endswith("w"):
        obj.build_offset_windows()
    return obj
