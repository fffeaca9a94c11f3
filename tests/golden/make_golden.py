"""Generate the golden fixtures in tests/golden/ from the reference itself.

Needs the reference library built from its own sources (``make -C oracle ref``,
which needs the TIMBIR tree) and, for the generator's known-answer table, the
environment variable TIMBIR_REFERENCE_SRC set to the tree's src directory.
Run from the repository root:

    TIMBIR_REFERENCE_SRC=<reference>/src python tests/golden/make_golden.py

Outputs (committed):
  park_miller_seed1.json   the known-answer table of the reference's generator,
                           read from the comment block of src/MBIR_4D/randlib.c
  stage_<name>.npz         per scenario of tests/scenarios.py: detector response,
                           mask, initial error sinogram and cost, and the state
                           after ICD iterations 1 and 3 of the reference schedule
  recon_small.npz          a full reconstruct() run of the reference driver
                           binary (object, cost trace) on a seeded 32x32x4 scan
  recon_rings.npz          the same with ring offsets in the data and
                           remove_rings 2 (object, offsets, cost trace)
  upsample.npz             the reference's x2 up-sampling between stages
                           (upsample_object_bilinear_2D / _3D) of seeded slices
  ingest.npz               the reference's data readers and view generator
                           (aps_data read_data, std_data read_ProjWeightData,
                           gen_interlaced_views_0_to_Inf) on seeded arrays,
                           through oracle/_ref/libref_io.so
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.bind import REF_BIN, REF_SO, Reference, reference_src  # noqa: E402
from timbir_b200 import synth  # noqa: E402

import scenarios  # noqa: E402

REF_SRC = reference_src()  # TIMBIR_REFERENCE_SRC: the reference tree's src directory


def park_miller_table():
    text = open(os.path.join(REF_SRC, "MBIR_4D", "randlib.c")).read()
    block = text[text.index("TABLE:"):]
    nums = [int(v) for v in re.findall(r"^\s*(\d+)\s*$", block, flags=re.M)[:20]]
    assert len(nums) == 20
    with open(os.path.join(HERE, "park_miller_seed1.json"), "w") as f:
        json.dump({"seed": 1, "values": nums, "source": "src/MBIR_4D/randlib.c:69-90"}, f, indent=1)


def stage_fixtures(names=None):
    for name in names or scenarios.SCENARIOS:
        wd = tempfile.mkdtemp()
        R = scenarios.make(name, Reference, workdir=wd)
        R.prepare()
        out = dict(hr=R.hr(), mask=R.mask()[0], e0=R.errorsino(), cost0=np.float64(R.cost()[0]))
        for it in (1, 2, 3):
            conv = R.iterate(it)
            if it in (1, 3):
                out[f"obj{it}"] = R.object()
                out[f"conv{it}"] = np.int32(conv)
                out[f"var{it}"] = np.float64(R.var_est())
        out["e3"] = R.errorsino()
        out["offset3"] = R.offset()
        out["cost3"] = np.float64(R.cost()[0])
        xs, ys = R.lines(0, 0, 0)
        out["hicd_x3"], out["hicd_y3"] = xs, ys
        xs, ys = R.lines(1, 0, 0)
        out["nhicd_x3"], out["nhicd_y3"] = xs, ys
        np.savez_compressed(os.path.join(HERE, f"stage_{name}.npz"), **out)
        print(name, {k: getattr(v, "shape", v) for k, v in out.items() if k.startswith("obj")})


RECON_ARGS = dict(sig_s=0.002, sig_t=1.0, c_s=1e-3, c_t=1e-3, convg_thresh=0.005, remove_rings=0,
                  quad_convex=1, huber_delta=0.5, huber_T=4.0)


def recon_fixture():
    scan = synth.ellipsoid_scan(32, 4, 48, seed=11)
    wd = tempfile.mkdtemp()
    scan.write_bin(wd)
    a = RECON_ARGS
    cmd = [REF_BIN, "--proj_rows", str(scan.proj_rows), "--proj_cols", str(scan.proj_cols), "--proj_num",
           str(scan.proj_num), "--recon_num", "1", "--vox_wid", str(scan.vox_wid), "--rot_center",
           str(scan.rot_center), "--sig_s", str(a["sig_s"]), "--sig_t", str(a["sig_t"]), "--c_s", str(a["c_s"]),
           "--c_t", str(a["c_t"]), "--convg_thresh", str(a["convg_thresh"]), "--remove_rings", "0", "--quad_convex"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    subprocess.run(cmd, cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    obj = np.fromfile(os.path.join(wd, "object_time_0.bin"), np.float32).reshape(4, 32, 32)
    cost = np.fromfile(os.path.join(wd, "cost.bin"), np.float64)
    np.savez_compressed(os.path.join(HERE, "recon_small.npz"), object=obj, cost=cost, threads=np.int32(4))
    print("recon", obj.shape, cost[-3:])


def recon_rings_fixture():
    """A full reference-driver run with ring correction (zero-mean offsets,
    remove_rings 2) and the quadratic data term: object, offsets, cost trace."""
    scan = synth.ellipsoid_scan(32, 4, 48, seed=13, ring_sigma=0.02)
    wd = tempfile.mkdtemp()
    scan.write_bin(wd)
    a = dict(RECON_ARGS, remove_rings=2)
    cmd = [REF_BIN, "--proj_rows", str(scan.proj_rows), "--proj_cols", str(scan.proj_cols), "--proj_num",
           str(scan.proj_num), "--recon_num", "1", "--vox_wid", str(scan.vox_wid), "--rot_center",
           str(scan.rot_center), "--sig_s", str(a["sig_s"]), "--sig_t", str(a["sig_t"]), "--c_s", str(a["c_s"]),
           "--c_t", str(a["c_t"]), "--convg_thresh", str(a["convg_thresh"]), "--remove_rings", "2", "--quad_convex"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    subprocess.run(cmd, cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    obj = np.fromfile(os.path.join(wd, "object_time_0.bin"), np.float32).reshape(4, 32, 32)
    off = np.fromfile(os.path.join(wd, "proj_offset.bin"), np.float32)
    cost = np.fromfile(os.path.join(wd, "cost.bin"), np.float64)
    np.savez_compressed(os.path.join(HERE, "recon_rings.npz"), object=obj, offset=off, cost=cost,
                        threads=np.int32(4))
    print("recon rings", obj.shape, off.shape, cost[-3:])


def upsample_fixture():
    """The reference's x2 up-sampling between stages on seeded random slices."""
    import ctypes as C
    lib = C.CDLL(REF_SO)
    lib.ref_upsample.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    rng = np.random.default_rng(31)
    out = {}
    for k, (nz, ny, nx) in enumerate([(4, 8, 8), (3, 5, 7), (2, 16, 2), (2, 2, 6)]):
        x = (rng.random((nz, ny, nx)) * 0.02).astype(np.float32)
        out[f"in{k}"] = x
        for z_too in (0, 1):
            oz = 2 * nz if z_too else nz
            y = np.zeros((oz, 2 * ny, 2 * nx), np.float32)
            lib.ref_upsample(x.ctypes.data, y.ctypes.data, nz, ny, nx, z_too)
            out[f"out{k}_{z_too}"] = y
    np.savez_compressed(os.path.join(HERE, "upsample.npz"), **out)
    print("upsample", sorted(out))


INGEST_CASES = {
    # name: (views, rows, cols, n_whites, n_darks, datafile_row0, proj_rows, proj_cols, proj_start, proj_num)
    "ratio1": (5, 8, 12, 4, 3, 0, 8, 12, 1, 3),
    "ratio2_trim": (6, 12, 27, 5, 4, 2, 4, 12, 0, 6),   # 27 columns: 3 trimmed, ratio 2
    "ratio3": (4, 9, 30, 6, 5, 0, 3, 10, 2, 2),
}
VIEW_CASES = [  # K, N_theta, proj_start, N_p, min_acq_time, rot_speed
    (16, 1024, 0, 1024, 0.0, 0.0), (32, 1024, 17, 200, 0.0, 0.0), (4, 256, 3, 150, 0.01, 1.5),
    (8, 24, 0, 40, 0.0, 0.0), (1, 64, 0, 70, 0.0, 0.0),
]


def ingest_fixture():
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_io.so"))
    VP, I = C.c_void_p, C.c_int
    lib.ref_read_aps.argtypes = [VP, I, VP, I, VP, I, I, I, I, I, I, I, I, VP, VP]
    lib.ref_read_std.argtypes = [VP, VP, I, I, I, I, I, I, I, I, VP, VP]
    lib.ref_gen_views.argtypes = [VP, VP, I, I, I, I, C.c_float, C.c_float]
    out = {}
    for k, (name, (n, rows, cols, nw, nd, r0, pr, pc, ps, pn)) in enumerate(sorted(INGEST_CASES.items())):
        rng = np.random.default_rng(70 + k)
        counts = rng.integers(50, 4000, size=(n, rows, cols)).astype(np.uint16)
        whites = rng.integers(4000, 6000, size=(nw, rows, cols)).astype(np.uint16)
        darks = rng.integers(0, 60, size=(nd, rows, cols)).astype(np.uint16)
        P = np.zeros((pn, pr, pc), np.float32)
        W = np.zeros_like(P)
        assert lib.ref_read_aps(counts.ctypes.data, n, whites.ctypes.data, nw, darks.ctypes.data, nd, rows, cols, r0,
                                pr, pc, ps, pn, P.ctypes.data, W.ctypes.data) == 0
        projs = rng.normal(1.0, 0.5, size=(n, rows, cols)).astype(np.float32)
        wts = rng.uniform(10, 1000, size=(n, rows, cols)).astype(np.float32)
        Ps = np.zeros_like(P)
        Ws = np.zeros_like(P)
        assert lib.ref_read_std(projs.ctypes.data, wts.ctypes.data, n, rows, cols, r0, pr, pc, ps, pn, Ps.ctypes.data,
                                Ws.ctypes.data) == 0
        for key, v in dict(counts=counts, whites=whites, darks=darks, aps_proj=P, aps_weight=W, std_in_proj=projs,
                           std_in_weight=wts, std_proj=Ps, std_weight=Ws,
                           params=np.array([n, rows, cols, nw, nd, r0, pr, pc, ps, pn], np.int32)).items():
            out[f"{name}/{key}"] = v
    for k, (K, Nt, ps, npv, mat, rs) in enumerate(VIEW_CASES):
        v = np.zeros(npv, np.float32)
        t = np.zeros(npv, np.float32)
        kept = lib.ref_gen_views(v.ctypes.data, t.ctypes.data, K, Nt, ps, npv, mat, rs)
        out[f"views{k}/angles"] = v
        out[f"views{k}/times"] = t
        out[f"views{k}/kept"] = np.int32(kept)
        out[f"views{k}/params"] = np.array([K, Nt, ps, npv, mat, rs], np.float64)
    np.savez_compressed(os.path.join(HERE, "ingest.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "ingest":
        ingest_fixture()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "upsample":
        upsample_fixture()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "recon_rings":
        recon_rings_fixture()
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[1] == "stage":  # named scenarios only
        stage_fixtures(sys.argv[2:])
        sys.exit(0)
    if not Reference.available():
        sys.exit("build the reference first: make -C oracle ref")
    park_miller_table()
    stage_fixtures()
    recon_fixture()
    recon_rings_fixture()
    upsample_fixture()
