#!/usr/bin/env python
"""Benchmark: ICD voxel-updates/s of the finest multi-resolution stage.

Workload (the 3-D single-GPU configuration): a seeded random-ellipsoid phantom
(10 ellipsoids, attenuation 0-0.02), volume 256 x 256 x 8, 256 views uniform
over 180 degrees, 256 detector columns x 8 rows, Poisson counts at I0 = 1e4
(weights = counts), qGGMRF p = 1.2, q = 2, c_s = 1 (T = 1), sigma_s = 0.002
(a tenth of the phantom's range), quadratic data term (quad_convex = 1), no
ring correction.  The stage starts warm, from the 2x-coarser phantom
up-sampled, as the multi-resolution driver hands it over.  A step is one outer
ICD iteration (updateVoxelsTimeSlices: HICD sweep, NHICD sweeps from the
second iteration, zero skipping).  The metric counts executed voxel updates.

Arms:
  (default)          the GPU engine (libtimbir_b200.so) through its C ABI
  --impl reference   the reference's own CPU implementation, built from its
                     sources (oracle/_ref/XT_Main_ref), in restart mode at the
                     same stage, all host threads; else the CPU restatement.

Under torchrun (N > 1 GPUs) every rank reconstructs its own copy of the
workload (independent problems, weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from timbir_b200 import synth  # noqa: E402

class Workload:
    """A benchmark configuration: scan, prior, warm start, stage count."""

    def __init__(self, name, desc, n_xy, rows, views, frames, prior, data):
        self.name, self.desc, self.n_xy, self.rows, self.views, self.frames = name, desc, n_xy, rows, views, frames
        self.prior, self.data = prior, data

    @property
    def stages(self):
        # multi-resolution stage count of reconstruct() (XT_Engine.c:111-141)
        n = max(2, min(8, int(np.log(self.n_xy / 64.0) / np.log(2.0) + 1)))
        return n

    def scan(self, seed_offset=0):
        if self.name == "3d":
            return synth.ellipsoid_scan(self.n_xy, self.rows, self.views, I0=1e4, seed=seed_offset)
        if self.name == "c5":
            # densities scaled by 256 / 2048 so that line integrals match the 3-D workload's
            return synth.moving_ellipsoid_scan(self.n_xy, self.rows, self.frames, 1536, 32, 4, I0=1e4,
                                               seed=seed_offset, vmax=0.02 * 256 / self.n_xy)
        return fourd_scan(self, seed_offset)

    def warm_start(self, scan):
        """The 2x-coarser phantom (mean over 2x2x2 cells) and its trilinear x2
        up-sampling onto the stage grid: the warm start both arms use."""
        if scan.phantom is None:  # no phantom kept: the stage starts from zero
            z = np.zeros((self.frames, self.rows, self.n_xy, self.n_xy), np.float32)
            return z, z
        coarse, fine = [], []
        for ph in scan.phantom:
            c, f = coarse_start_frame(ph)
            coarse.append(c)
            fine.append(f)
        return np.stack(coarse), np.stack(fine)


W3D = Workload("3d", "3d-shepp-logan-like 256x256x8, 256 views, I0=1e4, finest stage", 256, 8, 256, 1,
               dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=0, quad_convex=1,
                    huber_delta=0.5, huber_T=4.0),
               "synthetic (seeded random-ellipsoid phantom, Poisson counts)")
W4D = Workload("4d", "4d two-phase microstructure 16 x 256x256x16, 1024 interlaced views (K=16, 8 rotations), "
               "I0=5e3, 0.1% zingers, rings, finest stage", 256, 16, 1024, 16,
               dict(sig_s=0.002, sig_t=0.004, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=2, quad_convex=0,
                    huber_delta=0.5, huber_T=4.0),
               "synthetic (seeded Gaussian-random-field two-phase frames, Poisson counts, zingers, rings)")
WC5 = Workload("c5", "large 4d z-subset: 32 x 2048x2048 x 4 of 64 detector rows, 6144 interlaced views "
                "(K=32, 4 rotations of 1536, 192 per frame), densities 0-0.0025, I0=1e4, 0.1% zingers, rings, from "
                "zero; the full "
                "64-row configuration's time per iteration is this one's x 16 (extrapolated)", 2048, 4, 6144, 32,
               dict(sig_s=0.00025, sig_t=0.0005, c_s=1.0, c_t=1.0, convg_thresh=0.0, remove_rings=2, quad_convex=0,
                    huber_delta=0.5, huber_T=4.0),
               "synthetic (seeded drifting random ellipsoids, exact line integrals, Poisson counts, zingers, rings)")
W4DC = Workload("4dc", "4d two-phase microstructure 16 x 256x256x16 as the 4d workload (zingers and rings in the "
                "data), convex model: quadratic data term (quad_convex=1), no ring correction (remove_rings=0), "
                "finest stage", 256, 16, 1024, 16, dict(W4D.prior, quad_convex=1, remove_rings=0), W4D.data)
WORKLOADS = {"3d": W3D, "4d": W4D, "4dc": W4DC, "c5": WC5}


def finest_stage_switches(prior):
    """Stage switches of the finest multi-resolution stage (XT_Init.c:245-266,
    XT_Engine.c:111-141): ring offsets updated (mode 3, starting from the
    offsets handed over) when remove_rings > 0, the variance re-estimated
    when quad_convex = 0."""
    sw = {}
    if prior["remove_rings"]:
        sw["update_proj_offset"] = 3
    if not prior["quad_convex"]:
        sw["update_var"] = 1
        sw["var_est"] = 1.0
    return sw


def zero_offsets(scan):
    """Ring offsets [N_r][N_t] handed to the finest stage: zero (as
    PROJ_OFFSET_INIT leaves them on the reference's first stage)."""
    return np.zeros((scan.proj_cols, scan.proj_rows), np.float32)


def workload_stage(w, scan, sched, args, prior=None):
    """A finest-stage Stage of workload w with its schedule and switches."""
    import timbir_b200
    prior = prior or w.prior
    st = timbir_b200.Stage(scan, **prior, blocks=2 if w.rows < 8 else 8)
    st.set_switches(**finest_stage_switches(prior))
    if args.zgroup:
        st.set_sv_zgroup(args.zgroup)
    if getattr(args, "sv_alpha", 0.0):
        st.set_sv_relaxation(args.sv_alpha)
    if getattr(args, "sv_ctas", 0):
        st.set_sv_ctas(args.sv_ctas)
    st.set_schedule(sched, args.sv_side, args.warps_per_slice, args.acache)
    if sched and getattr(args, "nhicd", -1.0) >= 0:
        st.set_sv_nhicd(args.nhicd)
    return st


METRIC = "ICD voxel-updates/s"
# DRAM bytes (read + write) per voxel update of the super-voxel kernel, from
# one ncu capture of a full-sweep launch on the 3-D workload (217.6 MB read +
# 5.8 MB written over its 411,744 in-mask voxels); the line's roofline.traffic
# scales it to the average launch.
DRAM_BYTES_PER_UPDATE = {"3d": (218.342e6 + 5.682e6) / 411744}


def fourd_scan(w, seed_offset=0):
    """Config-2 stand-in: thresholded smoothed Gaussian random field coarsened
    by curvature-flow steps, 16 frames; views interlaced in K = 16 sub-frames,
    8 rotations of 128 views, 64 views per frame; line integrals of the
    voxelised frames (synth.project_frames, float64 on the CPU), Poisson counts
    at I0 = 5e3, 0.1% of readings x10 (zingers), per-(row, column) log offsets
    ~ N(0, 0.02) (rings)."""
    rng = np.random.default_rng(100 + seed_offset)
    frames = synth.two_phase_frames(w.n_xy, w.rows, w.frames, seed=seed_offset)
    angles = synth.interlaced_angles(16, w.views, 128)
    times = np.arange(w.views, dtype=np.float32)
    rt = np.linspace(0, w.views, w.frames + 1).astype(np.float32)
    li = synth.project_frames(frames, angles, rt, times, w.n_xy)
    proj, wts = synth.counts_to_data(li, 5e3, rng, zinger_frac=0.001, ring_sigma=0.02)
    return synth.Scan(proj, wts, angles, times, rt, w.rows, w.n_xy, w.views, w.frames, 1.0, w.n_xy / 2.0, frames)


def coarse_start_frame(ph):
    z, y, x = ph.shape
    coarse = ph.reshape(z // 2, 2, y // 2, 2, x // 2, 2).mean(axis=(1, 3, 5)).astype(np.float32)

    def up(a, axis):
        n = a.shape[axis]
        a = np.moveaxis(a, axis, 0)
        out = np.empty((2 * n,) + a.shape[1:], np.float64)
        out[0], out[-1] = a[0], a[-1]
        out[1] = (3.0 * a[0] + a[1]) / 4.0
        out[-2] = (a[-2] + 3.0 * a[-1]) / 4.0
        out[2:2 * n - 2:2] = (a[0:n - 2] + 3.0 * a[1:n - 1]) / 4.0
        out[3:2 * n - 2:2] = (3.0 * a[1:n - 1] + a[2:n]) / 4.0
        return np.moveaxis(out, 0, axis)

    fine = up(up(up(coarse.astype(np.float64), 2), 1), 0).astype(np.float32)
    return coarse, fine


def mean_amatrix_count(stage, scan):
    """Mean number of detector bins per (voxel line, view) of the A matrix over
    the in-mask lines (the c-bar of the algorithmic byte count), from the
    same index arithmetic as the kernels, in float64 numpy."""
    hr = stage.hr().astype(np.float64)
    n, dr = scan.proj_cols, scan.vox_wid
    R0 = -scan.rot_center * dr
    off_r = (dr / np.sqrt(2.0) + dr / 2.0) / 64
    k = np.arange(n)
    x = R0 + (k + 0.5) * dr
    y = -n * dr / 2.0 + (k + 0.5) * dr
    X, Y = np.meshgrid(x, y)
    m = stage.mask().astype(bool).reshape(X.shape)
    X, Y = X[m], Y[m]
    if len(X) > 20000:  # a seeded sample of lines on large images
        pick = np.random.default_rng(0).choice(len(X), 20000, replace=False)
        X, Y = X[pick], Y[pick]
    vstep = max(4, scan.proj_num // 256)
    total = 0
    for v in range(0, scan.proj_num, vstep):
        c, s = np.cos(np.float64(scan.proj_angles[v])), np.sin(np.float64(scan.proj_angles[v]))
        r = X * c - Y * s
        imin = np.maximum(np.floor((r - dr - R0) / dr), 0).astype(int)
        imax = np.minimum(np.floor((r + dr - R0) / dr), n - 1).astype(int)
        for d in range(0, 4):
            j = imin + d
            ok = j <= imax
            rc = R0 + (j + 0.5) * dr
            dd = np.abs(r - rc)
            idx = np.floor(dd / off_r).astype(int)
            ok &= (idx >= 0) & (idx < 64)
            idc = np.clip(idx, 0, 63)
            w1 = dd - idc * off_r
            f = (off_r - w1) * hr[v, idc] + w1 * hr[v, idc + 1]
            total += int(np.count_nonzero(ok & (f > 0)))
    return total / (len(X) * len(range(0, scan.proj_num, vstep)))


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons while the timed region
    runs: NVML polled every 2 ms from a thread (the timed region of a small
    workload lasts a few milliseconds, shorter than nvidia-smi's sampling
    period), nvidia-smi at 200 ms where NVML cannot be loaded.  Read-only
    queries; no setting of the GPU is touched."""

    Q = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    # NVML clock-event reason bits (nvml.h): HW slowdown 0x8, HW thermal 0x40,
    # SW thermal 0x20, SW power cap 0x4
    BITS = [0x8, 0x40, 0x20, 0x4]

    def __init__(self, index):
        self.index, self.rows, self.proc, self.nvml, self.stop = index, [], None, None, None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:  # the CUDA device's own PCI address (CUDA_VISIBLE_DEVICES renumbers devices)
            import torch
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            self.nvml, h = self._nvml_handle()
            nv = self.nvml
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def poll():
                while True:
                    sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                    self.rows.append((sm, r))
                    if self.stop.wait(0.002):
                        return

            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.stop is not None:
            self.stop.set()
            self.t.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        if self.nvml is not None:
            sm = [r[0] for r in self.rows]
            reasons = sorted({n for _, r in self.rows for n, b in zip(self.NAMES, self.BITS) if r & b})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, 2 ms polling"}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(self.rows[0][2]) if self.rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# --------------------------------------------------------------------- CPU --
def run_reference_binary(w, scan, coarse, iters, threads):
    """Reference driver in restart mode at the finest stage: the files a
    finished coarser stage leaves behind are written, then XT_Main_ref runs
    `iters` ICD iterations (ORACLE_MAX_ITERS).  Returns [(seconds, updates)]."""
    from oracle.bind import REF_BIN
    wd = tempfile.mkdtemp(prefix="timbir_ref_")
    scan.write_bin(wd)
    p = np.transpose(scan.projections, (0, 2, 1)).astype(np.float32)  # [view][col][row]
    wt = np.transpose(scan.weights, (0, 2, 1)).astype(np.float32)
    p.tofile(os.path.join(wd, "projs_runtime.bin"))
    wt.tofile(os.path.join(wd, "weights_runtime.bin"))
    np.array([1.0], np.float64).tofile(os.path.join(wd, "variance_estimate.bin"))
    np.zeros((scan.proj_cols, scan.proj_rows), np.float32).tofile(os.path.join(wd, "proj_offset.bin"))
    for f in range(scan.recon_num):
        coarse[f].astype(np.float32).tofile(os.path.join(wd, f"object_time_{f}.bin"))
    np.zeros(scan.recon_num * scan.proj_rows * scan.proj_cols * scan.proj_cols, np.float32).tofile(
        os.path.join(wd, "mag_update.bin"))
    np.array([w.stages - 1], np.int32).tofile(os.path.join(wd, "status.bin"))
    a = w.prior
    cmd = [REF_BIN, "--proj_rows", str(scan.proj_rows), "--proj_cols", str(scan.proj_cols), "--proj_num",
           str(scan.proj_num), "--recon_num", str(scan.recon_num), "--vox_wid", str(scan.vox_wid), "--rot_center",
           str(scan.rot_center), "--sig_s", str(a["sig_s"]), "--sig_t", str(a["sig_t"]), "--c_s", str(a["c_s"]),
           "--c_t", str(a["c_t"]), "--convg_thresh", str(a["convg_thresh"]), "--remove_rings",
           str(a["remove_rings"]), "--huber_delta", str(a["huber_delta"]), "--huber_T", str(a["huber_T"]),
           "--restart"] + (["--quad_convex"] if a["quad_convex"] else [])
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), ORACLE_MAX_ITERS=str(iters))
    r = subprocess.run(cmd, cwd=wd, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
                       timeout=1800)
    shutil.rmtree(wd, ignore_errors=True)
    out = []
    for line in r.stderr.splitlines():
        if line.startswith("ORACLE_ITER"):
            _, n, dt, upd = line.split()
            out.append((float(dt), int(upd)))
    if not out:
        raise RuntimeError("reference run produced no iterations: " + r.stderr[-500:])
    return out


def run_port(w, scan, coarse_fine, iters):
    """CPU restatement (single thread), when the reference build is absent."""
    from oracle.bind import Oracle
    o = Oracle(scan, **w.prior, blocks=2)
    o.prepare(coarse_fine)
    out = []
    last = 0
    for it in range(1, iters + 1):
        t0 = time.perf_counter()
        o.iterate(it)
        dt = time.perf_counter() - t0
        out.append((dt, o.update_count() - last))
        last = o.update_count()
    o.close()
    return out


def cpu_measure(w, scan, coarse, fine, warm, steps, threads):
    from oracle.bind import Reference
    if Reference.available() and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "XT_Main_ref")):
        its = run_reference_binary(w, scan, coarse, warm + steps, threads)
        kind, cores = "reference", threads
    else:
        its = run_port(w, scan, fine, warm + steps)
        kind, cores = "port", 1
    timed = its[warm:] if len(its) > warm else its
    secs = sum(t for t, _ in timed)
    upd = sum(u for _, u in timed)
    cpu_measure.iterations = its  # every iteration's (seconds, updates), warm-up included
    return upd / secs, kind, cores, len(timed), secs


def reference_time_to_map(w, scan, its, kind):
    """The reference's time-to-MAP on this host: its iterations to (1 + 1e-5) C*
    from the bench's warm start (counted where the fixture was made, from a
    fresh FP64 cost after each iteration of the reference library) times the
    iteration times this run measured -- the sum of the first ones when the run
    went that far, else their mean x the count (labelled extrapolated)."""
    ref = reference_map(w, scan)
    if not ref or not ref["ref_iterations"] or ref["ref_iterations"] < 0 or kind != "reference":
        return None
    n = ref["ref_iterations"]
    secs = [t for t, _ in its]
    if len(secs) >= n:
        v, how = sum(secs[:n]), f"measured: the first {n} iterations of this run"
    else:
        v, how = n * sum(secs) / len(secs), f"extrapolated: {n} x the mean of {len(secs)} measured iterations"
    return {"value": v, "unit": "s", "iterations": n, "target": "FP64 MAP cost <= (1 + 1e-5) C*",
            "cstar": ref["cstar"], "timed": how,
            "iterations_source": "reference library from the same warm start, fresh FP64 cost after each iteration "
                                 "(tests/golden/converged_%s.npz)" % w.name}


# ------------------------------------------------------------ batched (c3) --
C3_DESC = ("64 independent 3-D random-ellipsoid problems in one persistent launch per iteration (CUDA-graph "
           "replays): side from {128,192,256,384,512}, 4-32 slices (even), 1.5 x side views over 180 degrees, "
           "I0 log-uniform in [2e3, 5e4], seeds 0-63, from zero, plain ICD")
C3_PRIOR = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=1.0, remove_rings=0, quad_convex=1,
                huber_delta=0.5, huber_T=4.0)
C3_DATA = "synthetic (seeded random-ellipsoid phantoms, exact line integrals, Poisson counts)"


def c3_problem_workload(specs, k):
    sp = specs[k]
    prior = dict(C3_PRIOR, convg_thresh=0.0)
    return Workload("c3-sample", f"problem {k} of the batch: {sp['side']}x{sp['side']}x{sp['slices']}, "
                    f"{sp['views']} views, I0={sp['I0']:.0f}", sp["side"], sp["slices"], sp["views"], 1, prior, C3_DATA)


def c3_cpu_baseline(specs, weights, threads):
    """The reference's CPU rate on the batch: for each problem size, one ICD
    iteration (after one warm-up) of that size's problem with the fewest
    slices, run from zero; the per-size rates are combined as one sequential
    pass over every problem of the batch, each weighted by `weights` (its
    voxel updates per iteration), i.e. total updates / sum(updates / rate of
    its size).  Returns (rate, per-size dict, kind, cores, seconds)."""
    by_side = {}
    for k, sp in enumerate(specs):
        if sp["side"] not in by_side or sp["slices"] < specs[by_side[sp["side"]]]["slices"]:
            by_side[sp["side"]] = k
    per, kind, cores, secs_all = {}, None, None, 0.0
    for side, k in sorted(by_side.items()):
        sp = specs[k]
        w = c3_problem_workload(specs, k)
        scan = synth.ellipsoid_scan(sp["side"], sp["slices"], sp["views"], I0=sp["I0"], seed=sp["seed"])
        z = np.zeros((1, w.rows // 2, w.n_xy // 2, w.n_xy // 2), np.float32)
        zf = np.zeros((1, w.rows, w.n_xy, w.n_xy), np.float32)
        v, kind, cores, n, secs = cpu_measure(w, scan, z, zf, 1, 1, threads)
        per[str(side)] = {"value": v, "problem": k, "slices": sp["slices"], "views": sp["views"], "seconds": round(secs, 2)}
        secs_all += secs
    total = float(sum(weights))
    t = sum(float(weights[k]) / per[str(sp["side"])]["value"] for k, sp in enumerate(specs))
    return total / t, per, kind, cores, secs_all


def c3_build(specs, scans, tuned=None, autotune=True):
    """Stages of the batch (column cache, super-voxel schedule, prepared from
    zero); with `tuned` = {side: autotuner result} the schedule of each size
    is the tuned one, otherwise the representative of each size (most slices)
    is autotuned here and the others follow it."""
    import timbir_b200
    stages = [None] * len(specs)
    tune = {}
    reps = {}
    for k, sp in enumerate(specs):
        if sp["side"] not in reps or sp["slices"] > specs[reps[sp["side"]]]["slices"]:
            reps[sp["side"]] = k
    order = sorted(range(len(specs)), key=lambda k: (k not in reps.values(), k))
    for k in order:
        sp = specs[k]
        st = timbir_b200.Stage(scans[k], **C3_PRIOR, blocks=2)
        t = (tuned or tune).get(sp["side"])
        if t is None and not autotune:
            st.set_batch_schedule(0, 1, 1)
            st.prepare()
            info = st.schedule_info()
            t = {"sv_side": info["sv_side"], "warps_per_slice": info["warps_per_slice"],
                 "z_group": info["z_group"], "band_width": info["band_width"], "ns_per_update": 0.0}
            tune[sp["side"]] = t
        elif t is None:
            st.set_batch_schedule(0, 1, 1)
            st.prepare()
            t = st.autotune()
            tune[sp["side"]] = t
        else:
            st.set_batch_schedule(t["sv_side"], t["warps_per_slice"], 1)
            st.prepare()
        stages[k] = st
    return stages, (tuned or tune)


def c3_arm(args, rank, world, local_rank):
    import torch
    import timbir_b200
    torch.cuda.set_device(local_rank)
    specs = synth.batch_problem_specs(64, 0)[:args.problems]
    t0 = time.perf_counter()
    scans = [synth.ellipsoid_scan_device(sp["side"], sp["slices"], sp["views"], I0=sp["I0"], seed=sp["seed"],
                                         device="cuda") for sp in specs]
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    stages, tuned = c3_build(specs, scans, autotune=not args.no_tune)
    setup_s = time.perf_counter() - t0
    cbar = {}
    for k, sp in enumerate(specs):
        if sp["side"] not in cbar:
            cbar[sp["side"]] = mean_amatrix_count(stages[k], scans[k])
    b_vu = [sp["views"] * (cbar[sp["side"]] * 12 + 2 * cbar[sp["side"]] + 2) + 29 * 4 + 4 for sp in specs]
    # throughput: every problem iterating (convergence test off)
    for st in stages:
        st.set_convergence_threshold(0.0)
    batch = timbir_b200.Batch(stages)
    binfo = batch.info()
    for _ in range(args.warmup):
        batch.iterate(1)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)
    u0 = batch.stats()["updates"].copy()
    i0 = batch.info()
    step_ms = []
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            m0 = batch.info()["ms"]
            batch.iterate(1)
            step_ms.append(batch.info()["ms"] - m0)
    i1 = batch.info()
    du = batch.stats()["updates"] - u0
    updates = int(du.sum())
    total_ms = sum(step_ms)
    achieved = float(sum(int(du[k]) * b_vu[k] for k in range(len(specs)))) / (total_ms / 1e3) / 1e9
    batch.close()
    # time until every problem passes the reference's convergence test (1 %)
    ttc = None
    if not args.no_ttm:
        for st in stages:
            st.set_convergence_threshold(C3_PRIOR["convg_thresh"])
            st.prepare(st.fbp() if args.c3_start == "fbp" else None)
        batch = timbir_b200.Batch(stages)
        left = batch.iterate(200, check_every=1)
        bst = batch.stats()
        adj = [st.schedule_info()["stability_adjustments"] for st in stages]
        un = [k for k in range(len(specs)) if not bst["converged"][k]]
        ttc = {"value": batch.info()["ms"] / 1e3, "unit": "s", "iterations_max": int(bst["iterations"].max()),
               "iterations_mean": float(bst["iterations"].mean()), "unconverged": int(left),
               "unconverged_problems": [{"problem": k, "side": specs[k]["side"], "slices": specs[k]["slices"],
                                         "views": specs[k]["views"], "I0": round(specs[k]["I0"]),
                                         "last_pct": float(bst["percent"][k])} for k in un],
               "target": "every problem's convergence ratio below convg_thresh = 1 % (XT_ICD_update.c:1066-1103)",
               "start": "filtered backprojection (this library's FBP kernels)" if args.c3_start == "fbp" else "zero",
               "stability_adjustments": {"total": int(sum(adj)), "problems": int(sum(1 for a in adj if a))},
               "timed": "graph replays of the batched iterations and the per-problem cost guard (device events)"}
        batch.close()
    for st in stages:
        st.close()
    # end to end through the public API from pinned host buffers: stages,
    # schedules (the tuned ones), prologue, one batched iteration, objects back
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    pscans = [synth.Scan(pin(s.projections), pin(s.weights), pin(s.proj_angles), pin(s.proj_times),
                         pin(s.recon_times), s.proj_rows, s.proj_cols, s.proj_num, s.recon_num, s.vox_wid,
                         s.rot_center) for s in scans]
    h2d = sum(a.nbytes for s in pscans for a in (s.projections, s.weights, s.proj_angles, s.proj_times,
                                                  s.recon_times))
    d2h = sum(4 * sp["side"] ** 2 * sp["slices"] for sp in specs)
    pouts = [pin(np.zeros((1, sp["slices"], sp["side"], sp["side"]), np.float32)) for sp in specs]
    flush.fill_(0.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    # the whole solve a user runs: stages, the FBP start, the batched
    # iterations until every problem passes the 1 % test, objects back
    est, _ = c3_build(specs, pscans, tuned)
    for st in est:
        st.set_convergence_threshold(C3_PRIOR["convg_thresh"])
        if args.c3_start == "fbp":
            st.prepare(st.fbp())
    eb = timbir_b200.Batch(est)
    e_left = eb.iterate(200, check_every=1)
    e_st = eb.stats()
    e_upd = int(e_st["updates"].sum())
    e_iters = int(e_st["iterations"].max())
    eb.close()
    for st, o in zip(est, pouts):
        st.object(out=o)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    for st in est:
        st.close()
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    sizes = {}
    for sp, d in zip(specs, du):
        z = sizes.setdefault(str(sp["side"]), {"problems": 0, "updates_per_iteration": 0})
        z["problems"] += 1
        z["updates_per_iteration"] += int(d) // max(args.steps, 1)
    for side, t in tuned.items():
        sizes[str(side)].update({"views": (3 * side) // 2, "sv_side": t["sv_side"], "band_width": t["band_width"],
                                 "warps_per_slice": t["warps_per_slice"],
                                 "threads_per_voxel": 32 * t["warps_per_slice"], "z_group": t["z_group"],
                                 "ns_per_update_tuning": round(t["ns_per_update"], 3),
                                 "mean_bins_per_view": cbar[side]})
    line = {
        "metric": METRIC, "value": updates / (total_ms / 1e3), "unit": "voxel-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (A-matrix bin indices exact in FP64; convergence sums FP64)", "data": C3_DATA,
        "config": {"workload": C3_DESC + ("" if len(specs) == 64 else f"; the first {len(specs)} problems only")
                   + ("; default schedules, not autotuned" if args.no_tune else ""), "problems": len(specs), "voxels": int(sum(sp["side"] ** 2 * sp["slices"]
                                                                             for sp in specs)),
                   "schedule": "batched super-voxel (one persistent launch + one end kernel per iteration, "
                               "CUDA graph)", "ctas": binfo["ctas"], "smem_bytes_per_cta": binfo["smem_bytes"],
                   "autotuned_per_size": sizes, "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MB write)",
                   "setup_s": {"scan_generation": round(gen_s, 2), "stages_and_autotune": round(setup_s, 2)}},
        "e2e": {"value": e_upd / (e2e_ms / 1e3), "unit": "voxel-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "step_ms": [round(e2e_ms, 3)], "updates_per_step": e_upd,
                "includes": "64 stages from pinned host arrays, column caches, schedules, prologue, the start "
                            f"({'FBP' if args.c3_start == 'fbp' else 'zero'}), the batched iterations until every "
                            f"problem passes the 1 % test ({e_iters} at most, {e_left} left), 64 objects back into "
                            "pinned memory"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "bytes_per_update": "views x (c-bar x 14 + 2) + 120 per problem",
                     "kernel": "k_icd_sv (batched)", "kernel_ms": total_ms,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "gpu_launches": int(i1["launches"] - i0["launches"]),
        "clocks": clk.summary(),
    }
    if ttc:
        line["time_to_converge"] = ttc
    if not args.no_cpu:
        v, per, kind, cores, secs = c3_cpu_baseline(specs, [int(d) for d in du], os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": v, "unit": "voxel-updates/s", "cores": cores, "kind": kind,
                                "sample": "per problem size, one ICD iteration after one warm-up of its problem with "
                                          "the fewest slices (from zero), %.1f s in all; combined as one sequential pass "
                                          "over the batch weighted by each problem's updates" % secs,
                                "per_size": per}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ learned warm start --
C4_DESC = ("learned warm start: 3-D encoder-decoder network (4 levels, 16-128 channels, 1.33 M parameters) trained "
           "on (FBP, plain-ICD MBIR) pairs of seeded random-ellipsoid and two-phase Gaussian-random-field phantoms, "
           "256x256x16, 384 views, I0 log-uniform in [2e3, 5e4]; start = its output with the FBP's low frequencies "
           "(Gaussian low-pass of 1 slice x 4 x 4 voxels) kept; ICD from that start vs from FBP to (1 + 1e-5) C*")
C4_PRIOR = dict(W3D.prior)
C4_DATA = ("synthetic (seeded random-ellipsoid phantoms with exact line integrals, and two-phase Gaussian-random-field "
           "phantoms projected on the CPU; Poisson counts)")


def c4_scan(k, n_xy=256, rows=16, views=384):
    """Scan k of the learned-warm-start workload: even k a random-ellipsoid
    phantom, odd k a two-phase Gaussian-random-field phantom."""
    rng = np.random.default_rng(5000 + k)
    I0 = float(np.exp(rng.uniform(np.log(2e3), np.log(5e4))))
    if k % 2 == 0:
        return synth.ellipsoid_scan_device(n_xy, rows, views, I0=I0, seed=5000 + k)
    ph = synth.two_phase_frames(n_xy, rows, 1, seed=5000 + k)
    angles = (np.arange(views) * np.pi / views).astype(np.float32)
    times = np.arange(views, dtype=np.float32)
    rt = np.array([0.0, float(views)], np.float32)
    li = synth.project_frames(ph, angles, rt, times, n_xy)
    proj, wts = synth.counts_to_data(li, I0, rng)
    return synth.Scan(proj, wts, angles, times, rt, rows, n_xy, views, 1, 1.0, n_xy / 2.0, ph)


def c4_stage(scan, prior=None, blocks=2, acache=-1):
    import timbir_b200
    st = timbir_b200.Stage(scan, **(prior or C4_PRIOR), blocks=blocks)
    st.set_schedule(1, 0, 0, acache)
    return st


def icd_from(scan, start, cstar=None, max_iters=600, flat=1e-10, prior=None, blocks=2, acache=-1):
    """Plain GPU ICD from `start`: with cstar, device time and iterations
    until the FP64 cost is within (1 + 1e-5) cstar; without, iterations until
    two successive costs agree to `flat` (the converged cost C*).  Returns
    (iterations, ms of the ICD iterations, last cost, object)."""
    st = c4_stage(scan, prior, blocks, acache)
    st.prepare(start)
    ms, prev, c = 0.0, None, None
    for it in range(1, max_iters + 1):
        st.time_begin()
        st.iterate(it)
        ms += st.time_end()
        c = st.cost()[0]
        if cstar is not None and c <= (1.0 + 1e-5) * cstar:
            break
        if cstar is None and prev is not None and abs(prev - c) <= flat * abs(c):
            break
        prev = c
    x = st.object()
    st.close()
    return it, ms, c, x


def edge_weights(T, beta):
    """Per-voxel loss weights 1 + beta |grad T| / mean |grad T| of target
    volumes T (CUDA [N][D][H][W]; central differences, zero on the border):
    the loss leans on the MAP images' edges, where an ICD start's error
    decays slowest."""
    import torch
    g2 = torch.zeros_like(T)
    for ax in (1, 2, 3):
        n = T.shape[ax]
        if n < 3:
            continue
        d = (T.narrow(ax, 2, n - 2) - T.narrow(ax, 0, n - 2)) * 0.5
        g2.narrow(ax, 1, n - 2).add_(d * d)
    g = g2.sqrt()
    return (1.0 + beta * g / g.mean().clamp_min(1e-30)).contiguous()


def c4_arm(args, rank, world, local_rank, four_d=False, n_train=32, steps=2000):
    """Learned warm start: training pairs from the plain method, the network
    trained on them, then ICD from its output against ICD from FBP on held-out
    scans.  four_d: the 4-D workload (16 frames, 64 interlaced views per
    frame, zingers and rings), trained on 4-D scans of other seeds, evaluated
    on the bench's own 4-D scan, the warm run with FP16 A-matrix values."""
    import torch
    import timbir_b200
    from timbir_b200 import warm
    torch.cuda.set_device(local_rank)
    if four_d:
        w = W4D
        prior, blocks = w.prior, 8
        scan_of = lambda k: fourd_scan(w, 100 + k)  # noqa: E731
        held_out = [(fourd_scan(w, 0), "two-phase microstructure, 16 frames (the 4-D workload's scan)")]
        n_train, acache_warm = 4, -1
    else:
        prior, blocks, scan_of, acache_warm = C4_PRIOR, 2, c4_scan, -1
        held_out = [(c4_scan(1000), "random ellipsoids"), (c4_scan(1001), "two-phase Gaussian random field")]
    kw = dict(prior=prior, blocks=blocks)
    t0 = time.perf_counter()
    fbps, tgts = [], []
    target_iters = []
    for k in range(n_train):
        sc = scan_of(k)
        st = c4_stage(sc, prior, blocks)
        f = st.fbp()
        st.close()
        # target: the converged MAP image (ICD from the FBP until the cost is flat)
        n_it, _, _, x_map = icd_from(sc, f, max_iters=400, **kw)
        target_iters.append(n_it)
        fbps.extend(list(f))
        tgts.extend(list(x_map))
    data_s = time.perf_counter() - t0
    X = torch.from_numpy(np.stack(fbps)).cuda()
    T = torch.from_numpy(np.stack(tgts)).cuda()
    beta = float(getattr(args, "c4_edge_weight", 0.0))
    WT = edge_weights(T, beta) if beta > 0 else None
    net = warm.WarmNet(seed=7)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    hp = warm.BLEND_SIGMA if getattr(args, "c4_loss", "highpass") == "highpass" else None
    losses = warm.train(net, X, T, steps=steps, batch=4, patch=(16, 64, 64), lr=1e-3, seed=3, weights=WT,
                        highpass=hp)
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    pairs = int(X.shape[0])
    del X, T, WT
    results = []
    for sc, name in held_out:
        st = c4_stage(sc, prior, blocks)
        mask = st.mask().astype(np.float32)
        fbp = st.fbp()  # untimed first call
        warm.warm_start(net, fbp, mask)  # the network's buffers, allocated once
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        fbp = st.fbp()
        f1.record()
        torch.cuda.synchronize()
        fbp_ms = f0.elapsed_time(f1)
        st.close()
        f0.record()
        ws = warm.warm_start(net, fbp, mask)
        f1.record()
        torch.cuda.synchronize()
        net_ms = f0.elapsed_time(f1)
        n_star, _, cstar, x_star = icd_from(sc, fbp, max_iters=800, **kw)
        n_plain, ms_plain, c_plain, x_plain = icd_from(sc, fbp, cstar, **kw)
        n_warm, ms_warm, c_warm, x_warm = icd_from(sc, ws, cstar, acache=acache_warm, **kw)
        rng_ = float(x_star.max() - x_star.min())
        rm = lambda a: float(np.sqrt(np.mean((a - x_star) ** 2))) / rng_  # noqa: E731
        # how far ICD's iteration count moves with the start: the FBP's error
        # halved everywhere, and the FBP's low frequencies under the MAP
        # image's high frequencies (Gaussian low-pass, sigma 2 slices x 8 x 8)
        from scipy import ndimage
        lp = lambda a: ndimage.gaussian_filter(a.astype(np.float64), sigma=(0, 2, 8, 8)).astype(np.float32)  # noqa
        sens = {}
        # and the network's output as it is, and with the FBP's frequencies
        # kept under a wider low-pass than the warm start's (1 slice x 4 x 4)
        ws_raw = warm.warm_start(net, fbp, mask, blend=None)
        for key, s0 in (("fbp_error_halved", 0.5 * (fbp + x_star)),
                        ("map_high_frequencies_fbp_low", lp(fbp) + (x_star - lp(x_star))),
                        ("network_alone", ws_raw),
                        ("network_high_frequencies_fbp_low_2x8x8", lp(fbp) + (ws_raw - lp(ws_raw)))):
            s0 = (s0 * mask).astype(np.float32)
            n_s, _, _, _ = icd_from(sc, s0, cstar, **kw)
            sens[key] = {"iterations": n_s, "start_rmse_over_range": rm(s0)}
        results.append({
            "start_sensitivity": sens,
            "phantom": name, "cstar": cstar, "cstar_iterations": n_star,
            "plain": {"iterations": n_plain, "icd_ms": round(ms_plain, 2), "start_ms": round(fbp_ms, 2),
                      "total_ms": round(ms_plain + fbp_ms, 2), "a_matrix": "fp32"},
            "warm": {"iterations": n_warm, "icd_ms": round(ms_warm, 2), "start_ms": round(fbp_ms + net_ms, 2),
                     "total_ms": round(ms_warm + fbp_ms + net_ms, 2),
                     "a_matrix": "fp16" if acache_warm == 2 else "fp32"},
            "final_cost_over_cstar": {"plain": c_plain / cstar, "warm": c_warm / cstar},
            "speedup_total": (ms_plain + fbp_ms) / (ms_warm + fbp_ms + net_ms),
            "start_rmse_over_range": {"fbp": rm(fbp), "warm": rm(ws), "network_alone": rm(ws_raw)},
            "final_rmse_over_range": {"plain": rm(x_plain), "warm": rm(x_warm)},
        })
    net.close()
    line = {
        "metric": "time-to-MAP-cost (warm vs plain)", "value": float(np.mean([r["speedup_total"] for r in results])),
        "unit": "x (plain time / warm time, start images included)", "n_gpus": world, "higher_is_better": True,
        "config": {"workload": (W4D.desc + "; learned warm start (network trained on 4-D scans of other seeds)")
                   if four_d else C4_DESC,
                   "training_volumes": pairs,
                   "pair_target": "converged MAP image (plain ICD from FBP until two successive costs agree to 1e-10; "
                                  "mean %.0f iterations)" % float(np.mean(target_iters)),
                   "train_steps": steps, "train_batch": "4 patches 16x64x64", "params": int(net.n),
                   "loss": ("mean squared error" if beta <= 0 else
                            f"mean squared error weighted per voxel by 1 + {beta:g} |grad target| / "
                            "mean |grad target|")
                           + ("" if not hp else f" of the residual's high frequencies ((I - G) d, G a Gaussian "
                                                f"low-pass of {hp[0]:g} slice x {hp[1]:g} x {hp[1]:g} voxels)")},
        "training": {"ms": round(train_ms, 1), "ms_per_step": round(train_ms / steps, 3),
                     "loss_first_50": float(np.mean(losses[:50])), "loss_last_50": float(np.mean(losses[-50:])),
                     "pairs_s": round(data_s, 1)},
        "held_out": results, "target": "FP64 MAP cost <= (1 + 1e-5) C*, C* = the plain FP32 run's converged cost",
        "dtype": "network bf16 operands / fp32 accumulation; ICD f32",
        "data": W4D.data if four_d else C4_DATA,
    }
    print(json.dumps(line), flush=True)


def net_arm(args, rank, world, local_rank, shape=(4, 16, 64, 64)):
    """Training-step throughput of the warm-start network (forward, loss,
    backward, Adam) on a batch of patches of the training shape, random data;
    the tensor-core roofline of its convolutions (algorithmic FLOPs: per 3x3x3
    convolution 2 M 27 Cin Cout for the forward pass, the same again for the
    input gradient (every layer but the first) and for the weight gradient)."""
    import torch
    from timbir_b200 import warm
    torch.cuda.set_device(local_rank)
    B, D, H, Wd = shape
    flops = 0.0
    for k, (ci, co, lv) in enumerate(warm.LAYERS):
        M = B * (D >> lv) * (H >> lv) * (Wd >> lv)
        f = 2.0 * M * 27 * ci * co
        flops += f * (3 if k > 0 else 2)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(shape, generator=g, device="cuda") * 0.02
    t = x * 0.9
    net = warm.WarmNet(seed=1)
    for _ in range(args.warmup):
        net.gradients(x, t)
        net.adam_step(1e-4)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        net.gradients(x, t)
        net.adam_step(1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # the forward pass alone (its convolutions are forward ones only)
    fwd_flops = sum(2.0 * B * (D >> lv) * (H >> lv) * (Wd >> lv) * 27 * ci * co for ci, co, lv in warm.LAYERS)
    for _ in range(args.warmup):
        net.forward(x)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / args.steps
    net.close()

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = float(peaks.get("bf16_tflops", 1590.0))
    tf = flops / (ms / 1e3) / 1e12
    print(json.dumps({
        "metric": "warm-start network training steps/s", "value": 1e3 / ms, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "dtype": ("bf16 activations and operands, fp32 accumulation (convolutions and input gradients: "
                  "tcgen05.mma kind::f16 with TMA-loaded inputs and accumulators in tensor memory; weight "
                  "gradients: mma.sync m16n8k16); fp32 master weights and Adam state"),
        "data": "synthetic (random patches)",
        "forward": {"ms": fwd_ms, "tflops": fwd_flops / (fwd_ms / 1e3) / 1e12,
                    "note": "inference pass alone (15 convolutions, pooling, up-sampling; includes the "
                            "host-synchronised output copy of mbir_net_forward)"},
        "config": {"workload": f"one training step on {B} patches {D}x{H}x{Wd} (forward, loss, backward, Adam)",
                   "params": sum(27 * ci * co + co for ci, co, _ in warm.LAYERS)},
        "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s", "frac": tf / peak,
                     "flops_per_step": flops, "traffic": None,
                     "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"},
    }), flush=True)


# ------------------------------------------------------------ ingestion --
INGEST = dict(views=1536, rows=128, cols=4100, whites=22, darks=12, proj_rows=64, proj_cols=2048)
INGEST_DESC = ("APS raw-count normalisation (read_data): 1536 views of 128 x 4100 uint16 counts (4 edge columns "
               "trimmed, 2 x 2 down-sampling to 64 x 2048), 22 bright and 12 dark frames, beam-hardening 0.5")


def ingest_data(seed=0):
    c = INGEST
    rng = np.random.default_rng(seed)
    counts = rng.integers(200, 30000, size=(c["views"], c["rows"], c["cols"]), dtype=np.uint16)
    whites = rng.integers(30000, 40000, size=(c["whites"], c["rows"], c["cols"]), dtype=np.uint16)
    darks = rng.integers(0, 120, size=(c["darks"], c["rows"], c["cols"]), dtype=np.uint16)
    return counts, whites, darks


def ingest_reference_rate(counts, whites, darks, views):
    """The reference's read_data (oracle/_ref/libref_io.so: its sources
    compiled against an in-memory HDF5 stand-in) on the first `views` views:
    output samples / s (its normalisation loop is single-threaded)."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_io.so"))
    VP, I = C.c_void_p, C.c_int
    lib.ref_read_aps.argtypes = [VP, I, VP, I, VP, I, I, I, I, I, I, I, I, VP, VP]
    c = INGEST
    sub = np.ascontiguousarray(counts[:views])
    P = np.zeros((views, c["proj_rows"], c["proj_cols"]), np.float32)
    W = np.zeros_like(P)
    t0 = time.perf_counter()
    rc = lib.ref_read_aps(sub.ctypes.data, views, whites.ctypes.data, c["whites"], darks.ctypes.data, c["darks"],
                          c["rows"], c["cols"], 0, c["proj_rows"], c["proj_cols"], 0, views, P.ctypes.data,
                          W.ctypes.data)
    secs = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("reference read_data failed")
    return P.size / secs, secs


def ingest_arm(args, rank, world, local_rank):
    """Normalisation of raw counts (mbir_frame_mean_device +
    mbir_normalize_counts_device on device-resident stacks; e2e through
    mbir_normalize_counts from pinned host stacks); each rank its own scan."""
    import torch
    from timbir_b200 import ingest
    torch.cuda.set_device(local_rank)
    c = INGEST
    counts, whites, darks = ingest_data(rank)
    lib = ingest._lib()
    extras = c["cols"] % c["proj_cols"]
    ncols, ratio = c["cols"] - extras, (c["cols"] - extras) // c["proj_cols"]
    nrows = c["proj_rows"] * ratio
    win = lambda a, f0, nf: np.ascontiguousarray(a[f0:f0 + nf, :nrows, extras // 2:extras // 2 + ncols])  # noqa
    dc = torch.from_numpy(win(counts, 0, c["views"]).view(np.int16)).cuda()
    dw = torch.from_numpy(win(whites, 1, c["whites"] - 2).view(np.int16)).cuda()
    dd = torch.from_numpy(win(darks, 1, c["darks"] - 2).view(np.int16)).cuda()
    mw = torch.empty((nrows, ncols), dtype=torch.float32, device="cuda")
    md = torch.empty_like(mw)
    P = torch.empty((c["views"], c["proj_rows"], c["proj_cols"]), dtype=torch.float32, device="cuda")
    W = torch.empty_like(P)
    st = torch.cuda.current_stream().cuda_stream

    def step():
        rc = (lib.mbir_frame_mean_device(dw.data_ptr(), c["whites"] - 2, nrows, ncols, mw.data_ptr(), st) or
              lib.mbir_frame_mean_device(dd.data_ptr(), c["darks"] - 2, nrows, ncols, md.data_ptr(), st) or
              lib.mbir_normalize_counts_device(dc.data_ptr(), mw.data_ptr(), md.data_ptr(), c["views"], nrows, ncols,
                                               ratio, 0.5, P.data_ptr(), W.data_ptr(), st))
        if rc:
            raise RuntimeError(lib.mbir_ingest_last_error().decode())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            ev[2 * k].record()
            step()
            ev[2 * k + 1].record()
        torch.cuda.synchronize()
    ms = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    samples = P.numel()
    value = samples * args.steps / (sum(ms) / 1e3)
    # algorithmic bytes of a step: the counts window once, the bright / dark
    # stacks once, the two means written and read once, both outputs written
    byts = dc.numel() * 2 + (dw.numel() + dd.numel()) * 2 + 2 * 2 * mw.numel() * 4 + 2 * P.numel() * 4
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = byts / (sum(ms) / args.steps / 1e3) / 1e9
    # end to end: pinned host stacks -> the public call -> host outputs
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    pc, pw, pd = pin(counts), pin(whites), pin(darks)
    hp = pin(np.zeros((c["views"], c["proj_rows"], c["proj_cols"]), np.float32))
    hw = pin(np.zeros_like(hp))
    e2e_ms = []
    for k in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        _check = lib.mbir_normalize_counts(pc.ctypes.data, c["views"], pw.ctypes.data, c["whites"], pd.ctypes.data,
                                           c["darks"], c["rows"], c["cols"], 0, c["proj_rows"], c["proj_cols"], 0,
                                           c["views"], 0, 1, 0.5, hp.ctypes.data, hw.ctypes.data)
        if _check:
            raise RuntimeError(lib.mbir_ingest_last_error().decode())
        if k:  # the first call pays one-time set-up (context, module)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    same = bool(np.array_equal(hw, W.cpu().numpy()))
    line = {
        "metric": "projection samples normalised/s", "value": value, "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(ms) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16 counts, f32 sums (f64 fabs / log as the reference)",
        "data": "synthetic (seeded uniform counts, bright and dark fields)",
        "config": {"workload": INGEST_DESC, "l2": "inputs (1.6 GB of counts) larger than L2"},
        "e2e": {"value": samples / (statistics.median(e2e_ms) / 1e3), "unit": "samples/s",
                "h2d_bytes_per_step": int(c["views"] * nrows * ncols * 2 + (c["whites"] + c["darks"] - 4) * nrows *
                                          ncols * 2),
                "d2h_bytes_per_step": int(2 * P.numel() * 4), "step_ms": [round(v, 2) for v in e2e_ms],
                "step": "mbir_normalize_counts from pinned host stacks (hyperslab copies in, outputs back)",
                "weights_equal_device_path": same},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "bytes_per_step": byts, "kernel": "k_normalize + k_frame_mean", "traffic": None,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "gpu_launches": 3 * args.steps, "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        rate, secs = ingest_reference_rate(counts, whites, darks, 48)
        line["cpu_baseline"] = {"value": rate, "unit": "samples/s", "cores": 1, "kind": "reference",
                                "sample": f"the reference's read_data on the first 48 views, {secs:.1f} s "
                                          "(its normalisation loop is single-threaded)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ auxiliary kernels --
def kernels_arm(args, rank, world, local_rank):
    """Each kernel of the path besides the super-voxel sweep, run on the 4-D
    workload's sizes (sinogram-shaped arrays of 67 MB each, volume 67 MB:
    larger than L2 together) so that one command covers them for a profiler:
    the prologue's forward projection (k_forward_rows) and column cache
    (k_acache), the ring-offset update (k_offset_terms / k_offset_apply), the
    windowed ring-offset solve (k_offset_windows), the variance update
    (k_variance / k_variance_apply), the MAP cost (k_cost / k_sum_partials),
    the NHICD selection (k_vsc_filter / k_vsc_threshold / k_sv_nh_list) and
    pass, the stage hand-off up-sampling (k_upsample_xy / _xyz), the
    filtered backprojection (k_ramp / k_backproject) and, on the 3-D
    workload, one iteration of the reference schedule (k_icd_ref).  Prints
    the wall time of each call (the profiler gives per-kernel times)."""
    import torch
    import timbir_b200
    torch.cuda.set_device(local_rank)
    w = W4D
    scan = w.scan(0)
    _, fine = w.warm_start(scan)
    out = {}

    def timed(name, fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        out[name] = round((time.perf_counter() - t0) * 1e3, 3)
        return r

    st = workload_stage(w, scan, 1, args)
    timed("prologue (forward projection)", lambda: st.prepare(fine, zero_offsets(scan)))
    st.set_sv_nhicd(0.1)
    timed("iteration 1 (column cache, sweep, offsets, variance)", lambda: st.iterate(1))
    timed("iteration 2 (sweep, NHICD selection and pass, offsets, variance)", lambda: st.iterate(2))
    timed("MAP cost", st.cost)
    timed("ring-offset update (mode 2)", st.offset_update)
    timed("variance update", st.variance_update)
    x = st.object()
    st.close()
    s3 = workload_stage(w, scan, 1, args, prior=dict(w.prior, remove_rings=3))
    s3.set_offset_windows(True)
    s3.prepare(fine, zero_offsets(scan))
    timed("ring-offset update (mode 3, %d windows)" % s3.offset_window_count(), s3.offset_update)
    timed("filtered backprojection", s3.fbp)
    s3.close()
    coarse = np.ascontiguousarray(x[0, ::2, ::2, ::2])
    timed("up-sampling x2 (x, y)", lambda: timbir_b200.upsample(x[0], False))
    timed("up-sampling x2 (x, y, z)", lambda: timbir_b200.upsample(coarse, True))
    w3 = W3D
    scan3 = w3.scan(0)
    _, fine3 = w3.warm_start(scan3)
    sr = timbir_b200.Stage(scan3, **w3.prior, blocks=8)
    sr.prepare(fine3)
    timed("reference-schedule iteration (3-D workload)", lambda: sr.iterate(1))
    sr.close()
    print(json.dumps({"metric": "wall ms per call (profile for per-kernel device times)", "calls": out,
                      "config": {"workload": w.desc + "; reference schedule on " + w3.desc}}), flush=True)


# --------------------------------------------------------------------- GPU --
def reference_map(w, scan):
    """The converged MAP cost C* of workload w's scan from the reference library
    and the FP64 oracle (tests/golden/converged_<name>.npz, made by
    tests/golden/make_converged_full.py), with the reference's iterations to
    (1 + 1e-5) C* from the bench's warm start; None when there is no fixture
    for w or it was made for another scan (SHA-256 of projections and
    weights)."""
    import hashlib
    path = os.path.join(ROOT, "tests", "golden", f"converged_{w.name}.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    dig = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()  # noqa: E731
    if dig(scan.projections) != str(g["proj_sha256"]) or dig(scan.weights) != str(g["weight_sha256"]):
        return None
    n = int(g["ref_iterations_to_target"]) if "ref_iterations_to_target" in g.files else None
    return {"cstar": float(g["cstar"]), "ref_iterations": n, "ref_fresh_cost": float(g["ref_fresh_cost"]),
            "f64_fresh_cost": float(g["f64_fresh_cost"])}


def time_to_map(w, scan, fine, sched, args, max_iters=400):
    """Time-to-MAP of the GPU engine from the bench's warm start: device time of
    the ICD iterations (CUDA events on the stage's stream, host work inside an
    iteration included) until the MAP cost -- evaluated in FP64 on the GPU after
    each iteration, not timed -- is within (1 + 1e-5) of C*.  C* is the
    reference's converged cost (reference library to a flat cost, then the
    FP64 oracle; costs evaluated afresh in FP64) where a fixture exists for the
    workload, else the cost this schedule converges to (iterated until two
    successive costs agree to 1e-10 relative, at most max_iters iterations)."""
    def stage():
        st = workload_stage(w, scan, sched, args)
        st.prepare(fine, zero_offsets(scan) if w.prior["remove_rings"] else None)
        return st

    ref = reference_map(w, scan)
    if ref:
        cstar, n_star, source = ref["cstar"], None, "reference library + FP64 oracle, converged (fixture)"
    else:
        st = stage()
        prev, n_star = None, max_iters
        for it in range(1, max_iters + 1):
            st.iterate(it)
            c = st.cost()[0]
            if prev is not None and abs(prev - c) <= 1e-10 * abs(c):
                n_star = it
                break
            prev = c
        cstar, source = c, "this schedule's own converged cost"
        st.close()
    st = stage()
    ms, n = 0.0, None
    for it in range(1, max_iters + 1):
        st.time_begin()
        st.iterate(it)
        ms += st.time_end()
        if st.cost()[0] <= (1.0 + 1e-5) * cstar:
            n = it
            break
    st.close()
    out = {"value": ms / 1e3 if n else None, "unit": "s", "iterations": n, "target": "FP64 MAP cost <= (1 + 1e-5) C*",
           "cstar": cstar, "cstar_source": source,
           "start": "2x-coarser phantom up-sampled (the stage's warm start)",
           "timed": "ICD iterations only (cost evaluations excluded)"}
    if n_star is not None:
        out["cstar_iterations"] = n_star
    if n is None:
        out["not_reached_in"] = max_iters
    return out


def gpu_arm(args, rank, world, local_rank):
    import torch
    import timbir_b200
    if args.config == "c3":
        return c3_arm(args, rank, world, local_rank)
    if args.config in ("c4", "4d-warm"):
        return c4_arm(args, rank, world, local_rank, four_d=args.config == "4d-warm")
    if args.config == "net":
        return net_arm(args, rank, world, local_rank)
    if args.config == "kernels":
        return kernels_arm(args, rank, world, local_rank)
    if args.config == "ingest":
        return ingest_arm(args, rank, world, local_rank)
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    w = WORKLOADS[args.config]
    scan = w.scan(rank)
    coarse, fine = w.warm_start(scan)
    sched = 1 if args.schedule == "sv" else 0
    st = workload_stage(w, scan, sched, args)
    sched_info = st.schedule_info()
    big = w.name == "c5"  # hundreds of iterations of about a second, ~100 s per reference iteration
    if big and args.c5_start == "fbp":  # this library's filtered backprojection as the start
        fine = st.fbp()
    st.prepare(fine, zero_offsets(scan) if w.prior["remove_rings"] else None)
    cost_trace = [st.cost()[0]] if big else None
    for it in range(1, args.warmup + 1):
        st.iterate(it)
        if big:
            cost_trace.append(st.cost()[0])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)
    ms0, n_icd0, n_all0 = st.kernel_stats()
    upd0 = st.update_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            st.time_begin()
            st.iterate(args.warmup + 1 + k)
            step_ms.append(st.time_end())
            if big:  # the MAP cost after each iteration (outside the timed region)
                cost_trace.append(st.cost()[0])
    torch.cuda.synchronize()
    ms1, n_icd1, n_all1 = st.kernel_stats()
    updates = st.update_count() - upd0
    total_ms = sum(step_ms)
    icd_ms = ms1 - ms0
    if dist:
        t = torch.tensor([total_ms, float(updates)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        total_ms_max, updates_all = float(mx[0]), float(t[1])
    else:
        total_ms_max, updates_all = total_ms, float(updates)
    cbar = mean_amatrix_count(st, scan) if rank == 0 else 0.0
    st.close()

    # time to the MAP target (every rank: its iteration count sizes the e2e solve)
    ttm = time_to_map(w, scan, fine, sched, args) if not args.no_ttm and not big else None
    n_solve = ttm["iterations"] if ttm and ttm["iterations"] else args.steps

    # end to end through the public API with host buffers: every step is the
    # call a user makes -- the stage reconstructed from pinned host arrays
    # (set-up and H2D copies, prologue, n_solve ICD iterations: the iterations
    # the GPU needed to reach the MAP target) and its object read back into
    # pinned host memory (D2H); the same with one iteration reported beside it
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    pscan = synth.Scan(pin(scan.projections), pin(scan.weights), pin(scan.proj_angles), pin(scan.proj_times),
                       pin(scan.recon_times), scan.proj_rows, scan.proj_cols, scan.proj_num, scan.recon_num,
                       scan.vox_wid, scan.rot_center)
    pfine = pin(fine)
    pzero = pin(zero_offsets(scan)) if w.prior["remove_rings"] else None
    pout = pin(np.zeros_like(fine))
    h2d = sum(a.nbytes for a in (pscan.projections, pscan.weights, pscan.proj_angles, pscan.proj_times,
                                 pscan.recon_times, pfine) + ((pzero,) if pzero is not None else ()))
    d2h = fine.nbytes

    def e2e_run(n_iter, reps):
        # one untimed warm-up solve first (the process's first device
        # allocations of this size and the schedule cache), then `reps` timed
        # with the interpreter's cyclic garbage collector paused (as timeit
        # does), so that a collection of the bench's own objects does not
        # land inside a timed solve
        times, upd = [], 0
        gc.collect()
        gc.disable()
        try:
            return _e2e_reps(n_iter, reps, times, upd)
        finally:
            gc.enable()

    def _e2e_reps(n_iter, reps, times, upd):
        for rep in range(reps + 1):
            flush.fill_(0.0)
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record()
            s2 = workload_stage(w, pscan, sched, args)
            s2.prepare(pfine, pzero)
            for it in range(1, n_iter + 1):
                s2.iterate(it)
            s2.object(out=pout)
            t1.record()
            torch.cuda.synchronize()
            if rep > 0:
                times.append(t0.elapsed_time(t1))
                upd += s2.update_count()
            s2.close()
        return times, upd

    reps = max(1, min(args.steps, 5))
    e2e_ms, e2e_upd = e2e_run(n_solve, reps)
    one_ms, one_upd = e2e_run(1, reps)
    if dist:
        # a solve's median time (the slowest rank's) against the updates of
        # one solve on every rank
        t = torch.tensor([statistics.median(e2e_ms), float(e2e_upd) / len(e2e_ms)], dtype=torch.float64,
                         device="cuda")
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        e2e_value = float(t[1]) / (float(mx[0]) / 1e3)
        dist.barrier()
        dist.destroy_process_group()
    else:
        # the median solve: a solve's host-side work (set-up calls, one
        # synchronisation per iteration) is exposed to other tenants of the
        # host, which stretched single solves 2-3x; every solve's time is in
        # step_ms
        e2e_value = (e2e_upd / len(e2e_ms)) / (statistics.median(e2e_ms) / 1e3)
    if rank != 0:
        return
    value = updates_all / (total_ms_max / 1e3)
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    npf = w.views // w.frames
    b_vu = npf * (cbar * 1 * 12 + 2 * cbar + 2) + 29 * 4 + 4
    achieved = (updates * b_vu) / (icd_ms / 1e3) / 1e9 if icd_ms > 0 else 0.0
    n_icd = max(n_icd1 - n_icd0, 1)
    traffic, traffic_src = None, None
    if sched and args.config in DRAM_BYTES_PER_UPDATE:
        traffic = DRAM_BYTES_PER_UPDATE[args.config] * updates / n_icd
        traffic_src = "ncu dram__bytes_read.sum + dram__bytes_write.sum per update of a sweep launch, x updates per launch"
    line = {
        "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("f32, A-matrix values fp16" if sched_info.get("column_cache_values") == "fp16" else "f32")
        + " (A-matrix bin indices exact in FP64; cost and convergence sums FP64)",
        "data": w.data,
        "config": {"workload": w.desc, "volume": [w.frames, w.rows, w.n_xy, w.n_xy],
                   "views": w.views,
                   "schedule": ("super-voxel" if sched else "reference (checkerboard z-blocks)"),
                   "schedule_info": sched_info, "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MB write)"},
        "e2e": {"value": e2e_value, "unit": "voxel-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "step_ms": [round(v, 3) for v in e2e_ms],
                "statistic": f"median of {len(e2e_ms)} timed solves after one untimed",
                "updates_per_step": e2e_upd / max(len(e2e_ms), 1),
                "step": f"stage reconstructed from pinned host arrays: set-up, prologue, {n_solve} ICD iterations "
                        f"({'the GPU iterations to the MAP target' if ttm and ttm['iterations'] else 'steps'}), "
                        "object read back into pinned memory",
                "single_iteration": {"value": (one_upd / len(one_ms)) / (statistics.median(one_ms) / 1e3),
                                     "step_ms": [round(v, 3) for v in one_ms],
                                     "updates_per_step": one_upd / max(len(one_ms), 1)}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "bytes_per_update": b_vu, "mean_bins_per_view": cbar,
                     "kernel": "k_icd_sv" if sched else "k_icd_ref", "kernel_ms": icd_ms,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "gpu_launches": int(n_all1 - n_all0),
        "clocks": clk.summary(),
    }
    if ttm:
        line["time_to_map"] = ttm
    if big:
        line["cost_trace"] = {"start": "filtered backprojection" if args.c5_start == "fbp" else "zero",
                              "costs": [float(c) for c in cost_trace],
                              "note": "FP64 MAP cost after the prologue and after each warm-up and timed iteration",
                              "falling": bool(all(b <= a for a, b in zip(cost_trace, cost_trace[1:])))}
    if big:
        line["cpu_baseline"] = {"unavailable": "the reference's CPU code needs minutes per iteration at this size"}
    elif world > 1:
        line["cpu_baseline"] = {"unavailable": "measured on rank 0 of a one-GPU run only"}
    elif not args.no_cpu:
        v, kind, cores, n, secs = cpu_measure(w, scan, coarse, fine, 1, 1, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": v, "unit": "voxel-updates/s", "cores": cores, "kind": kind,
                                "sample": f"{n} ICD iteration(s) of the same stage after 1 warm-up, {secs:.1f} s"}
        rt = reference_time_to_map(w, scan, cpu_measure.iterations, kind)
        if rt:
            line["cpu_baseline"]["time_to_map"] = rt
    print(json.dumps(line), flush=True)


def reference_arm(args, rank):
    if rank != 0:
        return
    if args.config == "kernels":
        print(json.dumps({"impl": "reference", "unavailable": "a profiling helper of this library's kernels; no "
                          "reference counterpart"}), flush=True)
        return
    if args.config == "ingest":
        counts, whites, darks = ingest_data(0)
        rates = []
        for k in range(args.warmup + args.steps):
            r, secs = ingest_reference_rate(counts, whites, darks, 48)
            if k >= args.warmup:
                rates.append(r)
        v = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": "projection samples normalised/s", "value": v, "unit": "samples/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "config": {"workload": INGEST_DESC},
            "cpu_baseline": {"value": v, "unit": "samples/s", "cores": 1, "kind": "reference",
                             "sample": "the reference's read_data (its sources compiled against an in-memory HDF5 "
                                       "stand-in) on the first 48 views per step; single-threaded loop"},
            "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    if args.config in ("c4", "4d-warm", "net"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned warm start (its coarsest "
                          "stage starts from zero); the comparison is FBP-initialised ICD, in the same line"}),
              flush=True)
        return
    if args.config == "c3":
        # per-size samples combined over the batch (the reference runs one
        # problem per process; weights: the problems' voxel counts)
        specs = synth.batch_problem_specs(64, 0)
        threads = os.cpu_count() or 1
        v, per, kind, cores, secs = c3_cpu_baseline(specs, [sp["side"] ** 2 * sp["slices"] for sp in specs], threads)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "voxel-updates/s", "n_gpus": 0, "steps": 1,
            "warmup": 1, "ms_per_step": 1e3 * secs / max(len(per), 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 scalars)", "data": C3_DATA,
            "config": {"workload": C3_DESC, "threads": threads,
                       "sample": "one ICD iteration after one warm-up per problem size (its problem with the fewest "
                                 "slices), combined over the 64 problems weighted by voxels (bounded: one step)"},
            "cpu_baseline": {"value": v, "unit": "voxel-updates/s", "cores": cores, "kind": kind, "per_size": per,
                             "sample": "per-size samples, %.1f s" % secs},
            "e2e": {"value": v, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    else:
        w = WORKLOADS[args.config]
        scan = w.scan(0)
        coarse, fine = w.warm_start(scan)
    threads = os.cpu_count() or 1
    v, kind, cores, n, secs = cpu_measure(w, scan, coarse, fine, args.warmup, args.steps, threads)
    ttm = reference_time_to_map(w, scan, cpu_measure.iterations, kind) if args.config != "c3" else None
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "voxel-updates/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(n, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 scalars)",
            "data": w.data,
            "config": {"workload": w.desc, "volume": [w.frames, w.rows, w.n_xy, w.n_xy], "views": w.views,
                       "threads": threads},
            "cpu_baseline": {"value": v, "unit": "voxel-updates/s", "cores": cores, "kind": kind,
                             "sample": f"{n} ICD iterations after {args.warmup} warm-up, {secs:.1f} s"},
            "e2e": {"value": v, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if ttm:
        line["time_to_map"] = ttm
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-ttm", action="store_true", help="skip the time-to-MAP measurement")
    ap.add_argument("--schedule", default="sv", choices=["sv", "reference"])
    ap.add_argument("--c5-start", default="fbp", choices=["fbp", "zero"],
                    help="start of the large 4-D z-subset (c5)")
    ap.add_argument("--c3-start", default="fbp", choices=["fbp", "zero"],
                    help="start of the batched problems' convergence run (c3)")
    ap.add_argument("--config", default="3d", choices=sorted(WORKLOADS) + ["c3", "c4", "4d-warm", "net", "kernels", "ingest"],
                    help="3d: the single-GPU 3-D workload (default); 4d: 16-frame interlaced 4-D workload; "
                         "c3: 64 independent 3-D problems batched; c4: learned warm start (3-D); 4d-warm: learned warm "
                         "start on the 4-D workload; net: the network's training step; c5: large 4-D z-subset; "
                         "kernels: each auxiliary kernel once, for a profiler")
    ap.add_argument("--sv-side", type=int, default=0, help="super-voxel side (0: largest that fits)")
    ap.add_argument("--problems", type=int, default=64, help="c3: the first N of the 64 problems")
    ap.add_argument("--no-tune", action="store_true", help="c3: default schedules instead of the autotuner's")
    ap.add_argument("--warps-per-slice", type=int, default=0, help="1, 2 or 4 (0: automatic)")
    ap.add_argument("--zgroup", type=int, default=0, help="slices per super-voxel z-group (0: automatic)")
    ap.add_argument("--sv-alpha", type=float, default=0.0,
                    help="over-relaxation of the super-voxel schedule (0: automatic from the in-flight cap)")
    ap.add_argument("--sv-ctas", type=int, default=0, help="persistent CTAs per sweep (0: automatic)")
    ap.add_argument("--c4-loss", default="highpass", choices=["highpass", "mse"],
                    help="c4 / 4d-warm: train on the residual's high frequencies (those the start keeps) or on all")
    ap.add_argument("--c4-edge-weight", type=float, default=0.0,
                    help="c4 / 4d-warm: weight the training loss per voxel by 1 + BETA |grad target| / mean")
    ap.add_argument("--nhicd", type=float, default=-1.0,
                    help="share of each plane's lines the NHICD pass selects (default: the library's 0.1)")
    ap.add_argument("--a-fp16", dest="acache", action="store_const", const=2, default=-1,
                    help="A-matrix column cache with FP16 values (FP32 accumulation)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank)
    else:
        gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
