"""timbir_b200 -- B200-native MBIR ICD/NHICD engine behind TIMBIR's reconstruct() call.

Python host mirror of the native library's C ABI (libtimbir_b200.so, built from
timbir_b200/csrc by ``python -m timbir_b200.build``):

* :func:`reconstruct` -- the drop-in call, same argument names and meaning as
  the reference's ``reconstruct()`` (TIMBIR v0.0.2 src/include/mbir4d.h:35);
  it writes the same files in the working directory.
* :class:`Stage` -- one resolution stage on the GPU, exposing the stage-level
  entry points (set-up, ICD iteration, cost, ring offsets, variance) and state
  read-back in the reference's array layouts.

There is no CPU fallback: importing the package loads the native library and
raises if it is missing or if no CUDA device is usable when a call needs one.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtimbir_b200.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_VP = C.c_void_p

_lib = None
# int (*)(double *values, int32_t count, void *ctx): the sum over z-slab ranks
_ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int32, C.c_void_p)


def load_library() -> C.CDLL:
    """Load libtimbir_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"native library missing: {LIB_PATH} (run `python -m timbir_b200.build`)")
    lib = C.CDLL(LIB_PATH)
    fl, i32 = C.c_float, C.c_int32
    lib.mbir_init_stage.argtypes = [C.POINTER(_VP), _VP, _VP, _VP, _VP, _VP, i32, i32, i32, i32, fl, fl, fl, fl,
                                    fl, fl, fl, i32, i32, fl, fl, i32, i32, i32]
    lib.mbir_free_stage.argtypes = [_VP]
    lib.mbir_last_error.restype = C.c_char_p
    lib.mbir_set_stage_switches.argtypes = [_VP, i32, i32, C.c_double]
    lib.mbir_set_rng_state.argtypes = [_VP, C.c_uint32]
    lib.mbir_set_convergence_threshold.argtypes = [_VP, C.c_double]
    lib.mbir_get_rng_state.argtypes = [_VP]
    lib.mbir_get_rng_state.restype = C.c_uint32
    lib.mbir_icd_prepare.argtypes = [_VP, _VP, _VP, _VP]
    lib.mbir_update_voxels_time_slices.argtypes = [_VP, i32, C.POINTER(i32)]
    lib.mbir_compute_cost.argtypes = [_VP] + [C.POINTER(C.c_double)] * 3
    lib.mbir_update_sinogram_offset.argtypes = [_VP]
    lib.mbir_set_offset_windows.argtypes = [_VP, i32]
    lib.mbir_get_offset_windows.argtypes = [_VP]
    lib.mbir_update_variance_parameter.argtypes = [_VP]
    lib.mbir_set_device_bytes_cap.argtypes = [C.c_int64]
    lib.mbir_get_device_bytes.restype = C.c_int64
    lib.mbir_debug_sv_skip_tasks.argtypes = [_VP, i32]
    lib.mbir_set_z_slab.argtypes = [_VP, i32, i32, _ALLREDUCE_FN, _VP]
    lib.mbir_get_slab_faces.argtypes = [_VP, _VP, _VP]
    lib.mbir_set_slab_halo.argtypes = [_VP, _VP, _VP]
    lib.mbir_stage_dims.argtypes = [_VP, _i32p]
    for n in ("mbir_get_object", "mbir_set_object", "mbir_get_errorsino", "mbir_get_weight", "mbir_get_offset",
              "mbir_get_magmap", "mbir_get_hr"):
        getattr(lib, n).argtypes = [_VP, _f32p]
    lib.mbir_get_mask.argtypes = [_VP, _u8p]
    lib.mbir_get_lines.argtypes = [_VP, i32, i32, i32, _i32p, _i32p]
    for n in ("mbir_get_var_est", "mbir_get_update_percentage"):
        getattr(lib, n).argtypes = [_VP]
        getattr(lib, n).restype = C.c_double
    lib.mbir_get_update_count.argtypes = [_VP]
    lib.mbir_get_update_count.restype = C.c_longlong
    lib.mbir_forward_project.argtypes = [_VP, _f32p, _f32p]
    lib.mbir_fbp.argtypes = [_VP, _f32p]
    lib.mbir_get_kernel_stats.argtypes = [_VP, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                          C.POINTER(C.c_longlong)]
    lib.mbir_set_schedule.argtypes = [_VP, i32, i32, i32]
    lib.mbir_get_schedule.argtypes = [_VP] + [C.POINTER(i32)] * 6
    lib.mbir_set_acache.argtypes = [_VP, i32]
    lib.mbir_get_acache.argtypes = [_VP, C.POINTER(i32), C.POINTER(C.c_int64)]
    lib.mbir_get_acache_line.argtypes = [_VP, i32, i32, _i32p]
    lib.mbir_set_sv_ctas.argtypes = [_VP, i32]
    lib.mbir_set_sv_zgroup.argtypes = [_VP, i32]
    lib.mbir_get_sv_grid.argtypes = [_VP] + [C.POINTER(i32)] * 3 + [C.POINTER(C.c_double)]
    lib.mbir_set_sv_relaxation.argtypes = [_VP, C.c_double]
    lib.mbir_get_sv_adjustments.argtypes = [_VP]
    lib.mbir_set_sv_guard.argtypes = [_VP, i32]
    lib.mbir_set_sv_nhicd.argtypes = [_VP, C.c_double]
    lib.mbir_nhicd_select.argtypes = [_f32p, i32, i32, i32, _i32p, _u8p, _f32p]
    lib.mbir_upsample.argtypes = [_f32p, _f32p, i32, i32, i32, i32]
    lib.mbir_time_begin.argtypes = [_VP]
    lib.mbir_time_end.argtypes = [_VP, C.POINTER(C.c_double)]
    i64 = C.c_int64
    lib.mbir_batch_create.argtypes = [C.POINTER(_VP), C.POINTER(_VP), i32, i32]
    lib.mbir_batch_free.argtypes = [_VP]
    lib.mbir_batch_iterate.argtypes = [_VP, i32, i32, C.POINTER(i32)]
    lib.mbir_batch_stats.argtypes = [_VP, _VP, _VP, _VP, _VP, _VP]
    lib.mbir_batch_info.argtypes = [_VP, C.POINTER(C.c_double), C.POINTER(i64), C.POINTER(i64), C.POINTER(i32),
                                    C.POINTER(i64)]
    lib.mbir_autotune_stage.argtypes = [_VP] + [C.POINTER(i32)] * 3 + [C.POINTER(C.c_double)]
    lib.reconstruct.argtypes = [C.POINTER(C.POINTER(C.c_float))] + [_VP] * 5 + [i32] * 4 + [fl] * 7 + \
        [i32, i32, fl, fl, C.c_uint8, _VP]
    _lib = lib
    return lib


class MbirError(RuntimeError):
    pass


def _check(rc: int) -> None:
    if rc != 0:
        raise MbirError(load_library().mbir_last_error().decode(errors="replace"))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Stage:
    """One resolution stage on the GPU (include/timbir_b200.h).

    Constructed like the reference's initStatStructures + initDynStructures for
    a stage with voxel scales (mult_xy, mult_z); ``blocks`` is num_z_blocks."""

    def __init__(self, scan, sig_s, sig_t, c_s, c_t, convg_thresh=1.0, remove_rings=0, quad_convex=1,
                 huber_delta=0.5, huber_T=4.0, mult_xy=1, mult_z=1, blocks=2):
        lib = load_library()
        self.lib = lib
        self.scan = scan
        keep = [_f32(a) for a in (scan.projections, scan.weights, scan.proj_angles, scan.proj_times,
                                  scan.recon_times)]
        h = _VP()
        _check(lib.mbir_init_stage(C.byref(h), *[a.ctypes.data for a in keep], scan.proj_rows, scan.proj_cols,
                                   scan.proj_num, scan.recon_num, scan.vox_wid, scan.rot_center, sig_s, sig_t,
                                   c_s, c_t, convg_thresh, remove_rings, quad_convex, huber_delta, huber_T,
                                   mult_xy, mult_z, blocks))
        self.h = h
        d = np.zeros(9, np.int32)
        lib.mbir_stage_dims(self.h, d)
        (self.N_p, self.N_r, self.N_t, self.N_x, self.N_y, self.N_z, self.N_time, self.nblk,
         self.z_overlap) = [int(v) for v in d]

    def close(self):
        if self.h:
            self.lib.mbir_free_stage(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- driving -------------------------------------------------------
    def set_switches(self, update_proj_offset=0, update_var=0, var_est=0.0):
        _check(self.lib.mbir_set_stage_switches(self.h, update_proj_offset, update_var, var_est))

    def set_convergence_threshold(self, convg_thresh: float):
        """Convergence threshold of the iterations, percent (reconstruct()'s
        convg_thresh)."""
        _check(self.lib.mbir_set_convergence_threshold(self.h, convg_thresh))

    def set_rng_state(self, state: int):
        self.lib.mbir_set_rng_state(self.h, state)

    def rng_state(self) -> int:
        return self.lib.mbir_get_rng_state(self.h)

    SCHEDULE_REFERENCE = 0
    SCHEDULE_SUPERVOXEL = 1

    # --- z-slab sharding (XT_MPI.c:47-122) -------------------------------
    def set_z_slab(self, rank: int, ranks: int, allreduce=None):
        """Make this stage z-slab `rank` of `ranks` (its scan holds that slab's
        detector rows).  allreduce(values) sums a float64 numpy array over the
        ranks in place; the stage calls it where the reference reduces over
        its MPI ranks (cost, variance, convergence)."""
        if allreduce is None:
            cb = _ALLREDUCE_FN()
        else:
            def cb_py(ptr, n, _ctx):
                try:
                    v = np.ctypeslib.as_array(ptr, shape=(n,))
                    allreduce(v)
                    return 0
                except Exception:  # reported to the stage as a failed reduction
                    import traceback
                    traceback.print_exc()
                    return 1
            cb = _ALLREDUCE_FN(cb_py)
        self._allreduce_cb = cb  # kept alive while the stage may call it
        _check(self.lib.mbir_set_z_slab(self.h, rank, ranks, cb, None))

    def slab_faces(self):
        """This slab's slice 0 and slice N_z - 1 of every frame, as CUDA
        tensors [N_time][N_y][N_x] (the faces its neighbours take as halos)."""
        import torch
        lo = torch.empty((self.N_time, self.N_y, self.N_x), dtype=torch.float32, device="cuda")
        hi = torch.empty_like(lo)
        _check(self.lib.mbir_get_slab_faces(self.h, lo.data_ptr(), hi.data_ptr()))
        return lo, hi

    def set_slab_halo(self, lo=None, hi=None):
        """Halo slices from CUDA tensors [N_time][N_y][N_x]: lo = the slab
        below's top slice, hi = the slab above's bottom slice (None: kept)."""
        lo = None if lo is None else lo.contiguous()
        hi = None if hi is None else hi.contiguous()
        _check(self.lib.mbir_set_slab_halo(self.h, None if lo is None else lo.data_ptr(),
                                           None if hi is None else hi.data_ptr()))

    def set_schedule(self, schedule: int, sv_side: int = 0, warps_per_slice: int = 0, acache: int = -1):
        """0: the reference's checkerboard z-block schedule; 1: super-voxel
        schedule (sv_side 0 = largest side whose band fits shared memory;
        warps_per_slice 0 = automatic; acache: A-matrix column cache, -1 when
        it fits, 0 never, 1 always, 2 when it fits with FP16 values)."""
        _check(self.lib.mbir_set_acache(self.h, acache))
        _check(self.lib.mbir_set_schedule(self.h, schedule, sv_side, warps_per_slice))
        d = np.zeros(9, np.int32)
        self.lib.mbir_stage_dims(self.h, d)
        self.nblk = int(d[7])

    def schedule_info(self) -> dict:
        v = [C.c_int32() for _ in range(6)]
        self.lib.mbir_get_schedule(self.h, *[C.byref(x) for x in v])
        used, nbytes = C.c_int32(), C.c_int64()
        self.lib.mbir_get_acache(self.h, C.byref(used), C.byref(nbytes))
        d = dict(zip(("schedule", "sv_side", "z_group", "band_width", "phases", "warps_per_slice"),
                     [x.value for x in v]))
        d["column_cache_bytes"] = int(nbytes.value) if used.value else 0
        d["column_cache_values"] = {0: None, 1: "fp32", 2: "fp16"}[used.value]
        g = [C.c_int32() for _ in range(3)]
        rel = C.c_double()
        self.lib.mbir_get_sv_grid(self.h, *[C.byref(x) for x in g], C.byref(rel))
        d["ctas"], d["inflight_per_group"], d["resident_ctas"] = [x.value for x in g]
        d["relaxation"] = rel.value
        d["stability_adjustments"] = int(self.lib.mbir_get_sv_adjustments(self.h))
        return d

    def set_sv_relaxation(self, alpha: float):
        """Over-relaxation of the super-voxel schedule in (0, 2); 0 = automatic.
        Call before set_schedule."""
        _check(self.lib.mbir_set_sv_relaxation(self.h, alpha))

    def set_sv_zgroup(self, slices: int):
        """Slices per z-group of the super-voxel schedule (0 = automatic); call
        before set_schedule."""
        _check(self.lib.mbir_set_sv_zgroup(self.h, slices))

    def set_sv_guard(self, on: bool):
        """The super-voxel schedule's stability guard on (the default) or off."""
        _check(self.lib.mbir_set_sv_guard(self.h, 1 if on else 0))

    def set_sv_nhicd(self, fraction: float):
        """Share of each plane's in-mask lines the super-voxel schedule's NHICD
        pass selects (the reference's is 0.1; 0, the default, turns it off)."""
        _check(self.lib.mbir_set_sv_nhicd(self.h, fraction))

    def set_sv_ctas(self, ctas: int):
        """Persistent CTAs per super-voxel launch (0 = one per SM; 1 runs the
        super-voxels one after another, deterministically)."""
        _check(self.lib.mbir_set_sv_ctas(self.h, ctas))

    def acache_line(self, row: int, col: int):
        """Cached A-matrix columns of voxel line (row, col): per view the first
        detector column j0, the column count n and the values (n of them
        meaningful)."""
        mult = self.N_r // self.N_x  # mult_xy: columns per voxel
        eq = (2 * mult + 2 + 3) // 4  # 16-byte words per entry: ceil((1 + amax) / 4), amax = 2 mult + 1
        words = np.zeros((self.N_p, 4 * eq), np.int32)
        _check(self.lib.mbir_get_acache_line(self.h, row, col, words))
        j0 = words[:, 0] & 0xFFFF
        n = words[:, 0] >> 16
        return j0, n, words[:, 1:].view(np.float32)

    def prepare(self, obj=None, offset=None, magmap=None):
        arrs = [None if a is None else _f32(a) for a in (obj, offset, magmap)]
        _check(self.lib.mbir_icd_prepare(self.h, *[None if a is None else a.ctypes.data for a in arrs]))

    def iterate(self, it: int) -> int:
        conv = C.c_int32()
        _check(self.lib.mbir_update_voxels_time_slices(self.h, it, C.byref(conv)))
        return conv.value

    def cost(self):
        t, f, p = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.mbir_compute_cost(self.h, C.byref(t), C.byref(f), C.byref(p)))
        return t.value, f.value, p.value

    def offset_update(self):
        _check(self.lib.mbir_update_sinogram_offset(self.h))

    def set_offset_windows(self, on: bool = True):
        """Rectangular-patch constraint windows for ring-offset mode 3
        (mbir_set_offset_windows)."""
        _check(self.lib.mbir_set_offset_windows(self.h, 1 if on else 0))

    def build_offset_windows(self):
        self.set_offset_windows(True)

    def offset_window_count(self) -> int:
        return int(self.lib.mbir_get_offset_windows(self.h))

    def variance_update(self):
        _check(self.lib.mbir_update_variance_parameter(self.h))

    # --- state ---------------------------------------------------------
    def _get(self, fn, shape, dt=np.float32):
        out = np.zeros(shape, dt)
        _check(getattr(self.lib, fn)(self.h, out.reshape(-1)))
        return out

    def object(self, out=None):
        """The object [N_time][N_z][N_y][N_x]; `out` (float32, C-contiguous, e.g.
        pinned host memory) receives it when given."""
        if out is None:
            return self._get("mbir_get_object", (self.N_time, self.N_z, self.N_y, self.N_x))
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.N_time * self.N_z * self.N_y * self.N_x:
            raise ValueError("out must be a C-contiguous float32 array of the object's size")
        _check(self.lib.mbir_get_object(self.h, out.reshape(-1)))
        return out

    def set_object(self, x):
        _check(self.lib.mbir_set_object(self.h, _f32(x).reshape(-1)))

    def errorsino(self):
        return self._get("mbir_get_errorsino", (self.N_p, self.N_r, self.N_t))

    def weight(self):
        return self._get("mbir_get_weight", (self.N_p, self.N_r, self.N_t))

    def offset(self):
        return self._get("mbir_get_offset", (self.N_r, self.N_t))

    def magmap(self):
        return self._get("mbir_get_magmap", (self.N_time, self.nblk, self.N_y, self.N_x))

    def hr(self):
        return self._get("mbir_get_hr", (self.N_p, 65))

    def mask(self):
        return self._get("mbir_get_mask", (self.N_y, self.N_x), np.uint8)

    def lines(self, kind, frame, block):
        xs = np.zeros(self.N_x * self.N_y, np.int32)
        ys = np.zeros(self.N_x * self.N_y, np.int32)
        n = self.lib.mbir_get_lines(self.h, kind, frame, block, xs, ys)
        if n < 0:
            _check(n)
        return xs[:n].copy(), ys[:n].copy()

    def var_est(self) -> float:
        return self.lib.mbir_get_var_est(self.h)

    def update_percentage(self) -> float:
        return self.lib.mbir_get_update_percentage(self.h)

    def update_count(self) -> int:
        return self.lib.mbir_get_update_count(self.h)

    def kernel_stats(self):
        """(ICD kernel device ms, ICD kernel launches, all kernel launches)."""
        ms, n_icd, n_all = C.c_double(), C.c_longlong(), C.c_longlong()
        self.lib.mbir_get_kernel_stats(self.h, C.byref(ms), C.byref(n_icd), C.byref(n_all))
        return ms.value, n_icd.value, n_all.value

    def time_begin(self):
        _check(self.lib.mbir_time_begin(self.h))

    def time_end(self) -> float:
        ms = C.c_double()
        _check(self.lib.mbir_time_end(self.h, C.byref(ms)))
        return ms.value

    def fbp(self) -> np.ndarray:
        """Filtered backprojection of each frame [N_time][N_z][N_y][N_x]
        (zero outside the reconstruction mask)."""
        return self._get("mbir_fbp", (self.N_time, self.N_z, self.N_y, self.N_x))

    def forward_project(self, obj) -> np.ndarray:
        out = np.zeros((self.N_p, self.N_t, self.N_r), np.float32)
        _check(self.lib.mbir_forward_project(self.h, _f32(obj).reshape(-1), out.reshape(-1)))
        return out

    def set_batch_schedule(self, sv_side: int = 0, warps_per_slice: int = 1, acache: int = 1):
        """Super-voxel schedule that batched launches take: at least as many
        warps per slice as keep a lane's views at 8 or fewer, and the z-group
        and warps per slice filling the batched kernel's 256 threads
        (batch_split)."""
        views = -(-self.N_p // max(self.N_time, 1))  # views per frame (equal frames)
        wps = max(1, warps_per_slice)
        while wps < 4 and -(-views // (32 * wps)) > 8:
            wps *= 2
        wps, nz = batch_split(wps, self.N_z)
        self.set_sv_zgroup(nz)
        self.set_schedule(self.SCHEDULE_SUPERVOXEL, sv_side, wps, acache)

    def autotune(self) -> dict:
        """Pick the super-voxel side, warps per slice and z-group of the
        batched kernel for this stage by timing them (mbir_autotune_stage);
        the stage keeps the winner.  Call after prepare, before iterating."""
        side, wps, zg, ns = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _check(self.lib.mbir_autotune_stage(self.h, C.byref(side), C.byref(wps), C.byref(zg), C.byref(ns)))
        info = self.schedule_info()
        return {"sv_side": side.value, "warps_per_slice": wps.value, "z_group": zg.value,
                "band_width": info["band_width"], "ns_per_update": ns.value}


BATCH_WARPS = 8  # warps of the batched kernel's CTA (include/timbir_b200.h: 256 threads)


def batch_split(warps_per_slice: int, slices: int, warps: int = BATCH_WARPS):
    """(warps per slice, z-group) filling `warps` warps on a stack of
    `slices` slices, starting from `warps_per_slice` and widening it (up to
    4) when the stack is too short."""
    wps = warps_per_slice
    nz = min(warps // wps, slices)
    while nz * wps < warps and wps < 4:
        wps *= 2
        nz = min(warps // wps, slices)
    return wps, nz


class Batch:
    """Independent problems (prepared super-voxel stages with a column cache)
    iterated together: one persistent launch per iteration over all their
    super-voxels, replayed as a CUDA graph (include/timbir_b200.h,
    mbir_batch_*).  Each problem stops at its own convergence test."""

    def __init__(self, stages, uncapped: bool = False):
        self.lib = load_library()
        self.stages = list(stages)
        arr = (_VP * len(self.stages))(*[s.h for s in self.stages])
        h = _VP()
        _check(self.lib.mbir_batch_create(C.byref(h), arr, len(self.stages), 1 if uncapped else 0))
        self.h = h

    def iterate(self, max_iters: int = 1, check_every: int = 1) -> int:
        """Up to max_iters iterations (fewer once every problem has
        converged); returns the problems still iterating."""
        left = C.c_int32()
        _check(self.lib.mbir_batch_iterate(self.h, max_iters, check_every, C.byref(left)))
        return left.value

    def stats(self) -> dict:
        n = len(self.stages)
        it, cv = np.zeros(n, np.int32), np.zeros(n, np.int32)
        up, zs = np.zeros(n, np.int64), np.zeros(n, np.int64)
        pct = np.zeros(n, np.float64)
        _check(self.lib.mbir_batch_stats(self.h, it.ctypes.data, cv.ctypes.data, up.ctypes.data, zs.ctypes.data,
                                         pct.ctypes.data))
        return {"iterations": it, "converged": cv, "updates": up, "zero_skips": zs, "percent": pct}

    def info(self) -> dict:
        ms, rep, lau, ctas, sm = C.c_double(), C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
        _check(self.lib.mbir_batch_info(self.h, C.byref(ms), C.byref(rep), C.byref(lau), C.byref(ctas),
                                        C.byref(sm)))
        return {"ms": ms.value, "replays": rep.value, "launches": lau.value, "ctas": ctas.value,
                "smem_bytes": sm.value}

    def close(self):
        if self.h:
            self.lib.mbir_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nhicd_select(mag: np.ndarray, nsel) -> tuple:
    """The device NHICD line selection (mbir_nhicd_select) of magnitude maps
    mag [planes][N_y][N_x]: (selected-line byte map, per-plane thresholds)."""
    lib = load_library()
    mag = np.ascontiguousarray(mag, np.float32)
    planes, ny, nx = mag.shape
    nsel = np.ascontiguousarray(np.broadcast_to(np.asarray(nsel, np.int32), (planes,)))
    sel = np.zeros(mag.shape, np.uint8)
    th = np.zeros(planes, np.float32)
    _check(lib.mbir_nhicd_select(mag.reshape(-1), planes, ny, nx, nsel, sel.reshape(-1), th))
    return sel, th


def upsample(x: np.ndarray, z_too: bool) -> np.ndarray:
    """The GPU's x2 up-sampling between multi-resolution stages (mbir_upsample)
    of x [n_z][n_y][n_x]."""
    lib = load_library()
    x = np.ascontiguousarray(x, np.float32)
    nz, ny, nx = x.shape
    out = np.zeros(((2 if z_too else 1) * nz, 2 * ny, 2 * nx), np.float32)
    _check(lib.mbir_upsample(x.reshape(-1), out.reshape(-1), nz, ny, nx, 1 if z_too else 0))
    return out


def _malloc_copy(a: np.ndarray) -> C.c_void_p:
    """Copy into a malloc'd block: reconstruct() free()s its inputs."""
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    a = _f32(a)
    p = libc.malloc(max(a.nbytes, 4))
    if not p:
        raise MemoryError
    C.memmove(p, a.ctypes.data, a.nbytes)
    return C.c_void_p(p)


def reconstruct(projections, weights, proj_angles, proj_times, recon_times, proj_rows, proj_cols, proj_num,
                recon_num, vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh, remove_rings,
                quad_convex, huber_delta, huber_T, restart=0, debug_log: str | None = None) -> int:
    """The drop-in reconstruct() on numpy arrays; outputs go to the working
    directory (object_time_<t>.bin, proj_offset.bin, ...).  Returns the C
    call's status (0 on success, -1 on failure)."""
    lib = load_library()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fp = libc.fopen((debug_log or os.devnull).encode(), b"a")
    obj = C.POINTER(C.c_float)()
    try:
        return lib.reconstruct(C.byref(obj), _malloc_copy(projections), _malloc_copy(weights),
                               _malloc_copy(proj_angles), _malloc_copy(proj_times), _malloc_copy(recon_times),
                               proj_rows, proj_cols, proj_num, recon_num, vox_wid, rot_center, sig_s, sig_t, c_s,
                               c_t, convg_thresh, remove_rings, quad_convex, huber_delta, huber_T, restart,
                               C.c_void_p(fp))
    finally:
        libc.fclose(fp)
