"""ctypes bindings to the CPU oracles (test infrastructure only).

* ``Oracle`` wraps oracle/_build/liboracle.so (or liboracle64.so): the C
  restatement of the reference hot path in oracle/mbir_oracle.c.
* ``Reference`` wraps oracle/_ref/libmbir4d_ref.so: the reference library
  itself (TIMBIR v0.0.2 src/MBIR_4D, unmodified) plus the flat driver in
  oracle/ref/ref_shim.c.  It exists only where oracle/Makefile could build it
  (it needs the reference sources); ``Reference.available()`` says whether it
  does.

Both expose the same methods, so a test can run one scenario through either
and compare.  Arrays come back in the reference layouts (sinogram-shaped
arrays [N_p][N_r][N_t], object [N_time][N_z][N_y][N_x]).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
ORACLE64_SO = os.path.join(HERE, "_build", "liboracle64.so")
REF_SO = os.path.join(HERE, "_ref", "libmbir4d_ref.so")
REF_BIN = os.path.join(HERE, "_ref", "XT_Main_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def reference_src() -> str:
    """The reference tree's src/ directory, from TIMBIR_REFERENCE_SRC ('' if unset)."""
    return os.environ.get("TIMBIR_REFERENCE_SRC", "")


def build_reference(ref_src: str = "") -> bool:
    """Compile the reference where its sources lie (ref_src, else
    TIMBIR_REFERENCE_SRC); False if they are absent."""
    ref_src = ref_src or reference_src()
    if not ref_src or not os.path.isdir(os.path.join(ref_src, "MBIR_4D")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_src}"], check=True)
    return True


class _Lib:
    prefix = ""

    def _bind(self, lib):
        p = self.prefix
        f = lambda n: getattr(lib, p + n)  # noqa: E731
        f("create").restype = C.c_void_p
        f("prepare").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        f("iterate").argtypes = [C.c_void_p, C.c_int]
        f("cost").restype = C.c_double
        f("set_switches").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        for n in ("offset_update", "variance_update", "random_select", "vsc_select"):
            f(n).argtypes = [C.c_void_p]
        f("dims").argtypes = [C.c_void_p, _i32p]
        f("scalars").argtypes = [C.c_void_p, _f64p]
        f("view_map").argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p]
        for n in ("get_object", "get_errorsino", "get_weight", "get_offset", "get_magmap", "get_hr"):
            f(n).argtypes = [C.c_void_p, _f32p]
        f("set_magmap").argtypes = [C.c_void_p, _f32p]
        f("get_projselect").argtypes = [C.c_void_p, _u8p]
        f("get_mask").argtypes = [C.c_void_p, _u8p]
        f("get_lines").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _i32p, _i32p]
        f("amatrix").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _i32p, _f64p, C.c_int]
        f("functional_substitution").argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _f64p, _u8p, _f64p, _u8p]
        f("functional_substitution").restype = C.c_double
        f("build_offset_windows").argtypes = [C.c_void_p]
        f("get_offset_windows").argtypes = [C.c_void_p, C.c_void_p]
        f("get_offset_windows").restype = C.c_int
        f("var_est").argtypes = [C.c_void_p]
        f("var_est").restype = C.c_double
        f("num_z_blocks").argtypes = [C.c_void_p]
        f("srandom2").argtypes = [C.c_uint32]
        f("random2").restype = C.c_double
        f("randomized_select").argtypes = [_f32p, C.c_uint32, C.c_uint32]
        f("randomized_select").restype = C.c_double
        self._f = f

    def __init__(self, scan, sig_s, sig_t, c_s, c_t, convg_thresh=1.0, remove_rings=0, quad_convex=1,
                 huber_delta=0.5, huber_T=4.0, mult_xy=1, mult_z=1, blocks=2):
        self.scan = scan
        self.h = self._create(scan, sig_s, sig_t, c_s, c_t, convg_thresh, remove_rings, quad_convex,
                              huber_delta, huber_T, mult_xy, mult_z, blocks)
        if not self.h:
            raise RuntimeError("set-up failed")
        d = np.zeros(9, np.int32)
        self._f("dims")(self.h, d)
        (self.N_p, self.N_r, self.N_t, self.N_x, self.N_y, self.N_z, self.N_time, self.nblk,
         self.z_overlap) = [int(v) for v in d]

    def _args(self, s, sig_s, sig_t, c_s, c_t, convg, rr, qc, hd, hT):
        fp = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(C.c_void_p)  # noqa: E731
        self._keep = [np.ascontiguousarray(a, np.float32) for a in
                      (s.projections, s.weights, s.proj_angles, s.proj_times, s.recon_times)]
        ptrs = [a.ctypes.data_as(C.c_void_p) for a in self._keep]
        return ptrs + [C.c_int(s.proj_rows), C.c_int(s.proj_cols), C.c_int(s.proj_num), C.c_int(s.recon_num),
                       C.c_float(s.vox_wid), C.c_float(s.rot_center), C.c_float(sig_s), C.c_float(sig_t),
                       C.c_float(c_s), C.c_float(c_t), C.c_float(convg), C.c_int(rr), C.c_int(qc),
                       C.c_float(hd), C.c_float(hT)]

    # --- driving -------------------------------------------------------
    def set_switches(self, update_proj_offset=0, update_var=0, var_est=0.0):
        self._f("set_switches")(self.h, update_proj_offset, update_var, var_est)

    def prepare(self, obj=None, offset=None):
        self._obj = None if obj is None else np.ascontiguousarray(obj, np.float32)
        self._off = None if offset is None else np.ascontiguousarray(offset, np.float32)
        r = self._f("prepare")(self.h, None if self._obj is None else self._obj.ctypes.data,
                               None if self._off is None else self._off.ctypes.data)
        if r != 0:
            raise RuntimeError("prepare failed")

    def iterate(self, it):
        return self._f("iterate")(self.h, it)

    def cost(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        v = self._cost(a, b, c)
        return v, a.value, b.value, c.value

    def offset_update(self):
        self._f("offset_update")(self.h)

    def variance_update(self):
        self._f("variance_update")(self.h)

    def random_select(self):
        self._f("random_select")(self.h)

    def vsc_select(self):
        self._f("vsc_select")(self.h)

    # --- state ---------------------------------------------------------
    def scalars(self):
        s = np.zeros(47, np.float64)
        self._f("scalars")(self.h, s)
        return s

    def view_map(self, frame):
        n = C.c_int()
        self._f("view_map")(self.h, frame, C.byref(n), None)
        out = np.zeros(max(n.value, 1), np.int32)
        self._f("view_map")(self.h, frame, C.byref(n), out.ctypes.data)
        return out[: n.value]

    def _get(self, name, shape, dt=np.float32):
        out = np.zeros(shape, dt)
        self._f(name)(self.h, out.reshape(-1))
        return out

    def object(self):
        return self._get("get_object", (self.N_time, self.N_z, self.N_y, self.N_x))

    def errorsino(self):
        return self._get("get_errorsino", (self.N_p, self.N_r, self.N_t))

    def weight(self):
        return self._get("get_weight", (self.N_p, self.N_r, self.N_t))

    def projselect(self):
        return self._get("get_projselect", (self.N_p, self.N_r, self.N_t), np.uint8)

    def offset(self):
        return self._get("get_offset", (self.N_r, self.N_t))

    def magmap(self):
        return self._get("get_magmap", (self.N_time, self.nblk, self.N_y, self.N_x))

    def set_magmap(self, m):
        self._f("set_magmap")(self.h, np.ascontiguousarray(m, np.float32).reshape(-1))

    def hr(self):
        return self._get("get_hr", (self.N_p, 65))

    def mask(self):
        return self._get("get_mask", (self.N_time, self.N_y, self.N_x), np.uint8)

    def lines(self, kind, frame, block):
        xs = np.zeros(self.N_x * self.N_y, np.int32)
        ys = np.zeros(self.N_x * self.N_y, np.int32)
        n = self._f("get_lines")(self.h, kind, frame, block, xs, ys)
        return xs[:n].copy(), ys[:n].copy()

    def amatrix(self, row, col, view):
        idx = np.zeros(512, np.int32)
        val = np.zeros(512, np.float64)
        n = self._f("amatrix")(self.h, row, col, view, idx, val, 512)
        return idx[:n].copy(), val[:n].copy()

    def functional_substitution(self, V, th1, th2, sn, sf, tn, tf):
        return self._f("functional_substitution")(
            self.h, V, th1, th2, np.ascontiguousarray(sn, np.float64).reshape(-1),
            np.ascontiguousarray(sf, np.uint8).reshape(-1), np.ascontiguousarray(tn, np.float64),
            np.ascontiguousarray(tf, np.uint8))

    def build_offset_windows(self):
        """Build the rectangular-patch constraint windows of offset mode 3."""
        self._f("build_offset_windows")(self.h)

    def offset_windows(self):
        """The constraint windows [M][N_r][N_t] (M = 0: none built)."""
        m = self._f("get_offset_windows")(self.h, None)
        out = np.zeros((m, self.N_r, self.N_t), np.float32)
        if m:
            self._f("get_offset_windows")(self.h, out.ctypes.data)
        return out

    def var_est(self):
        return self._f("var_est")(self.h)

    # --- RNG -----------------------------------------------------------
    def srandom2(self, seed):
        self._f("srandom2")(seed)

    def random2(self):
        return self._f("random2")()

    def randomized_select(self, a, i):
        a = np.ascontiguousarray(a, np.float32).copy()
        return self._f("randomized_select")(a, len(a), i)


class Oracle(_Lib):
    """The C restatement (liboracle.so; f64=True -> liboracle64.so)."""

    prefix = "orc_"
    _libs: dict = {}

    def __init__(self, scan, *a, f64=False, **k):
        path = ORACLE64_SO if f64 else ORACLE_SO
        if path not in Oracle._libs:
            if not os.path.exists(path):
                build_oracle()
            Oracle._libs[path] = C.CDLL(path)
        self.lib = Oracle._libs[path]
        self._bind(self.lib)
        self.lib.orc_cost.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
        self.lib.orc_last_update_percentage.restype = C.c_double
        self.lib.orc_last_update_percentage.argtypes = [C.c_void_p]
        self.lib.orc_update_count.restype = C.c_longlong
        self.lib.orc_update_count.argtypes = [C.c_void_p]
        self.lib.orc_destroy.argtypes = [C.c_void_p]
        self.lib.orc_set_lines.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _i32p, _i32p]
        super().__init__(scan, *a, **k)

    def _create(self, s, sig_s, sig_t, c_s, c_t, convg, rr, qc, hd, hT, mxy, mz, blocks):
        args = self._args(s, sig_s, sig_t, c_s, c_t, convg, rr, qc, hd, hT)
        return self.lib.orc_create(*args, C.c_int(mxy), C.c_int(mz), C.c_int(blocks))

    def _cost(self, a, b, c):
        return self.lib.orc_cost(self.h, C.byref(a), C.byref(b), C.byref(c))

    def last_update_percentage(self):
        return self.lib.orc_last_update_percentage(self.h)

    def update_count(self):
        return self.lib.orc_update_count(self.h)

    def set_lines(self, frame, block, xs, ys):
        self.lib.orc_set_lines(self.h, frame, block, len(xs), np.ascontiguousarray(xs, np.int32),
                               np.ascontiguousarray(ys, np.int32))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None


class Reference(_Lib):
    """The reference library built from its own sources (oracle/_ref)."""

    prefix = "ref_"
    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self, scan, *a, blocks=2, workdir=None, **k):
        if Reference._lib is None:
            Reference._lib = C.CDLL(REF_SO)
        self.lib = Reference._lib
        self._bind(self.lib)
        self.lib.ref_cost.argtypes = [C.c_void_p]
        self.lib.ref_cost_parts.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
        self.lib.ref_create.argtypes = None
        self._workdir = workdir
        super().__init__(scan, *a, blocks=blocks, **k)

    def _create(self, s, sig_s, sig_t, c_s, c_t, convg, rr, qc, hd, hT, mxy, mz, blocks):
        # num_z_blocks follows omp_get_max_threads() (XT_Init.c:389-398); pick
        # the smallest thread count that yields `blocks`.
        threads = max(2, blocks) * s.recon_num
        args = self._args(s, sig_s, sig_t, c_s, c_t, convg, rr, qc, hd, hT)
        cwd = os.getcwd()
        if self._workdir:
            os.chdir(self._workdir)
        try:
            libc = C.CDLL(None)
            libc.fopen.restype = C.c_void_p
            libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
            log = libc.fopen(b"/dev/null", b"w")
            return self.lib.ref_create(*args, C.c_int(mxy), C.c_int(mz), C.c_int(threads), C.c_void_p(log))
        finally:
            os.chdir(cwd)

    def _cost(self, a, b, c):
        v = self.lib.ref_cost(self.h)
        self.lib.ref_cost_parts(self.h, C.byref(a), C.byref(b), C.byref(c))
        return v

    def prepare(self, obj=None, offset=None):
        cwd = os.getcwd()
        if self._workdir:
            os.chdir(self._workdir)
        try:
            super().prepare(obj, offset)
        finally:
            os.chdir(cwd)

    def close(self):
        self.h = None
