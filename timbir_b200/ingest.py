"""Data ingestion before reconstruct() (include/timbir_b200.h, ingestion
section): the APS driver's normalisation of raw counts by bright and dark
fields, the standard driver's down-sampling of projections and weights, and
the interlaced view generator, on the GPU through the native library
(TIMBIR src/reconstruct/aps_data/XT_HDFIO.c, XT_Views.c,
std_data/XT_HDFIO.c).  The HDF5 reading is the caller's (h5py or any other
reader): pass the datasets' arrays as stored, [frames][rows][cols]."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load_library

_done = False


def _lib():
    global _done
    lib = load_library()
    if not _done:
        VP, I32, F = C.c_void_p, C.c_int32, C.c_float
        lib.mbir_ingest_last_error.restype = C.c_char_p
        lib.mbir_normalize_counts.argtypes = [VP, I32, VP, I32, VP, I32] + [I32] * 9 + [C.c_double, VP, VP]
        lib.mbir_downsample_projections.argtypes = [VP, VP] + [I32] * 10 + [C.c_double, VP, VP]
        lib.mbir_gen_interlaced_views.argtypes = [VP, VP, I32, I32, I32, I32, F, F]
        lib.mbir_gen_interlaced_views.restype = I32
        lib.mbir_frame_mean_device.argtypes = [VP, I32, I32, I32, VP, VP]
        lib.mbir_normalize_counts_device.argtypes = [VP, VP, VP, I32, I32, I32, I32, C.c_double, VP, VP, VP]
        _done = True
    return lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(_lib().mbir_ingest_last_error().decode(errors="replace"))


BH_APS = 0.5  # BH_QUAD_COEF of the APS driver (aps_data/XT_Constants.h)
BH_STD = 0.0  # of the standard driver (std_data/XT_Constants.h)


def normalize_counts(counts, whites, darks, proj_rows, proj_cols, proj_start=0, proj_num=None, datafile_row0=0,
                     rank=0, ranks=1, bh=BH_APS):
    """read_data of the APS driver on uint16 stacks [frames][rows][cols];
    returns (projections, weights), each [proj_num][proj_rows / ranks][proj_cols]."""
    counts = np.ascontiguousarray(counts, np.uint16)
    whites = np.ascontiguousarray(whites, np.uint16)
    darks = np.ascontiguousarray(darks, np.uint16)
    n, rows, cols = counts.shape
    if whites.shape[1:] != (rows, cols) or darks.shape[1:] != (rows, cols):
        raise ValueError("bright and dark stacks must have the counts' rows and columns")
    if proj_num is None:
        proj_num = n - proj_start
    out = [np.zeros((proj_num, proj_rows // ranks, proj_cols), np.float32) for _ in range(2)]
    _check(_lib().mbir_normalize_counts(counts.ctypes.data, n, whites.ctypes.data, whites.shape[0],
                                        darks.ctypes.data, darks.shape[0], rows, cols, datafile_row0, proj_rows,
                                        proj_cols, proj_start, proj_num, rank, ranks, bh, out[0].ctypes.data,
                                        out[1].ctypes.data))
    return out[0], out[1]


def downsample_projections(projs, wts, proj_rows, proj_cols, proj_start=0, proj_num=None, datafile_row0=0, rank=0,
                           ranks=1, bh=BH_STD):
    """read_ProjWeightData of the standard driver on float [views][rows][cols]."""
    projs = np.ascontiguousarray(projs, np.float32)
    wts = np.ascontiguousarray(wts, np.float32)
    n, rows, cols = projs.shape
    if wts.shape != projs.shape:
        raise ValueError("projections and weights must have the same shape")
    if proj_num is None:
        proj_num = n - proj_start
    out = [np.zeros((proj_num, proj_rows // ranks, proj_cols), np.float32) for _ in range(2)]
    _check(_lib().mbir_downsample_projections(projs.ctypes.data, wts.ctypes.data, n, rows, cols, datafile_row0,
                                              proj_rows, proj_cols, proj_start, proj_num, rank, ranks, bh,
                                              out[0].ctypes.data, out[1].ctypes.data))
    return out[0], out[1]


def interlaced_views(K, N_theta, N_p, proj_start=0, min_acq_time=0.0, rot_speed=0.0):
    """gen_interlaced_views_0_to_Inf: (angles, times, kept views generated)."""
    v = np.zeros(N_p, np.float32)
    t = np.zeros(N_p, np.float32)
    n = _lib().mbir_gen_interlaced_views(v.ctypes.data, t.ctypes.data, K, N_theta, proj_start, N_p, min_acq_time,
                                         rot_speed)
    if n < 0:
        raise ValueError("invalid interlaced-view parameters")
    return v, t, int(n)
