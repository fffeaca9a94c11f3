"""CPU oracle of the data-ingestion path (test infrastructure only): numpy
restatements of the reference's APS reader normalisation (read_data,
src/reconstruct/aps_data/XT_HDFIO.c:46-236), standard reader down-sampling
(read_ProjWeightData, std_data/XT_HDFIO.c:41-158) and interlaced view
generator (gen_interlaced_views_0_to_Inf, aps_data/XT_Views.c:41-80), with
the C code's float / double roundings.  Pinned against the reference itself
(tests/golden/ingest.npz from the reference's sources compiled against an
in-memory HDF5 stand-in, oracle/ref/h5_shim.c).  log is numpy's, which can
differ from the C library's in a double's last bit."""
from __future__ import annotations

import math

import numpy as np


def _window(rows, cols, datafile_row0, proj_rows, proj_cols, rank, ranks):
    extras = cols % proj_cols  # XT_HDFIO.c:94-125
    ncols = cols - extras
    ratio = ncols // proj_cols
    prows = proj_rows // ranks
    nrows = prows * ratio
    row0 = datafile_row0 + rank * nrows
    return ratio, extras // 2, ncols, row0, nrows, prows


def _frame_mean(stack):
    s = np.zeros(stack.shape[1:], np.float32)
    for f in stack:  # float sums in frame order, then / n (float)
        s = (s + f.astype(np.float32)).astype(np.float32)
    return (s / np.float32(stack.shape[0])).astype(np.float32)


def normalize_counts(counts, whites, darks, proj_rows, proj_cols, proj_start, proj_num, datafile_row0=0, rank=0,
                     ranks=1, bh=0.5):
    rows, cols = counts.shape[1:]
    ratio, c0, nc, r0, nr, prows = _window(rows, cols, datafile_row0, proj_rows, proj_cols, rank, ranks)
    sel = np.s_[r0:r0 + nr, c0:c0 + nc]
    white = _frame_mean(whites[1:-1][(slice(None),) + sel])
    dark = _frame_mean(darks[1:-1][(slice(None),) + sel])
    cnt = counts[proj_start:proj_start + proj_num][(slice(None),) + sel]
    P = np.zeros((proj_num, prows, proj_cols), np.float32)
    W = np.zeros_like(P)
    w = np.zeros((proj_num, prows, proj_cols), np.float32)
    wd = np.zeros((prows, proj_cols), np.float32)
    for m in range(ratio):
        for q in range(ratio):
            c = cnt[:, m::ratio, q::ratio].astype(np.float32)
            d = dark[m::ratio, q::ratio]
            wh = white[m::ratio, q::ratio]
            w = (w.astype(np.float64) + np.abs((c - d).astype(np.float32)).astype(np.float64)).astype(np.float32)
            wd = (wd.astype(np.float64) + np.abs((wh - d).astype(np.float32)).astype(np.float64)).astype(np.float32)
    t = np.log((wd[None] / w).astype(np.float32).astype(np.float64)).astype(np.float32).astype(np.float64)
    P[:] = (bh * t * t + t).astype(np.float32)
    W[:] = w
    return P, W


def downsample_projections(projs, wts, proj_rows, proj_cols, proj_start, proj_num, datafile_row0=0, rank=0, ranks=1,
                           bh=0.0):
    rows, cols = projs.shape[1:]
    ratio, c0, nc, r0, nr, prows = _window(rows, cols, datafile_row0, proj_rows, proj_cols, rank, ranks)
    p = projs[proj_start:proj_start + proj_num, r0:r0 + nr, c0:c0 + nc].astype(np.float32)
    ww = wts[proj_start:proj_start + proj_num, r0:r0 + nr, c0:c0 + nc].astype(np.float32)
    t = np.zeros((proj_num, prows, proj_cols), np.float32)
    w = np.zeros_like(t)
    for m in range(ratio):
        for q in range(ratio):
            t = (t + p[:, m::ratio, q::ratio]).astype(np.float32)
            w = (w + ww[:, m::ratio, q::ratio]).astype(np.float32)
    t = (t / np.float32(ratio * ratio)).astype(np.float32).astype(np.float64)
    return (bh * t * t + t).astype(np.float32), w


def interlaced_views(K, N_theta, N_p, proj_start=0, min_acq_time=0.0, rot_speed=0.0):
    L = N_theta // K
    bits = int(math.floor(math.log(K) / math.log(2.0) + 0.5))
    dth = np.float32(math.pi / N_theta)
    min_d = np.float32(np.float32(rot_speed) * np.float32(min_acq_time))
    ang, tim = [], []
    i = 0
    while len(ang) < proj_start + N_p:
        q = (i // L) % K
        r = 0
        for b in range(bits):
            if q & (1 << b):
                r |= 1 << (bits - 1 - b)
        a = np.float32(i * K + r)
        t = np.float32(a / np.float32(K))
        av = np.float32(a * dth)
        if i == 0 or np.float32(av - ang[-1]) > min_d:
            ang.append(av)
            tim.append(t)
        i += 1
    return (np.array(ang[proj_start:], np.float32), np.array(tim[proj_start:], np.float32), len(ang))
