"""Fault injection on the GPU without a GPU fault: an exhausted device
(the library's allocator under a cap) and a device-side wait that runs out
(a super-voxel whose conflicting predecessor never runs).  Each must end in
an error the host reports, leave no device memory behind, and leave the
CUDA context usable for the next reconstruction."""
import time

import numpy as np
import pytest

import timbir_b200
from timbir_b200 import synth

pytestmark = pytest.mark.gpu

PRIOR = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0, blocks=2)


def scan():
    return synth.ellipsoid_scan(48, 8, 72, seed=4)


def lib():
    return timbir_b200.load_library()


def test_allocation_failure_is_reported_and_nothing_leaks():
    held = lib().mbir_get_device_bytes()
    lib().mbir_set_device_bytes_cap(held + (1 << 20))  # 1 MiB more than now
    st = None
    try:
        with pytest.raises(timbir_b200.MbirError):
            st = timbir_b200.Stage(scan(), **PRIOR)
            st.set_schedule(1)
            st.prepare()
    finally:
        lib().mbir_set_device_bytes_cap(0)
        if st is not None:
            st.close()
    assert lib().mbir_get_device_bytes() == held  # what the failed set-up took is freed
    st = timbir_b200.Stage(scan(), **PRIOR)
    st.set_schedule(1)
    st.prepare()
    c0 = st.cost()[0]
    st.iterate(1)
    assert st.cost()[0] < c0
    st.close()


def test_a_dependency_wait_that_runs_out_is_an_error_not_a_hang():
    st = timbir_b200.Stage(scan(), **PRIOR)
    st.set_schedule(1)
    st.prepare()
    st.iterate(1)
    _check = lib().mbir_debug_sv_skip_tasks(st.h, 1)  # the first super-voxel of the next sweep never runs
    assert _check == 0
    t0 = time.time()
    with pytest.raises(timbir_b200.MbirError, match="dependency wait timed out"):
        st.iterate(2)
    assert time.time() - t0 < 30.0
    st.close()
    # the context is usable: a new stage reconstructs as before
    st = timbir_b200.Stage(scan(), **PRIOR)
    st.set_schedule(1)
    st.prepare()
    c0 = st.cost()[0]
    for it in range(1, 4):
        st.iterate(it)
    c3 = st.cost()[0]
    st.close()
    assert np.isfinite(c3) and c3 < c0
