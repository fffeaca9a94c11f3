"""The ring-offset update that allocates no device memory.

Callers that cannot allocate device memory -- an application that reserves
all of the GPU's memory for its own pool at start-up, or a loop that must not
take cudaMalloc's device-wide synchronisation -- use
mbir_update_sinogram_offset_noalloc() on device arrays they own; its scratch
is a fixed array inside the library.  This test gives it the state of a stage
(the test itself may allocate: it plays the caller's framework, with torch as
its allocator), calls it twice in a row through the C ABI, and checks each
result against the stage-level entry point mbir_update_sinogram_offset() on
the same state, within the tolerance of the other offset tests (1e-5
relative).  It also checks that oversized detectors are refused.

The file is named to be collected last, so a failure here comes after every
other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import scenarios
import timbir_b200

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def bind():
    lib = timbir_b200.load_library()
    f = lib.mbir_update_sinogram_offset_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                  C.c_float, C.c_float, C.c_void_p]
    f.restype = C.c_int
    lib.mbir_noalloc_last_error.restype = C.c_char_p
    return lib, f


@pytest.mark.parametrize("name", ["rings1", "rings2", "rings3", "zinger_var"])
def test_noalloc_offset_update_matches_stage_entry_point(name):
    import torch
    lib, noalloc = bind()
    s = scenarios.make(name, timbir_b200.Stage)
    rng = np.random.default_rng(17)
    x = (0.01 + 0.005 * rng.standard_normal((s.N_time, s.N_z, s.N_y, s.N_x))).astype(np.float32)
    off = (0.01 * rng.standard_normal((s.N_r, s.N_t))).astype(np.float32)
    s.prepare(x, off)
    dev = torch.device("cuda", 0)
    # the caller's device arrays, in the device layouts the entry point takes
    e = torch.from_numpy(np.ascontiguousarray(np.transpose(s.errorsino(), (2, 0, 1)))).to(dev)
    w = torch.from_numpy(np.ascontiguousarray(np.transpose(s.weight(), (2, 0, 1)))).to(dev)
    d = torch.from_numpy(np.ascontiguousarray(s.offset().T)).to(dev)
    _, kw, _, _, _, _ = scenarios.SCENARIOS[name]
    args = dict(scenarios.BASE, **kw)
    for call in range(2):
        s.offset_update()
        torch.cuda.synchronize()
        rc = noalloc(e.data_ptr(), w.data_ptr(), d.data_ptr(), s.N_p, s.N_r, s.N_t, args["remove_rings"],
                     args.get("quad_convex", 1), args.get("huber_delta", 0.5), args.get("huber_T", 4.0), None)
        assert rc == 0, lib.mbir_noalloc_last_error().decode()
        e_na = np.transpose(e.cpu().numpy(), (1, 2, 0))
        d_na = d.cpu().numpy().T
        assert rel(d_na, s.offset()) < 1e-5, f"call {call + 1}: offsets"
        assert rel(e_na, s.errorsino()) < 1e-5, f"call {call + 1}: error sinogram"


def test_noalloc_rejects_detectors_beyond_its_scratch():
    lib, noalloc = bind()
    rows, cols = 2048, 1024  # 2 Mi detector elements > MBIR_NOALLOC_MAX_ELEMS
    rc = noalloc(None, None, None, 16, cols, rows, 2, 1, 0.5, 4.0, None)
    assert rc == -1
    assert b"exceeds the no-allocation limit" in lib.mbir_noalloc_last_error()
