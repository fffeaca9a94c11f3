"""Host-side fault injection (no GPU needed: these checks run before any
device work): non-finite or negative inputs and out-of-range switches are
refused with an error, as the failure plan of the engine prescribes (error
codes, never a crash or a NaN reconstruction)."""
import numpy as np
import pytest

import timbir_b200
from timbir_b200 import synth

PRIOR = dict(sig_s=0.002, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=1.0, blocks=2)


@pytest.mark.parametrize("field,index,value", [("projections", 5, np.nan), ("weights", 17, np.inf),
                                               ("weights", 3, -1.0), ("projections", 0, -np.inf)])
def test_non_finite_or_negative_inputs_are_refused(field, index, value):
    scan = synth.ellipsoid_scan(16, 4, 24, seed=1)
    arr = getattr(scan, field).copy()
    arr.reshape(-1)[index] = value
    setattr(scan, field, arr)
    with pytest.raises(timbir_b200.MbirError, match="not finite"):
        timbir_b200.Stage(scan, **PRIOR)


@pytest.mark.parametrize("kw,msg", [(dict(remove_rings=4), "remove_rings"), (dict(quad_convex=2), "quad_convex"),
                                    (dict(blocks=3), "num_z_blocks")])
def test_out_of_range_switches_are_refused(kw, msg):
    scan = synth.ellipsoid_scan(16, 4, 24, seed=1)
    args = dict(PRIOR)
    args.update(kw)
    with pytest.raises(timbir_b200.MbirError, match=msg):
        timbir_b200.Stage(scan, **args)
