"""The multi-resolution hand-off on the device.

Between the stages of one reconstruct() call the next stage's start object
and update-magnitude map are the previous stage's, up-sampled x2 on the GPU
(initObject, XT_ICD_update.c:540-651) instead of written to files, read back
and up-sampled on the host.  The up-sampling must equal the reference's own
(upsample_object_bilinear_2D / _3D, XT_ICD_update.c:359-498) bit for bit:
tests/golden/upsample.npz holds the reference's results on seeded slices
(made by tests/golden/make_golden.py from the reference library).
"""
import os

import numpy as np
import pytest

import timbir_b200

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("z_too", [0, 1], ids=["xy", "xyz"])
def test_device_upsampling_is_the_references(z_too):
    g = np.load(os.path.join(GOLD, "upsample.npz"))
    for k in range(4):
        x = g[f"in{k}"]
        np.testing.assert_array_equal(timbir_b200.upsample(x, bool(z_too)), g[f"out{k}_{z_too}"],
                                      err_msg=f"shape {x.shape}")
