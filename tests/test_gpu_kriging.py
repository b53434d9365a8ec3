"""Kriging weights built on the device (k_kriging_rows) against the host builder
(dr_kriging_matrix, FP64 Cholesky / QR): identical sparsity, weights within
1e-7 absolute (both are FP64 solves rounded to float).  Cases: isotropic and
anisotropic grids, an ill-conditioned spectrum, and a covariance with
variance above 1, where K is not positive definite and rows fall back to QR."""
import os

import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import api, synth

pytestmark = pytest.mark.gpu

CASES = {
    "c1_like": dict(dims=(20, 20, 18), voxel=1.0, theta=(0.806, 0.132, 1.0), radius=6.9),
    "aniso_1p5": dict(dims=(16, 18, 14), voxel=1.5, theta=(1.0, 0.4, 1.5), radius=6.9),
    "smooth": dict(dims=(18, 16, 16), voxel=1.0, theta=(0.95, 0.05, 2.0), radius=5.0),
    "variance_above_1": dict(dims=(14, 14, 12), voxel=1.0, theta=(1.6, 0.3, 1.0), radius=3.5),
    "rotated_aniso": dict(dims=(18, 18, 14), voxel=1.0, theta=(0.9, 0.3, 1.2), radius=6.9, rotate=True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_kriging_matches_host(name, monkeypatch):
    c = CASES[name]
    vol = synth.make_volume(c["dims"], c["voxel"], c["theta"], 0.5, 0.3, c["radius"], "ellipsoid", 0.65, 9)
    if c.get("rotate"):
        vol = synth.rotated(vol)
    monkeypatch.delenv("DRB_HOST_KRIGING", raising=False)
    dv = d.MultiResData.from_volume(vol)
    rp, col, val = dv.W()
    hr = np.where(vol.hmask == 0, 0, vol.highres) if vol.hmask is not None else vol.highres
    hrp, hcol, hval = api.kriging_matrix(hr, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
    assert np.array_equal(rp, hrp)
    assert np.array_equal(col, hcol)
    assert np.abs(val - hval).max() < 1e-7
    # and the same volume built with the host solves gives the same sampler inputs
    monkeypatch.setenv("DRB_HOST_KRIGING", "1")
    dh = d.MultiResData.from_volume(vol)
    rp2, col2, val2 = dh.W()
    assert np.array_equal(rp2, rp) and np.array_equal(col2, col)
    assert np.abs(val2 - val).max() < 1e-7
    dv.close()
    dh.close()
