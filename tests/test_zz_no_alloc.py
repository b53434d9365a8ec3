"""dr_log_posterior_noalloc: the evaluation entry point that allocates no device
memory, for callers that may not call cudaMalloc/cudaFree (device memory owned by
another allocator, or a loop that has stopped allocating).  Its scratch is one
library-owned device array, so two consecutive calls must both agree with the
allocating entry point dr_log_posterior.  This file is collected last on purpose."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative, the bar used for the log posterior in the parity tests


def _case(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    import dualres_b200 as d
    vol = d.MultiResData(g["highres"], g["qform_hr"], g["stdres"], g["qform_sr"], tuple(g["theta"]),
                         float(g["radius"]))
    return g, vol


@pytest.mark.parametrize("name", ["g1_rbf_e1", "g3_rbf_aniso"])
def test_noalloc_matches_allocating_entry_point_twice(name):
    import torch

    import dualres_b200 as d
    g, vol = _case(name)
    chains = d.MultiResParameters(vol, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=3, seed=1), 1)
    sh, ss = (float(x) for x in g["sigma"])
    mu = g["mu"]
    chains.set_state(0, mu, (sh, ss))
    lp, ll = chains.log_prior_likelihood(0, mu)
    dmu = torch.from_numpy(np.ascontiguousarray(mu, np.complex64).view(np.float32).ravel().copy()).to("cuda:0")
    for _ in range(2):
        lp2, ll2 = d.api.log_posterior_noalloc(vol, dmu.data_ptr(), sh, ss)
        assert abs(lp2 / lp - 1) < TOL, (lp2, lp)
        assert abs(ll2 / ll - 1) < TOL, (ll2, ll)
    # a different field after the first: the shared scratch must not leak state
    mu2 = (mu * 0.5).astype(np.complex64)
    chains.set_state(0, mu2, (sh, ss))
    lp_b, ll_b = chains.log_prior_likelihood(0, mu2)
    dmu2 = torch.from_numpy(mu2.view(np.float32).ravel().copy()).to("cuda:0")
    lp3, ll3 = d.api.log_posterior_noalloc(vol, dmu2.data_ptr(), sh, ss)
    assert abs(lp3 / lp_b - 1) < TOL and abs(ll3 / ll_b - 1) < TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import dualres_b200 as d
    from dualres_b200 import synth
    # single resolution, 70 x 40 x 40 latent grid -> 256 x 128 x 128 embedding (2^22 points > 2^21)
    v = synth.make_volume((70, 40, 40), 1.0, (1.0, 0.3, 1.0), 0.5, 0.3, 2.0, "full", 1.0, 3, dual=False)
    vol = d.MultiResData(v.highres, v.qform_hr, covariance=v.theta)
    assert vol.N > 2 ** 21
    dmu = torch.zeros(2 * vol.N, dtype=torch.float32, device="cuda:0")
    with pytest.raises(d.DrError) as e:
        d.api.log_posterior_noalloc(vol, dmu.data_ptr(), 1.0, 1.0)
    assert e.value.code == d.api.DR_ERR_UNSUPPORTED
    assert "scratch limit" in str(e.value)
