"""The benchmark's plain single-chain GPU comparator (bench.PlainGPU: the reference
algorithm with four cuFFT transforms per leapfrog step) computes the same
gradient and log posterior as the library at identical inputs, so the ratio the
benchmark reports compares two implementations of one algorithm.  Tolerance:
norm-wise rel 1e-4 (both FP32 transforms; the comparator sums in its own order)."""
import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import synth

pytestmark = pytest.mark.gpu


def test_plain_gpu_gradient_matches_library():
    import torch

    import bench
    vol = synth.small_volume(seed=61, dims=(14, 12, 10))
    data = d.MultiResData.from_volume(vol)
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=3, seed=1), 1)
    rng = np.random.default_rng(4)
    mu = ((rng.standard_normal(data.shape) + 1j * rng.standard_normal(data.shape)) * 0.3).astype(np.complex64)
    sh, ss = 1.7, 4.2
    ch.set_state(0, mu, (sh, ss))
    g_lib = ch.gradient(0, mu)
    lp, ll = ch.log_prior_likelihood(0, mu)
    pg = bench.PlainGPU(data)
    mt = torch.tensor(mu, device="cuda:0")
    g_plain = pg.gradient(mt, sh, ss).cpu().numpy()
    rel = np.linalg.norm(g_plain - g_lib) / np.linalg.norm(g_lib)
    assert rel < 1e-4, rel
    h, _, _ = pg.log_post(mt, sh, ss)
    assert abs(float(h) / (lp + ll) - 1) < 1e-5
    r, ms = bench.plain_gpu_rate(data, 5, 3)
    assert r > 0 and ms > 0
    ch.close()
    data.close()
