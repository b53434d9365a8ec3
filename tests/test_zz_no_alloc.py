"""dr_log_posterior_noalloc: the evaluation entry point that allocates no device
memory, for callers that may not call cudaMalloc/cudaFree (device memory owned by
another allocator, or a loop that has stopped allocating).  Its scratch is one
library-owned device array, so two consecutive calls must both agree with the
allocating entry point dr_log_posterior and with the FP64 oracle, and a call
after the first must leave the device's free memory, the default memory pool's
high-water mark and that of the library's own pool (from which every other
library allocation comes) where they were.  This file is collected last on
purpose."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative, the bar used for the log posterior in the parity tests
CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7
CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


def _case(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    import dualres_b200 as d
    vol = d.MultiResData(g["highres"], g["qform_hr"], g["stdres"], g["qform_sr"], tuple(g["theta"]),
                         float(g["radius"]))
    return g, vol


class _DriverMemory:
    """Free device memory (cuMemGetInfo) and the default pool's in-use bytes and high-water mark, read through the
    driver API so that the library's own runtime is not involved."""

    def __init__(self, device=0):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int(0)
        assert self.cu.cuDeviceGet(ctypes.byref(dev), device) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def _attr(self, a):
        v = ctypes.c_uint64(0)
        assert self.cu.cuMemPoolGetAttribute(self.pool, a, ctypes.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = ctypes.c_uint64(0)  # setting the high-water mark to 0 resets it to the current use
        assert self.cu.cuMemPoolSetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH, ctypes.byref(zero)) == 0

    def snapshot(self):
        free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
        assert self.cu.cuMemGetInfo_v2(ctypes.byref(free), ctypes.byref(total)) == 0
        return dict(free=free.value, used=self._attr(CU_MEMPOOL_ATTR_USED_MEM_CURRENT),
                    high=self._attr(CU_MEMPOOL_ATTR_USED_MEM_HIGH))


@pytest.mark.parametrize("name", ["g1_rbf_e1", "g3_rbf_aniso"])
def test_noalloc_matches_allocating_entry_point_twice(oracle, name):
    import torch

    import dualres_b200 as d
    g, vol = _case(name)
    chains = d.MultiResParameters(vol, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=3, seed=1), 1)
    sh, ss = (float(x) for x in g["sigma"])
    mu = g["mu"]
    chains.set_state(0, mu, (sh, ss))
    lp, ll = chains.log_prior_likelihood(0, mu)
    # the FP64 oracle on the same input
    W = (g["W_rowptr"], g["W_col"], g["W_val"])
    m = oracle.Model(g["D"], g["Yh"], g["qform_hr"], tuple(g["theta"]), g["Ys"], W, g["O"])
    m.set_sigma(sh, ss)
    lp64, ll64 = m.log_prior(mu), m.log_likelihood(mu)
    dmu = torch.from_numpy(np.ascontiguousarray(mu, np.complex64).view(np.float32).ravel().copy()).to("cuda:0")
    torch.cuda.synchronize()
    for _ in range(2):
        lp2, ll2 = d.api.log_posterior_noalloc(vol, dmu.data_ptr(), sh, ss)
        assert abs(lp2 / lp - 1) < TOL, (lp2, lp)
        assert abs(ll2 / ll - 1) < TOL, (ll2, ll)
        assert abs(lp2 / lp64 - 1) < TOL and abs(ll2 / ll64 - 1) < TOL, (lp2, lp64, ll2, ll64)
    # a different field after the first: the shared scratch must not leak state
    mu2 = (mu * 0.5).astype(np.complex64)
    chains.set_state(0, mu2, (sh, ss))
    lp_b, ll_b = chains.log_prior_likelihood(0, mu2)
    dmu2 = torch.from_numpy(mu2.view(np.float32).ravel().copy()).to("cuda:0")
    torch.cuda.synchronize()
    lp3, ll3 = d.api.log_posterior_noalloc(vol, dmu2.data_ptr(), sh, ss)
    assert abs(lp3 / lp_b - 1) < TOL and abs(ll3 / ll_b - 1) < TOL
    assert abs(lp3 / m.log_prior(mu2) - 1) < TOL and abs(ll3 / m.log_likelihood(mu2) - 1) < TOL


def test_noalloc_allocates_nothing_on_the_32cubed_volume(oracle):
    """The 32^3 volume (64^3 embedding, 2.47 M kriging nonzeros): two calls against the FP64 oracle; the second
    leaves the free device memory and the default pool's in-use bytes and high-water mark unchanged."""
    import torch

    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.config_c1()
    data = d.MultiResData.from_volume(vol)
    prep = oracle.prepare(vol.highres)
    rp, col, val = data.W()
    _, ys = data.data()
    m = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, (rp, col, val.astype(np.float64)),
                     prep["O"])
    sh, ss = 4.0, 11.0
    m.set_sigma(sh, ss)
    rng = np.random.default_rng(3)
    mu = ((rng.standard_normal(m.shape) + 1j * rng.standard_normal(m.shape)) * 0.3).astype(np.complex64)
    dmu = torch.from_numpy(mu.view(np.float32).ravel().copy()).to("cuda:0")
    torch.cuda.synchronize()
    lp64, ll64 = m.log_prior(mu), m.log_likelihood(mu)
    mem = _DriverMemory(0)
    first = d.api.log_posterior_noalloc(data, dmu.data_ptr(), sh, ss)  # warms up: finds the scratch array
    torch.cuda.synchronize()
    mem.reset_high()
    before = mem.snapshot()
    lib_before = d.api.pool_usage(0, reset_high=True)
    second = d.api.log_posterior_noalloc(data, dmu.data_ptr(), sh, ss)
    torch.cuda.synchronize()
    after = mem.snapshot()
    lib_after = d.api.pool_usage(0)
    for lp, ll in (first, second):
        assert abs(lp / lp64 - 1) < TOL and abs(ll / ll64 - 1) < TOL, (lp, lp64, ll, ll64)
    assert after["free"] == before["free"], (before, after)
    assert after["used"] == before["used"] and after["high"] == before["used"], (before, after)
    assert lib_before[0] > 0 and lib_after[0] == lib_before[0] and lib_after[1] == lib_before[0], (lib_before,
                                                                                                  lib_after)
    assert torch.cuda.current_device() == 0
    data.close()


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
