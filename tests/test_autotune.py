"""Per-shape autotuning of the chain-set configuration (update path and
kriging-product grid): a tuned chain set reports one of the candidates and the
time it measured, a second chain set of the same shape reuses the choice, and
the switches that turn tuning off or force a path are honoured.  The sampler's
results on any configuration are covered by the parity tests, which run every
path against the oracle."""
import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import synth

pytestmark = pytest.mark.gpu


def _chains(vol, C, leapfrog):
    data = d.MultiResData.from_volume(vol)
    return data, d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=leapfrog, seed=2), C)


def test_tuned_choice_is_cached_per_shape(monkeypatch):
    for k in ("DRB_AUTOTUNE", "DRB_NO_PLANE", "DRB_PLANE_PREFETCH", "DRB_FFT_PLAN"):
        monkeypatch.delenv(k, raising=False)
    vol = synth.small_volume(seed=51, dims=(12, 12, 10))
    data, a = _chains(vol, 3, 7)
    ca = a.config()
    assert ca["path"] in d.MultiResParameters.PATHS and ca["blocks_per_sm"] in (2, 4, 8)
    assert ca["tuned_ms"] > 0
    b = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=7, seed=9), 3)
    assert b.config() == ca  # same shape: the cached choice, not a new measurement
    a.run()
    st = a.stats()
    assert all(s["done"] == 1 for s in st)
    assert np.all(np.isfinite(a.summary(-1)["mean"]))
    a.close(), b.close(), data.close()


def test_switches(monkeypatch):
    vol = synth.small_volume(seed=52, dims=(12, 12, 10))
    monkeypatch.setenv("DRB_AUTOTUNE", "0")
    monkeypatch.delenv("DRB_NO_PLANE", raising=False)
    monkeypatch.delenv("DRB_PLANE_PREFETCH", raising=False)
    data, a = _chains(vol, 2, 5)
    assert a.config() == {"path": "plane", "blocks_per_sm": 8, "tuned_ms": 0.0, "tensor_products": False,
                          "tma_row_gather": False, "z_tile_chains": 1, "fft_plan": 0}
    monkeypatch.setenv("DRB_NO_PLANE", "1")
    b = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=5, seed=2), 2)
    assert b.config()["path"] == "lines"
    a.close(), b.close(), data.close()


def test_tuner_chooses_the_z_tile_shape(monkeypatch):
    """With 8 or more chains the tuner also times the z passes' tile shape (4 lines x 8 chains against 32 lines of
    one chain); DRB_ZTILE forces either, and both give the same gradient bit for bit (the tile only changes which
    lines a block transforms)."""
    for k in ("DRB_AUTOTUNE", "DRB_NO_PLANE", "DRB_PLANE_PREFETCH", "DRB_ZTILE"):
        monkeypatch.delenv(k, raising=False)
    vol = synth.small_volume(seed=53, dims=(12, 12, 10))
    data, a = _chains(vol, 8, 5)
    assert a.config()["z_tile_chains"] in (1, 8)
    monkeypatch.setenv("DRB_AUTOTUNE", "0")
    rng = np.random.default_rng(4)
    mu = ((rng.standard_normal(data.shape) + 1j * rng.standard_normal(data.shape)) * 0.3).astype(np.complex64)
    grads = {}
    for zt in ("8", "1"):
        monkeypatch.setenv("DRB_ZTILE", zt)
        ch = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=5, seed=2), 8)
        assert ch.config()["z_tile_chains"] == int(zt)
        ch.set_state(6, mu, (1.5, 3.0))
        grads[zt] = ch.gradient(6, mu)
        ch.close()
    assert np.array_equal(grads["8"].view(np.uint32), grads["1"].view(np.uint32))
    a.close(), data.close()


def test_tuner_chooses_the_fft_plan(monkeypatch, oracle):
    """On a 64^3 embedding (transforms of 64 points) the tuner also times the second radix plan (16 x 4 against
    8 x 8) of the inverse and forward z passes; DRB_FFT_PLAN forces the plans (bits: 1 inverse z, 2 forward z, 4 the
    x-line kernel). Both plans are FP32 transforms of the same sums in a different order, so the gradient agrees
    with the FP64 oracle within the parity bar on each."""
    for k in ("DRB_AUTOTUNE", "DRB_NO_PLANE", "DRB_PLANE_PREFETCH", "DRB_ZTILE", "DRB_FFT_PLAN"):
        monkeypatch.delenv(k, raising=False)
    vol = synth.small_volume(seed=54, dims=(22, 20, 18))
    data = d.MultiResData.from_volume(vol)
    assert data.E == (64, 64, 64)
    a = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=5, seed=2), 2)
    assert a.config()["fft_plan"] in range(8)
    a.close()
    monkeypatch.setenv("DRB_AUTOTUNE", "0")
    rng = np.random.default_rng(5)
    mu = ((rng.standard_normal(data.shape) + 1j * rng.standard_normal(data.shape)) * 0.3).astype(np.complex64)
    prep = oracle.prepare(vol.highres)
    rp, col, val = data.W()
    _, ys = data.data()
    m = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, (rp, col, val.astype(np.float64)),
                     prep["O"])
    m.set_sigma(1.5, 3.0)
    g64 = m.gradient(mu)
    for plan in ("0", "7"):
        for path in ("plane", "lines"):
            monkeypatch.setenv("DRB_FFT_PLAN", plan)
            if path == "lines":
                monkeypatch.setenv("DRB_NO_PLANE", "1")
            else:
                monkeypatch.delenv("DRB_NO_PLANE", raising=False)
            ch = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=3, thin=1, leapfrog=5, seed=2), 2)
            assert ch.config()["fft_plan"] == int(plan) and ch.config()["path"] == path
            ch.set_state(1, mu, (1.5, 3.0))
            g = ch.gradient(1, mu)
            rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
            assert rel < 1e-5, (plan, path, rel)
            ch.close()
    monkeypatch.delenv("DRB_NO_PLANE", raising=False)
    data.close()
