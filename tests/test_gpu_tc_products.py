"""GPU parity of the tensor-core kriging products (tcgen05, kind::tf32 in three
split passes) against the FP64 oracle and against the CSR products.

Tolerances:
  * gradient at identical inputs: norm-wise rel 1e-5 against the FP64 oracle
    (the bar of the CSR path), and rel 2e-6 against the CSR products on the
    same chain set shape (both FP32; only the summation order and the
    split-operand rounding differ);
  * fixed-momentum leapfrog: norm-wise rel 1e-4 against the oracle;
  * log likelihood: rel 1e-5 against the oracle;
  * a full run: every chain finishes, no device wait gave up, posterior means
    within 4 combined standard errors of a CSR run at 97 % of output voxels.
"""
import numpy as np
import pytest

from test_gpu_parity import rel

pytestmark = pytest.mark.gpu


@pytest.fixture
def products(monkeypatch):
    monkeypatch.setenv("DRB_AUTOTUNE", "0")
    monkeypatch.delenv("DRB_NO_PLANE", raising=False)
    monkeypatch.delenv("DRB_PLANE_PREFETCH", raising=False)

    def make(data, n_chains, tc, **kw):
        import dualres_b200 as d
        monkeypatch.setenv("DRB_TC_PRODUCTS", "1" if tc else "0")
        hmc = d.HMCParameters(burnin=kw.pop("burnin", 4), nsave=kw.pop("nsave", 4), thin=1,
                              leapfrog=kw.pop("leapfrog", 5), seed=kw.pop("seed", 3))
        ch = d.MultiResParameters(data, hmc, n_chains)
        assert ch.config()["tensor_products"] == tc
        return ch
    return make


def _pair(oracle, vol):
    import dualres_b200 as d
    dv = d.MultiResData.from_volume(vol)
    prep = oracle.prepare(vol.highres, vol.hmask, vol.omask)
    W = oracle.kriging(prep["masked"], vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
    s = vol.stdres.ravel()
    Ys = s[~(np.isnan(s) | (s == 0))]
    theta32 = tuple(float(np.float32(t)) for t in vol.theta)
    m = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, theta32, Ys, W, prep["O"])
    return dv, m


def _field(shape, rng, scale):
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * scale).astype(np.complex64)


@pytest.mark.parametrize("n_chains", [16, 64, 100, 200])
def test_gradient_and_leapfrog_match_oracle(oracle, products, n_chains):
    from dualres_b200 import synth
    vol = synth.small_volume(seed=61, dims=(14, 13, 12), radius=4.2)
    dv, m = _pair(oracle, vol)
    ch = products(dv, n_chains, True)
    rng = np.random.default_rng(n_chains)
    sh, ss = 1.3, 3.1
    m.set_sigma(sh, ss)
    # every chain holds its own state, so the products mix per-chain halves of mu_D
    mus = [_field(m.shape, rng, 0.3) for _ in range(n_chains)]
    for c in range(n_chains):
        ch.set_state(c, mus[c], (sh, ss))
    for c in sorted({0, 1, n_chains // 2, n_chains - 1}):
        mu64 = mus[c].astype(np.complex128)
        assert rel(ch.gradient(c, mus[c]), m.gradient(mu64)) < 1e-5
        lp, ll = ch.log_prior_likelihood(c, mus[c])
        assert abs(ll / m.log_likelihood(mu64) - 1) < 1e-5
    p = _field(m.shape, rng, 2.0)
    c = n_chains - 1
    muL, pL, _ = ch.leapfrog(c, mus[c], p, 0.05, 4)
    mo, po = m.leapfrog(mus[c].astype(np.complex128), p.astype(np.complex128), 0.05, 4)
    assert rel(muL, mo) < 1e-4 and rel(pL, po) < 1e-4
    ch.close()
    dv.close()


def test_c1_tensor_products_match_csr(products):
    """The 32^3 C1 volume (W: 2298 x 19660, 2.47 M nonzeros; tiles split over all SMs, several segments per
    tile): the tensor-core gradient equals the CSR gradient to FP32 summation-order accuracy."""
    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.config_c1()
    data = d.MultiResData.from_volume(vol)
    a = products(data, 64, True)
    b = products(data, 64, False)
    rng = np.random.default_rng(5)
    shape = data.shape
    for c in (0, 37, 63):
        mu = _field(shape, rng, 0.3)
        for ch in (a, b):
            ch.set_state(c, mu, (1.7, 4.2))
        ga, gb = a.gradient(c, mu), b.gradient(c, mu)
        assert rel(ga, gb) < 2e-6, rel(ga, gb)
        la, lb = a.log_prior_likelihood(c, mu), b.log_prior_likelihood(c, mu)
        assert abs(la[1] / lb[1] - 1) < 1e-6
    a.close(), b.close(), data.close()


def test_tma_row_gathers_equal_thread_gathers(products, monkeypatch):
    """W^T rs with the chain vectors brought in by TMA row gathers (tile::gather4) and with the gather warps' own
    loads: the MMA operands are the same, so the gradients are bit-identical."""
    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.small_volume(seed=63, dims=(16, 15, 13), radius=4.2)
    data = d.MultiResData.from_volume(vol)
    rng = np.random.default_rng(9)
    mus = [_field(data.shape, rng, 0.3) for _ in range(3)]
    grads = {}
    for tg in ("1", "0"):
        monkeypatch.setenv("DRB_TC_TMA_GATHER", tg)
        ch = products(data, 64, True)
        assert ch.config()["tma_row_gather"] == (tg == "1")
        for c, mu in zip((0, 20, 63), mus):
            ch.set_state(c, mu, (1.3, 2.9))
        grads[tg] = [ch.gradient(c, mu) for c, mu in zip((0, 20, 63), mus)]
        ch.close()
    for a, b in zip(grads["1"], grads["0"]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    data.close()


@pytest.mark.parametrize("n_chains", [32, 200])
def test_full_run_matches_csr_run(products, n_chains):
    """A full run of the sampler with the tensor-core products against one with the CSR products; 200 chains run
    the 256-chain product (two stages in shared memory, two gather groups)."""
    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.small_volume(seed=62, dims=(16, 14, 12), radius=4.2)
    data = d.MultiResData.from_volume(vol)
    means = {}
    for tc in (True, False):
        ch = products(data, n_chains, tc, burnin=80, nsave=80, leapfrog=8, seed=11 if tc else 12)
        ch.run()
        st = ch.stats()
        assert all(s["done"] == 1 for s in st)
        x = np.array([ch.summary(c)["mean"] for c in range(n_chains)], np.float64)
        means[tc] = (x.mean(axis=0), x.std(axis=0, ddof=1) / np.sqrt(n_chains))
        ch.close()
    (ma, sa), (mb, sb) = means[True], means[False]
    z = np.abs(ma - mb) / np.sqrt(sa ** 2 + sb ** 2 + 1e-12)
    assert np.mean(z < 4.0) >= 0.97, (np.mean(z < 4.0), np.median(z))
    data.close()
