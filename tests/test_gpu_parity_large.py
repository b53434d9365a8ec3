"""Oracle parity at the benchmark and large-embedding configurations, through the sampler's own kernels.

The gradient and log posterior entry points (dr_gradient, dr_log_posterior) run step 0 of the sampler's leapfrog
sequence -- the kriging products of the chain set's path, the inverse z pass and the plane or x-line kernel -- so
every check below exercises the kernels the sampler runs, on these configurations:

  * the 32^3 volume at 1 mm (RBF 0.806 / 0.132 / 1, 64^3 embedding) with 64 chains: the plane kernel at E = 64 and
    the kriging products on the tensor cores, the batched configuration the throughput is quoted on; chains 0, 31
    and 63 each hold their own state;
  * the 64x64x48 volume at 1.5 mm (RBF 1.0 / 0.4 / 1.5, 128^3 embedding, smoothed-noise mask): the plane kernel at
    E = 128 with the CSR products (1 chain) and with the tensor-core products (16 chains);
  * an 80x80x64 volume at 1 mm (256x256x128 embedding): the x-line kernel at E0 = 256 with separate y passes.

The kriging sparsity of each volume is compared bit for bit with the oracle's own build
(kriging_matrix.h:148-343); both sides then use the library's weights, which are checked against the host builder
elsewhere. Bars (norm-wise relative): log prior, log likelihood and gradient 1e-5 against the FP64 oracle;
fixed-momentum leapfrog 1e-4, with its step-0 energies at 1e-5 and its final energies at 1e-4; posterior mean and
variance on identical draws 1e-4 / 1e-3.
"""
import numpy as np
import pytest

from test_posterior_mean_fp64 import _device_step, _drive, _flat, _rel

pytestmark = pytest.mark.gpu


@pytest.fixture
def defaults(monkeypatch):
    """The chain sets' default configuration (no tuning), optionally with the products forced."""
    monkeypatch.setenv("DRB_AUTOTUNE", "0")
    for k in ("DRB_NO_PLANE", "DRB_PLANE_PREFETCH", "DRB_TC_PRODUCTS"):
        monkeypatch.delenv(k, raising=False)
    return monkeypatch


def _x256_volume():
    from dualres_b200 import synth
    # the largest class of the uneven batch: 80x80x64 latent grid -> 256x256x128 embedding
    return synth.make_volume((80, 80, 64), 1.0, (1.0, 0.35, 1.4), 0.6, 0.4, 6.9, "ellipsoid", 0.60, 5, name="x256")


def _setup(oracle, vol):
    """Library volume and FP64 oracle model of the same images; the kriging sparsity is checked bit for bit."""
    import dualres_b200 as d
    data = d.MultiResData.from_volume(vol)
    prep = oracle.prepare(vol.highres)
    rp, col, val = data.W()
    orp, ocol, _ = oracle.kriging(prep["masked"], vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius,
                                  solve=False)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    d_idx, o_idx = data.indices()
    _, ys = data.data()
    m = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, (rp, col, val.astype(np.float64)), prep["O"])
    assert tuple(m.E) == tuple(data.E)
    assert np.array_equal(d_idx, _flat(prep["D"], m.E))
    return data, m, prep


def _prior_draw(m, prep, rng):
    """A prior-typical field plus the data (the fixtures' recipe): FFT(sqrt(lambda / N) w) on live modes + Yh."""
    lam = m.lam().real
    w = rng.standard_normal(m.shape) + 1j * rng.standard_normal(m.shape)
    mu = np.fft.fftn(np.where(lam > 0, np.sqrt(np.abs(lam) / m.N), 0.0) * w)
    mu.ravel()[_flat(prep["D"], m.E)] += prep["Yh"]
    return mu.astype(np.complex64)


def _momentum(m, rng):
    return (rng.standard_normal(m.shape) + 1j * rng.standard_normal(m.shape)).astype(np.complex64)


def _check_point(ch, m, c, mu, tol_grad=1e-5):
    mu64 = mu.astype(np.complex128)
    lp, ll = ch.log_prior_likelihood(c, mu)
    assert abs(lp / m.log_prior(mu64) - 1) < 1e-5, (lp, m.log_prior(mu64))
    assert abs(ll / m.log_likelihood(mu64) - 1) < 1e-5, (ll, m.log_likelihood(mu64))
    g = ch.gradient(c, mu)
    r = _rel(g.astype(np.complex128), m.gradient(mu64))
    assert r < tol_grad, r
    return r


def _check_leapfrog(ch, m, c, mu, p, eps, L):
    muL, pL, en = ch.leapfrog(c, mu, p, eps, L)
    mo, po = m.leapfrog(mu.astype(np.complex128), p.astype(np.complex128), eps, L)
    rm, rp = _rel(muL.astype(np.complex128), mo), _rel(pL.astype(np.complex128), po)
    assert rm < 1e-4 and rp < 1e-4, (rm, rp)
    mu64, p64 = mu.astype(np.complex128), p.astype(np.complex128)
    for got, want in ((en[0], m.log_prior(mu64)), (en[1], m.log_likelihood(mu64)), (en[2], m.kinetic(p64))):
        assert abs(got / want - 1) < 1e-5, (got, want)
    for got, want in ((en[3], m.log_prior(mo)), (en[4], m.log_likelihood(mo)), (en[5], m.kinetic(po))):
        assert abs(got / want - 1) < 1e-4, (got, want)
    return rm, rp


def test_32cubed_64_chains_plane_and_tensor_products(oracle, defaults):
    """The batched configuration: 64 chains on the 32^3 volume, plane kernel E = 64, tcgen05 kriging products."""
    import dualres_b200 as d
    from dualres_b200 import synth
    data, m, prep = _setup(oracle, synth.config_c1())
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=4, thin=1, leapfrog=25, seed=2), 64)
    cfg = ch.config()
    assert cfg["path"] == "plane" and cfg["tensor_products"], cfg
    rng = np.random.default_rng(64)
    sh, ss = 4.0, 11.0
    m.set_sigma(sh, ss)
    mus = {c: _prior_draw(m, prep, rng) for c in (0, 31, 63)}
    for c, mu in mus.items():
        ch.set_state(c, mu, (sh, ss))
    for c, mu in mus.items():
        r = _check_point(ch, m, c, mu)
        rm, rp = _check_leapfrog(ch, m, c, mu, _momentum(m, rng), 0.05, 25)
        print(f"32^3 x 64 chains, chain {c}: gradient rel {r:.2e}, leapfrog mu {rm:.2e} p {rp:.2e}")
    ch.close()
    data.close()


@pytest.mark.parametrize("n_chains", [1, 16])
def test_128_embedding_plane_kernel(oracle, defaults, n_chains):
    """The 64x64x48 volume at 1.5 mm: plane kernel at E = 128; CSR products for 1 chain, tensor cores for 16."""
    import dualres_b200 as d
    from dualres_b200 import synth
    data, m, prep = _setup(oracle, synth.config_c2())
    assert tuple(data.E) == (128, 128, 128)
    if n_chains >= 16:
        defaults.setenv("DRB_TC_PRODUCTS", "1")  # the default turns them on from 32 chains
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=4, thin=1, leapfrog=10, seed=2), n_chains)
    cfg = ch.config()
    assert cfg["path"] == "plane" and cfg["tensor_products"] == (n_chains >= 16), cfg
    rng = np.random.default_rng(128 + n_chains)
    sh, ss = 2.0, 8.0
    m.set_sigma(sh, ss)
    c = n_chains - 1
    mu = _prior_draw(m, prep, rng)
    ch.set_state(c, mu, (sh, ss))
    r = _check_point(ch, m, c, mu)
    rm, rp = _check_leapfrog(ch, m, c, mu, _momentum(m, rng), 0.01, 10)
    print(f"128^3, {n_chains} chain(s): gradient rel {r:.2e}, leapfrog mu {rm:.2e} p {rp:.2e}")
    ch.close()
    data.close()


def test_128_embedding_posterior_moments_on_identical_draws(oracle, defaults):
    """Posterior mean and variance of Re mu at the output voxels over 8 transitions (L = 10) of the device chain
    and the FP64 oracle chain on the same momentum normals and accept uniforms, at fixed sigma."""
    import dualres_b200 as d
    from dualres_b200 import synth
    data, m, prep = _setup(oracle, synth.config_c2())
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=10, seed=1), 1)
    sh, ss = 2.0, 8.0
    m.set_sigma(sh, ss)
    mu0 = np.zeros(m.shape, np.complex64)
    mu0.ravel()[_flat(prep["D"], m.E)] = prep["Yh"]
    ch.set_state(0, mu0, (sh, ss))
    oi = _flat(prep["O"], m.E)
    eps, L = 0.01, 10
    (m64, v64), (m32, v32), flips, rate = _drive(m, _device_step(ch, eps, L), mu0, oi, eps, L, 8, 1)
    print(f"128^3: posterior mean rel {_rel(m32, m64):.2e}, variance rel {_rel(v32, v64):.2e}, accept {rate:.3f}")
    assert flips == 0 and rate > 0.3, (flips, rate)
    assert _rel(m32, m64) < 1e-4, _rel(m32, m64)
    assert _rel(v32, v64) < 1e-3, _rel(v32, v64)
    ch.close()
    data.close()


def test_256_embedding_xline_kernel(oracle, defaults):
    """The 80x80x64 volume (256x256x128 embedding): the x-line kernel at E0 = 256 and the separate y passes."""
    import dualres_b200 as d
    data, m, prep = _setup(oracle, _x256_volume())
    assert tuple(data.E) == (256, 256, 128)
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=4, nsave=4, thin=1, leapfrog=3, seed=2), 1)
    assert ch.config()["path"] == "lines"
    rng = np.random.default_rng(256)
    sh, ss = 2.5, 6.0
    m.set_sigma(sh, ss)
    mu = _prior_draw(m, prep, rng)
    ch.set_state(0, mu, (sh, ss))
    r = _check_point(ch, m, 0, mu)
    rm, rp = _check_leapfrog(ch, m, 0, mu, _momentum(m, rng), 0.01, 3)
    print(f"256x256x128: gradient rel {r:.2e}, leapfrog mu {rm:.2e} p {rp:.2e}")
    ch.close()
    data.close()
