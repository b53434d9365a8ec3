"""GPU parity of the model variants against the FP64 oracle:

  * single-resolution mode (no std-res image: MultiResData.h:81-93 and the
    n_datasets == 1 branches of MultiResParameters.h:357-358, 488-514);
  * the rational-quadratic covariance (kernels.inl:59-74);
  * posterior moments of full fits against the oracle's own sampler, within
    Monte Carlo standard error.

Tolerances: eigenvalues rel 1e-10 (FP64 both sides); log prior, log
likelihood and kinetic energy rel 1e-5; gradient norm-wise rel 1e-5;
fixed-momentum leapfrog norm-wise rel 1e-4; posterior means within 4 combined
standard errors at 97 % of the output voxels.
"""
import numpy as np
import pytest

from test_gpu_parity import rel, update_path  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _pair(oracle, vol, covfun):
    """The product's volume and the oracle model built independently from the same images."""
    import dualres_b200 as d
    dv = d.MultiResData(vol.highres, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius,
                        hmask=vol.hmask, omask=vol.omask, covfun=covfun)
    prep = oracle.prepare(vol.highres, vol.hmask, vol.omask)
    if vol.stdres is not None:
        W = oracle.kriging(prep["masked"], vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
        s = vol.stdres.ravel()
        Ys = s[~(np.isnan(s) | (s == 0))]
    else:
        W, Ys = None, None
    # the C ABI takes the covariance parameters in float, as dualgpmf does
    theta32 = tuple(float(np.float32(t)) for t in vol.theta)
    m = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, theta32, Ys, W, prep["O"], covfun=covfun)
    return dv, m, prep


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    mu = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.3
    p = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 2.0
    return mu.astype(np.complex64), p.astype(np.complex64)


CASES = {
    "single_res_rbf": dict(dual=False, covfun=0, theta=(0.9, 0.35, 1.3)),
    "dual_res_rq": dict(dual=True, covfun=1, theta=(1.1, 0.4, 1.5)),
    "single_res_rq": dict(dual=False, covfun=1, theta=(0.8, 0.25, 1.0)),
    # scanner-like geometry: rotated qform, 1.8 x 1.8 x 2.3 mm voxels, qfac -1 (std-res at twice the size)
    "rotated_aniso_rbf": dict(dual=True, covfun=0, theta=(0.9, 0.3, 1.2), rotate=True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_variant_matches_oracle(oracle, case, update_path):  # noqa: F811
    import dualres_b200 as d
    from dualres_b200 import synth
    c = CASES[case]
    vol = synth.small_volume(seed=21, theta=c["theta"], dual=c["dual"])
    if c.get("rotate"):
        vol = synth.rotated(vol)
    dv, m, prep = _pair(oracle, vol, c["covfun"])
    assert tuple(dv.E) == m.E
    assert dv.n_stdres == (0 if not c["dual"] else dv.n_stdres) and dv.n_highres == len(prep["Yh"])
    assert dv.info.n_nonpositive == m.n_S
    assert rel(dv.lambda_re(), m.lam().real) < 1e-10
    mu, p = _fields(m.shape, 5)
    sh, ss = 1.7, 4.2
    m.set_sigma(sh, ss)
    ch = d.MultiResParameters(dv, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=3, seed=2), 1)
    ch.set_state(0, mu, (sh, ss))
    lp, ll = ch.log_prior_likelihood(0, mu)
    mu64, p64 = mu.astype(np.complex128), p.astype(np.complex128)
    assert abs(lp / m.log_prior(mu64) - 1) < 1e-5
    assert abs(ll / m.log_likelihood(mu64) - 1) < 1e-5
    tol_g = 1e-3 if m.n_S > 0.1 * m.N else 1e-5
    assert rel(ch.gradient(0, mu), m.gradient(mu64)) < tol_g
    eps, L = 0.05, 4
    muL, pL, en = ch.leapfrog(0, mu, p, eps, L)
    mo, po = m.leapfrog(mu64, p64, eps, L)
    tol = 1e-3 if m.n_S > 0.1 * m.N else 1e-4
    assert rel(muL, mo) < tol and rel(pL, po) < tol
    assert abs(en[2] / m.kinetic(p64) - 1) < 1e-5
    ch.close()
    dv.close()


def _chain_means(out_mean_per_chain):
    x = np.asarray(out_mean_per_chain, np.float64)
    return x.mean(axis=0), x.std(axis=0, ddof=1) / np.sqrt(x.shape[0])


@pytest.mark.parametrize("dual", [True, False])
def test_posterior_mean_within_mcse_of_oracle(oracle, dual):
    """Posterior means of independent GPU chains against independent FP64 oracle
    chains (its own sampler and RNG) on the same volume."""
    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.small_volume(seed=33, dual=dual)
    dv, m, prep = _pair(oracle, vol, 0)
    burnin, nsave, thin, L, n_chains = 150, 150, 1, 8, 16
    ch = d.MultiResParameters(dv, d.HMCParameters(burnin=burnin, nsave=nsave, thin=thin, leapfrog=L,
                                                  mhtarget=0.65, seed=17), n_chains)
    ch.run()
    gpu = [ch.summary(c)["mean"] for c in range(n_chains)]
    n_out = dv.n_output
    orc = []
    for s in range(8):
        r = m.fit(burnin, nsave, thin, L, 0.65, 1000 + s, n_out)
        orc.append(r["mean"])
    mg, sg = _chain_means(gpu)
    mo, so = _chain_means(orc)
    z = np.abs(mg - mo) / np.sqrt(sg ** 2 + so ** 2 + 1e-12)
    assert np.mean(z < 4.0) >= 0.97, (np.mean(z < 4.0), np.median(z))
    # the pooled summary is the mean of the per-chain means (equal sample counts)
    pooled = ch.summary(-1)["mean"]
    assert np.abs(pooled - mg).max() < 1e-4 * max(1.0, np.abs(mg).max())
    ch.close()
    dv.close()
