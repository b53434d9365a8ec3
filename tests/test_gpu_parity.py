"""GPU parity of the CUDA path against the FP64 oracle and the golden fixtures.

dr_log_posterior and dr_gradient run step 0 of the sampler's own leapfrog
sequence (kriging products, inverse z pass, plane or x-line kernel), so these
bars apply to the kernels the sampler runs, on each of its update paths.

Tolerances (stated per check):
  * eigenvalues: FP64 on both sides, rel 1e-10;
  * log prior / log likelihood at identical inputs: rel 1e-5 (the accuracy bar for this path);
  * gradient: norm-wise rel 1e-5 on well-conditioned spectra; on the fixture
    with 1940/4096 non-positive modes (g2) the bar is 1e-3, because FP32
    rounding of u = IFFT(mu) is amplified by 1/lambda_min.  There the
    reference's own FP32 arithmetic (the oracle's FP32 build: four FP32 FFTs
    and an FP32 spectrum) is off by 0.22 on the same input, and the device
    must stay at least 100x closer to FP64 than that;
  * fixed-momentum leapfrog: norm-wise rel 1e-4 (the trajectory bar for this path);
  * kriging sparsity: bit-exact; weights abs 1e-6.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases

pytestmark = pytest.mark.gpu


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(params=["plane", "prefetch", "lines"])
def update_path(request, monkeypatch):
    """The three device update paths: the fused xy-plane kernel (E0 == E1 <= 128,
    the default), the same kernel with bulk-copy prefetch of the state planes,
    and the x-line kernel with separate y passes (every other embedding)."""
    monkeypatch.delenv("DRB_NO_PLANE", raising=False)
    monkeypatch.delenv("DRB_PLANE_PREFETCH", raising=False)
    monkeypatch.setenv("DRB_AUTOTUNE", "0")  # the path under test, not the tuner's choice
    if request.param == "lines":
        monkeypatch.setenv("DRB_NO_PLANE", "1")
    elif request.param == "prefetch":
        monkeypatch.setenv("DRB_PLANE_PREFETCH", "1")
    return request.param


def volume_of(g):
    import dualres_b200 as d
    return d.MultiResData(g["highres"], g["qform_hr"], g["stdres"], g["qform_sr"], tuple(g["theta"]),
                          float(g["radius"]))


def chains_of(vol, n=1, **kw):
    import dualres_b200 as d
    hmc = d.HMCParameters(burnin=kw.pop("burnin", 10), nsave=kw.pop("nsave", 10), thin=kw.pop("thin", 1),
                          leapfrog=kw.pop("leapfrog", 5), seed=kw.pop("seed", 3), **kw)
    return d.MultiResParameters(vol, hmc, n)


def oracle_model(oracle, g, precision="d"):
    W = (g["W_rowptr"], g["W_col"], g["W_val"])
    m = oracle.Model(g["D"], g["Yh"], g["qform_hr"], tuple(g["theta"]), g["Ys"], W, g["O"], precision=precision)
    m.set_sigma(*g["sigma"])
    return m


@pytest.mark.parametrize("name", golden_cases())
def test_volume_setup(name):
    g = load(name)
    v = volume_of(g)
    assert tuple(v.E) == tuple(int(e) for e in g["E"])
    assert v.info.n_nonpositive == int(g["n_S"])
    lam = v.lambda_re()
    assert rel(lam, g["lam"].real) < 1e-10
    d_idx, o_idx = v.indices()
    E = g["E"]
    D = g["D"]
    assert np.array_equal(d_idx, D[:, 2] * E[0] * E[1] + D[:, 1] * E[0] + D[:, 0])
    rp, col, val = v.W()
    assert np.array_equal(rp, g["W_rowptr"]) and np.array_equal(col, g["W_col"])
    assert np.abs(val - g["W_val"]).max() < 1e-6
    yh, ys = v.data()
    assert np.array_equal(yh, g["Yh"]) and np.array_equal(ys, g["Ys"])


@pytest.mark.parametrize("name", golden_cases())
def test_log_posterior_and_gradient(oracle, name, update_path):
    g = load(name)
    v = volume_of(g)
    p = chains_of(v)
    sh, ss = g["sigma"]
    mu = g["mu"]
    p.set_state(0, mu, (sh, ss))
    lp, ll = p.log_prior_likelihood(0, mu)
    assert abs(lp / float(g["log_prior"]) - 1) < 1e-5
    assert abs(ll / float(g["log_likelihood"]) - 1) < 1e-5
    grad = p.gradient(0, mu)
    ill = int(g["n_S"]) > 0.1 * mu.size
    tol = 1e-3 if ill else 1e-5
    r = rel(grad, g["grad"])
    assert r < tol, r
    # the oracle (FP64) agrees with the fixture
    m = oracle_model(oracle, g)
    assert abs(m.log_prior(mu) / lp - 1) < 1e-5
    if ill:
        # the reference's FP32 arithmetic on the same input, for scale
        r32 = rel(oracle_model(oracle, g, "f").gradient(mu), g["grad"])
        print(f"{name}: device gradient rel {r:.2e}, reference FP32 arithmetic rel {r32:.2e}")
        assert r < 0.01 * r32, (r, r32)


@pytest.mark.parametrize("name", golden_cases())
def test_fixed_momentum_leapfrog(oracle, name, update_path):
    g = load(name)
    v = volume_of(g)
    p = chains_of(v)
    sh, ss = g["sigma"]
    p.set_state(0, g["mu"], (sh, ss))
    eps, L = float(g["eps"]), int(g["L"])
    muL, pL, en = p.leapfrog(0, g["mu"], g["p"], eps, L)
    tol = 1e-3 if int(g["n_S"]) > 0.1 * g["mu"].size else 1e-4
    assert rel(muL, g["mu_L"]) < tol
    assert rel(pL, g["p_L"]) < tol
    assert abs(en[0] / float(g["log_prior"]) - 1) < 1e-5
    assert abs(en[1] / float(g["log_likelihood"]) - 1) < 1e-5
    assert abs(en[2] / float(g["kinetic"]) - 1) < 1e-5
    assert abs(en[3] / float(g["log_prior_L"]) - 1) < 10 * tol
    assert abs(en[4] / float(g["log_likelihood_L"]) - 1) < 10 * tol
    assert abs(en[5] / float(g["kinetic_L"]) - 1) < 10 * tol
    # and against the oracle directly at FP64
    m = oracle_model(oracle, g)
    mo, po = m.leapfrog(g["mu"].astype(np.complex128), g["p"].astype(np.complex128), eps, L)
    assert rel(muL, mo) < tol


def test_dual_averaging_matches_oracle(oracle):
    import dualres_b200 as d
    rng = np.random.default_rng(0)
    for (burnin, L) in [(40, 7), (0, 3), (25, 1)]:
        rates = rng.uniform(0, 1, 80).astype(np.float32)
        rates[:3] = [0.9, 0.95, 0.2]
        eps, steps = d.debug_dual_averaging(burnin, 20, 2, L, 1.0 / L, 0.65, rates)
        h = oracle.lib()
        import ctypes
        st = oracle_hmc = None
        hs = _OracleHmc(oracle, burnin, 20, 2, L, float(np.float32(1.0 / L)), 0.65)
        for i, r in enumerate(rates):
            hs.update(float(r))
            assert abs(hs.eps() - eps[i]) <= 1e-12 * max(1.0, abs(eps[i])), (burnin, i)
            assert hs.steps() == steps[i]


class _OracleHmc:
    def __init__(self, oracle, burnin, nsave, thin, L, eps0, target):
        import ctypes as C

        class H(C.Structure):
            _fields_ = [(n, C.c_int) for n in ("warmup", "eps_start_found", "burnin", "integrator_steps",
                                               "iteration", "n_save", "thin")] + \
                       [(n, C.c_double) for n in ("A", "eps", "eps0", "eps_bar", "eps_target", "gamma", "h_bar",
                                                  "mh_running_sum", "mh_target", "t0", "kappa")]
        self.C = C
        self.h = H()
        self.L = oracle.lib()
        self.L.orc_hmc_init.argtypes = [C.POINTER(H), C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        self.L.orc_hmc_update.argtypes = [C.POINTER(H), C.c_double]
        self.L.orc_hmc_integrator_steps.argtypes = [C.POINTER(H)]
        assert self.L.orc_hmc_init(C.byref(self.h), burnin, nsave, thin, L, eps0, target) == 0

    def update(self, r):
        self.L.orc_hmc_update(self.C.byref(self.h), r)

    def eps(self):
        return self.h.eps

    def steps(self):
        return self.L.orc_hmc_integrator_steps(self.C.byref(self.h))


def test_sampler_runs_and_counts(update_path):
    import dualres_b200 as d
    g = load("g1_rbf_e1")
    v = volume_of(g)
    p = chains_of(v, 3, burnin=12, nsave=6, thin=2, leapfrog=6)
    p.run()
    st = p.stats()
    for s in st:
        assert s["iteration"] == 12 + 2 * 6
        assert s["saved"] == 6 and s["done"] == 1
        assert 0 < s["grad_evals"] <= 24 * 7
        assert np.isfinite(s["sigma_hr"]) and np.isfinite(s["sigma_sr"])
        assert 0.0 <= s["mh_rate"] <= 1.0
    summ = p.summary(-1)
    assert summ["mean"].shape == (v.n_output,)
    assert np.all(np.isfinite(summ["mean"])) and np.all(summ["var"] >= -1e-6)


def test_chain_is_independent_of_batch(update_path):
    """Chain 0 of a 4-chain set follows the same trajectory as a 1-chain set
    with the same seed (RNG keyed by (seed, chain, iteration), never by slot)."""
    import dualres_b200 as d
    g = load("g3_rbf_aniso")
    v = volume_of(g)
    p1 = chains_of(v, 1, burnin=6, nsave=4, thin=1, leapfrog=4, seed=11)
    p4 = chains_of(v, 4, burnin=6, nsave=4, thin=1, leapfrog=4, seed=11)
    p1.update(3)
    p4.update(3)
    a, sa = p1.get_state(0)
    b, sb = p4.get_state(0)
    assert rel(b, a) < 1e-4
    assert abs(sa[0] / sb[0] - 1) < 1e-4


def test_evaluation_leaves_the_chain_state_unchanged(update_path):
    """dr_gradient and dr_log_posterior run the sampler's step 0 in the proposal half of the chain's buffers: the
    accepted state, sigma and the next iterations are those of a chain set that was never evaluated."""
    import dualres_b200 as d
    g = load("g1_rbf_e1")
    v = volume_of(g)
    a = chains_of(v, 2, burnin=4, nsave=4, thin=1, leapfrog=4, seed=17)
    b = chains_of(v, 2, burnin=4, nsave=4, thin=1, leapfrog=4, seed=17)
    a.update(2)
    b.update(2)
    other = (g["mu"] * 0.7).astype(np.complex64)
    for c in (0, 1):
        a.gradient(c, other)
        a.log_prior_likelihood(c, other)
    for c in (0, 1):
        (ma, sa), (mb, sb) = a.get_state(c), b.get_state(c)
        assert np.array_equal(ma, mb) and np.array_equal(sa, sb)
    a.update(3)
    b.update(3)
    for c in (0, 1):
        (ma, _), (mb, _) = a.get_state(c), b.get_state(c)
        assert np.array_equal(ma, mb)
    assert [s["iteration"] for s in a.stats()] == [s["iteration"] for s in b.stats()]
