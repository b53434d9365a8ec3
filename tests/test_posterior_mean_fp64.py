"""Posterior means and variances of the FP32 sampler against the FP64 oracle on identical draws.

Two Markov chains with independent random streams agree on a posterior mean only within Monte Carlo
error (checked in test_gpu_modes.py). To measure what FP32 arithmetic does to the posterior moments,
both chains here consume the same randomness: per iteration the same 2N standard normals z (the
momentum draw of MultiResParameters.h:784-815, turned into p by the FP64 oracle) and the same accept
uniform u (MultiResParameters.h:680-705), at fixed sigma (the conditional posterior; the Gibbs step is
left out on both sides). The FP64 side is the oracle's transition (four FFTs per leapfrog step,
MultiResParameters.h:674-727). The FP32 side is the device: dr_leapfrog_fixed runs the trajectory
through the sampler's own kernels and returns the initial and final log prior, log likelihood and
kinetic energy, from which the same Metropolis ratio is formed. The running means and variances of
Re mu at the output voxels are compared at the end.

Bars: posterior mean rel 1e-4 and variance rel 1e-3 (norm-wise over output voxels) on the
well-conditioned fixtures and the 32^3 / 64^3-embedding volume; 1e-3 / 1e-2 on the fixture with
1940/4096 non-positive modes, where FP32 rounding is amplified by 1/lambda_min. The CPU test runs the
oracle's own FP32 build (the `dualgpmf` arithmetic) against its FP64 build on the same draws, which
shows the size of the error FP32 alone makes (about 3e-7 on the fixtures).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def _flat(ijk, E):
    ijk = np.asarray(ijk).reshape(-1, 3)
    return ijk[:, 2] * E[0] * E[1] + ijk[:, 1] * E[0] + ijk[:, 0]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class _Moments:
    def __init__(self, n):
        self.k, self.s, self.s2 = 0, np.zeros(n), np.zeros(n)

    def add(self, x):
        x = np.asarray(x, np.float64)
        self.k += 1
        self.s += x
        self.s2 += x * x

    def mean_var(self):
        m = self.s / self.k
        return m, self.s2 / self.k - m * m


def _drive(fp64, fp32_step, mu0, oi, eps, L, iters, seed):
    """Runs the FP64 oracle chain and an FP32 chain on the same draws.

    fp32_step(mu, p, u, E0z) -> (mu_next, accepted) advances the FP32 side."""
    rng = np.random.default_rng(seed)
    fp64.set_mu(mu0)
    mu = mu0.astype(np.complex64)
    a, b = _Moments(len(oi)), _Moments(len(oi))
    flips = acc = 0
    for _ in range(iters):
        z = rng.standard_normal(2 * fp64.N).astype(np.float32)
        u = float(rng.random())
        p, e0z = fp64.momentum(z)
        _, out, _ = fp64.transition(z, u, eps, L)
        mu, acc32 = fp32_step(mu, p, u, e0z, z)
        flips += int(bool(out[1]) != acc32)
        acc += int(out[1])
        a.add(fp64.get_mu().ravel()[oi].real)
        b.add(mu.ravel()[oi].real)
    return a.mean_var(), b.mean_var(), flips, acc / iters


CASES = {"g1_rbf_e1": (1e-4, 1e-3), "g3_rbf_aniso": (1e-4, 1e-3), "g2_rbf_e2_negative_modes": (1e-3, 1e-2)}


def _oracle_model(oracle, g, precision):
    W = (g["W_rowptr"], g["W_col"], g["W_val"])
    m = oracle.Model(g["D"], g["Yh"], g["qform_hr"], tuple(g["theta"]), g["Ys"], W, g["O"], precision=precision)
    m.set_sigma(*g["sigma"])
    return m


@pytest.mark.parametrize("name", ["g1_rbf_e1", "g3_rbf_aniso"])
def test_oracle_fp32_build_keeps_posterior_moments_of_fp64(oracle, name):
    g = _load(name)
    md, mf = _oracle_model(oracle, g, "d"), _oracle_model(oracle, g, "f")
    oi = _flat(g["O"], g["E"])
    mf.set_mu(g["mu"])

    def step(mu, p, u, e0z, z):
        _, out, _ = mf.transition(z, u, float(g["eps"]), int(g["L"]))
        return mf.get_mu(), bool(out[1])

    (m64, v64), (m32, v32), flips, rate = _drive(md, step, g["mu"], oi, float(g["eps"]), int(g["L"]), 200, 5)
    assert flips == 0 and rate > 0.3
    assert _rel(m32, m64) < 1e-5 and _rel(v32, v64) < 1e-4


def _device_step(chains, eps, L):
    def step(mu, p, u, e0z, z):
        muL, _, en = chains.leapfrog(0, mu, p.astype(np.complex64), eps, L)
        log_r = (en[3] + en[4] + en[5]) - (e0z + en[0] + en[1])   # proposed energy - E0, in FP64
        accept = bool(np.log(u) < log_r)                           # u < exp(log_r); NaN rejects
        return (muL if accept else mu), accept
    return step


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_posterior_moments_match_fp64_oracle_on_identical_draws(oracle, name):
    import dualres_b200 as d
    g = _load(name)
    vol = d.MultiResData(g["highres"], g["qform_hr"], g["stdres"], g["qform_sr"], tuple(g["theta"]),
                         float(g["radius"]))
    chains = d.MultiResParameters(vol, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=3, seed=1), 1)
    sh, ss = (float(x) for x in g["sigma"])
    chains.set_state(0, g["mu"], (sh, ss))
    md = _oracle_model(oracle, g, "d")
    eps, L = float(g["eps"]), int(g["L"])
    oi = _flat(g["O"], g["E"])
    (m64, v64), (m32, v32), flips, rate = _drive(md, _device_step(chains, eps, L), g["mu"], oi, eps, L, 200, 5)
    tol_m, tol_v = CASES[name]
    print(f"{name}: posterior mean rel {_rel(m32, m64):.2e}, variance rel {_rel(v32, v64):.2e}, accept {rate:.3f}")
    assert flips == 0 and rate > 0.3, (flips, rate)
    assert _rel(m32, m64) < tol_m, _rel(m32, m64)
    assert _rel(v32, v64) < tol_v, _rel(v32, v64)
    chains.close()
    vol.close()


@pytest.mark.gpu
def test_device_posterior_mean_on_the_32cubed_volume(oracle):
    """The 32^3 latent grid at 1 mm (64^3 embedding, RBF 0.806 / 0.132 / 1, kriging radius 6.9 mm, L = 25);
    both sides use the library's kriging matrix (its sparsity and weights are checked separately)."""
    import dualres_b200 as d
    from dualres_b200 import synth
    vol = synth.config_c1()
    data = d.MultiResData.from_volume(vol)
    chains = d.MultiResParameters(data, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=25, seed=1), 1)
    prep = oracle.prepare(vol.highres)
    rp, col, val = data.W()
    _, ys = data.data()
    md = oracle.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, (rp, col, val.astype(np.float64)),
                      prep["O"])
    sh, ss = 4.0, 11.0
    md.set_sigma(sh, ss)
    mu0 = np.zeros(md.shape, np.complex64)
    mu0.ravel()[_flat(prep["D"], md.E)] = prep["Yh"]
    chains.set_state(0, mu0, (sh, ss))
    oi = _flat(prep["O"], md.E)
    eps, L = 0.05, 25
    (m64, v64), (m32, v32), flips, rate = _drive(md, _device_step(chains, eps, L), mu0, oi, eps, L, 30, 1)
    print(f"32^3 volume: posterior mean rel {_rel(m32, m64):.2e}, variance rel {_rel(v32, v64):.2e}, accept {rate:.3f}")
    assert flips == 0 and rate > 0.3, (flips, rate)
    assert _rel(m32, m64) < 1e-4, _rel(m32, m64)
    assert _rel(v32, v64) < 1e-3, _rel(v32, v64)
    chains.close()
    data.close()
