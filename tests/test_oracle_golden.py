"""The CPU oracle against the golden fixtures (independent numpy restatement)
and against analytic known-answer tests."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def test_fft_known_answers(oracle):
    rng = np.random.default_rng(0)
    x = rng.standard_normal((8, 16, 4)) + 1j * rng.standard_normal((8, 16, 4))
    f = oracle.fft3d(x, False)
    assert rel(f, np.fft.fftn(x)) < 1e-13
    b = oracle.fft3d(f, True)
    assert rel(b, x * x.size) < 1e-13              # IFFT(FFT(x)) = N x
    c = np.ones((4, 4, 4), complex)
    fc = oracle.fft3d(c)
    assert abs(fc[0, 0, 0] - 64) < 1e-12 and np.abs(fc.ravel()[1:]).max() < 1e-12
    k = np.zeros((4, 8, 16), complex)
    z, y, xg = np.meshgrid(np.arange(4), np.arange(8), np.arange(16), indexing="ij")
    k[:] = np.exp(2j * np.pi * (3 * xg / 16 + 1 * y / 8))   # single frequency -> one spike
    fk = oracle.fft3d(k)
    assert abs(fk[0, 1, 3] - k.size) < 1e-9
    assert rel(oracle.fft3d(x, False, "f"), np.fft.fftn(x)) < 1e-6


@pytest.mark.parametrize("shape", [(2, 4, 8), (32, 2, 1), (1, 128, 2), (256, 1, 4), (2, 2, 512), (64, 64, 64)])
def test_fft_radix_stages_against_numpy(oracle, shape):
    """Every power-of-two length (odd and even log2, so with and without the radix-2 stage) on every axis,
    lines fewer and more than the 16 the passes transform at once."""
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert rel(oracle.fft3d(x, False), np.fft.fftn(x)) < 1e-13
    assert rel(oracle.fft3d(x, True), np.fft.ifftn(x) * x.size) < 1e-13
    assert rel(oracle.fft3d(x, False, "f"), np.fft.fftn(x)) < 2e-6


def test_embedding_rule(oracle):
    E = np.zeros(3, np.int32)
    assert oracle.lib().orc_embedding_dims(np.array([32, 32, 32], np.int32), E) == 0
    assert tuple(E) == (64, 64, 64)
    oracle.lib().orc_embedding_dims(np.array([64, 64, 48], np.int32), E)
    assert tuple(E) == (128, 128, 128)   # 2*47 = 94 -> 128 (reference rule)
    oracle.lib().orc_embedding_dims(np.array([80, 80, 64], np.int32), E)
    assert tuple(E) == (256, 256, 128)
    assert oracle.lib().orc_embedding_dims(np.array([1, 5, 5], np.int32), E) == -1


def test_neighborhood_counts(oracle):
    I = np.eye(4, dtype=np.float32)
    assert len(oracle.neighborhood(I, 6.9)) == 1357
    Q15 = np.diag([1.5, 1.5, 1.5, 1.0]).astype(np.float32)
    assert len(oracle.neighborhood(Q15, 6.9)) == 437
    P = oracle.neighborhood(I, 1.0)
    # i fastest, then j, then k
    assert P.tolist() == [[0, 0, -1], [0, -1, 0], [-1, 0, 0], [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]


@pytest.mark.parametrize("name", golden_cases())
def test_prepare_and_kriging_sparsity(oracle, name):
    g = load(name)
    prep = oracle.prepare(g["highres"])
    assert np.array_equal(prep["D"], g["D"])
    assert np.array_equal(prep["O"], g["O"])
    assert np.array_equal(prep["Yh"], g["Yh"])
    rp, col, val = oracle.kriging(prep["masked"], g["qform_hr"], g["stdres"], g["qform_sr"],
                                  tuple(g["theta"]), float(g["radius"]))
    assert np.array_equal(rp, g["W_rowptr"])          # bit-exact sparsity
    assert np.array_equal(col, g["W_col"])
    # FP64 column-pivoted QR vs FP64 LU; the exponent-2 case is ill-conditioned (cond ~ 1e8)
    assert np.abs(val - g["W_val"]).max() < 1e-6


@pytest.mark.parametrize("name", golden_cases())
@pytest.mark.parametrize("prec", ["d", "f"])
def test_model_against_golden(oracle, name, prec):
    g = load(name)
    W = (g["W_rowptr"], g["W_col"], g["W_val"])
    m = oracle.Model(g["D"], g["Yh"], g["qform_hr"], tuple(g["theta"]), g["Ys"], W, g["O"], precision=prec)
    assert tuple(m.E) == tuple(g["E"])
    assert m.n_S == int(g["n_S"])
    sh, ss = g["sigma"]
    m.set_sigma(sh, ss)
    tol = 1e-8 if prec == "d" else 1e-4  # g2 amplifies rounding by 1/lambda_min
    lam = m.lam()
    assert rel(lam, g["lam"]) < (1e-12 if prec == "d" else 1e-5)
    mu, p = g["mu"].astype(np.complex128), g["p"].astype(np.complex128)
    well_posed = int(g["n_S"]) < 0.1 * mu.size
    if prec == "d" or well_posed:
        assert abs(m.log_prior(mu) / float(g["log_prior"]) - 1) < tol
    assert abs(m.log_likelihood(mu) / float(g["log_likelihood"]) - 1) < tol
    if prec == "d" or well_posed:
        assert rel(m.gradient(mu), g["grad"]) < tol
        assert abs(m.kinetic(p) / float(g["kinetic"]) - 1) < tol
    if prec == "d":
        muL, pL = m.leapfrog(mu, p, float(g["eps"]), int(g["L"]))
        assert rel(muL, g["mu_L"]) < 1e-9
        assert rel(pL, g["p_L"]) < 1e-9


def test_transition_identities(oracle):
    """eps -> 0 leaves H unchanged except for the reference's S-mode quirk:
    E0 = -1/2 sum |z|^2 runs over all N modes (MultiResParameters.h:787-799) while
    the final kinetic term skips lambda_mass == 0 (:558-572), so
    log R = 1/2 sum_{k in S} |w_k|^2 with w = IFFT(z)/sqrt(N)."""
    for name in ("g3_rbf_aniso", "g1_rbf_e1"):
        g = load(name)
        W = (g["W_rowptr"], g["W_col"], g["W_val"])
        m = oracle.Model(g["D"], g["Yh"], g["qform_hr"], tuple(g["theta"]), g["Ys"], W, g["O"])
        m.set_sigma(*g["sigma"])
        m.set_mu(g["mu"])
        z = np.random.default_rng(3).standard_normal(2 * m.N)
        r, out, norms = m.transition(z, 0.5, 1e-6, 3)
        zc = (z[0::2] + 1j * z[1::2]).reshape(m.shape)
        w = np.fft.ifftn(zc) * np.sqrt(zc.size)
        S = g["lam"].real <= 0
        expect = 0.5 * float((np.abs(w[S]) ** 2).sum())
        assert out[1] == 1.0
        assert abs(np.log(out[0]) - expect) < 1e-4 * max(1.0, expect)
        assert norms[0] > 0 and norms[1] > 0
