"""Generate the golden fixtures in tests/golden/*.npz.

An independent numpy (FP64) restatement of the reference's sampler math is
used for this, written separately from the C oracle. The CPU tests check the
oracle against these fixtures, and the GPU tests check the CUDA path against
both. The reference itself ships no golden vectors and cannot be compiled in
this image, so parity stays "unpinned" in the strict sense.

Sources restated (paths relative to the reference project root):
  include/dualres/impl/circulant_base.inl:30-89   circulant base
  include/dualres/MultiResParameters.h:173-300     lambda, S, data indices
  include/dualres/MultiResParameters.h:337-376     gradient
  include/dualres/MultiResParameters.h:429-514     log prior / likelihood
  include/dualres/MultiResParameters.h:551-603     kinetic term
  include/dualres/MultiResParameters.h:674-700     leapfrog
  include/dualres/kriging_matrix.h:41-343          kriging CSR
  src/dualgpm.cpp:125-155,288 + gaussian_process_model.h:104-117  masks/indices

Run:  python tests/golden/gen_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from dualres_b200 import synth  # noqa: E402


# ---------------------------------------------------------------- indices
def nonzero(img):
    return ~(np.isnan(img) | (img == 0))


def ijk_of(img, mask):
    z, y, x = np.nonzero(mask)
    order = np.argsort(x + img.shape[2] * (y + img.shape[1] * z), kind="stable")
    return np.stack([x[order], y[order], z[order]], axis=1).astype(np.int64)


def prepare(hr, hmask=None, omask=None):
    hr = hr.copy()
    hm = (hr if hmask is None else hmask).astype(np.float32).copy()
    om = (hr if omask is None else omask).astype(np.float32).copy()
    hr[(hm == 0) | np.isnan(hr)] = 0
    union = hm + om
    uz, uy, ux = np.nonzero(nonzero(union))
    bbmin = np.array([ux.min(), uy.min(), uz.min()])
    bbmax = np.array([ux.max(), uy.max(), uz.max()])
    ijk = ijk_of(hr, nonzero(hr))
    inbox = np.all((ijk >= bbmin) & (ijk <= bbmax), axis=1)
    D = ijk[inbox] - bbmin
    Yh = hr.ravel()[nonzero(hr).ravel()]
    oijk = ijk_of(om, nonzero(om))
    oin = np.all((oijk >= bbmin) & (oijk <= bbmax), axis=1)
    O = oijk[oin] - bbmin
    return hr, D, Yh.astype(np.float32), O


# ---------------------------------------------------------------- spectrum
def embedding(g):
    return synth.embedding_dims(g)


def covf(d, theta, covfun=0):
    v, b, e = theta
    if covfun == 0:
        return v * np.exp(-b * np.abs(d) ** e)
    return v * (1.0 + b / e * d * d) ** (-e)


def lam_of(E, Q, theta, covfun=0):
    o = []
    for n in E:
        t = np.arange(n)
        o.append(np.where(t <= n // 2, t, n - t).astype(np.float32))
    Z, Y, X = np.meshgrid(o[2], o[1], o[0], indexing="ij")
    Q3 = Q[:3, :3].astype(np.float32)
    q = [Q3[r, 0] * X + Q3[r, 1] * Y + Q3[r, 2] * Z for r in range(3)]
    d = np.sqrt((q[0] * q[0] + q[1] * q[1] + q[2] * q[2]).astype(np.float32)).astype(np.float64)
    return np.fft.fftn(covf(d, theta, covfun))


# ---------------------------------------------------------------- model
class NpModel:
    def __init__(self, D, Yh, Q, theta, Ys=None, W=None, O=None, covfun=0):
        g = D.max(axis=0) + 1
        self.E = embedding(tuple(int(v) for v in g))
        self.shape = (self.E[2], self.E[1], self.E[0])
        self.N = int(np.prod(self.E))
        self.lam = lam_of(self.E, Q, theta, covfun)
        self.S = self.lam.real <= 0
        self.Dflat = D[:, 2] * self.E[0] * self.E[1] + D[:, 1] * self.E[0] + D[:, 0]
        self.Yh = Yh.astype(np.float64)
        self.Ys = None if Ys is None else Ys.astype(np.float64)
        self.W = None
        if W is not None:
            rp, col, val = W
            Wd = np.zeros((len(rp) - 1, len(Yh)))
            for r in range(len(rp) - 1):
                Wd[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
            self.W = Wd
        self.sig = [1.0, 1.0]

    def ifft(self, x):
        return np.fft.ifftn(x) * self.N

    def log_prior(self, mu):
        u = self.ifft(mu)
        a = np.where(self.S, 0, np.conj(u) * u / np.where(self.S, 1, self.lam)).sum()
        return -0.5 * (a.real + a.imag) / self.N

    def _data(self, mu):
        m = mu.ravel()[self.Dflat].real
        rh = self.Yh - m
        rs = None if self.W is None else self.Ys - self.W @ m
        return m, rh, rs

    def log_likelihood(self, mu):
        _, rh, rs = self._data(mu)
        ll = self.sig[0] * (rh @ rh)
        if rs is not None:
            ll += self.sig[1] * (rs @ rs)
        return -0.5 * ll

    def gradient(self, mu):
        u = self.ifft(mu)
        t = np.where(self.S, 0, u / (-self.N * np.where(self.S, 1, self.lam)))
        g = np.fft.fftn(t)
        _, rh, rs = self._data(mu)
        sub = self.sig[0] * rh
        if rs is not None:
            sub = sub + self.sig[1] * (self.W.T @ rs)
        gf = g.ravel()
        gf[self.Dflat] += sub
        return gf.reshape(self.shape)

    def lam_mass(self):
        return np.where(self.S, 0, 1.0 / np.where(self.S, 1, self.lam) + self.sig[0])

    def kinetic(self, p):
        lm = self.lam_mass()
        u = self.ifft(p)
        a = np.where(lm != 0, np.conj(u) * u / np.where(lm != 0, lm, 1), 0).sum()
        return -0.5 * (a.real + a.imag) / self.N

    def leapfrog(self, mu, p, eps, L):
        lm = self.lam_mass()
        mu = mu.copy()
        p = p + 0.5 * eps * self.gradient(mu)
        for s in range(L):
            k = 0.5 if s == L - 1 else 1.0
            t = self.ifft(p)
            t = np.where(self.S, 0, t / (np.where(self.S, 1, lm) * (self.N / eps)))
            mu = mu + np.fft.fftn(t)
            p = p + k * eps * self.gradient(mu)
        return mu, p


# ---------------------------------------------------------------- kriging
def neighborhood(Q, radius):
    Q = Q.astype(np.float32)
    vd = np.sqrt((Q[:, :3] ** 2).sum(axis=0)).astype(np.float32)
    nr = (np.float32(radius) / vd).astype(np.int64)
    K, J, I = np.meshgrid(np.arange(-nr[2], nr[2] + 1), np.arange(-nr[1], nr[1] + 1),
                          np.arange(-nr[0], nr[0] + 1), indexing="ij")
    P = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1)
    q = (P.astype(np.float32) @ Q[:3, :3].T.astype(np.float32)).astype(np.float32)
    keep = np.sqrt((q * q).sum(axis=1)) <= np.float32(radius)
    return P[keep]


def kriging(hr, Qhr, sr, Qsr, theta, radius):
    P = neighborhood(Qhr, radius)
    Ph = P @ Qhr[:3, :3].astype(np.float64).T
    dd = np.sqrt(((Ph[:, None, :] - Ph[None, :, :]) ** 2).sum(-1))
    K = covf(dd, theta)
    np.fill_diagonal(K, 1.0)
    nz, ny, nx = hr.shape
    hz, hy, hx = np.nonzero(nonzero(hr))
    bbmin = np.array([hx.min(), hy.min(), hz.min()])
    bbmax = np.array([hx.max(), hy.max(), hz.max()])
    bd = bbmax - bbmin + 1
    sub = hr[bbmin[2]:bbmax[2] + 1, bbmin[1]:bbmax[1] + 1, bbmin[0]:bbmax[0] + 1]
    bmask = nonzero(sub).ravel()
    bmap = np.full(bmask.size, -1, dtype=np.int64)
    bmap[bmask] = np.arange(bmask.sum())
    mp = np.linalg.inv(Qhr.astype(np.float64)) @ Qsr.astype(np.float64)
    sijk = ijk_of(sr, nonzero(sr))
    rowptr = [0]
    cols, vals = [], []
    hrf = hr.ravel()
    for s in sijk:
        sv = np.array([s[0], s[1], s[2], 1.0])
        base = np.trunc((mp @ sv)[:3]).astype(np.int64)
        h = base[None, :] + P
        flat = h[:, 2] * ny * nx + h[:, 1] * nx + h[:, 0]
        ok = (flat >= 0) & (flat < hr.size)
        idx = np.nonzero(ok)[0]
        idx = idx[nonzero(hrf[flat[idx]])]
        rel = h[idx] - bbmin
        bhr = rel[:, 2] * bd[0] * bd[1] + rel[:, 1] * bd[0] + rel[:, 0]
        assert np.all((bhr >= 0) & (bhr < bmap.size))
        good = bmap[bhr] >= 0
        idx = idx[good]
        c = bmap[bhr[good]]
        if len(idx):
            sm = (Qsr.astype(np.float64) @ sv)[:3]
            hm = (Qhr.astype(np.float64) @ np.concatenate([h[idx], np.ones((len(idx), 1))], axis=1).T).T[:, :3]
            kp = covf(np.sqrt(((sm[None, :] - hm) ** 2).sum(1)) + 1e-5, theta)
            w = np.linalg.solve(K[np.ix_(idx, idx)], kp)
            ws = w.sum()
            if ws == 0:
                ws = 1.0
            if not np.isnan(ws):
                cols.append(c)
                vals.append(w / ws)
                rowptr.append(rowptr[-1] + len(c))
                continue
        rowptr.append(rowptr[-1])
    col = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
    val = np.concatenate(vals) if vals else np.zeros(0)
    return np.array(rowptr, np.int32), col, val


# ---------------------------------------------------------------- fixtures
def make_case(name, vol, seed, eps, L, covfun=0):
    rng = np.random.default_rng(seed)
    # the reference carries the covariance parameters as float (dualgpmf)
    vol.theta = tuple(float(np.float32(t)) for t in vol.theta)
    hr, D, Yh, O = prepare(vol.highres)
    W = kriging(hr, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
    Ys = vol.stdres.ravel()[nonzero(vol.stdres).ravel()].astype(np.float32)
    m = NpModel(D, Yh, vol.qform_hr, vol.theta, Ys, W, O, covfun)
    m.sig = [float(np.float32(1.7)), float(np.float32(4.3))]
    shp = m.shape
    # a prior-typical mu plus data, and a unit momentum draw
    w = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    mu = np.fft.fftn(np.where(m.S, 0, np.sqrt(np.abs(m.lam) / m.N)) * w)
    mu.ravel()[m.Dflat] += Yh
    mu = mu.astype(np.complex64).astype(np.complex128)
    p = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64).astype(np.complex128)
    muL, pL = m.leapfrog(mu, p, eps, L)
    return dict(
        name=name, highres=vol.highres, qform_hr=vol.qform_hr, stdres=vol.stdres, qform_sr=vol.qform_sr,
        theta=np.array(vol.theta), radius=np.float64(vol.radius), covfun=np.int32(covfun),
        D=D.astype(np.int32), Yh=Yh, O=O.astype(np.int32), Ys=Ys,
        W_rowptr=W[0], W_col=W[1], W_val=W[2], E=np.array(m.E, np.int32),
        lam=m.lam, n_S=np.int64(m.S.sum()), sigma=np.array(m.sig),
        mu=mu.astype(np.complex64), p=p.astype(np.complex64),
        log_prior=np.float64(m.log_prior(mu)), log_likelihood=np.float64(m.log_likelihood(mu)),
        grad=m.gradient(mu), kinetic=np.float64(m.kinetic(p)),
        eps=np.float64(eps), L=np.int32(L), mu_L=muL, p_L=pL,
        log_prior_L=np.float64(m.log_prior(muL)), log_likelihood_L=np.float64(m.log_likelihood(muL)),
        kinetic_L=np.float64(m.kinetic(pL)),
    )


def cases():
    v1 = synth.make_volume((8, 6, 5), 1.0, (0.8, 0.3, 1.0), 0.5, 0.3, 2.6, "ellipsoid", 0.75, 11, name="g1")
    # exponent 2 (Gaussian) on a coarse grid: the embedding has non-positive eigenvalues (S not empty)
    v2 = synth.make_volume((8, 7, 6), 1.0, (1.0, 0.05, 2.0), 0.6, 0.4, 2.3, "ellipsoid", 0.7, 12, name="g2")
    # anisotropic voxels
    v3 = synth.make_volume((7, 8, 6), 1.5, (0.9, 0.4, 1.5), 0.7, 0.35, 3.1, "smooth", 0.6, 13, name="g3")
    return [("g1_rbf_e1", v1, 21, 0.05, 6, 0), ("g2_rbf_e2_negative_modes", v2, 22, 0.02, 4, 0),
            ("g3_rbf_aniso", v3, 23, 0.04, 5, 0)]


def main():
    for name, vol, seed, eps, L, cf in cases():
        d = make_case(name, vol, seed, eps, L, cf)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **d)
        print(f"{path}: E={tuple(d['E'])} n_h={len(d['Yh'])} n_s={len(d['Ys'])} nnz={len(d['W_col'])} "
              f"n_S={int(d['n_S'])} lp={float(d['log_prior']):.6g} ll={float(d['log_likelihood']):.6g}")


if __name__ == "__main__":
    main()
