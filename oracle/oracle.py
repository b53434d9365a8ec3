"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the dualres_b200 package.

Parity status: unpinned. The reference has no golden vectors and cannot be
compiled in this image (Eigen, FFTW3 and Boost are absent); the oracle is a
restatement cross-checked against tests/golden (numpy) and analytic tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    """Compile the oracle with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _declare(_lib)
    return _lib


_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _declare(L):
    L.orc_nonzero_indices.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _i32p, C.c_int]
    L.orc_nonzero_indices.restype = C.c_int
    L.orc_embedding_dims.argtypes = [_i32p, _i32p]
    L.orc_embedding_dims.restype = C.c_int
    L.orc_neighborhood.argtypes = [_f32p, C.c_float, _i32p, C.c_int]
    L.orc_neighborhood.restype = C.c_int
    L.orc_prepare_highres.argtypes = [_f32p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      _i32p, _f32p, _i32p, C.POINTER(C.c_int), C.c_int]
    L.orc_prepare_highres.restype = C.c_int
    L.orc_kriging_build.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, _f32p, C.c_int, C.c_int,
                                    C.c_int, _f32p, _f32p, C.c_float, C.c_int, _i32p, C.c_int, _i32p,
                                    _f64p, C.c_int64, C.POINTER(C.c_int)]
    L.orc_kriging_build.restype = C.c_int64
    L.orc_cov.argtypes = [C.c_int, C.c_double, _f64p]
    L.orc_cov.restype = C.c_double
    L.orc_mce_offsets.argtypes = [C.c_void_p, C.c_int]
    L.orc_mce_offsets.restype = C.c_int
    L.orc_mce_summary.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_mce_summary.restype = C.c_int
    for sfx, rp, rt in (("_d", _f64p, C.c_double), ("_f", _f32p, C.c_float)):
        g = lambda n: getattr(L, n + sfx)
        g("orc_fft3d").argtypes = [rp, _i32p, C.c_int]
        g("orc_model_create").argtypes = [C.c_int, _i32p, _f32p, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, _f32p, _f64p, C.c_int, C.c_int,
                                          _i32p, C.POINTER(C.c_int)]
        g("orc_model_create").restype = C.c_void_p
        g("orc_model_free").argtypes = [C.c_void_p]
        g("orc_model_info").argtypes = [C.c_void_p, _i32p, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
        g("orc_model_lambda").argtypes = [C.c_void_p, _f64p]
        g("orc_model_set_sigma").argtypes = [C.c_void_p, rt, rt]
        g("orc_model_get_sigma").argtypes = [C.c_void_p, rp]
        g("orc_model_set_mu").argtypes = [C.c_void_p, rp]
        g("orc_model_get_mu").argtypes = [C.c_void_p, rp]
        for n in ("orc_log_prior", "orc_log_likelihood", "orc_kinetic"):
            g(n).argtypes = [C.c_void_p, rp]
            g(n).restype = C.c_double
        g("orc_gradient").argtypes = [C.c_void_p, rp, rp]
        g("orc_leapfrog").argtypes = [C.c_void_p, rp, rp, rt, C.c_int]
        g("orc_transition").argtypes = [C.c_void_p, rp, C.c_double, rt, C.c_int, _f64p, _f64p]
        g("orc_transition").restype = C.c_double
        g("orc_momentum").argtypes = [C.c_void_p, rp, rp]
        g("orc_momentum").restype = C.c_double
        g("orc_fit").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                 _f64p, _f64p, _f64p, _f64p]
        g("orc_fit").restype = C.c_int
        g("orc_run_iterations").argtypes = [C.c_void_p, C.c_int, C.c_int, rt, C.c_uint64]
        g("orc_run_iterations").restype = C.c_int64
        g("orc_set_threads").argtypes = [C.c_int]


def _img(a):
    return np.ascontiguousarray(a, dtype=np.float32).ravel()


def fft3d(field, inverse=False, precision="d"):
    """Unnormalised 3D DFT of a complex field shaped (E2, E1, E0)."""
    dt = np.complex128 if precision == "d" else np.complex64
    a = np.ascontiguousarray(field, dtype=dt)
    E = np.array(a.shape[::-1], dtype=np.int32)
    buf = a.view(np.float64 if precision == "d" else np.float32).ravel().copy()
    getattr(lib(), "orc_fft3d_" + precision)(buf, E, 1 if inverse else 0)
    return buf.view(dt).reshape(a.shape)


def nonzero_indices(img):
    nz, ny, nx = img.shape
    out = np.zeros(3 * img.size, dtype=np.int32)
    n = lib().orc_nonzero_indices(_img(img), nx, ny, nz, out, img.size)
    return out[: 3 * n].reshape(n, 3)


def neighborhood(Q, radius):
    out = np.zeros(3 * 20000, dtype=np.int32)
    n = lib().orc_neighborhood(np.ascontiguousarray(Q, dtype=np.float32).ravel(), radius, out, 20000)
    if n < 0:
        raise RuntimeError(f"orc_neighborhood failed ({n})")
    return out[: 3 * n].reshape(n, 3)


def prepare(hr, hmask=None, omask=None):
    """Masking + bbox + data/output indices, as dualgpm.cpp + fit_model do."""
    nz, ny, nx = hr.shape
    h = _img(hr).copy()
    hm = None if hmask is None else _img(hmask)
    om = None if omask is None else _img(omask)
    D = np.zeros(3 * h.size, dtype=np.int32)
    O = np.zeros(3 * h.size, dtype=np.int32)
    Yh = np.zeros(h.size, dtype=np.float32)
    no = C.c_int(0)
    hm_p = hm.ctypes.data_as(C.c_void_p) if hm is not None else None
    om_p = om.ctypes.data_as(C.c_void_p) if om is not None else None
    nh = lib().orc_prepare_highres(h, hm_p, om_p, nx, ny, nz, D, Yh, O, C.byref(no), h.size)
    if nh < 0:
        raise RuntimeError(f"orc_prepare_highres failed ({nh})")
    return dict(D=D[: 3 * nh].reshape(nh, 3), Yh=Yh[:nh].copy(), O=O[: 3 * no.value].reshape(no.value, 3),
                masked=h.reshape(hr.shape))


def kriging(hr_masked, Qhr, sr, Qsr, theta, radius, solve=True, max_nnz=None):
    nz, ny, nx = hr_masked.shape
    sz, sy, sx = sr.shape
    nrows_cap = int(np.count_nonzero(~np.isnan(sr) & (sr != 0))) + 1
    if max_nnz is None:
        max_nnz = nrows_cap * len(neighborhood(Qhr, radius)) + 1
    rowptr = np.zeros(nrows_cap + 1, dtype=np.int32)
    col = np.zeros(max_nnz, dtype=np.int32)
    val = np.zeros(max_nnz, dtype=np.float64)
    nr = C.c_int(0)
    nnz = lib().orc_kriging_build(_img(hr_masked), nx, ny, nz, np.ascontiguousarray(Qhr, np.float32).ravel(),
                                  _img(sr), sx, sy, sz, np.ascontiguousarray(Qsr, np.float32).ravel(),
                                  np.asarray(theta, dtype=np.float32), float(radius), 1 if solve else 0,
                                  rowptr, nrows_cap, col, val, max_nnz, C.byref(nr))
    if nnz < 0:
        raise RuntimeError(f"orc_kriging_build failed ({nnz})")
    n = nr.value
    return rowptr[: n + 1].copy(), col[:nnz].copy(), val[:nnz].copy()


class Model:
    """Oracle MultiResParameters + MultiResData (precision 'd' or 'f')."""

    def __init__(self, D, Yh, Qhr, theta, Ys=None, W=None, O=None, covfun=0, precision="d"):
        self.p = precision
        self.rdt = np.float64 if precision == "d" else np.float32
        self.cdt = np.complex128 if precision == "d" else np.complex64
        L = lib()
        self._f = lambda n: getattr(L, n + "_" + precision)
        D = np.ascontiguousarray(D, dtype=np.int32).ravel()
        Yh = np.ascontiguousarray(Yh, dtype=np.float32)
        O = D if O is None else np.ascontiguousarray(O, dtype=np.int32).ravel()
        st = C.c_int(0)
        self._keep = []
        if W is not None:
            rowptr, col, val = W
            rowptr = np.ascontiguousarray(rowptr, np.int32)
            col = np.ascontiguousarray(col, np.int32)
            val = np.ascontiguousarray(val, self.rdt)
            Ys = np.ascontiguousarray(Ys, np.float32)
            self._keep += [rowptr, col, val, Ys]
            args = (len(Ys), Ys.ctypes.data_as(C.c_void_p), rowptr.ctypes.data_as(C.c_void_p),
                    col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p))
        else:
            args = (0, None, None, None, None)
        self.h = self._f("orc_model_create")(len(Yh), D, Yh, *args,
                                              np.ascontiguousarray(Qhr, np.float32).ravel(),
                                              np.asarray(theta, np.float64), covfun, len(O) // 3, O, C.byref(st))
        if not self.h:
            raise RuntimeError(f"orc_model_create failed ({st.value})")
        E = np.zeros(3, np.int32)
        N = C.c_int64(0)
        nS = C.c_int(0)
        self._f("orc_model_info")(self.h, E, C.byref(N), C.byref(nS))
        self.E = tuple(int(e) for e in E)
        self.N = int(N.value)
        self.n_S = int(nS.value)
        self.shape = (self.E[2], self.E[1], self.E[0])

    def __del__(self):
        if getattr(self, "h", None):
            self._f("orc_model_free")(self.h)
            self.h = None

    def _c(self, x):
        a = np.ascontiguousarray(x, dtype=self.cdt).reshape(self.shape)
        return a.view(self.rdt).ravel().copy()

    def _back(self, buf):
        return buf.view(self.cdt).reshape(self.shape)

    def lam(self):
        out = np.zeros(2 * self.N)
        self._f("orc_model_lambda")(self.h, out)
        return out.view(np.complex128).reshape(self.shape)

    def set_sigma(self, sh, ss):
        self._f("orc_model_set_sigma")(self.h, sh, ss)

    def log_prior(self, mu):
        return self._f("orc_log_prior")(self.h, self._c(mu))

    def log_likelihood(self, mu):
        return self._f("orc_log_likelihood")(self.h, self._c(mu))

    def gradient(self, mu):
        out = np.zeros(2 * self.N, self.rdt)
        self._f("orc_gradient")(self.h, self._c(mu), out)
        return self._back(out)

    def kinetic(self, p):
        return self._f("orc_kinetic")(self.h, self._c(p))

    def leapfrog(self, mu, p, eps, L):
        m = self._c(mu)
        q = self._c(p)
        self._f("orc_leapfrog")(self.h, m, q, eps, L)
        return self._back(m), self._back(q)

    def set_mu(self, mu):
        self._f("orc_model_set_mu")(self.h, self._c(mu))

    def get_mu(self):
        out = np.zeros(2 * self.N, self.rdt)
        self._f("orc_model_get_mu")(self.h, out)
        return self._back(out)

    def transition(self, z, u, eps, L):
        out = np.zeros(6)
        norms = np.zeros(2)
        r = self._f("orc_transition")(self.h, np.ascontiguousarray(z, self.rdt).ravel(), u, eps, L, out, norms)
        return r, out, norms

    def momentum(self, z):
        """p and E0 from injected normals z (2N reals), as transition() draws them."""
        out = np.zeros(2 * self.N, self.rdt)
        e0 = self._f("orc_momentum")(self.h, np.ascontiguousarray(z, self.rdt).ravel(), out)
        return self._back(out), e0

    def fit(self, burnin, n_save, thin, L, mh_target, seed, n_out):
        mean = np.zeros(n_out)
        var = np.zeros(n_out)
        act = np.zeros(n_out)
        stats = np.zeros(4)
        n = self._f("orc_fit")(self.h, burnin, n_save, thin, L, mh_target, seed, mean, var, act, stats)
        return dict(mean=mean, var=var, activation=act, mh_rate=stats[0], eps=stats[1],
                    grad_evals=stats[2], iterations=stats[3], samples=n)

    def run_iterations(self, iters, L, eps, seed):
        return int(self._f("orc_run_iterations")(self.h, iters, L, eps, seed))


def mce_offsets():
    """perturbation_matrix_3d offsets (n x 3, int32)."""
    n = lib().orc_mce_offsets(None, 0)
    P = np.zeros(3 * n, np.int32)
    lib().orc_mce_offsets(P.ctypes.data_as(C.c_void_p), n)
    return P.reshape(n, 3)


def mce_summary(img, Q, P=None):
    """compute_mce_summary_data: distance, covariance, npairs and the raw double sums per offset."""
    if P is None:
        P = mce_offsets()
    nz, ny, nx = img.shape
    n = len(P)
    dist = np.zeros(n, np.float32)
    cov = np.zeros(n, np.float32)
    npairs = np.zeros(n, np.int32)
    sums = np.zeros(3 * n)
    P = np.ascontiguousarray(P, np.int32)
    lib().orc_mce_summary(_img(img), nx, ny, nz, np.ascontiguousarray(Q, np.float32).ravel(),
                          P.ctypes.data_as(C.c_void_p), n, dist.ctypes.data_as(C.c_void_p),
                          cov.ctypes.data_as(C.c_void_p), npairs.ctypes.data_as(C.c_void_p),
                          sums.ctypes.data_as(C.c_void_p))
    return dict(distance=dist, covariance=cov, npairs=npairs, sums=sums.reshape(n, 3))


def set_threads(n):
    lib().orc_set_threads_d(n)
    lib().orc_set_threads_f(n)
