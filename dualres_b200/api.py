"""Python mirror of the sampler's C ABI (include/dualres_b200.h).

The class names follow the reference's C++ API so that calling code reads
like the reference (include/dualres/*.h):

* ``MultiResData``        -> a device volume (images, masks, kriging matrix, spectrum)
* ``HMCParameters``       -> the sampler options (burnin, nsave, thin, leapfrog, mhtarget, seed)
* ``MultiResParameters``  -> a set of chains on one volume (state, energies, gradient, update)
* ``fit_model``           -> the fit loop, returning an ``mcmc_summary``

Errors raise ``DrError`` with the library's code and message, the way the
reference throws std::domain_error / std::logic_error.  The library is CUDA
only: loading works without a GPU (for the host-side kriging builder), but
every device call needs one and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

DR_OK = 0
DR_ERR_INVALID = -1
DR_ERR_CUDA = -2
DR_ERR_NOMEM = -3
DR_ERR_DOMAIN = -4
DR_ERR_UNSUPPORTED = -5
DR_ERR_STATE = -6
DR_ERR_TIMEOUT = -7
DR_COV_RBF = 0
DR_COV_RQ = 1

_ERR_NAMES = {DR_ERR_INVALID: "INVALID", DR_ERR_CUDA: "CUDA", DR_ERR_NOMEM: "NOMEM", DR_ERR_DOMAIN: "DOMAIN",
              DR_ERR_UNSUPPORTED: "UNSUPPORTED", DR_ERR_STATE: "STATE", DR_ERR_TIMEOUT: "TIMEOUT"}


class DrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{_ERR_NAMES.get(code, code)}] {msg}")
        self.code = code


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


class VolumeDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("highres", _fp), ("qform_hr", _fp),
                ("hmask", _fp), ("omask", _fp), ("sx", C.c_int), ("sy", C.c_int), ("sz", C.c_int),
                ("stdres", _fp), ("qform_sr", _fp), ("smask", _fp), ("covariance", C.c_float * 3),
                ("covfun", C.c_int), ("neighborhood", C.c_float), ("device", C.c_int)]


class VolumeInfo(C.Structure):
    _fields_ = [("E", C.c_int * 3), ("N", C.c_int64), ("box", C.c_int * 3), ("n_highres", C.c_int),
                ("n_stdres", C.c_int), ("n_output", C.c_int), ("kriging_nnz", C.c_int64),
                ("n_nonpositive", C.c_int), ("max_eigenvalue", C.c_double), ("setup_seconds", C.c_double),
                ("kriging_seconds", C.c_double), ("neighborhood", C.c_float), ("device_bytes", C.c_int64),
                ("kriging_plan_seconds", C.c_double), ("kriging_solve_seconds", C.c_double),
                ("kriging_device_rows", C.c_int), ("kriging_host_rows", C.c_int)]


class HmcOpts(C.Structure):
    _fields_ = [("burnin", C.c_int), ("nsave", C.c_int), ("thin", C.c_int), ("leapfrog", C.c_int),
                ("mhtarget", C.c_float), ("starting_eps", C.c_float), ("seed", C.c_uint64),
                ("store_samples", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_int64), ("max_active", C.c_int),
                ("iterations_per_round", C.c_int), ("host_threads", C.c_int), ("max_chains_in_flight", C.c_int)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int), ("error", C.c_int), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("finish_s", C.c_double), ("grad_evals", C.c_int64), ("mh_rate", C.c_float),
                ("n_output", C.c_int), ("device_bytes", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("done", C.c_int64), ("failed", C.c_int64), ("running", C.c_int64),
                ("grad_evals", C.c_int64), ("peak_device_bytes", C.c_int64), ("peak_running", C.c_int),
                ("busy_s", C.c_double), ("kernel_launches", C.c_int64)]


JOB_QUEUED, JOB_READY, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_PREEMPTED = range(6)


class ChainStats(C.Structure):
    _fields_ = [("iteration", C.c_int), ("saved", C.c_int), ("integrator_steps", C.c_int), ("eps", C.c_float),
                ("mh_rate", C.c_float), ("sigma_hr", C.c_float), ("sigma_sr", C.c_float),
                ("last_log_ratio", C.c_double), ("accepted", C.c_int64), ("grad_evals", C.c_int64),
                ("done", C.c_int), ("last_eps", C.c_float), ("initial_energy", C.c_double),
                ("proposed_energy", C.c_double)]


_lib = None


def lib_path():
    """The library this process loads: the bounds-checked build when DRB_LIBRARY=checked, else the release build."""
    return _build.LIB_CHECKED if os.environ.get("DRB_LIBRARY") == "checked" else _build.LIB


def lib(build_if_missing=True):
    """Load the in-tree shared library (building it if it is missing or stale)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if build_if_missing:
            _build.build(checked=path == _build.LIB_CHECKED)
        if not os.path.exists(path):
            raise DrError(DR_ERR_STATE, f"CUDA library not built: {path}")
        L = C.CDLL(path)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    vp = C.c_void_p
    L.dr_last_error.restype = C.c_char_p
    L.dr_version.restype = C.c_char_p
    L.dr_kernel_launches.argtypes = [C.c_int]
    L.dr_kernel_launches.restype = C.c_int64
    L.dr_volume_create.argtypes = [C.POINTER(VolumeDesc), C.POINTER(vp)]
    L.dr_volume_info_get.argtypes = [vp, C.POINTER(VolumeInfo)]
    L.dr_volume_kriging_get.argtypes = [vp, vp, vp, vp]
    L.dr_volume_lambda_get.argtypes = [vp, vp]
    L.dr_volume_indices_get.argtypes = [vp, vp, vp]
    L.dr_volume_data_get.argtypes = [vp, vp, vp]
    L.dr_volume_destroy.argtypes = [vp]
    L.dr_volume_destroy.restype = None
    L.dr_chainset_create.argtypes = [vp, C.c_int, C.POINTER(HmcOpts), C.POINTER(vp)]
    L.dr_chainset_config_get.argtypes = [vp, _ip, _ip, _dp, _ip]
    L.dr_chainset_ztile_get.argtypes = [vp, _ip]
    L.dr_chainset_fft_plan_get.argtypes = [vp, _ip]
    L.dr_chainset_checkpoint_size.argtypes = [vp, C.POINTER(C.c_int64)]
    L.dr_chainset_checkpoint_save.argtypes = [vp, vp, C.c_int64]
    L.dr_chainset_checkpoint_restore.argtypes = [vp, vp, C.c_int64]
    L.dr_chainset_destroy.argtypes = [vp]
    L.dr_chainset_destroy.restype = None
    L.dr_step.argtypes = [vp, C.c_int]
    L.dr_step_timed.argtypes = [vp, C.c_int, vp]
    L.dr_run.argtypes = [vp]
    L.dr_chain_stats_get.argtypes = [vp, vp]
    L.dr_summary_get.argtypes = [vp, C.c_int, vp, vp, vp]
    L.dr_samples_get.argtypes = [vp, C.c_int, vp, C.c_int, _ip]
    L.dr_set_state.argtypes = [vp, C.c_int, vp, C.c_float, C.c_float]
    L.dr_get_state.argtypes = [vp, C.c_int, vp, vp]
    L.dr_log_posterior.argtypes = [vp, C.c_int, vp, vp]
    L.dr_gradient.argtypes = [vp, C.c_int, vp, vp]
    L.dr_leapfrog_fixed.argtypes = [vp, C.c_int, vp, vp, C.c_float, C.c_int, vp, vp, vp]
    L.dr_kriging_matrix.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int, vp, vp,
                                    C.c_float, _ip, C.POINTER(C.c_int64), C.POINTER(_ip), C.POINTER(_ip),
                                    C.POINTER(_fp)]
    L.dr_debug_time_kernel.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp]
    L.dr_debug_tc_layout.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, vp, vp]
    L.dr_debug_bounded_wait.argtypes = [C.c_int, C.c_double, _ip, _dp]
    L.dr_server_preempt.argtypes = [vp, C.c_uint64, C.c_double]
    L.dr_server_resume.argtypes = [vp, C.c_uint64]
    L.dr_debug_pool_usage.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.dr_log_posterior_noalloc.argtypes = [vp, vp, C.c_float, C.c_float, vp]
    L.dr_free.argtypes = [vp]
    L.dr_free.restype = None
    L.dr_mce_offsets.argtypes = [vp, C.c_int, _ip]
    L.dr_mce_summary.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp, vp]
    L.dr_fit_rbf_parameters.argtypes = [vp, vp, vp, C.c_int, vp]
    L.dr_estimate_covariance.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp]
    L.dr_sample_records_get.argtypes = [vp, C.c_int, vp, C.c_int, _ip]
    L.dr_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(vp)]
    L.dr_server_submit.argtypes = [vp, C.POINTER(VolumeDesc), C.POINTER(HmcOpts), C.c_int, C.POINTER(C.c_uint64)]
    L.dr_server_status.argtypes = [vp, C.c_uint64, C.POINTER(JobStatus)]
    L.dr_server_result.argtypes = [vp, C.c_uint64, vp, vp, vp]
    L.dr_server_wait.argtypes = [vp, C.c_uint64, C.c_double]
    L.dr_server_drain.argtypes = [vp, C.c_double]
    L.dr_server_stats_get.argtypes = [vp, C.POINTER(ServerStats)]
    L.dr_server_forget.argtypes = [vp, C.c_uint64]
    L.dr_server_destroy.argtypes = [vp]
    L.dr_server_destroy.restype = None
    L.dr_debug_dual_averaging.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, vp,
                                          vp, vp, C.c_int]


def check(rc):
    if rc != DR_OK:
        msg = lib().dr_last_error()
        raise DrError(rc, msg.decode() if msg else "")
    return rc


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def kriging_matrix(highres, qform_hr, stdres, qform_sr, covariance, neighborhood):
    """Host-side get_sparse_kriging_matrix_data (kriging_matrix.h:148-343); highres must be masked."""
    L = lib()
    hr, sr = _f32(highres), _f32(stdres)
    nz, ny, nx = hr.shape
    sz, sy, sx = sr.shape
    qh, qs = _f32(qform_hr), _f32(qform_sr)
    th = _f32(covariance)
    nrows = C.c_int(0)
    nnz = C.c_int64(0)
    rp, cl, vl = _ip(), _ip(), _fp()
    check(L.dr_kriging_matrix(_ptr(hr), nx, ny, nz, _ptr(qh), _ptr(sr), sx, sy, sz, _ptr(qs), _ptr(th),
                              float(neighborhood), C.byref(nrows), C.byref(nnz), C.byref(rp), C.byref(cl),
                              C.byref(vl)))
    try:
        n, z = nrows.value, nnz.value
        rowptr = np.ctypeslib.as_array(rp, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(cl, shape=(max(z, 1),))[:z].copy()
        val = np.ctypeslib.as_array(vl, shape=(max(z, 1),))[:z].copy()
    finally:
        L.dr_free(rp)
        L.dr_free(cl)
        L.dr_free(vl)
    return rowptr, col, val


def _volume_desc(keep, highres, qform_hr, stdres, qform_sr, covariance, neighborhood, hmask, omask, smask,
                 covfun, device):
    """A dr_volume_desc over float32 copies of the images (kept alive in ``keep``)."""
    hr = _f32(highres)
    nz, ny, nx = hr.shape
    d = VolumeDesc()
    d.nx, d.ny, d.nz = nx, ny, nz

    def fp(a):
        if a is None:
            return None
        a = _f32(a)
        keep.append(a)
        return a.ctypes.data_as(_fp)

    d.highres = fp(hr)
    d.qform_hr = fp(qform_hr)
    d.hmask = fp(hmask)
    d.omask = fp(omask)
    if stdres is not None:
        sr = _f32(stdres)
        d.sz, d.sy, d.sx = sr.shape
        d.stdres = fp(sr)
        d.qform_sr = fp(qform_sr)
        d.smask = fp(smask)
    for i in range(3):
        d.covariance[i] = float(covariance[i])
    d.covfun = covfun
    d.neighborhood = float(neighborhood)
    d.device = device
    return d


class MultiResData:
    """A volume on the GPU: the inputs of MultiResData<T> (MultiResData.h:96-127) plus
    the one-time part of the MultiResParameters<T> constructor."""

    def __init__(self, highres, qform_hr, stdres=None, qform_sr=None, covariance=(1.0, 0.6, 1.5),
                 neighborhood=-1.0, hmask=None, omask=None, smask=None, covfun=DR_COV_RBF, device=0):
        L = lib()
        self._keep = []
        d = _volume_desc(self._keep, highres, qform_hr, stdres, qform_sr, covariance, neighborhood, hmask, omask,
                         smask, covfun, device)
        h = C.c_void_p()
        check(L.dr_volume_create(C.byref(d), C.byref(h)))
        self._keep = []
        self.h = h
        info = VolumeInfo()
        check(L.dr_volume_info_get(self.h, C.byref(info)))
        self.info = info
        self.E = tuple(info.E)
        self.N = int(info.N)
        self.shape = (self.E[2], self.E[1], self.E[0])
        self.n_highres = info.n_highres
        self.n_stdres = info.n_stdres
        self.n_output = info.n_output

    @classmethod
    def from_volume(cls, vol, device=0, **kw):
        """Build from a ``dualres_b200.synth.Volume``."""
        return cls(vol.highres, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius,
                   hmask=vol.hmask, omask=vol.omask, device=device, **kw)

    def close(self):
        if getattr(self, "h", None):
            lib().dr_volume_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def W(self):
        """Kriging matrix as (rowptr, col, val)."""
        rp = np.zeros(self.n_stdres + 1, np.int32)
        z = int(self.info.kriging_nnz)
        col = np.zeros(max(z, 1), np.int32)
        val = np.zeros(max(z, 1), np.float32)
        check(lib().dr_volume_kriging_get(self.h, _ptr(rp), _ptr(col), _ptr(val)))
        return rp, col[:z], val[:z]

    def lambda_re(self):
        out = np.zeros(self.N, np.float64)
        check(lib().dr_volume_lambda_get(self.h, _ptr(out)))
        return out.reshape(self.shape)

    def indices(self):
        d = np.zeros(self.n_highres, np.int32)
        o = np.zeros(max(self.n_output, 1), np.int32)
        check(lib().dr_volume_indices_get(self.h, _ptr(d), _ptr(o)))
        return d, o[: self.n_output]

    def data(self):
        yh = np.zeros(self.n_highres, np.float32)
        ys = np.zeros(max(self.n_stdres, 1), np.float32)
        check(lib().dr_volume_data_get(self.h, _ptr(yh), _ptr(ys)))
        return yh, ys[: self.n_stdres]


@dataclass
class HMCParameters:
    """HMCParameters<T>(burnin, n_save, thin, integrator_steps, starting_eps, mh_target)
    (HMCParameters.h:97-149) plus --seed; defaults of GPMCommandParser.inl:210-226."""

    burnin: int = 1000
    nsave: int = 1000
    thin: int = 3
    leapfrog: int = 25
    mhtarget: float = 0.65
    starting_eps: float = -1.0
    seed: int = 1
    store_samples: bool = False

    def c(self):
        o = HmcOpts()
        o.burnin, o.nsave, o.thin, o.leapfrog = self.burnin, self.nsave, self.thin, self.leapfrog
        o.mhtarget, o.starting_eps, o.seed = self.mhtarget, self.starting_eps, self.seed
        o.store_samples = 1 if self.store_samples else 0
        return o


class MultiResParameters:
    """n independent chains on one volume (MultiResParameters<float> x n)."""

    def __init__(self, data: MultiResData, hmc: HMCParameters, n_chains=1):
        self.data = data
        self.hmc = hmc
        self.n_chains = n_chains
        h = C.c_void_p()
        o = hmc.c()
        check(lib().dr_chainset_create(data.h, n_chains, C.byref(o), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().dr_chainset_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _field(self, x):
        a = np.ascontiguousarray(x, dtype=np.complex64).reshape(self.data.shape)
        return a

    PATHS = ("plane", "plane+prefetch", "lines")

    def config(self):
        """The chain set's update path, kriging-product blocks per SM, tuned iteration time (ms, 0 if untuned),
        whether the kriging products run on the tensor cores, the z passes' tile shape and the radix plan of the z
        (and x-line) transforms."""
        p, g, ms, tc = C.c_int(0), C.c_int(0), C.c_double(0), C.c_int(0)
        check(lib().dr_chainset_config_get(self.h, C.byref(p), C.byref(g), C.byref(ms), C.byref(tc)))
        zt, fp = C.c_int(0), C.c_int(0)
        check(lib().dr_chainset_ztile_get(self.h, C.byref(zt)))
        check(lib().dr_chainset_fft_plan_get(self.h, C.byref(fp)))
        return dict(path=self.PATHS[p.value], blocks_per_sm=g.value, tuned_ms=ms.value,
                    tensor_products=bool(tc.value), tma_row_gather=tc.value == 2, z_tile_chains=zt.value,
                    fft_plan=fp.value)

    def update(self, iterations=1):
        check(lib().dr_step(self.h, iterations))

    def checkpoint(self):
        """The chain set's sampler state as bytes (dr_chainset_checkpoint_save)."""
        n = C.c_int64(0)
        check(lib().dr_chainset_checkpoint_size(self.h, C.byref(n)))
        buf = np.zeros(n.value, np.uint8)
        check(lib().dr_chainset_checkpoint_save(self.h, _ptr(buf), n.value))
        return buf.tobytes()

    def restore(self, state):
        """Continue from a checkpoint of a chain set of the same volume, options and chain count."""
        buf = np.frombuffer(state, np.uint8).copy()
        check(lib().dr_chainset_checkpoint_restore(self.h, _ptr(buf), len(buf)))

    def update_timed(self, iterations=1):
        """Advance and return the device time (ms, CUDA events on the library's stream)."""
        ms = np.zeros(1, np.float64)
        check(lib().dr_step_timed(self.h, iterations, _ptr(ms)))
        return float(ms[0])

    def run(self):
        check(lib().dr_run(self.h))

    def stats(self):
        arr = (ChainStats * self.n_chains)()
        check(lib().dr_chain_stats_get(self.h, arr))
        return [{f: getattr(s, f) for f, _ in ChainStats._fields_} for s in arr]

    def summary(self, chain=-1):
        n = self.data.n_output
        m = np.zeros(max(n, 1), np.float32)
        v = np.zeros(max(n, 1), np.float32)
        a = np.zeros(max(n, 1), np.float32)
        check(lib().dr_summary_get(self.h, chain, _ptr(m), _ptr(v), _ptr(a)))
        return dict(mean=m[:n], var=v[:n], activation=a[:n])

    def samples(self, chain, max_saved=None):
        max_saved = max_saved or self.hmc.nsave
        out = np.zeros((max_saved, max(self.data.n_output, 1)), np.float32)
        ns = C.c_int(0)
        check(lib().dr_samples_get(self.h, chain, _ptr(out), max_saved, C.byref(ns)))
        return out[: ns.value, : self.data.n_output]

    def set_state(self, chain, mu, sigma_sq_inv):
        a = self._field(mu)
        check(lib().dr_set_state(self.h, chain, _ptr(a), float(sigma_sq_inv[0]), float(sigma_sq_inv[1])))

    def get_state(self, chain):
        mu = np.zeros(self.data.shape, np.complex64)
        s = np.zeros(2, np.float32)
        check(lib().dr_get_state(self.h, chain, _ptr(mu), _ptr(s)))
        return mu, s

    def log_prior_likelihood(self, chain, mu):
        a = self._field(mu)
        out = np.zeros(2, np.float64)
        check(lib().dr_log_posterior(self.h, chain, _ptr(a), _ptr(out)))
        return float(out[0]), float(out[1])

    def log_posterior(self, chain, mu):
        lp, ll = self.log_prior_likelihood(chain, mu)
        return lp + ll

    def gradient(self, chain, mu):
        a = self._field(mu)
        g = np.zeros(self.data.shape, np.complex64)
        check(lib().dr_gradient(self.h, chain, _ptr(a), _ptr(g)))
        return g

    def leapfrog(self, chain, mu0, p0, eps, L):
        a, b = self._field(mu0), self._field(p0)
        mo = np.zeros(self.data.shape, np.complex64)
        po = np.zeros(self.data.shape, np.complex64)
        en = np.zeros(6, np.float64)
        check(lib().dr_leapfrog_fixed(self.h, chain, _ptr(a), _ptr(b), float(eps), int(L), _ptr(mo), _ptr(po),
                                      _ptr(en)))
        return mo, po, en


def fit_model(data: MultiResData, hmc: HMCParameters, n_chains=1):
    """gpp_approx::fit_model (gaussian_process_model.h:88-177): run to nsave samples and summarise."""
    p = MultiResParameters(data, hmc, n_chains)
    p.run()
    out = p.summary(-1)
    st = p.stats()
    out["mh_rate"] = float(np.mean([s["mh_rate"] for s in st]))
    out["eps"] = float(np.mean([s["eps"] for s in st]))
    out["stats"] = st
    out["chains"] = p
    return out


def debug_dual_averaging(burnin, nsave, thin, L, starting_eps, mhtarget, rates, device=0):
    r = np.ascontiguousarray(rates, np.float32)
    e = np.zeros(len(r), np.float64)
    s = np.zeros(len(r), np.int32)
    check(lib().dr_debug_dual_averaging(burnin, nsave, thin, L, starting_eps, mhtarget, len(r), _ptr(r), _ptr(e),
                                        _ptr(s), device))
    return e, s


KERNEL_NAMES = ["state update (k_xyplane when E0 == E1 <= 128, else k_xline)", "forward y pass (k_pass)", "forward z pass + gather (k_pass)",
                "W product (k_tc_product + k_tc_finish from 16 chains, else k_spmv_w)",
                "W^T product (k_tc_product + k_tc_finish from 16 chains, else k_spmv_wt)", "inverse z pass (k_pass)",
                "inverse y pass (k_pass)"]


def time_kernel(chains, which, step=1, reps=20):
    """Mean CUDA-event duration (ms) and algorithmic bytes of one kernel of the leapfrog step."""
    ms = np.zeros(1, np.float64)
    b = np.zeros(1, np.float64)
    check(lib().dr_debug_time_kernel(chains.h, which, step, reps, _ptr(ms), _ptr(b)))
    return float(ms[0]), float(b[0])


def pool_usage(device=0, reset_high=False):
    """(bytes in use, high-water mark) of the library's device memory pool (dr_debug_pool_usage)."""
    u, h = C.c_uint64(0), C.c_uint64(0)
    check(lib().dr_debug_pool_usage(device, 1 if reset_high else 0, C.byref(u), C.byref(h)))
    return int(u.value), int(h.value)


def bounded_wait(limit_ms=200.0, device=0):
    """One device wait that nothing completes (dr_debug_bounded_wait): (gave_up, waited_ms)."""
    g, w = C.c_int(-1), C.c_double(0)
    check(lib().dr_debug_bounded_wait(device, float(limit_ms), C.byref(g), C.byref(w)))
    return bool(g.value == 1), w.value


def zorder_keys(ijk):
    """Z-order keys of integer coordinates (n x 3, 10 bits each), as the tensor-core products order tile rows."""
    ijk = np.asarray(ijk, np.int64)
    k = np.zeros(len(ijk), np.uint32)
    for b in range(10):
        for a in range(3):
            k |= (((ijk[:, a] >> b) & 1) << (3 * b + a)).astype(np.uint32)
    return k


def tc_layout(rowptr, col, val, n_cols, keys, g_max):
    """Host-only check of the tensor-core products' dense-tile layout (dr_debug_tc_layout): the dense matrix read
    back from the tiles, and the layout's statistics (tiles, chunks, segments, CTAs, chunks covered once, rows
    covered once, index tables consistent)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    keys = np.ascontiguousarray(keys, np.uint32)
    n_rows = len(rowptr) - 1
    dense = np.empty((n_rows, int(n_cols)), np.float32)
    stats = np.zeros(7, np.int64)
    check(lib().dr_debug_tc_layout(n_rows, int(n_cols), _ptr(rowptr), _ptr(col), _ptr(val), _ptr(keys), int(g_max),
                                   _ptr(dense), _ptr(stats)))
    return dense, dict(zip(("tiles", "chunks", "segments", "ctas", "chunks_once", "rows_once", "consistent"),
                           (int(x) for x in stats)))


def log_posterior_noalloc(data: MultiResData, mu_device_ptr: int, s_hr: float, s_sr: float):
    """(log prior, log likelihood) of a device-resident field without any device allocation.

    For callers that cannot call cudaMalloc/cudaFree (their device memory is owned by
    another allocator, or their loop has stopped allocating).  mu_device_ptr points to
    2N float32 values (re, im) on the volume's device.  Calls share one library-owned
    scratch array: do not overlap them on the GPU.
    """
    out = np.zeros(2, np.float64)
    check(lib().dr_log_posterior_noalloc(data.h, C.c_void_p(int(mu_device_ptr)), float(s_hr), float(s_sr),
                                         _ptr(out)))
    return float(out[0]), float(out[1])


def kernel_launches(reset=False):
    return int(lib().dr_kernel_launches(1 if reset else 0))


@dataclass
class JobResult:
    mean: np.ndarray
    var: np.ndarray
    activation: np.ndarray
    mh_rate: float
    grad_evals: int
    latency_s: float          # submission to result on the host
    queue_s: float            # submission to admission on the device
    device_bytes: int


class Server:
    """Continuous batching of independent fits on one GPU (dr_server_*).

    ``submit`` copies the images and returns a job id at once; host set-up runs
    on worker threads, and a scheduler thread admits prepared jobs while their
    device footprint fits ``hbm_budget_bytes``, advancing resident jobs
    ``iterations_per_round`` iterations per round on their own streams, the
    earliest admitted first while their chains fit ``max_chains_in_flight``.
    A job's result does not depend on what else runs beside it."""

    def __init__(self, device=0, hbm_budget_bytes=0, max_active=64, iterations_per_round=8, host_threads=4,
                 max_chains_in_flight=0):
        L = lib()
        o = ServerOpts(device, int(hbm_budget_bytes), max_active, iterations_per_round, host_threads,
                       int(max_chains_in_flight))
        h = C.c_void_p()
        check(L.dr_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self.device = device

    def submit(self, highres, qform_hr, stdres=None, qform_sr=None, covariance=(1.0, 0.6, 1.5), neighborhood=-1.0,
               hmask=None, omask=None, smask=None, covfun=DR_COV_RBF, hmc: HMCParameters | None = None,
               n_chains=1):
        keep = []
        d = _volume_desc(keep, highres, qform_hr, stdres, qform_sr, covariance, neighborhood, hmask, omask, smask,
                         covfun, self.device)
        o = (hmc or HMCParameters()).c()
        jid = C.c_uint64(0)
        check(lib().dr_server_submit(self.h, C.byref(d), C.byref(o), int(n_chains), C.byref(jid)))
        return int(jid.value)

    def submit_volume(self, vol, hmc: HMCParameters | None = None, n_chains=1):
        """Submit a ``dualres_b200.synth.Volume``."""
        return self.submit(vol.highres, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius,
                           hmask=vol.hmask, omask=vol.omask, hmc=hmc, n_chains=n_chains)

    def preempt(self, job, timeout_s=600.0):
        """Checkpoint a resident job at its next round boundary and release its device memory (dr_server_preempt)."""
        check(lib().dr_server_preempt(self.h, job, float(timeout_s)))

    def resume(self, job):
        """Re-admit a preempted job; it continues from its checkpoint (dr_server_resume)."""
        check(lib().dr_server_resume(self.h, job))

    def status(self, job):
        st = JobStatus()
        check(lib().dr_server_status(self.h, job, C.byref(st)))
        return st

    def wait(self, job, timeout=600.0):
        check(lib().dr_server_wait(self.h, job, float(timeout)))

    def drain(self, timeout=3600.0):
        check(lib().dr_server_drain(self.h, float(timeout)))

    def result(self, job, forget=False):
        st = self.status(job)
        n = st.n_output
        mean, var, act = (np.empty(n, np.float32) for _ in range(3))
        check(lib().dr_server_result(self.h, job, _ptr(mean), _ptr(var), _ptr(act)))
        if forget:
            check(lib().dr_server_forget(self.h, job))
        return JobResult(mean, var, act, float(st.mh_rate), int(st.grad_evals), st.finish_s - st.submit_s,
                         st.admit_s - st.submit_s, int(st.device_bytes))

    def stats(self):
        s = ServerStats()
        check(lib().dr_server_stats_get(self.h, C.byref(s)))
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().dr_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ covariance estimation
def mce_offsets():
    """perturbation_matrix_3d offsets, (n, 3) int32."""
    L = lib()
    n = C.c_int(0)
    check(L.dr_mce_offsets(None, 0, C.byref(n)))
    P = np.zeros(3 * n.value, np.int32)
    check(L.dr_mce_offsets(_ptr(P), n.value, C.byref(n)))
    return P.reshape(-1, 3)


def mce_summary(img, qform, device=0, with_sums=False):
    """compute_mce_summary_data on the GPU: distance, covariance and pair count per offset."""
    L = lib()
    a = _f32(img)
    nz, ny, nx = a.shape
    n = C.c_int(0)
    check(L.dr_mce_offsets(None, 0, C.byref(n)))
    n = n.value
    dist, cov = np.zeros(n, np.float32), np.zeros(n, np.float32)
    npairs = np.zeros(n, np.int32)
    sums = np.zeros(3 * n) if with_sums else None
    check(L.dr_mce_summary(_ptr(a), nx, ny, nz, _ptr(_f32(qform)), device, _ptr(dist), _ptr(cov), _ptr(npairs),
                           _ptr(sums)))
    out = dict(distance=dist, covariance=cov, npairs=npairs)
    if with_sums:
        out["sums"] = sums.reshape(n, 3)
    return out


def fit_rbf_parameters(distance, covariance, npairs, theta0=(1.0, 0.6, 1.5)):
    """compute_rbf_parameters (host): COBYLA fit of the RBF model to an MCE summary."""
    th = np.asarray(theta0, np.float64).copy()
    d, c = _f32(distance), _f32(covariance)
    n = np.ascontiguousarray(npairs, np.int32)
    check(lib().dr_fit_rbf_parameters(_ptr(d), _ptr(c), _ptr(n), len(d), _ptr(th)))
    return tuple(float(x) for x in th)


def estimate_covariance(img, qform, theta0=(1.0, 0.6, 1.5), device=0):
    """compute_covar_parameters_if_needed: MCE summary on the GPU, then the COBYLA fit."""
    th = np.asarray(theta0, np.float64).copy()
    a = _f32(img)
    nz, ny, nx = a.shape
    check(lib().dr_estimate_covariance(_ptr(a), nx, ny, nz, _ptr(_f32(qform)), device, _ptr(th)))
    return tuple(float(x) for x in th)


def cli_path():
    """The dualgpmf command line (built next to the library)."""
    _build.build()
    return _build.CLI
