"""Host-side parts of the dualgpmf command line and of covariance estimation
(no GPU): the MCE offsets against the oracle, the COBYLA fit against scipy's
COBYLA on the same objective, NIfTI reading (qform from quaternions), and the
command line's option handling (GPMCommandParser.inl:219-606)."""
import os
import subprocess

import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import api, nifti, synth


def test_mce_offsets_match_oracle(oracle):
    P = api.mce_offsets()
    assert P.shape == (25348, 3)
    assert np.array_equal(P, oracle.mce_offsets())
    assert P[0].tolist() == [0, 0, 0] and P[-1].tolist() == [0, 0, 25]


def _objective(summary):
    dist = summary["distance"].astype(np.float64)
    cov = summary["covariance"].astype(np.float64)
    m = (np.arange(len(dist)) >= 1) & (summary["npairs"] != 0) & (dist <= 1e6)
    x, y = np.abs(dist[m]), cov[m]
    _, inv, cnt = np.unique(x, return_inverse=True, return_counts=True)
    w = np.sqrt(1.0 / cnt[inv])
    return lambda t: float(np.sum((w * (y - t[0] * np.exp(-t[1] * x ** t[2]))) ** 2) / len(x))


@pytest.mark.parametrize("theta", [(1.0, 0.3, 1.4), (0.8, 0.15, 1.0), (1.2, 0.5, 1.8)])
def test_rbf_fit_reaches_the_constrained_minimum(oracle, theta):
    """compute_rbf_parameters: our COBYLA and scipy's COBYLA minimise the same
    weighted least squares under the same bounds and bandwidth <= exponent."""
    from scipy.optimize import minimize
    vol = synth.make_volume((24, 24, 20), 1.0, theta, 0.2, 0.3, 6.9, "ellipsoid", 0.8, 5, dual=False)
    s = oracle.mce_summary(vol.highres, vol.qform_hr)
    th = api.fit_rbf_parameters(s["distance"], s["covariance"], s["npairs"])
    f = _objective(s)
    tau = float(s["covariance"][0])
    assert 1e-5 - 1e-9 <= th[0] <= tau + 1e-9
    assert th[1] >= 1e-5 - 1e-9 and th[1] <= th[2] + 1e-7 and th[2] <= 2 - 1e-5 + 1e-9
    res = minimize(f, [min(1.0, tau), 0.6, 1.5], method="COBYLA",
                   constraints=[{"type": "ineq", "fun": lambda t: t[2] - t[1]}],
                   bounds=[(1e-5, tau), (1e-5, None), (1e-5, 2 - 1e-5)],
                   options={"rhobeg": 0.1, "tol": 1e-10, "maxiter": 20000})
    assert f(th) <= res.fun * (1 + 1e-4) + 1e-12, (th, res.x, f(th), res.fun)
    # the minimiser is well determined in variance and exponent
    assert abs(th[0] / res.x[0] - 1) < 2e-2 and abs(th[2] / res.x[2] - 1) < 2e-2


def test_rbf_fit_rejects_bad_starts():
    s = dict(distance=np.array([0, 1, 2], np.float32), covariance=np.array([1.0, 0.5, 0.2], np.float32),
             npairs=np.array([10, 9, 8], np.int32))
    with pytest.raises(d.DrError):
        api.fit_rbf_parameters(s["distance"], s["covariance"], s["npairs"], theta0=(1.0, 1.8, 1.5))
    z = dict(s, covariance=np.zeros(3, np.float32))
    with pytest.raises(d.DrError):
        api.fit_rbf_parameters(z["distance"], z["covariance"], z["npairs"])


@pytest.mark.parametrize("suffix", [".nii", ".nii.gz"])
def test_nifti_round_trip(tmp_path, suffix):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((5, 6, 7)).astype(np.float32)
    p = str(tmp_path / ("x" + suffix))
    nifti.write(p, a, pixdim=(1.8, 1.8, 2.3), quatern=(0.2895, -0.866, -0.2865), qoffset=(10, -4, 3), qfac=-1)
    b, Q, h = nifti.read(p)
    assert np.array_equal(a, b) and h["qform_code"] == 1
    # column norms of the rotation part are the voxel sizes
    assert np.allclose(np.linalg.norm(Q[:3, :3], axis=0), [1.8, 1.8, 2.3], rtol=1e-5)
    assert np.allclose(Q[:3, 3], [10, -4, 3])
    assert np.linalg.det(Q[:3, :3]) < 0  # qfac = -1 flips the third axis


def _run(args, cwd):
    cli = api.cli_path()
    return subprocess.run([cli, *args], cwd=cwd, capture_output=True, text=True, timeout=300)


def test_cli_help_and_option_errors(tmp_path):
    r = _run(["--help"], tmp_path)
    assert r.returncode == 0 and "--highres" in r.stderr and "--rational-quadratic" in r.stderr
    assert _run([], tmp_path).returncode == 1
    r = _run(["--bogus"], tmp_path)
    assert r.returncode == 1 and "Unrecognized option: --bogus" in r.stderr
    r = _run(["--highres", str(tmp_path / "missing.nii.gz")], tmp_path)
    assert r.returncode == 1 and "nifti-1 standard" in r.stderr
    a = np.ones((4, 4, 4), np.float32)
    nifti.write(str(tmp_path / "a.nii"), a)
    for bad in (["--mhtarget", "1.5"], ["--covariance", "1", "2"], ["--burnin", "x"], ["--seed"]):
        assert _run(["--highres", str(tmp_path / "a.nii"), *bad], tmp_path).returncode == 1, bad


def test_cli_reads_rotated_images_up_to_the_device(tmp_path):
    """The command line reads and masks both images, derives the neighbourhood
    from the high-res qform (3 x the largest voxel dimension), prints the
    settings, and stops with an error at the first device call on a machine
    without a GPU."""
    rng = np.random.default_rng(2)
    hr = rng.standard_normal((10, 12, 12)).astype(np.float32)
    sr = rng.standard_normal((5, 6, 6)).astype(np.float32)
    q = (0.2895, -0.866, -0.2865)
    nifti.write(str(tmp_path / "hr.nii.gz"), hr, pixdim=(1.8, 1.8, 2.3), quatern=q, qfac=-1)
    nifti.write(str(tmp_path / "sr.nii.gz"), sr, pixdim=(3.6, 3.6, 4.6), quatern=q, qfac=-1)
    r = _run(["--highres", "hr.nii.gz", "--stdres", "sr.nii.gz", "--covariance", "0.8", "0.2", "1.0",
              "--burnin", "5", "--nsave", "5", "--output", "out"], tmp_path)
    assert "High-resolution file: hr.nii.gz" in r.stdout and "Standard-resolution file: sr.nii.gz" in r.stdout
    assert "Neighborhood: 6.9 (mm)" in r.stdout
    assert "Covariance parameters: (0.8, 0.2, 1)" in r.stdout
    if not _has_gpu():
        assert r.returncode == 1 and "Exception caught" in r.stderr


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_cli_rejects_invalid_covariance(tmp_path):
    a = np.ones((4, 4, 4), np.float32)
    nifti.write(str(tmp_path / "a.nii"), a)
    r = _run(["--highres", "a.nii", "--covariance", "1", "0.5", "2.5"], tmp_path)
    assert r.returncode == 1
    assert "Third covariance parameter (exponent) must be in (0, 2]" in r.stderr


def test_cli_exists_next_to_the_library():
    assert os.path.dirname(api.cli_path()) == os.path.dirname(api.lib_path())


# Every option the reference's parser accepts (include/dualres/impl/CommandParser/GPMCommandParser.inl:219-606)
REFERENCE_OPTIONS = ["--burnin", "--covariance", "--debug", "--help", "--highres", "--hmask", "--leapfrog",
                     "--mhtarget", "--monitor", "--neighborhood", "--nsave", "--omask", "--output",
                     "--rational-quadratic", "--samples", "--seed", "--smask", "--stdres", "--theta", "--thin",
                     "--threads"]


def test_cli_accepts_every_reference_option(tmp_path):
    r = _run(["--help"], tmp_path)
    assert r.returncode == 0                        # --help itself is accepted; the others are listed
    missing = [o for o in REFERENCE_OPTIONS if o != "--help" and o not in r.stderr + r.stdout]
    assert not missing, missing
