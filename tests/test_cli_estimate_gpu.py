"""GPU parts of covariance estimation and the dualgpmf command line.

  * the device MCE summary against the oracle: distances and pair counts
    bit-exact, double sums rel 1e-12, float covariances rel 1e-6;
  * dr_estimate_covariance equals the host fit of the oracle's summary;
  * the command line end to end: its posterior mean image equals the
    library's fit with the same seed and settings (bit-exact), the residual
    image is data minus mean, and --samples writes one line per saved
    iteration with mu, sigma per dataset, tau and the log likelihood.
"""
import os
import subprocess

import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import api, nifti, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,rot", [((20, 22, 24), False), ((13, 17, 11), True)])
def test_mce_summary_matches_oracle(oracle, shape, rot):
    rng = np.random.default_rng(3)
    img = rng.standard_normal(shape).astype(np.float32)
    img[img < -1.2] = 0.0
    img[rng.uniform(size=shape) < 0.02] = np.nan
    Q = nifti.quatern_to_qform(0.2895, -0.866, -0.2865, (1.8, 1.8, 2.3), (0, 0, 0), -1) if rot else \
        np.diag([1.5, 1.5, 2.0, 1.0]).astype(np.float32)
    g = api.mce_summary(img, Q, with_sums=True)
    o = oracle.mce_summary(img, Q)
    assert np.array_equal(g["distance"], o["distance"])
    assert np.array_equal(g["npairs"], o["npairs"])
    scale = np.abs(o["sums"]).max(axis=0) + 1e-300
    assert (np.abs(g["sums"] - o["sums"]) / scale).max() < 1e-12
    m = np.abs(o["covariance"]) > 1e-3
    assert np.abs(g["covariance"][m] / o["covariance"][m] - 1).max() < 1e-6


def test_estimate_covariance_equals_host_fit_of_oracle_summary(oracle):
    vol = synth.make_volume((24, 24, 20), 1.0, (1.0, 0.3, 1.4), 0.2, 0.3, 6.9, "ellipsoid", 0.8, 5, dual=False)
    th_gpu = api.estimate_covariance(vol.highres, vol.qform_hr)
    s = oracle.mce_summary(vol.highres, vol.qform_hr)
    th_host = api.fit_rbf_parameters(s["distance"], s["covariance"], s["npairs"])
    assert np.allclose(th_gpu, th_host, rtol=1e-3), (th_gpu, th_host)


def _write_volume(tmp, vol):
    nifti.write_like(os.path.join(tmp, "hr.nii.gz"), vol.highres, vol.qform_hr)
    args = ["--highres", "hr.nii.gz"]
    if vol.stdres is not None:
        nifti.write_like(os.path.join(tmp, "sr.nii.gz"), vol.stdres, vol.qform_sr)
        args += ["--stdres", "sr.nii.gz"]
    if vol.hmask is not None:
        nifti.write_like(os.path.join(tmp, "hm.nii.gz"), vol.hmask, vol.qform_hr)
        args += ["--hmask", "hm.nii.gz"]
    if vol.omask is not None:
        nifti.write_like(os.path.join(tmp, "om.nii.gz"), vol.omask, vol.qform_hr)
        args += ["--omask", "om.nii.gz"]
    return args


def _cli(args, cwd):
    return subprocess.run([api.cli_path(), *args], cwd=cwd, capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("dual", [True, False])
def test_cli_matches_library_fit(tmp_path, dual):
    vol = synth.small_volume(seed=41, dual=dual)
    tmp = str(tmp_path)
    args = _write_volume(tmp, vol) + ["--covariance", *[str(t) for t in vol.theta], "--neighborhood",
                                      str(vol.radius), "--burnin", "30", "--nsave", "12", "--thin", "2",
                                      "--leapfrog", "6", "--seed", "77", "--samples", "--output", "run"]
    r = _cli(args, tmp)
    assert r.returncode == 0, r.stderr + r.stdout
    for suffix in ("_posterior_mean", "_posterior_variance", "_posterior_activation", "_residual"):
        assert os.path.exists(os.path.join(tmp, "run" + suffix + ".nii.gz"))
    data = d.MultiResData.from_volume(vol)
    fit = d.fit_model(data, d.HMCParameters(burnin=30, nsave=12, thin=2, leapfrog=6, seed=77, store_samples=True), 1)
    mean_img, Q, _ = nifti.read(os.path.join(tmp, "run_posterior_mean.nii.gz"))
    om = vol.omask if vol.omask is not None else vol.highres
    sel = ~np.isnan(om) & (om != 0)
    assert np.allclose(Q, vol.qform_hr)
    np.testing.assert_array_equal(mean_img[sel], fit["mean"])
    var_img, _, _ = nifti.read(os.path.join(tmp, "run_posterior_variance.nii.gz"))
    assert np.allclose(var_img[sel], fit["var"], rtol=0, atol=0) or np.array_equal(var_img[sel], fit["var"])
    res_img, _, _ = nifti.read(os.path.join(tmp, "run_residual.nii.gz"))
    hr = np.where(np.isnan(vol.highres), 0, vol.highres)
    if vol.hmask is not None:
        hr = np.where(vol.hmask == 0, 0, hr)
    both = sel & (hr != 0)
    np.testing.assert_allclose(res_img[both], hr[both] - fit["mean"][both[sel]], rtol=0, atol=1e-6)
    assert np.all(res_img[~sel] == 0)
    lines = open(os.path.join(tmp, "run_samples.dat")).read().split("\n")
    assert len(lines) == 12
    cols = [len(ln.split("\t")) for ln in lines]
    assert set(cols) == {data.n_output + (2 if dual else 1) + 2}
    last = np.array(lines[-1].split("\t"), np.float64)
    smp = fit["chains"].samples(0)
    np.testing.assert_allclose(last[: data.n_output], smp[-1], rtol=1e-5, atol=1e-6)
    assert abs(last[-2] - np.sqrt(vol.theta[0])) < 1e-5  # tau = sqrt(1 / tau^-2), tau^-2 = 1 / variance
    stats = open(os.path.join(tmp, "run_stats.csv")).read().split("\n")
    assert stats[0] == "MHrate,SamplingTime,StepSize"
    mh, _, eps = (float(x) for x in stats[1].split(","))
    assert abs(mh - fit["mh_rate"]) < 1e-5 and abs(eps - fit["eps"]) < 1e-5 * max(1, abs(eps))
    assert "Metropolis-Hastings rate was" in r.stdout
    data.close()


def test_cli_estimates_covariance_when_absent(tmp_path):
    vol = synth.small_volume(seed=42, dims=(14, 14, 12))
    tmp = str(tmp_path)
    args = _write_volume(tmp, vol) + ["--burnin", "10", "--nsave", "5", "--thin", "1", "--leapfrog", "4",
                                      "--seed", "3", "--output", "est"]
    r = _cli(args, tmp)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "Estimating covariance parameters... Done!" in r.stdout
    line = [ln for ln in r.stdout.split("\n") if ln.startswith("Covariance parameters:")][0]
    th = [float(x) for x in line.split("(")[1].rstrip(")").split(",")]
    assert th[0] > 0 and 0 < th[1] <= th[2] + 1e-6 and th[2] <= 2
    # estimated from the std-res image, as the reference does when it is given
    s = api.mce_summary(vol.stdres, vol.qform_sr)
    th2 = api.fit_rbf_parameters(s["distance"], s["covariance"], s["npairs"])
    assert np.allclose(th, th2, rtol=1e-4)


def test_cli_patient_sized_rotated_volume(tmp_path):
    """A clinical-sized input: 120 x 120 x 72 high-res voxels of 1.8 x 1.8 x 2.3 mm under a rotated qform with
    qfac -1, std-res at twice the voxel size (256^3 embedding, x-line update path)."""
    vol = synth.rotated(synth.make_volume((120, 120, 72), 1.0, (1.0, 0.3, 1.5), 0.5, 0.3, 6.9, "ellipsoid", 0.6, 17))
    tmp = str(tmp_path)
    nifti.write(os.path.join(tmp, "hr.nii.gz"), vol.highres, pixdim=(1.8, 1.8, 2.3),
                quatern=(0.2895, -0.866, -0.2865), qoffset=(-90.0, 120.0, -40.0), qfac=-1)
    _, Qh, _ = nifti.read(os.path.join(tmp, "hr.nii.gz"))
    assert np.allclose(Qh, vol.qform_hr, atol=1e-5)
    Qs = vol.qform_sr.astype(np.float64)
    nifti.write(os.path.join(tmp, "sr.nii.gz"), vol.stdres, pixdim=(3.6, 3.6, 4.6),
                quatern=(0.2895, -0.866, -0.2865), qoffset=tuple(Qs[:3, 3]), qfac=-1)
    r = _cli(["--highres", "hr.nii.gz", "--stdres", "sr.nii.gz", "--covariance", "1", "0.3", "1.5",
              "--burnin", "5", "--nsave", "3", "--thin", "1", "--leapfrog", "3", "--seed", "4", "--output", "big"], tmp)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "Neighborhood: 6.9 (mm)" in r.stdout
    mean, Q, _ = nifti.read(os.path.join(tmp, "big_posterior_mean.nii.gz"))
    assert np.allclose(Q, vol.qform_hr, atol=1e-5)
    sel = vol.highres != 0
    assert np.all(np.isfinite(mean[sel])) and np.count_nonzero(mean[sel]) > 0.99 * sel.sum()


def test_cli_monitor_prints_every_transition(tmp_path):
    """--monitor prints one line per iteration, as MultiResParameters::update does (MultiResParameters.h:706-713):
    the initial and proposed energy, the step size and the MH ratio R = exp(proposed - initial); and the fit is the
    same as without it."""
    import re
    vol = synth.small_volume(seed=43)
    tmp = str(tmp_path)
    base = _write_volume(tmp, vol) + ["--covariance", *[str(t) for t in vol.theta], "--neighborhood",
                                      str(vol.radius), "--burnin", "12", "--nsave", "5", "--thin", "2",
                                      "--leapfrog", "4", "--seed", "5"]
    r = _cli(base + ["--monitor", "--output", "mon"], tmp)
    assert r.returncode == 0, r.stderr + r.stdout
    pat = re.compile(r"^Energy Transition \((\S+) -> (\S+)\);  step size \((\S+)\);  MH = \((\S+)\)$")
    lines = [m for m in (pat.match(x) for x in r.stdout.splitlines()) if m]
    assert len(lines) == 12 + 2 * 5, r.stdout
    for m in lines:
        e0, ep, eps, mh = (float(x) for x in m.groups())
        assert eps > 0
        # printed with 4 significant digits: compare R with exp(ep - e0) where the difference is resolved
        if abs(ep - e0) < 5 and abs(e0) < 1e3:
            assert abs(mh - np.exp(ep - e0)) <= 0.05 * max(1.0, mh) + 1e-3, (e0, ep, mh)
    q = _cli(base + ["--output", "plain"], tmp)
    assert q.returncode == 0, q.stderr + q.stdout
    a = nifti.read(os.path.join(tmp, "mon_posterior_mean.nii.gz"))[0]
    b = nifti.read(os.path.join(tmp, "plain_posterior_mean.nii.gz"))[0]
    assert np.array_equal(a, b)
