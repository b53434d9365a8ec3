"""Host-side pieces of bench.py that the reported numbers rest on (no GPU).

The ESS estimator (Geyer's initial monotone sequence over FFT autocorrelations)
is checked against processes whose effective sample size is known in closed
form: iid draws (ESS = n) and AR(1) chains x_t = phi x_{t-1} + e_t, whose
integrated autocorrelation time is (1 + phi) / (1 - phi).
"""
import numpy as np
import pytest

import bench


def _ar1(n, phi, cols, seed):
    rng = np.random.default_rng(seed)
    e = rng.standard_normal((n, cols))
    x = np.empty_like(e)
    x[0] = e[0] / np.sqrt(1 - phi * phi)
    for t in range(1, n):
        x[t] = phi * x[t - 1] + e[t]
    return x


def test_ess_of_iid_draws_is_the_sample_size():
    n = 20000
    x = np.random.default_rng(1).standard_normal((n, 64))
    ess = bench.ess_geyer(x)
    assert ess.shape == (64,)
    assert abs(np.median(ess) / n - 1) < 0.1, np.median(ess)


@pytest.mark.parametrize("phi", [0.5, 0.8])
def test_ess_of_ar1_chains_matches_closed_form(phi):
    n = 40000
    x = _ar1(n, phi, 32, seed=int(phi * 10))
    tau = (1 + phi) / (1 - phi)
    ess = bench.ess_geyer(x)
    assert abs(np.median(ess) / (n / tau) - 1) < 0.15, (np.median(ess), n / tau)


def test_ess_of_a_constant_voxel_is_zero():
    x = np.random.default_rng(2).standard_normal((500, 3))
    x[:, 1] = 4.0
    ess = bench.ess_geyer(x)
    assert ess[1] == 0.0 and ess[0] > 0 and ess[2] > 0


def test_config_names_the_workload_and_its_sizes():
    cfg = bench.config_of("batched64")
    assert cfg["workload"] == "batched64"
    assert cfg["chains"] == 64 and cfg["leapfrog"] == 25
    assert (cfg["burnin"], cfg["nsave"], cfg["thin"]) == (500, 500, 3)


def test_reference_byte_model_on_the_32cubed_volume():
    # 64^3 embedding, 2,467,584 kriging nonzeros shared by 64 chains, 19,660 / 2,298 data voxels
    b = bench.reference_bytes_per_step(64 ** 3, 2467584, 64, 19660, 2298)
    assert abs(b - (104 * 262144 + 16 * 2467584 / 64 + 12 * 19660 + 8 * 2298)) < 1e-6
    assert 28.0e6 < b < 28.3e6
