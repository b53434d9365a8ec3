"""Continuous-batching server (dr_server_*): a job's result is the same alone
and in a mix, admission keeps resident jobs inside the HBM budget, and a failed
job does not disturb the others."""
import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import synth

pytestmark = pytest.mark.gpu

HMC = dict(burnin=30, nsave=20, thin=2, leapfrog=6, mhtarget=0.65)


def _jobs():
    """Three volumes of different sizes and seeds (so their graphs differ)."""
    return [
        (synth.small_volume(seed=7), d.HMCParameters(seed=11, **HMC), 2),
        (synth.small_volume(seed=8, dims=(14, 12, 9)), d.HMCParameters(seed=12, **HMC), 3),
        (synth.small_volume(seed=9, dims=(12, 12, 12)), d.HMCParameters(seed=13, **HMC), 1),
    ]


def test_job_alone_equals_job_in_mix_and_direct_fit():
    jobs = _jobs()
    vol, hmc, C = jobs[0]
    with d.Server(iterations_per_round=3) as sv:
        alone = sv.result(_submit_wait(sv, vol, hmc, C))
    with d.Server(iterations_per_round=2) as sv:
        ids = [sv.submit_volume(v, h, c) for v, h, c in jobs]
        sv.drain(600)
        mixed = [sv.result(i) for i in ids]
        st = sv.stats()
    assert st.done == 3 and st.failed == 0
    assert st.peak_running >= 2, "jobs did not overlap on the device"
    assert st.kernel_launches > 0
    np.testing.assert_array_equal(alone.mean, mixed[0].mean)
    np.testing.assert_array_equal(alone.var, mixed[0].var)
    np.testing.assert_array_equal(alone.activation, mixed[0].activation)
    assert alone.mh_rate == mixed[0].mh_rate and alone.grad_evals == mixed[0].grad_evals
    # the server runs the same iteration graph as a direct fit
    data = d.MultiResData.from_volume(vol)
    fit = d.fit_model(data, hmc, n_chains=C)
    np.testing.assert_array_equal(fit["mean"], mixed[0].mean)
    np.testing.assert_array_equal(fit["var"], mixed[0].var)
    data.close()
    for r, (v, h, c) in zip(mixed, jobs):
        assert np.all(np.isfinite(r.mean)) and np.all(r.var >= 0)
        assert 0 < r.grad_evals <= c * (h.burnin + h.nsave * h.thin) * (h.leapfrog + 1)
        assert r.latency_s >= r.queue_s >= 0


def test_chain_budget_runs_the_earliest_jobs_first():
    """With room for 3 chains in flight, the jobs of 2, 3 and 1 chains cannot all advance at once: the first and the
    third run together, the second starts when the first has finished. Every result equals the one without a
    budget (the order of the rounds does not enter a job's arithmetic)."""
    jobs = _jobs()
    with d.Server(iterations_per_round=2) as sv:
        ids = [sv.submit_volume(v, h, c) for v, h, c in jobs]
        sv.drain(600)
        free = [sv.result(i) for i in ids]
    with d.Server(iterations_per_round=2, max_chains_in_flight=3) as sv:
        ids = [sv.submit_volume(v, h, c) for v, h, c in jobs]
        sv.drain(600)
        held = [sv.result(i) for i in ids]
        st = [sv.status(i) for i in ids]
    assert all(s.state == d.api.JOB_DONE for s in st)
    assert st[1].finish_s > st[0].finish_s
    for a, b in zip(free, held):
        np.testing.assert_array_equal(a.mean, b.mean)
        np.testing.assert_array_equal(a.var, b.var)
        assert a.grad_evals == b.grad_evals


def test_preempted_job_resumes_bit_for_bit():
    """A job preempted while it runs (its checkpoint saved, its device memory released) and resumed later gives the
    same result as an uninterrupted run of the same job, while another job keeps running beside it."""
    import time
    jobs = _jobs()
    vol, hmc, C = jobs[1]
    with d.Server(iterations_per_round=2) as sv:
        ref = sv.result(_submit_wait(sv, vol, hmc, C))
    with d.Server(iterations_per_round=2) as sv:
        other = sv.submit_volume(*jobs[0])
        j = sv.submit_volume(vol, hmc, C)
        t0 = time.time()
        while sv.status(j).state != d.api.JOB_RUNNING and time.time() - t0 < 120:
            time.sleep(0.005)
        sv.preempt(j)
        st = sv.status(j)
        assert st.state == d.api.JOB_PREEMPTED and st.device_bytes == 0
        sv.wait(other, 600)
        sv.resume(j)
        sv.wait(j, 600)
        got = sv.result(j)
        with pytest.raises(d.DrError):
            sv.resume(j)  # only a preempted job can be resumed
    np.testing.assert_array_equal(ref.mean, got.mean)
    np.testing.assert_array_equal(ref.var, got.var)
    assert ref.grad_evals == got.grad_evals and ref.mh_rate == got.mh_rate


def _submit_wait(sv, vol, hmc, C):
    j = sv.submit_volume(vol, hmc, C)
    sv.wait(j, 600)
    return j


def test_admission_respects_budget():
    jobs = _jobs() * 2
    with d.Server(iterations_per_round=4) as sv:
        sizes = []
        for v, h, c in jobs[:3]:
            j = _submit_wait(sv, v, h, c)
            sizes.append(sv.status(j).device_bytes)
    budget = max(sizes) + min(sizes) // 4  # room for exactly one resident job
    with d.Server(hbm_budget_bytes=budget, iterations_per_round=4) as sv:
        ids = [sv.submit_volume(v, h, c) for v, h, c in jobs]
        sv.drain(600)
        st = sv.stats()
        assert st.done == len(jobs) and st.failed == 0
        assert st.peak_device_bytes <= budget + max(sizes)
        assert st.peak_running <= 2
        for i in ids:
            assert sv.status(i).state == d.api.JOB_DONE


def test_failed_job_is_isolated():
    vol, hmc, C = _jobs()[0]
    with d.Server(iterations_per_round=4) as sv:
        with pytest.raises(d.DrError):
            sv.submit_volume(vol, hmc, 0)  # rejected at submission
        bad = d.HMCParameters(**{**HMC, "mhtarget": 1.5})
        with pytest.raises(d.DrError):
            sv.submit_volume(vol, bad, 1)
        empty = np.zeros_like(vol.highres)  # no data voxel: set-up fails on a worker
        jb = sv.submit(empty, vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius, hmc=hmc, n_chains=1)
        jg = sv.submit_volume(vol, hmc, C)
        with pytest.raises(d.DrError):
            sv.wait(jb, 600)
        sv.wait(jg, 600)
        assert sv.status(jb).state == d.api.JOB_FAILED
        assert sv.status(jg).state == d.api.JOB_DONE
        with pytest.raises(d.DrError):
            sv.result(jb)
        r = sv.result(jg, forget=True)
        assert np.all(np.isfinite(r.mean))
        with pytest.raises(d.DrError):
            sv.status(jg)  # forgotten
        st = sv.stats()
        assert st.failed == 1 and st.done == 1


def test_volume_released_before_its_chain_set():
    """A volume destroyed while a chain set still uses it stays alive until that chain set goes."""
    vol, hmc, C = _jobs()[0]
    data = d.MultiResData.from_volume(vol)
    p = d.MultiResParameters(data, hmc, C)
    data.close()
    p.update(3)
    assert all(s["iteration"] == 3 for s in p.stats())
    p.close()
    data2 = d.MultiResData.from_volume(vol)  # later calls see no stale error
    data2.close()
