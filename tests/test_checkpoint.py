"""Checkpoint and resume of a chain set (dr_chainset_checkpoint_*): a chain set restored from a checkpoint on a
fresh chain set of the same volume, options and chain count continues bit for bit as the saved one would have
(posterior summary, chain statistics and stored samples), during the step-size search and after it, and a
checkpoint of another shape is refused."""
import numpy as np
import pytest

import dualres_b200 as d
from dualres_b200 import synth

pytestmark = pytest.mark.gpu


def _hmc(store=False):
    return d.HMCParameters(burnin=12, nsave=10, thin=2, leapfrog=6, seed=21, store_samples=store)


@pytest.mark.parametrize("cut", [3, 17])  # inside the step-size search / after burn-in
def test_resume_is_bit_identical(cut):
    vol = synth.small_volume(seed=61, dims=(12, 11, 10))
    data = d.MultiResData.from_volume(vol)
    total = 12 + 2 * 10
    ref = d.MultiResParameters(data, _hmc(store=True), 3)
    ref.update(total)
    want = ref.summary(-1), ref.stats(), [ref.samples(c) for c in range(3)]
    a = d.MultiResParameters(data, _hmc(store=True), 3)
    a.update(cut)
    ck = a.checkpoint()
    a.close()
    b = d.MultiResParameters(data, _hmc(store=True), 3)
    b.restore(ck)
    b.update(total - cut)
    got = b.summary(-1), b.stats(), [b.samples(c) for c in range(3)]
    for k in ("mean", "var"):
        np.testing.assert_array_equal(want[0][k], got[0][k])
    for s0, s1 in zip(want[1], got[1]):
        assert s0 == s1
    for x0, x1 in zip(want[2], got[2]):
        np.testing.assert_array_equal(x0, x1)
    ref.close(), b.close(), data.close()


def test_checkpoint_of_another_shape_is_refused():
    vol = synth.small_volume(seed=62, dims=(12, 11, 10))
    data = d.MultiResData.from_volume(vol)
    a = d.MultiResParameters(data, _hmc(), 2)
    a.update(2)
    ck = a.checkpoint()
    b = d.MultiResParameters(data, _hmc(), 3)
    with pytest.raises(d.DrError):
        b.restore(ck)
    with pytest.raises(d.DrError):
        a.restore(b"\0" * 64)
    a.close(), b.close(), data.close()
