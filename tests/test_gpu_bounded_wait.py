"""The time-out path of the device pipelines: a bounded mbarrier wait that
nothing completes gives up after its limit (the global-timer bound), reports
it, and leaves the context usable for the next launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_gives_up_and_device_stays_usable():
    import dualres_b200 as d
    from dualres_b200 import api, synth
    gave_up, waited = api.bounded_wait(200.0)
    assert gave_up and 200.0 <= waited < 2000.0, waited
    vol = synth.small_volume(seed=71)
    data = d.MultiResData.from_volume(vol)
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=3, nsave=2, thin=1, leapfrog=3, seed=1), 2)
    ch.run()
    assert np.all(np.isfinite(ch.summary(-1)["mean"]))
    ch.close()
    data.close()
