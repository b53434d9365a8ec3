"""The performance switches change when and how the kernels run, never what they compute: a 64-chain fit on the
64^3 embedding (tensor-core products, plane kernel) and a 4-chain fit on a non-square embedding (x-line kernel, CSR
products) give bit-identical posterior summaries and chain statistics with programmatic dependent launch and the L2
prefetch of the update state each turned off.  Each setting runs in a subprocess, since the library reads the
switches once per process."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SNIPPET = r"""
import hashlib, json, os
os.environ["DRB_AUTOTUNE"] = "0"
import dualres_b200 as d
from dualres_b200 import synth
out = {}
for name, vol, C in (("plane", synth.small_volume(seed=71, dims=(22, 20, 18)), 64),
                     ("lines", synth.small_volume(seed=72, dims=(24, 14, 10)), 4)):
    data = d.MultiResData.from_volume(vol)
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=8, nsave=6, thin=1, leapfrog=5, seed=3), C)
    ch.update(14)
    s = ch.summary(-1)
    h = hashlib.sha256(s["mean"].tobytes() + s["var"].tobytes())
    h.update(json.dumps(ch.stats(), sort_keys=True).encode())
    cfg = ch.config()
    out[name] = [h.hexdigest(), cfg["path"], cfg["tensor_products"]]
    ch.close(), data.close()
print(json.dumps(out))
"""


def _run(extra):
    env = dict(os.environ, **extra)
    r = subprocess.run([sys.executable, "-c", SNIPPET], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_switches_leave_results_bit_identical():
    base = _run({})
    assert base["plane"][1] == "plane" and base["plane"][2] is True
    assert base["lines"][1] == "lines"
    for extra in ({"DRB_PDL": "0"}, {"DRB_L2_PREFETCH": "0"}):
        assert _run(extra) == base, extra
