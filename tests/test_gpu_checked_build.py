"""The bounds-checked library (DRB_LIBRARY=checked, built with DRB_BOUNDS_CHECK) on a cross-section of the GPU
tests: every data-dependent index of the kernels (the box-to-voxel maps, the kriging columns and tile rows, the
gathered field indices, each block's plane or lines of the state) is tested before its access, and a failure ends
the call with an error.  The same parity tests must pass with it: the update paths on the fixtures, the tensor-core
products, the x-line path on the 256x256x128 embedding and the server.  This is the stand-in for a memory checker:
every check records a failure and skips the access, so nothing here faults or traps the GPU."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SELECTION = [
    "tests/test_gpu_parity.py::test_log_posterior_and_gradient",
    "tests/test_gpu_parity.py::test_fixed_momentum_leapfrog",
    "tests/test_gpu_parity.py::test_sampler_runs_and_counts",
    "tests/test_gpu_tc_products.py::test_gradient_and_leapfrog_match_oracle",
    "tests/test_gpu_parity_large.py::test_256_embedding_xline_kernel",
    "tests/test_server.py::test_job_alone_equals_job_in_mix_and_direct_fit",
]


def test_parity_cross_section_passes_with_the_bounds_checked_library():
    env = dict(os.environ, DRB_LIBRARY="checked")
    code = ("import dualres_b200 as d; v = d.lib().dr_version(); "
            "assert b'bounds-checked' in v, v; print(v.decode())")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider", *SELECTION], cwd=ROOT,
                       env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
