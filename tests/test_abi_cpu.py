"""CPU-side checks of the C ABI: the library loads without a GPU, exports every
entry point declared in include/*.h, and its host-side kriging builder matches
the oracle (sparsity bit-exact)."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_cases


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(dr_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import dualres_b200 as d
    L = d.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_library_reports_version():
    import dualres_b200 as d
    assert b"sm_100a" in d.lib().dr_version()


def test_bounds_checked_library_loads_and_exports_the_same_symbols():
    """The checked build (DRB_BOUNDS_CHECK: every data-dependent index tested before its access, a failure recorded
    and the access skipped) is a second library with the same entry points, selected by DRB_LIBRARY=checked."""
    import ctypes

    from dualres_b200 import build as b
    b.build(checked=True)
    L = ctypes.CDLL(b.LIB_CHECKED)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    L.dr_version.restype = ctypes.c_char_p
    assert b"bounds-checked" in L.dr_version()


@pytest.mark.parametrize("name", golden_cases())
def test_host_kriging_matches_oracle(oracle, name):
    import dualres_b200 as d
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    prep = oracle.prepare(g["highres"])
    rp, col, val = d.kriging_matrix(prep["masked"], g["qform_hr"], g["stdres"], g["qform_sr"], g["theta"],
                                    float(g["radius"]))
    assert np.array_equal(rp, g["W_rowptr"])
    assert np.array_equal(col, g["W_col"])
    assert np.abs(val - g["W_val"]).max() < 1e-6


def test_host_kriging_c1_sparsity_matches_oracle(oracle):
    """Config-1 geometry (1 mm, r = 6.9 mm, 1357 offsets): pattern bit-exact."""
    import dualres_b200 as d
    from dualres_b200 import synth
    v = synth.make_volume((20, 18, 16), 1.0, (0.806, 0.132, 1.0), 0.5, 0.3, 6.9, "ellipsoid", 0.6, 5)
    prep = oracle.prepare(v.highres)
    rp, col, val = d.kriging_matrix(prep["masked"], v.qform_hr, v.stdres, v.qform_sr, v.theta, v.radius)
    rp2, col2, _ = oracle.kriging(prep["masked"], v.qform_hr, v.stdres, v.qform_sr, v.theta, v.radius, solve=False)
    assert np.array_equal(rp, rp2) and np.array_equal(col, col2)
    # each kept row's weights sum to one (kriging_matrix.h:318-327)
    sums = np.add.reduceat(val.astype(np.float64), rp[:-1][np.diff(rp) > 0])
    assert np.allclose(sums, 1.0, atol=1e-5)


def test_host_kriging_errors():
    import dualres_b200 as d
    hr = np.zeros((6, 6, 6), np.float32)
    hr[2:4, 2:4, 2:4] = 1
    sr = np.zeros((3, 3, 3), np.float32)
    sr[1, 1, 1] = 1
    Q = np.eye(4, dtype=np.float32)
    with pytest.raises(d.DrError) as e:
        d.kriging_matrix(hr, Q, sr, Q, (1, 0.5, 1), -1.0)
    assert e.value.code == d.api.DR_ERR_INVALID
    with pytest.raises(d.DrError) as e:          # > 5000 offsets (kriging_matrix.h:172-174)
        d.kriging_matrix(hr, Q, sr, Q, (1, 0.5, 1), 11.0)
    assert e.value.code == d.api.DR_ERR_DOMAIN


def test_device_calls_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import dualres_b200 as d
    from dualres_b200 import synth
    with pytest.raises(d.DrError):
        d.MultiResData.from_volume(synth.small_volume())
