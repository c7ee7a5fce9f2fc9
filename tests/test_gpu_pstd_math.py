"""pine's pstd numerics as the kernels run them (math_mode = pine), evaluated on the GPU
and checked against pine's own outputs (tests/golden/pstd_math.npz, produced by running
pine's src/pstd/math.h:142-351): the functions on the hit-distance and sampling paths
(sqrt, log2, log, pow) bit for bit, the series-based ones to the accuracy the C
restatement holds against pine (pine's -ffast-math build folds its Taylor divisions into
reciprocal multiplications)."""

import numpy as np
import pytest

from conftest import golden

import oracle
import pine_b200 as pb

pytestmark = pytest.mark.gpu

BITEXACT = ["sqrt", "log2", "log", "pow"]


def _domain(name, a, b):
    if name in ("cos", "sin", "exp"):
        return np.abs(a) <= 20
    if name == "tan":
        return (np.abs(a) <= 20) & (np.abs(np.cos(a)) > 0.1)
    if name in ("acos", "asin"):
        return np.abs(a) <= 1
    if name == "atan":
        return np.abs(a) <= 4
    return (np.abs(a) <= 4) & (np.abs(b) > 0.25)


@pytest.mark.parametrize("k,name", list(enumerate(oracle.MATH_NAMES)))
def test_device_pstd_math_against_reference(pglib, k, name):
    z = golden("pstd_math.npz")
    inp, out = z["inputs"], z["outputs"]
    dev = pb.pstd_math_device(inp)[:, k]
    ref = out[:, k]
    if name in BITEXACT:
        same = (dev.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(dev) & np.isnan(ref))
        assert same.all(), f"{name}: {np.count_nonzero(~same)} of {same.size} differ"
        return
    a, b = inp[:, 0], inp[:, 1]
    dom = _domain(name, a, b)
    d = np.abs(dev.astype(np.float64) - ref) / np.maximum(1.0, np.abs(ref))
    assert np.nanmax(d[dom]) < (1e-5 if name == "tan" else 2e-6), name
