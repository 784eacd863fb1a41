"""The table-driven FP64 exp of the evaluation kernels (csrc/fexp.cuh, Tang's
method) against the CUDA library exp and the host libm exp: at most 2 ulp
apart over [-700, 700] (both references are within 1 ulp of exp)."""
import numpy as np
import pytest

import closures_b200 as cb

pytestmark = pytest.mark.gpu


def ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_fast_exp_accuracy():
    rng = np.random.default_rng(3)
    x = np.concatenate([np.linspace(-700.0, 700.0, 1_000_001),
                        rng.uniform(-1.0, 1.0, 500_000),
                        rng.uniform(-60.0, 5.0, 500_000),
                        np.array([0.0, -0.0, 1e-300, -1e-300, np.log(2.0), -np.log(2.0),
                                  700.0, -700.0, 709.0, -745.0, 710.0])])
    fast, ref = cb.exp_check(x)
    ok = np.isfinite(ref) & (ref > 0)
    assert ulps(fast[ok], ref[ok]).max() <= 2
    assert ulps(fast[ok], np.exp(x[ok])).max() <= 2
    assert ulps(fast[ok], ref[ok]).mean() < 0.5
    # outside the table range the library exp is used
    big = np.abs(x) > 700
    assert (fast[big] == ref[big]).all()
