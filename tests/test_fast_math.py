"""The FP64 reciprocal and reciprocal square root of the pair loops (hardware
approximation refined by two Newton-Raphson steps) against the correctly rounded
1/x and 1/sqrt(x), over the input range of the per-pair denominators."""
import ctypes as C

import numpy as np
import pytest

import lenstool_hpc_b200 as lt

pytestmark = pytest.mark.gpu


def ulp_diff(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_rcp_rsqrt_within_few_ulp():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    L = lt.load_library()
    dp = C.POINTER(C.c_double)
    L.lt_eval_fast_math.argtypes = [C.c_int, C.c_int, dp, dp, dp]
    rng = np.random.default_rng(1)
    x = np.concatenate([10.0 ** rng.uniform(-12, 12, 200000), rng.uniform(0.5, 2.0, 100000),
                        np.array([1.0, 2.0, 4.0, 0.25, 3.0, 1e-300, 1e300])])
    rcp = np.empty_like(x)
    rsq = np.empty_like(x)
    assert L.lt_eval_fast_math(0, x.size, x.ctypes.data_as(dp), rcp.ctypes.data_as(dp), rsq.ctypes.data_as(dp)) == 0
    assert ulp_diff(rcp, 1.0 / x).max() <= 2
    # reference 1/sqrt(x) in extended precision, rounded once
    ref = (1.0 / np.sqrt(x.astype(np.longdouble))).astype(np.float64)
    assert ulp_diff(rsq, ref).max() <= 2
