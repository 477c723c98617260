"""The FP64 reciprocal and reciprocal square root of the pair loops (hardware
approximation refined by one third-order step) against the correctly rounded 1/x and
1/sqrt(x), over the input range of the per-pair denominators."""
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


def _fast_math32(L, y, x):
    fp = C.POINTER(C.c_float)
    L.lt_eval_fast_math32.argtypes = [C.c_int, C.c_int, fp, fp, fp, fp, fp, fp]
    y = np.ascontiguousarray(y, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    outs = [np.empty(y.size, np.float32) for _ in range(4)]
    ptr = lambda a: a.ctypes.data_as(fp)  # noqa: E731
    assert L.lt_eval_fast_math32(0, y.size, ptr(y), ptr(x), *[ptr(o) for o in outs]) == 0
    return outs  # atan2 (own), atan2f (CUDA), sqrt(x), atanh(y)


def test_fp32_atan2_and_sqrt():
    """The FP32 atan2 of the compensated potential (own polynomial) against FP64 atan2 and
    CUDA's atan2f, and its approximate square root against FP64 sqrt, over the operand
    range of the pair loops (|x|, |y| in [1e-6, 1e3], every quadrant and the axes)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    L = lt.load_library()
    rng = np.random.default_rng(2)
    n = 400000
    y = (rng.standard_normal(n) * 10.0 ** rng.uniform(-6, 3, n)).astype(np.float32)
    x = (rng.standard_normal(n) * 10.0 ** rng.uniform(-6, 3, n)).astype(np.float32)
    y[:4] = [0., -0., 1., -1.]
    x[:4] = [1., -1., 0., 0.]
    own, cuda, _, _ = _fast_math32(L, y, x)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    err = np.abs(own.astype(np.float64) - ref)
    assert err.max() <= 4e-7
    assert np.max(err / np.maximum(np.abs(ref), 1e-30)) <= 4e-7
    assert np.max(np.abs(own.astype(np.float64) - cuda.astype(np.float64))) <= 6e-7
    ax = np.abs(x)
    big = ax > 1e-30
    rs = np.sqrt(ax[big].astype(np.float64))
    # sqrt of |x| (the loops take roots of non-negative operands only)
    _, _, sq2, _ = _fast_math32(L, y, ax)
    assert np.max(np.abs(sq2[big].astype(np.float64) - rs) / rs) <= 2.4e-7


def test_fp32_atanh_third():
    """The atanh polynomial of the FP32 deflection and potential (log(1 + t)/2 = atanh s for
    |s| <= 1/3) against FP64 atanh, relative error, over |s| in [1e-30, 1/3]."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    L = lt.load_library()
    rng = np.random.default_rng(3)
    m = np.concatenate([rng.uniform(0., 1. / 3., 200000), 10.0 ** rng.uniform(-30, np.log10(1. / 3.), 200000)])
    s = (m * np.where(rng.random(m.size) < 0.5, -1., 1.)).astype(np.float32)
    s = s[s != 0]
    s = s[np.abs(s) <= np.float32(1. / 3.)]
    th = _fast_math32(L, s, np.ones_like(s))[3]
    ref = np.arctanh(s.astype(np.float64))
    assert np.max(np.abs(th.astype(np.float64) - ref) / np.abs(ref)) <= 2.4e-7


def test_fp32_approx_rcp_rsqrt_log():
    """The approximate FP32 reciprocal, reciprocal square root and logarithm of the pair
    loops (the .ftz instruction forms) over normal operands from 1e-30 to 1e30: reciprocal
    and reciprocal square root within 2^-22 relative of the FP64 values, the logarithm (on
    its domain in the loops, x >= 2) within 3e-7 relative of FP64 log and of CUDA's logf."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    L = lt.load_library()
    fp = C.POINTER(C.c_float)
    L.lt_eval_approx32.argtypes = [C.c_int, C.c_int, fp, fp, fp, fp, fp]
    rng = np.random.default_rng(4)
    x = np.concatenate([10.0 ** rng.uniform(-30, 30, 300000), rng.uniform(2., 4., 100000),
                        np.array([1., 2., 3., 4., 1e30])]).astype(np.float32)
    outs = [np.empty(x.size, np.float32) for _ in range(4)]
    ptr = lambda a: a.ctypes.data_as(fp)  # noqa: E731
    assert L.lt_eval_approx32(0, x.size, ptr(x), *[ptr(o) for o in outs]) == 0
    rcp, rsq, lg, lg_cuda = (o.astype(np.float64) for o in outs)
    xd = x.astype(np.float64)
    assert np.max(np.abs(rcp * xd - 1.)) <= 2. ** -22
    assert np.max(np.abs(rsq * np.sqrt(xd) - 1.)) <= 2. ** -22
    dom = xd >= 2.
    ref = np.log(xd[dom])
    assert np.max(np.abs(lg[dom] - ref) / ref) <= 3e-7
    assert np.max(np.abs(lg[dom] - lg_cuda[dom]) / ref) <= 3e-7
