"""lt_hessian_maps_noalloc (the LT_FP32C Hessian-map call whose recomputation list is a
static device array) through the C ABI, against lt_hessian_maps in LT_FP32C on the same
inputs, on two calls in a row.  Same kernels, so the planes agree to the test tolerance
(1e-12 of max(|ref|, RMS); they are expected to be identical)."""
import ctypes as C

import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

from conftest import max_rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
KINDS = ("kappa", "gamma1", "gamma2", "mu", "ampli1")


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    lib = lt.load_library()
    fn = lib.lt_hessian_maps_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(lt._Grid), C.c_int32, C.c_double, C.c_double,
                   C.POINTER(lt._MapReq), C.c_int32, C.c_void_p]
    fn.restype = C.c_int
    ctx = lt.Context(0)
    yield ctx, fn
    ctx.close()


def _call(ctx, fn, cat, g, outs, D, kmap=0, mult=1.0):
    req = (lt._MapReq * len(outs))(*[lt._MapReq(lt.MAP[k], o.data_ptr()) for k, o in outs.items()])
    return fn(ctx.handle, cat.handle, C.byref(lt._grid(g)), kmap, D, mult, req, len(outs), None)


def test_noalloc_matches_hessian_maps_twice(env):
    import torch
    ctx, fn = env
    cat, _ = catalog.workload("maps_1000h_4096")
    g = catalog.Grid.square(150., 1024)
    dcat = ctx.upload(cat)
    D = 0.6
    ref = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in KINDS}
    ctx.hessian_maps(dcat, g, list(KINDS), precision="fp32c", dlsds=D, out=list(ref.values()))
    ctx.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items()}
    for call in range(2):
        outs = {k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda") for k in KINDS}
        st = _call(ctx, fn, dcat, g, outs, D)
        assert st == 0, (call, lt.STATUS.get(st), ctx._lib.lt_last_error(ctx.handle))
        ctx.synchronize()
        for k, v in outs.items():
            got = v.cpu().numpy()
            assert np.all(np.isfinite(got)), (call, k)
            assert max_rel_err(got, ref[k]) <= TOL, (call, k)


def test_noalloc_allocates_nothing_and_uses_its_list(env):
    """On a warmed context, repeated calls leave the device's free memory unchanged, and
    the grid has pixels near critical curves (|mu| > 100, always recomputed in FP64), so
    the equality with lt_hessian_maps shows the static list at work."""
    import torch
    ctx, fn = env
    cat, _ = catalog.workload("maps_1000h_4096")
    g = catalog.Grid.square(150., 1024)
    dcat = ctx.upload(cat)
    D = 0.6
    outs = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in KINDS}
    assert _call(ctx, fn, dcat, g, outs, D) == 0
    ctx.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _call(ctx, fn, dcat, g, outs, D) == 0
    ctx.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    mu = outs["mu"].cpu().numpy()
    assert np.count_nonzero(np.abs(mu) > 100) > 100


def test_noalloc_kmap(env):
    """The Kmap form (per-halo D_LS/D_OS weights, two source planes) against
    lt_hessian_maps with kmap, on two calls in a row."""
    import torch
    ctx, fn = env
    cat = catalog.cluster_galaxy_catalog(2, 300, 11)
    cat.dlsds = np.where(np.arange(cat.n) < 150, 0.55, 0.75)
    g = catalog.Grid.square(100., 768)
    dcat = ctx.upload(cat)
    kinds = ("hess_a", "hess_b", "mass", "mu")
    ref = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in kinds}
    ctx.hessian_maps(dcat, g, list(kinds), precision="fp32c", kmap=True, dlsds=1.0, mult=1.3,
                     out=list(ref.values()))
    ctx.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items()}
    for call in range(2):
        outs = {k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda") for k in kinds}
        st = _call(ctx, fn, dcat, g, outs, 1.0, kmap=1, mult=1.3)
        assert st == 0, (call, lt.STATUS.get(st), ctx._lib.lt_last_error(ctx.handle))
        ctx.synchronize()
        for k, v in outs.items():
            got = v.cpu().numpy()
            assert max_rel_err(got, ref[k]) <= TOL, (call, k)


def test_noalloc_rejects_what_it_cannot_serve(env):
    import torch
    ctx, fn = env
    dcat = ctx.upload(catalog.cluster_galaxy_catalog(1, 20, 3))
    big = catalog.Grid.square(100., 2049)  # above the 2048^2-pixel limit
    outs = {"kappa": torch.empty((8, 8), dtype=torch.float64, device="cuda")}
    assert _call(ctx, fn, dcat, big, outs, 0.6) == 1  # LT_ERR_INVALID_ARGUMENT
    assert b"limit" in ctx._lib.lt_last_error(ctx.handle)
    g = catalog.Grid.square(10., 16)
    host = np.zeros((16, 16))
    req = (lt._MapReq * 1)(lt._MapReq(lt.MAP["kappa"], host.ctypes.data))
    assert fn(ctx.handle, dcat.handle, C.byref(lt._grid(g)), 0, 0.6, 1.0, req, 1, None) == 1
