"""Posterior samples applied on the device (lt_catalog_update) against a fresh upload of
the same sample: with the host's cos/sin the re-packed records are the upload's bit for
bit, so every map is identical; with the device's own cos/sin they agree to the
rounding of cos/sin.  A batch graph holding the catalogue sees the update; a sample that
changes a halo's FP32C class or leaves a profile's domain is reported."""
import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

from conftest import max_rel_err

pytestmark = pytest.mark.gpu
KINDS = ["kappa", "gamma1", "gamma2", "mu"]


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    c = lt.Context(0)
    yield c
    c.close()


def _maps(ctx, cat, g, prec):
    import torch
    outs = [torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for _ in KINDS]
    ctx.hessian_maps(cat, g, KINDS, precision=prec, dlsds=0.6, out=outs)
    ax, ay = (torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for _ in range(2))
    ctx.gradient_grid(cat, g, precision=prec, out=(ax, ay))
    ctx.synchronize()
    return [o.cpu().numpy() for o in outs + [ax, ay]]


@pytest.mark.parametrize("cluster_type", [catalog.DPIE, catalog.PIEMD])
def test_update_equals_upload(ctx, cluster_type):
    rng = np.random.Generator(np.random.PCG64(12))
    base = catalog.cluster_galaxy_parameters(2, 120, 31, cluster_type=cluster_type)
    sample = base.perturbed(rng)
    g = catalog.Grid.square(100., 200)
    d = ctx.upload(base.catalog())
    fresh = ctx.upload(sample.catalog())
    d.update(*sample.update_args())
    for prec in ("fp64", "fp32c"):
        got, exp = _maps(ctx, d, g, prec), _maps(ctx, fresh, g, prec)
        for k, (a, b) in enumerate(zip(got, exp)):
            assert np.array_equal(a, b), (prec, k)
    # cos/sin of the angle computed on the device (CUDA's sincos, within 2 ulp of the host's):
    # the rotated coordinates of pixels near a halo's axis amplify that rounding, so the maps
    # agree to the FP64 path's tolerance, 1e-12, not bit for bit
    d2 = ctx.upload(base.catalog())
    d2.update(*sample.update_args()[:7])
    got, exp = _maps(ctx, d2, g, "fp64"), _maps(ctx, fresh, g, "fp64")
    for k, (a, b) in enumerate(zip(got[:3] + got[4:], exp[:3] + exp[4:])):
        assert max_rel_err(a, b) <= 1e-12, k


def test_update_under_a_batch_graph(ctx):
    import torch
    rng = np.random.Generator(np.random.PCG64(5))
    base = catalog.cluster_galaxy_parameters(2, 80, 7)
    g = catalog.Grid.square(100., 128)
    d = ctx.upload(base.catalog())
    out = {"kappa": torch.empty((128, 128), dtype=torch.float64, device="cuda")}
    b = ctx.batch([lt.Request(d, g, out, dlsds=0.6)], precision="fp32c")
    for _ in range(3):
        sample = base.perturbed(rng)
        d.update(*sample.update_args())
        b.launch()
        ctx.synchronize()
        exp = torch.empty((128, 128), dtype=torch.float64, device="cuda")
        ctx.hessian_maps(ctx.upload(sample.catalog()), g, ["kappa"], precision="fp32c", dlsds=0.6, out=[exp])
        ctx.synchronize()
        assert np.array_equal(out["kappa"].cpu().numpy(), exp.cpu().numpy())
    b.destroy()


def test_update_class_change_and_domain(ctx):
    base = catalog.cluster_galaxy_parameters(1, 20, 3)
    d = ctx.upload(base.catalog())
    big = base.perturbed(np.random.Generator(np.random.PCG64(1)), rel=0.)
    big.vdisp[5] = 3000.   # a galaxy becomes cluster-scale (b0 >= 5"): leaves the FP32 class
    big.ellipticity[7] = 0.  # nearly circular (epot 1e-5 < 1e-3): leaves the FP32 class
    d.update(*big.update_args())
    g = catalog.Grid.square(100., 200)
    fresh = ctx.upload(big.catalog())
    got, exp = _maps(ctx, d, g, "fp32c"), _maps(ctx, fresh, g, "fp64")
    mu = exp[3]
    mask = np.isfinite(mu) & (np.abs(mu) <= 100)
    for k, (a, b) in enumerate(zip(got, exp)):  # FP64 proxies: the FP32C bound
        assert max_rel_err(a, b, mask) <= 1e-6, k
    bad = base.perturbed(np.random.Generator(np.random.PCG64(1)), rel=0.)
    bad.rcut[3] = bad.rcore[3] * 0.5  # rcut < rcore
    d.update(*bad.update_args())
    with pytest.raises(lt.LensError) as e:
        ctx.synchronize()
    assert e.value.status == 3
    with pytest.raises(lt.LensError):
        d.update(*[a[:-1] for a in base.update_args()[:7]])  # wrong length is caught on the host
