"""Strong-lensing chi2 on the GPU (lt_delense, lt_chi2, lt_chi2_batch) against the oracle
(itself pinned to the reference's delense_barycenter and chi_computation by
tests/test_chi2_oracle.py).

The GPU deflection grid agrees with the reference's to <= 1e-12; fed with the same
deflections, the GPU inclusion tests, barycentres and linking round exactly as the
reference's, so the predicted images must be identical and chi2 equal to 1e-12."""
import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog
from lenstool_hpc_b200.images import generate_systems

pytestmark = pytest.mark.gpu
FRAME = (-100., 100., -100., 100.)


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


@pytest.fixture(scope="module")
def setup(ctx):
    cat = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    ic = int(np.argmax(cat.b0))
    dcat = ctx.upload(cat)
    systems = generate_systems(lambda bx, by, dr: ctx.delense(dcat, FRAME, 1024, bx, by, dr), 10, 21, dr=0.6,
                               centre=(cat.position_x[ic], cat.position_y[ic]), source_radius=8.)
    return cat, dcat, systems


def test_delense_matches_oracle_on_the_same_deflections(ctx, setup, oracle_lib):
    cat, dcat, s = setup
    n = 300
    g = catalog.Grid(*FRAME, n, n)
    ax, ay = ctx.gradient_grid(dcat, g, precision="fp64")
    bx, by = s.source_x, s.source_y
    nf, fx, fy = ctx.delense(dcat, FRAME, n, bx, by, s.dr)
    onf, ofx, ofy = oracle_lib.delense(n, FRAME, ax, ay, bx, by, s.dr)
    assert np.array_equal(nf, onf)
    for k in range(s.nsys):
        assert np.array_equal(fx[k, :nf[k]], ofx[k, :nf[k]]) and np.array_equal(fy[k, :nf[k]], ofy[k, :nf[k]])
    assert np.all(nf >= 1)


@pytest.mark.parametrize("which", ["true", "perturbed"])
def test_chi2_matches_oracle(ctx, setup, oracle_lib, which):
    cat, dcat, s = setup
    model = cat if which == "true" else catalog.perturb_catalog(cat, np.random.Generator(np.random.PCG64(4)))
    n = 512
    chi, found = ctx.chi2(ctx.upload(model), FRAME, n, s)
    ref = oracle_lib.chi2(model, FRAME, n, s.nimg, s.x, s.y, s.dr)
    assert found == ref["images_found"]
    assert abs(chi - ref["chi2"]) <= 1e-12 * max(1., abs(ref["chi2"]))
    if which == "true":
        assert chi < 1000.


def test_chi2_batch_equals_single_models(ctx, setup):
    cat, dcat, s = setup
    rng = np.random.Generator(np.random.PCG64(8))
    models = [cat] + [catalog.perturb_catalog(cat, rng) for _ in range(5)]
    handles = [ctx.upload(m) for m in models]
    chi, found = ctx.chi2(handles, FRAME, 256, s)
    for m, h in enumerate(handles):
        c1, f1 = ctx.chi2(h, FRAME, 256, s)
        assert c1 == chi[m] and f1 == found[m]
    assert chi[0] == min(chi)


def test_chi2_rejects_bad_systems(ctx, setup):
    _, dcat, s = setup
    from lenstool_hpc_b200.images import ImageSystems
    bad = ImageSystems(np.array([0], np.int32), np.zeros(0), np.zeros(0), np.array([0.6]))
    with pytest.raises(lt.LensError) as e:
        ctx.chi2(dcat, FRAME, 64, bad)
    assert e.value.status == 1
    with pytest.raises(lt.LensError):
        ctx.chi2(dcat, (0., -1., 0., 1.), 64, s)


def test_chi2_fp32c_deflections(ctx, setup):
    """The deflection grid in LT_FP32C (within 1e-6 of the FP64 grid), the sources,
    delensing and chi2 in FP64.  A predicted image is the image-plane barycentre of a grid
    triangle whose source-plane image contains the source (src/delense_CPU.cpp:117-118), so
    the grid's deflections enter only through the inclusion tests: chi2 changes only where
    a source lies within ~1e-5" of a source-plane triangle's edge, which none of these
    models' sources does (the same images, chi2 equal well inside 1e-3)."""
    cat, dcat, s = setup
    rng = np.random.Generator(np.random.PCG64(9))
    handles = [dcat] + [ctx.upload(catalog.perturb_catalog(cat, rng)) for _ in range(7)]
    for n in (512, 1024):
        c64, f64 = ctx.chi2(handles, FRAME, n, s)
        c32, f32 = ctx.chi2(handles, FRAME, n, s, precision="fp32c")
        rel = np.abs(c32 - c64) / np.maximum(np.abs(c64), 1.)
        print(n, "found", f64.tolist(), f32.tolist(), "max rel chi2 diff", rel.max())
        assert np.array_equal(f32, f64)
        assert rel.max() <= 1e-3


def test_chi2_fp64fast_deflections(ctx, setup):
    """The deflection grid in LT_FP64_FAST (the dPIE deflection through log(1 + eps), within
    2e-12 of the reference's arithmetic), the rest as in LT_FP64: the same images found and
    chi2 within 1e-9 (a deflection change of 1e-12 moves no inclusion test here)."""
    cat, dcat, s = setup
    rng = np.random.Generator(np.random.PCG64(10))
    handles = [dcat] + [ctx.upload(catalog.perturb_catalog(cat, rng)) for _ in range(3)]
    c64, f64 = ctx.chi2(handles, FRAME, 512, s)
    cf, ff = ctx.chi2(handles, FRAME, 512, s, precision="fp64fast")
    rel = np.abs(cf - c64) / np.maximum(np.abs(c64), 1.)
    print("found", f64.tolist(), ff.tolist(), "max rel chi2 diff", rel.max())
    assert np.array_equal(ff, f64)
    assert rel.max() <= 1e-9
