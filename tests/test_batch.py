"""Batches (lt_batch_*): many requests in one graph-captured persistent launch.

Every request's Hessian maps must equal, bit for bit, the single-grid call of the same
precision on the same inputs: the work-queue kernel evaluates each pixel with the same
pair loops, chunk order and epilogue (LT_FP32C: including the FP64 recomputation of the
pixels with |mu| above the flag threshold; LT_FP64: the reference-order Hessian).  The
deflection and potential planes agree to the compiler's FMA contraction
(conftest.plane_close)."""
import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

from conftest import plane_close

pytestmark = pytest.mark.gpu


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


def _same(got, exp, kind, precision):
    return plane_close(got, exp, kind, precision)


def _dev(g):
    import torch
    return torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda")


def _requests(seed=7):
    """Mixed requests: perturbed cluster catalogues, PIEMD/SIS variants, odd and even grids,
    Hessian maps, potential, deflection and Kmap mass and magnification maps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    base = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    cats = [catalog.perturb_catalog(base, rng) for _ in range(3)]
    cats.append(catalog.cluster_galaxy_catalog(1, 60, 11, cluster_type=catalog.PIEMD))
    sis = catalog.cluster_galaxy_catalog(1, 40, 12)
    sis.type[:] = 5
    sis = sis.sorted_by_type()
    cats.append(sis)
    grids = [catalog.Grid.square(100., 256), catalog.Grid(-100., 100., -80., 90., 131, 97),
             catalog.Grid.square(60., 192), catalog.Grid(-50., 50., -50., 50., 64, 200),
             catalog.Grid.square(30., 129)]
    specs = [
        (["kappa", "mu"], {}),
        (["kappa", "gamma1", "gamma2", "mu", "potential"], {}),
        (["deflection_x", "deflection_y", "ampli1"], {}),
        (["shear2", "ampli3", "hess_a", "hess_d"], {}),
        (["mass", "mu"], {"kmap": True, "mult": 0.37}),
    ]
    out = []
    for cat, g, (kinds, kw) in zip(cats, grids, specs):
        out.append((cat, g, kinds, kw))
    return out


def _single(ctx, cat, g, kinds, kw, precision, D=0.6, scale=1.3):
    """The same planes from the single-grid calls."""
    import torch
    res = {}
    hk = [k for k in kinds if k not in ("potential", "deflection_x", "deflection_y")]
    if hk:
        outs = [_dev(g) for _ in hk]
        ctx.hessian_maps(cat, g, hk, precision=precision, dlsds=D, kmap=kw.get("kmap", False),
                         mult=kw.get("mult", 1.0), out=outs)
        res.update(zip(hk, outs))
    if "potential" in kinds:
        o = _dev(g)
        ctx.potential_grid(cat, g, precision=precision, scale=scale, out=o)
        res["potential"] = o
    if "deflection_x" in kinds:
        ax, ay = _dev(g), _dev(g)
        ctx.gradient_grid(cat, g, precision=precision, scale=scale, out=(ax, ay))
        res["deflection_x"], res["deflection_y"] = ax, ay
    ctx.synchronize()
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in res.items()}


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_batch_equals_single_calls(ctx, precision):
    import torch
    ctx.synchronize()
    ctx.recompute_count()  # count from here on
    reqs, planes, expect = [], [], []
    for cat, g, kinds, kw in _requests():
        h = ctx.upload(cat)
        outs = {k: _dev(g) for k in kinds}
        reqs.append(lt.Request(h, g, outs, dlsds=0.6, scale=1.3, **kw))
        planes.append(outs)
        expect.append(_single(ctx, h, g, kinds, kw, precision))
    b = ctx.batch(reqs, precision=precision)
    assert len(b) == len(reqs)
    ctx.synchronize()
    single_recomputed = ctx.recompute_count()
    n0 = lt.launch_count()
    b.launch()
    ctx.synchronize()
    torch.cuda.synchronize()
    assert lt.launch_count() - n0 == 2  # queue reset + persistent kernel
    # the batch recomputes in FP64 exactly the pixels the single calls recomputed
    assert ctx.recompute_count() == single_recomputed
    if precision == "fp32c":
        assert single_recomputed > 0
    for i, (outs, exp) in enumerate(zip(planes, expect)):
        for k, o in outs.items():
            got = o.cpu().numpy()
            assert _same(got, exp[k], k, precision), (precision, i, k)
    # replaying the graph (outputs cleared first) gives the same planes
    for outs in planes:
        for o in outs.values():
            o.fill_(np.nan)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())  # the fills come before the batch's writes
    b.launch(stream=s)
    s.synchronize()
    ctx.synchronize()
    for i, (outs, exp) in enumerate(zip(planes, expect)):
        for k, o in outs.items():
            assert _same(o.cpu().numpy(), exp[k], k, precision), ("replay", precision, i, k)
    b.destroy()


def test_batch_many_small_items(ctx):
    """More requests than CTAs, uneven grids: every item is evaluated exactly once."""
    import torch
    rng = np.random.Generator(np.random.PCG64(3))
    base = catalog.cluster_galaxy_catalog(1, 30, 5)
    reqs, outs, cats, grids = [], [], [], []
    for i in range(400):
        c = ctx.upload(catalog.perturb_catalog(base, rng))
        n = int(rng.choice([8, 33, 64, 90]))
        g = catalog.Grid.square(40., n)
        o = {"kappa": _dev(g), "mu": _dev(g)}
        reqs.append(lt.Request(c, g, o, dlsds=0.7))
        outs.append(o)
        cats.append(c)
        grids.append(g)
    b = ctx.batch(reqs, precision="fp32c")
    b.launch()
    ctx.synchronize()
    torch.cuda.synchronize()
    for i in range(0, 400, 37):
        exp = _single(ctx, cats[i], grids[i], ["kappa", "mu"], {}, "fp32c", D=0.7)
        for k in ("kappa", "mu"):
            assert np.array_equal(outs[i][k].cpu().numpy(), exp[k]), (i, k)
    for o in outs:
        for v in o.values():
            assert not torch.isnan(v).any()
    b.destroy()


def test_batch_empty_catalogue(ctx):
    import torch
    empty = catalog.cluster_galaxy_catalog(1, 5, 1).subset(np.array([], dtype=np.int64))
    h = ctx.upload(empty)
    g = catalog.Grid.square(10., 48)
    o = {"kappa": _dev(g), "mu": _dev(g), "deflection_x": _dev(g)}
    b = ctx.batch([lt.Request(h, g, o, dlsds=0.5)], precision="fp32c")
    b.launch()
    ctx.synchronize()
    torch.cuda.synchronize()
    assert np.all(o["kappa"].cpu().numpy() == 0.)
    assert np.all(o["mu"].cpu().numpy() == 1.)
    assert np.all(o["deflection_x"].cpu().numpy() == 0.)
    b.destroy()


def test_batch_rejects_bad_requests(ctx):
    cat = ctx.upload(catalog.cluster_galaxy_catalog(1, 5, 1))
    g = catalog.Grid.square(10., 16)
    with pytest.raises(lt.LensError) as e:
        ctx.batch([lt.Request(cat, g, {"kappa": np.zeros((16, 16))})])  # host output
    assert e.value.status == 1
    with pytest.raises(lt.LensError) as e:
        ctx.batch([lt.Request(cat, g, {"kappa": _dev(g)})], precision="fp64fast")
    assert e.value.status == 1
    with pytest.raises(lt.LensError):
        ctx.batch([lt.Request(cat, g, {99: _dev(g)})])


def test_autotune_shape_is_applied_to_batches():
    """lt_autotune searches the FP32C configurations (pixels per thread, CTAs per SM,
    threads per CTA, halo records per stage) on a grid over the catalogue and keeps the
    fastest; the maps in the tuned configuration stay within 1e-6 of LT_FP64, and a batch
    built afterwards runs its persistent kernel with the tuned pixels per thread (its
    lt_batch_config) and equals the single calls in that configuration bit for bit."""
    import torch
    from conftest import max_rel_err
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    c = lt.Context(0)
    try:
        cat = c.upload(catalog.cluster_galaxy_catalog(2, 198, 20261203))
        default = c.kernel_config("fp32c", "hessian")
        ppt, cps, ms = c.autotune(cat, "fp32c", "hessian", grid_n=384)
        cfg = c.kernel_config("fp32c", "hessian")
        assert ms > 0 and (ppt, cps) == (cfg["pixels_per_thread"], cfg["ctas_per_sm"])
        assert cfg["threads"] in (128, 256) and cfg["chunk"] in (32, 64, 128)
        print("default", default, "tuned", cfg, f"{ms:.3f} ms")
        g = catalog.Grid(-100., 100., -100., 100., 300, 260)
        kinds = ["kappa", "gamma1", "mu"]
        tuned = _single(c, cat, g, kinds, {}, "fp32c", D=0.62)
        ref = _single(c, cat, g, kinds, {}, "fp64", D=0.62)
        mask = np.abs(ref["mu"]) <= 100
        for k in kinds:
            assert max_rel_err(tuned[k], ref[k], mask) <= 1e-6, k
        outs = {k: _dev(g) for k in kinds}
        b = c.batch([lt.Request(cat, g, outs, dlsds=0.62)], precision="fp32c")
        bc = b.config()
        assert bc["pixels_per_thread"] == cfg["pixels_per_thread"]
        b.launch()
        c.synchronize()
        torch.cuda.synchronize()
        for k in kinds:
            assert np.array_equal(outs[k].cpu().numpy(), tuned[k]), k
        b.destroy()
        # every built configuration can be set; unbuilt ones are refused
        c.set_kernel_config("fp32c", "hessian", 2, 3, 128, 32)
        with pytest.raises(lt.LensError):
            c.set_kernel_config("fp32c", "hessian", 2, 3, 256, 64)
        with pytest.raises(lt.LensError):
            c.set_kernel_config("fp64", "hessian", 2, 2, 128, 64)
    finally:
        c.close()
