"""bayes.dat rows applied on the device (lt_bayes_apply) against uploads of the state the
reference's own setbayesmapmodels produces for the same rows (pinned bit for bit by
test_bayes_oracle.py): with host rows the catalogues are the uploads' bit for bit, so
every map is identical; device rows (cos/sin of the angles taken on the device) agree to
the FP64 tolerance.  A batch graph over the catalogues sees each new set of rows."""
import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import bayes, catalog

from conftest import max_rel_err
from test_bayes_oracle import _model

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


def _fp64_class(st, types):
    """Halos the FP32C path sums in FP64 everywhere (b0 >= 5, rcore >= 1, epot < 1e-3)."""
    nsis = types != 5
    return (st["b0"] >= 5.) | (nsis & (st["rcore"] >= 1.)) | (nsis & (st["epot"] < 1e-3))


def test_rows_equal_reference_state_uploads(ctx):
    model, pots, cols, flags, pot_free, nh = _model(seed=4)
    rows = bayes.synthetic_rows(model, cols, 4, np.random.Generator(np.random.PCG64(21)), potfiles=pots)
    base = bayes.catalog_from_state(model, bayes.base_state(model, pots))
    cats = [ctx.upload(base) for _ in range(rows.shape[0])]
    b = ctx.bayes(model, cols, pots)
    b.apply(rows, cats)
    g = catalog.Grid.square(60., 160)
    base_class = _fp64_class(bayes.base_state(model, pots), model.type)
    for r in range(rows.shape[0]):
        st = bayes.reference_state(model, pots, cols, rows[r])
        fresh = ctx.upload(bayes.catalog_from_state(model, st))
        for prec in ("fp64", "fp32c"):
            got, exp = _maps(ctx, cats[r], g, prec), _maps(ctx, fresh, g, prec)
            same_class = np.array_equal(_fp64_class(st, model.type), base_class)
            for k, (a, e) in enumerate(zip(got, exp)):
                if prec == "fp64" or same_class:
                    assert np.array_equal(a, e), (r, prec, k)
                else:  # a halo left the FP32 class: its FP64 proxy sums it in FP64
                    assert max_rel_err(a, e) <= 1e-6, (r, prec, k)
    b.destroy()


def test_device_rows(ctx):
    import torch
    model, pots, cols, flags, pot_free, nh = _model(seed=5)
    rows = bayes.synthetic_rows(model, cols, 3, np.random.Generator(np.random.PCG64(22)), potfiles=pots)
    base = bayes.catalog_from_state(model, bayes.base_state(model, pots))
    cats = [ctx.upload(base) for _ in range(3)]
    b = ctx.bayes(model, cols, pots)
    b.apply(torch.tensor(rows, device="cuda"), cats)
    g = catalog.Grid.square(60., 128)
    for r in range(3):
        fresh = ctx.upload(bayes.catalog_from_state(model, bayes.reference_state(model, pots, cols, rows[r])))
        got, exp = _maps(ctx, cats[r], g, "fp64"), _maps(ctx, fresh, g, "fp64")
        for k in (0, 1, 2, 4, 5):
            assert max_rel_err(got[k], exp[k]) <= 1e-12, (r, k)
    b.destroy()


def test_batch_graph_sees_new_rows(ctx):
    import torch
    p = catalog.cluster_galaxy_parameters(2, 150, 9)
    model = bayes.model_from_parameters(p)
    n = model.n
    model.mag = np.concatenate([np.zeros(2), np.random.Generator(np.random.PCG64(1)).uniform(18., 23., n - 2)])
    pots = [bayes.Potfile(2, n - 2, mag0=20., sigma=150., cut=25., core=0.12)]
    B = bayes
    cols = bayes.columns_from_free([{B.X, B.Y, B.EMASS, B.THETA, B.RCORE, B.VDISP}] * 2, 0, [(True, True)])
    g = catalog.Grid.square(100., 128)
    rng = np.random.Generator(np.random.PCG64(3))
    rows = bayes.synthetic_rows(model, cols, 2, rng, potfiles=pots)
    cats = [ctx.upload(bayes.catalog_from_state(model, bayes.reference_state(model, pots, cols, rows[r])))
            for r in range(2)]
    outs = [{"kappa": torch.empty((128, 128), dtype=torch.float64, device="cuda")} for _ in range(2)]
    batch = ctx.batch([lt.Request(c, g, o, dlsds=0.6) for c, o in zip(cats, outs)], precision="fp64")
    b = ctx.bayes(model, cols, pots)
    for _ in range(3):
        rows = bayes.synthetic_rows(model, cols, 2, rng, potfiles=pots)
        b.apply(rows, cats)
        batch.launch()
        ctx.synchronize()
        for r in range(2):
            fresh = ctx.upload(bayes.catalog_from_state(model, bayes.reference_state(model, pots, cols, rows[r])))
            exp = torch.empty((128, 128), dtype=torch.float64, device="cuda")
            ctx.hessian_maps(fresh, g, ["kappa"], precision="fp64", dlsds=0.6, out=[exp])
            ctx.synchronize()
            assert np.array_equal(outs[r]["kappa"].cpu().numpy(), exp.cpu().numpy())
    batch.destroy()
    b.destroy()


def test_bad_rows_and_catalogues(ctx):
    model, pots, cols, flags, pot_free, nh = _model(seed=6)
    rows = bayes.synthetic_rows(model, cols, 1, np.random.Generator(np.random.PCG64(2)), potfiles=pots)
    base = bayes.catalog_from_state(model, bayes.base_state(model, pots))
    cat = ctx.upload(base)
    b = ctx.bayes(model, cols, pots)
    bad = rows.copy()
    rcut_col = int(np.where(cols[:, 0] == bayes.RCUT)[0][0])
    rc_col = int(np.where((cols[:, 0] == bayes.RCORE) & (cols[:, 1] == cols[rcut_col, 1]))[0][0])
    bad[0, rcut_col] = 0.5 * bad[0, rc_col]  # rcut < rcore for a dPIE
    b.apply(bad, [cat])
    with pytest.raises(lt.LensError) as e:
        ctx.synchronize()
    assert e.value.status == 3
    other = ctx.upload(catalog.cluster_galaxy_catalog(1, 10, 2))
    with pytest.raises(lt.LensError):
        b.apply(rows, [other])  # not the model's halos
    with pytest.raises(lt.LensError):
        ctx.bayes(model, np.array([[bayes.X, model.n]], np.int32), pots)  # no such halo
    with pytest.raises(lt.LensError):
        ctx.bayes(model, np.array([[bayes.VDISP, pots[0].first]], np.int32), pots)  # a potfile galaxy
    b.destroy()
