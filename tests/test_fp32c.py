"""FP32-compensated maps against the FP64 path (itself pinned to the oracle by
test_gpu_parity.py).

Bound: per pixel |fp32c - fp64| <= 1e-6 * max(|fp64|, RMS(fp64 map)), pixels with
|mu| > 100 excluded (they are reported separately), as the accuracy target of the
compensated path states."""
import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

pytestmark = pytest.mark.gpu
TOL32 = 1e-6


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


def rel_errors(got, ref, mask):
    g = got[mask]
    r = ref[mask]
    rms = np.sqrt(np.mean(r * r))
    e = np.abs(g - r) / np.maximum(np.abs(r), rms)
    return float(e.max())


def _maps(ctx, cat, g, precision, D=0.6, kinds=("kappa", "gamma1", "gamma2", "mu")):
    import torch
    outs = [torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for _ in kinds]
    ctx.hessian_maps(cat, g, list(kinds), precision=precision, dlsds=D, out=outs)
    ctx.synchronize()
    return {k: o.cpu().numpy() for k, o in zip(kinds, outs)}


def test_fp32c_workload_maps(ctx):
    """The 1000-halo 4096^2 workload through the fused lens-maps call (the benchmarked
    step): kappa, gamma1, gamma2, mu and psi of LT_FP32C within 1e-6 of LT_FP64 (whose
    Hessian equals the reference's CPU arithmetic bit for bit and whose potential is the
    reference's pi05), pixels with |mu| > 100 reported on their own."""
    import torch
    from lenstool_hpc_b200.accuracy import map_errors
    cat, g = catalog.workload("maps_1000h_4096")
    dls, dos, _ = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos  # lens at z 0.35, sources at z 1.5, as in the benchmark
    dcat = ctx.upload(cat)
    names = ("kappa", "gamma1", "gamma2", "mu", "psi")
    res = {}
    for prec in ("fp64", "fp32c"):
        res[prec] = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in names}
        ctx.lens_maps(dcat, g, precision=prec, dlsds=D, out=res[prec])
        ctx.synchronize()
    errs = map_errors(res["fp32c"], res["fp64"])
    for k, e in errs.items():
        print(f"fp32c {k}: max {e['max']:.3e} rms {e['rms']:.3e} over {e['pixels']} px; |mu|>100: "
              f"max {e['max_mu_gt_cut']:.3e} rms {e['rms_mu_gt_cut']:.3e} over {e['pixels_mu_gt_cut']} px")
    for k in names:
        assert errs[k]["max"] <= TOL32, (k, errs[k])
    # the excluded pixels are few: the critical curves of a 4096^2 map
    assert errs["mu"]["pixels_mu_gt_cut"] < 1e-2 * g.npix
    # and their Hessian maps come from the FP64 recomputation (the closed forms in FP64)
    for k in ("kappa", "gamma1", "gamma2"):
        assert errs[k]["max_mu_gt_cut"] <= 1e-10, (k, errs[k])


@pytest.mark.parametrize("cluster_type", [81, 8, 5])
def test_fp32c_mixed_profiles(ctx, cluster_type):
    cat = catalog.cluster_galaxy_catalog(2, 150, 99, cluster_type=cluster_type)
    g = catalog.Grid.square(100., 512)
    m64 = _maps(ctx, cat, g, "fp64", kinds=("kappa", "gamma1", "gamma2", "mu", "ampli3", "shear2"))
    m32 = _maps(ctx, cat, g, "fp32c", kinds=("kappa", "gamma1", "gamma2", "mu", "ampli3", "shear2"))
    mask = np.isfinite(m64["mu"]) & (np.abs(m64["mu"]) <= 100)
    for k in m64:
        assert rel_errors(m32[k], m64[k], mask) <= TOL32, k


def test_fp32c_sis_galaxies_and_kmap(ctx):
    rng = np.random.default_rng(4)
    n = 120
    t = np.where(np.arange(n) < 60, 5, 81)
    cat = catalog.make_catalog(t, rng.uniform(-60, 60, n), rng.uniform(-60, 60, n),
                               np.exp(rng.uniform(np.log(80), np.log(300), n)), rng.uniform(0, 0.5, n),
                               rng.uniform(0, np.pi, n), rng.uniform(0.05, 0.2, n), rng.uniform(5, 50, n))
    cat.dlsds = np.where(np.arange(n) < 40, 0.5, 0.8)
    g = catalog.Grid.square(80., 384)
    import torch
    o64 = [torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for _ in range(3)]
    o32 = [torch.empty_like(o64[0]) for _ in range(3)]
    kinds = ["hess_a", "hess_b", "mass"]
    ctx.hessian_maps(cat, g, kinds, precision="fp64", kmap=True, mult=1.7, out=o64)
    ctx.hessian_maps(cat, g, kinds, precision="fp32c", kmap=True, mult=1.7, out=o32)
    ctx.synchronize()
    mask = np.ones((g.ny, g.nx), bool)
    for a, b, k in zip(o32, o64, kinds):
        assert rel_errors(a.cpu().numpy(), b.cpu().numpy(), mask) <= TOL32, k


def test_fp32c_host_outputs_and_potential(ctx):
    """lens_maps in FP32C through host buffers, the potential included."""
    cat = catalog.cluster_galaxy_catalog(2, 80, 7)
    g = catalog.Grid.square(100., 200)
    a = ctx.lens_maps(cat, g, precision="fp32c", dlsds=0.6)
    b = ctx.lens_maps(cat, g, precision="fp64", dlsds=0.6)
    mask = np.isfinite(b["mu"]) & (np.abs(b["mu"]) <= 100)
    for k in ("kappa", "gamma1", "gamma2", "mu"):
        assert rel_errors(a[k], b[k], mask) <= TOL32, k
    e = rel_errors(a["psi"], b["psi"], np.ones_like(mask))
    print("fp32c psi max rel err (82 halos):", e)
    assert e <= TOL32


@pytest.mark.parametrize("ptype", [81, 8, 5])
def test_fp32c_potential_single_galaxies(ctx, ptype):
    """The FP32 potential (deflection-based form) of lone galaxy-scale halos against the
    LT_FP64 potential (the reference's pi05), over mass ellipticities 0.02-0.6 and core /
    cut radii 0.01-0.8 / 5-50 arcsec (the FP32 class needs rc < 1), on a field reaching
    150 arcsec from the centre; every pixel counts (the FP64 fallback regions included;
    no pixel at a halo centre, where the reference's pi05 is 0/0)."""
    import torch
    cases = [(0.02, 0.1, 20.), (0.3, 0.05, 10.), (0.6, 0.01, 5.), (0.2, 0.8, 50.), (0.45, 0.3, 30.)]
    g = catalog.Grid(-150., 150., -150., 150., 301, 301)
    worst = 0.
    for i, (em, rc, rcut) in enumerate(cases):
        x0, y0 = 0.37 * (i + 1), -0.21 * (i + 1)
        cat = catalog.make_catalog([ptype], [x0], [y0], [120.], [em], [0.4 + 0.5 * i], [rc], [rcut])
        res = {}
        for prec in ("fp32c", "fp64"):
            psi = torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")
            ctx.potential_grid(cat, g, precision=prec, out=psi)
            ctx.synchronize()
            res[prec] = psi.cpu().numpy()
        e = rel_errors(res["fp32c"], res["fp64"], np.ones((g.ny, g.nx), bool))
        print(f"fp32c psi, lone type-{ptype} halo e_mass {em} rc {rc} rcut {rcut}: {e:.3e}")
        worst = max(worst, e)
        assert e <= TOL32, (ptype, em, rc, rcut, e)
    print(f"fp32c psi max rel err, lone type-{ptype} halos: {worst}")


@pytest.mark.parametrize("workload", ["grad_200h_1024", "maps_1000h_4096"])
def test_fp32c_deflection(ctx, workload):
    """FP32C deflection (core - cut difference as log(1 + eps) in FP32, cluster-scale
    halos and near-field pairs in FP64) against LT_FP64, on the workload catalogues over
    their fields at 768^2."""
    import torch
    cat, g0 = catalog.workload(workload)
    g = catalog.Grid(g0.xmin, g0.xmax, g0.ymin, g0.ymax, 768, 768)
    res = {}
    for prec in ("fp32c", "fp64"):
        ax = torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")
        ay = torch.empty_like(ax)
        ctx.gradient_grid(cat, g, precision=prec, out=(ax, ay))
        ctx.synchronize()
        res[prec] = (ax.cpu().numpy(), ay.cpu().numpy())
    mask = np.ones((g.ny, g.nx), bool)
    errs = [rel_errors(res["fp32c"][i], res["fp64"][i], mask) for i in range(2)]
    print(f"fp32c deflection max rel err {workload}: {errs}")
    for i in range(2):
        assert errs[i] <= TOL32, (workload, i)


def test_fp32c_per_term_errors_of_lone_galaxies(ctx):
    """The FP32 closed forms term by term: lone galaxy-scale cut dPIEs at random mass
    ellipticity (0.01-0.6), core (0.01-0.8") and cut (5-50") radii, each alone on a near
    field (4 rcut) and a far field (150"); outside the halo's FP64 disc every pixel is one
    FP32 term.  Relative errors against LT_FP64: convergence and the potential against
    their own values, the shear components against |gamma1| + |gamma2|, the deflection
    against |alpha|."""
    import torch
    rng = np.random.default_rng(7)
    worst = {"kappa": 0., "gamma": 0., "alpha": 0., "psi": 0.}
    n = 0
    while n < 16:
        sig = float(np.exp(rng.uniform(np.log(80), np.log(300))))
        em, th = float(rng.uniform(0.01, 0.6)), float(rng.uniform(0, np.pi))
        rc = float(np.exp(rng.uniform(np.log(0.01), np.log(0.8))))
        rcut = float(rng.uniform(5, 50))
        x0, y0 = float(rng.uniform(-1, 1)), float(rng.uniform(-1, 1))
        cat = catalog.make_catalog([81], [x0], [y0], [sig], [em], [th], [rc], [rcut])
        b0, e = float(cat.b0[0]), float(cat.ellipticity_potential[0])
        if b0 >= 5 or e < 1e-3:
            continue
        n += 1
        for half in (4 * rcut, 150.):
            g = catalog.Grid.square(half, 385)
            res = {}
            for prec in ("fp32c", "fp64"):
                o = [torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for _ in range(6)]
                ctx.hessian_maps(cat, g, ["hess_a", "hess_b", "hess_c"], precision=prec, out=o[:3])
                ctx.gradient_grid(cat, g, precision=prec, out=(o[3], o[4]))
                ctx.potential_grid(cat, g, precision=prec, out=o[5])
                ctx.synchronize()
                res[prec] = [x.cpu().numpy() for x in o]
            a, b, c, ax, ay, ps = res["fp64"]
            a2, b2, c2, ax2, ay2, ps2 = res["fp32c"]
            px, py = g.coords()
            r2 = (px.reshape(g.ny, g.nx) - x0) ** 2 + (py.reshape(g.ny, g.nx) - y0) ** 2
            m = r2 >= max(b0 / 0.2, 3 * rc) ** 2 * 1.001  # outside the FP64 disc
            k, k2 = (a + c) / 2, (a2 + c2) / 2
            g1, g12, g2, g22 = (a - c) / 2, (a2 - c2) / 2, b, b2
            errs = {"kappa": np.abs(k2 - k) / np.abs(k),
                    "gamma": np.maximum(np.abs(g12 - g1), np.abs(g22 - g2)) / (np.abs(g1) + np.abs(g2)),
                    "alpha": np.hypot(ax2 - ax, ay2 - ay) / np.hypot(ax, ay),
                    "psi": np.abs(ps2 - ps) / np.abs(ps)}
            for key, err in errs.items():
                worst[key] = max(worst[key], float(err[m].max()))
    print("fp32c per-term relative errors, lone dPIEs:", worst)
    assert worst["kappa"] <= 1.2e-6 and worst["gamma"] <= 1.2e-6
    assert worst["alpha"] <= 2e-6 and worst["psi"] <= 1.5e-6


@pytest.mark.parametrize("precision", ["fp32c", "fp64", "fp64fast"])
def test_host_outputs_in_bands_equal_device_outputs(ctx, precision):
    """Host-output calls run the grid in bands of rows (the copy of one band overlaps the next
    band's kernels); the bands start on the kernels' tile rows, so the maps equal a
    device-output call over the whole grid bit for bit."""
    import torch
    cat = catalog.cluster_galaxy_catalog(2, 120, 31)
    g = catalog.Grid(-90., 90., -60., 70., 600, 523)
    host = ctx.lens_maps(cat, g, precision=precision, dlsds=0.63)
    dev = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in host}
    ctx.lens_maps(cat, g, precision=precision, dlsds=0.63, out=dev)
    ctx.synchronize()
    for k in host:
        assert np.array_equal(host[k], dev[k].cpu().numpy()), (precision, k)


def test_recompute_count(ctx):
    """lt_recompute_count: the pixels a call recomputes in FP64 (its flagged pixels, some of
    this field's); a call without determinant-sensitive maps recomputes none."""
    cat, _ = catalog.workload("maps_1000h_4096")
    g = catalog.Grid.square(150., 512)
    dcat = ctx.upload(cat)
    ctx.recompute_count()
    _maps(ctx, dcat, g, "fp32c")
    n = ctx.recompute_count()
    print("recomputed", n, "of", g.npix)
    assert 0 < n < g.npix
    _maps(ctx, dcat, g, "fp32c", kinds=("kappa", "gamma1"))
    assert ctx.recompute_count() == 0


@pytest.mark.parametrize("seed", range(8))
def test_fp32c_random_fields_hold_the_bound(ctx, seed):
    """The error estimate (three standard deviations of the FP32 terms' independent errors,
    against a tolerance of half the target) over random cluster + galaxy fields of different
    richness and magnification: kappa, gamma1, gamma2 and mu within 1e-6 of LT_FP64 on a
    1024^2 grid, pixels with |mu| > 100 excluded."""
    rng = np.random.default_rng(100 + seed)
    nc = int(rng.integers(1, 5))
    ng = int(rng.integers(100, 800))
    cat = catalog.cluster_galaxy_catalog(nc, ng, 1000 + seed)
    g = catalog.Grid.square(float(rng.uniform(60., 160.)), 1024)
    D = float(rng.uniform(0.3, 0.9))
    dcat = ctx.upload(cat)
    m64 = _maps(ctx, dcat, g, "fp64", D=D)
    m32 = _maps(ctx, dcat, g, "fp32c", D=D)
    keep = np.abs(m64["mu"]) <= 100
    errs = {k: rel_errors(m32[k], m64[k], keep) for k in m32}
    print(seed, nc, ng, f"D={D:.2f}", "max errors", {k: f"{v:.2e}" for k, v in errs.items()},
          "|mu|>100 pixels", int((~keep).sum()))
    for k, e in errs.items():
        assert e <= TOL32, (k, e)


@pytest.mark.parametrize("nx,ny", [(1, 1), (1, 37), (41, 1), (3, 5), (65, 9), (130, 17)])
def test_fp32c_degenerate_grids(ctx, nx, ny):
    """Grids smaller than a tile or a warp's pixel box in either direction, with partial
    tiles at both edges: every map within the bound of LT_FP64 (the kernels clamp the
    pixels beyond the grid and store none of them), host and device outputs alike."""
    import torch
    cat = catalog.cluster_galaxy_catalog(2, 150, 77)
    g = catalog.Grid(-37.3, 25.1, -12.7, 31.9, nx, ny, dx=62.4 / max(nx - 1, 1), dy=44.6 / max(ny - 1, 1))
    dcat = ctx.upload(cat)
    kinds = ("kappa", "gamma1", "gamma2", "mu")
    m64 = _maps(ctx, dcat, g, "fp64", kinds=kinds)
    m32 = _maps(ctx, dcat, g, "fp32c", kinds=kinds)
    keep = np.abs(m64["mu"]) <= 100
    for k in kinds:
        assert m32[k].shape == (ny, nx)
        if keep.any():
            assert rel_errors(m32[k], m64[k], keep) <= TOL32, k
    host = ctx.lens_maps(dcat, g, precision="fp32c", dlsds=0.6)
    dev = {k: torch.empty((ny, nx), dtype=torch.float64, device="cuda") for k in host}
    ctx.lens_maps(dcat, g, precision="fp32c", dlsds=0.6, out=dev)
    ctx.synchronize()
    for k in host:
        assert np.array_equal(host[k], dev[k].cpu().numpy()), k
