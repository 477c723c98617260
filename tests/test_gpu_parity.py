"""FP64 parity of the CUDA path (through the C ABI) with the reference's golden vectors
and the oracle.  Tolerance: |gpu - ref| <= 1e-12 * max(|ref|, RMS(map)) per pixel."""
import numpy as np
import pytest

from conftest import catalog_from_npz, golden, grid_from_npz, max_rel_err

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

pytestmark = pytest.mark.gpu
TOL = 1e-12


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


def test_kat_dpie95(ctx):
    z = golden("kat_dpie95.npz")
    cat = catalog_from_npz(z)
    px, py = float(z["px"]), float(z["py"])
    g = catalog.Grid(px, px + 1., py, py + 1., 1, 1, dx=1., dy=1.)
    ax, ay = ctx.gradient_grid(cat, g)
    want = z["lenstool_grad"]
    assert abs(ax[0, 0] - want[0]) <= 1e-12 * abs(want[0])
    assert abs(ay[0, 0] - want[1]) <= 1e-12 * abs(want[1])


@pytest.mark.parametrize("name", ["90Pot81", "90Pot", "90PotSIS", "MarkusBenchmark"])
def test_par_gradient(ctx, name):
    z = golden(f"par_{name}.npz")
    cat, g = catalog_from_npz(z), grid_from_npz(z)
    ax, ay = ctx.gradient_grid(cat, g)
    assert max_rel_err(ax, z["grad"][0]) <= TOL
    assert max_rel_err(ay, z["grad"][1]) <= TOL


def test_par_dpie_hessian_potential_kmap(ctx):
    z = golden("par_90Pot81.npz")
    cat, g = catalog_from_npz(z), grid_from_npz(z)
    m = ctx.hessian_maps(cat, g, ["hess_a", "hess_b", "hess_c", "hess_d", "ampli5"])
    for k, name in enumerate(["hess_a", "hess_b", "hess_c", "hess_d"]):
        # bit-identical to the reference's gradient2_grid_CPU
        assert np.array_equal(m[name], z["hess"][k]), name
    assert max_rel_err(m["ampli5"], z["amplif5"]) <= TOL
    psi = ctx.potential_grid(cat, g)
    assert max_rel_err(psi, z["pot"]) <= TOL
    kcat = catalog_from_npz(z)
    kcat.dlsds = np.array(z["kmap_dlsds"])
    mk = ctx.hessian_maps(kcat, g, ["hess_a", "hess_b", "hess_c", "hess_d"], kmap=True)
    for k, name in enumerate(["hess_a", "hess_b", "hess_c", "hess_d"]):
        # bit-identical to the reference's Kmap kernel (run on the host)
        assert np.array_equal(mk[name], z["kmap"][k]), name


def _cat(cluster_type=81, n_gal=198, seed=20261203):
    return catalog.cluster_galaxy_catalog(2, n_gal, seed, cluster_type=cluster_type)


@pytest.mark.parametrize("cluster_type", [81, 8, 5])
@pytest.mark.parametrize("shape", [(128, 96, 0, 0), (77, 51, 3, 5), (1, 1, 0, 0), (130, 9, 0, 2)])
def test_grid_vs_oracle(ctx, oracle_lib, cluster_type, shape):
    nx, ny, i0, j0 = shape
    cat = _cat(cluster_type, n_gal=60)
    g = catalog.Grid(-100., 100., -90., 80., nx, ny, i0, j0, dx=200. / 127, dy=170. / 95)
    ax, ay = ctx.gradient_grid(cat, g)
    ox, oy = oracle_lib.grad_grid(cat, g)
    assert max_rel_err(ax, ox) <= TOL and max_rel_err(ay, oy) <= TOL
    # LT_FP64_FAST: the dPIE deflection as log(1 + eps) away from its 0/0 points
    fx, fy = ctx.gradient_grid(cat, g, precision="fp64fast")
    assert max_rel_err(fx, ox) <= TOL and max_rel_err(fy, oy) <= TOL
    h = ctx.hessian_maps(cat, g, ["hess_a", "hess_b", "hess_c", "hess_d"])
    oh = oracle_lib.hess_grid(cat, g)
    for k, name in enumerate(["hess_a", "hess_b", "hess_c", "hess_d"]):
        # LT_FP64 reproduces the reference's rounding sequence: bit-identical planes
        assert np.array_equal(h[name], oh[k]), (name, max_rel_err(h[name], oh[k]))
    hf = ctx.hessian_maps(cat, g, ["hess_a", "hess_b", "hess_c"], precision="fp64fast")
    for k, name in enumerate(["hess_a", "hess_b", "hess_c"]):
        assert max_rel_err(hf[name], oh[k]) <= TOL, name
    psi = ctx.potential_grid(cat, g)
    opsi = oracle_lib.pot_grid(cat, g)
    assert max_rel_err(psi, opsi) <= TOL
    # LT_FP64_FAST takes the potential through the deflection (N+- form near its 0/0 points)
    assert max_rel_err(ctx.potential_grid(cat, g, precision="fp64fast"), opsi) <= TOL


@pytest.mark.parametrize("ptype", [81, 8])
def test_fp64fast_potential_near_removable_points(ctx, oracle_lib, ptype):
    """LT_FP64_FAST takes the potential through the deflection (x . alpha plus one log per
    radius), whose complex quotients are 0/0 at u = 0, v = 2 sqrt(e) r.  It keeps the N+-
    form within 0.0316 rc of the core point and within 0.02 rcut of the cut point, and
    (dPIE) takes log z_c - log z_t within 0.02 rcut of the core point.
    Pixels on the points and at offsets from 1e-12 r up to beyond each switch, on both
    sides of it, each relative to its own value, against pi05 in extended precision (the
    oracle's x87 build): the reference's pi05 in FP64 is itself off by up to ~1e-12 of
    the small potential close to a dPIE's centre."""
    import oracle
    x0, y0, ang = 3.3, -1.7, 0.7
    rc, rcut = 0.4, 15.
    cat = catalog.make_catalog([ptype], [x0], [y0], [180.], [0.3], [ang], [rc], [rcut])
    e = float(cat.ellipticity_potential[0])
    cs, sn = float(cat.anglecos[0]), float(cat.anglesin[0])
    # (radius of the point, switch radii around it)
    points = [(rc, [0.0316 * rc, 0.02 * rcut]), (rcut, [0.02 * rcut])] if ptype == 81 else [(rc, [0.0316 * rc])]
    for r, edges in points:
        offsets = [0., 1e-12 * r, 1e-8 * r, 1e-5 * r, 3e-3 * r] + [f * x for x in edges for f in (0.99, 1.01, 1.5)]
        pts = []
        for d in offsets:
            for a in np.linspace(0., 2. * np.pi, 5, endpoint=False):
                u = d * np.cos(a)
                v = 2. * np.sqrt(e) * r + d * np.sin(a)
                pts.append((x0 + u * cs - v * sn, y0 + u * sn + v * cs))
        px = np.array([p[0] for p in pts])
        py = np.array([p[1] for p in pts])
        got = np.array([ctx.potential_grid(cat, catalog.Grid(x, x + 1., y, y + 1., 1, 1, dx=1., dy=1.),
                                           precision="fp64fast")[0, 0] for x, y in zip(px, py)])
        want = oracle.Oracle(oracle.ORACLE_LD_SO).pot_points(cat, px, py)
        err = np.abs(got - want) / np.abs(want)
        assert err.max() <= TOL, (ptype, r, err.max(), offsets[int(np.argmax(err)) // 5])
        # and the FP64 oracle (pi05 as the reference rounds it) agrees to its own error
        ref64 = oracle_lib.pot_points(cat, px, py)
        assert np.max(np.abs(got - ref64) / np.abs(ref64)) <= 2e-12


def test_fp64fast_deflection_workload(ctx):
    """LT_FP64_FAST deflection (log(1 + eps) for dPIE pairs, the reference's form within
    0.02 rcut of the 0/0 points) against LT_FP64 on the 1000-halo workload field at 768^2."""
    import torch
    cat, g0 = catalog.workload("maps_1000h_4096")
    g = catalog.Grid(g0.xmin, g0.xmax, g0.ymin, g0.ymax, 768, 768)
    res = {}
    for prec in ("fp64", "fp64fast"):
        ax = torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")
        ay = torch.empty_like(ax)
        ctx.gradient_grid(cat, g, precision=prec, out=(ax, ay))
        ctx.synchronize()
        res[prec] = (ax.cpu().numpy(), ay.cpu().numpy())
    for i in range(2):
        assert max_rel_err(res["fp64fast"][i], res["fp64"][i]) <= TOL, i


def test_every_map_kind_vs_oracle(ctx, oracle_lib):
    cat = _cat(81, n_gal=80)
    g = catalog.Grid.square(60., 64)
    D = 0.62
    a, b, c, d = oracle_lib.hess_grid(cat, g)
    kinds = ["ampli1", "ampli2", "ampli3", "ampli4", "ampli5", "ampli6", "shear1", "shear2"]
    m = ctx.hessian_maps(cat, g, kinds, dlsds=D)
    for k in kinds:
        ref = oracle_lib.map(k, a, b, c, D).reshape(g.ny, g.nx)
        if k == "ampli3":
            # -2.5 log10|det|: CUDA's log10 and the C library's are each within a couple
            # of ulp of the exact value, so the two agree to a few ulp of the result
            assert max_rel_err(m[k], ref) <= TOL, k
        else:
            # every other kind is +, -, *, / and sqrt, correctly rounded on both sides, in
            # the reference's operation order on identical Hessian planes
            assert np.array_equal(m[k], ref), (k, max_rel_err(m[k], ref))
    kinds = ["shear3", "shear4", "kappa", "gamma1", "gamma2", "mu", "mass"]
    m = ctx.hessian_maps(cat, g, kinds, dlsds=D, mult=3.5)
    for k in kinds:
        ref = oracle_lib.map("scale" if k == "mass" else k, a, b, c, D, 3.5).reshape(g.ny, g.nx)
        assert np.array_equal(m[k], ref), (k, max_rel_err(m[k], ref))


def test_lens_maps_fused_equals_separate(ctx, oracle_lib):
    cat = _cat(81, n_gal=100)
    g = catalog.Grid.square(150., 96)
    D = 0.7
    out = ctx.lens_maps(cat, g, dlsds=D)
    a, b, c, d = oracle_lib.hess_grid(cat, g)
    for k in ("kappa", "gamma1", "gamma2", "mu"):
        ref = oracle_lib.map(k, a, b, c, D).reshape(g.ny, g.nx)
        assert np.array_equal(out[k], ref), (k, max_rel_err(out[k], ref))
    assert max_rel_err(out["psi"], D * oracle_lib.pot_grid(cat, g)) <= TOL


@pytest.mark.parametrize("precision", ["fp64", "fp64fast"])
def test_c0_gradient_full_grid_vs_reference(ctx, ref_lib, precision):
    """The plain FP64 deflection workload at its own size: 200 halos (2 PIEMD cluster
    halos + 198 cut-dPIE galaxies) on the full 1024^2 grid over 200"x200", against the
    reference's own gradient_grid_CPU (src/grid_gradient_CPU.cpp:33-100, compiled from its
    sources) at 1e-12 of max(|ref|, RMS) on every pixel."""
    import torch
    cat, g = catalog.workload("grad_200h_1024")
    assert (cat.n, g.nx, g.ny) == (200, 1024, 1024)
    ax = torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")
    ay = torch.empty_like(ax)
    ctx.gradient_grid(cat, g, precision=precision, out=(ax, ay))
    ctx.synchronize()
    rx, ry = ref_lib.grad_grid(cat, g)
    ex = max_rel_err(ax.cpu().numpy(), rx)
    ey = max_rel_err(ay.cpu().numpy(), ry)
    print(f"C0 {precision}: max rel err alpha_x {ex:.3e} alpha_y {ey:.3e}")
    assert ex <= TOL and ey <= TOL


def test_device_outputs_and_stream(ctx, oracle_lib):
    import torch
    cat = _cat(81, n_gal=50)
    g = catalog.Grid.square(100., 100)
    s = torch.cuda.Stream()
    ax = torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")
    ay = torch.empty_like(ax)
    dcat = ctx.upload(cat)
    ctx.gradient_grid(dcat, g, out=(ax, ay), stream=s)
    ctx.synchronize(s)
    ox, oy = oracle_lib.grad_grid(cat, g)
    assert max_rel_err(ax.cpu().numpy(), ox) <= TOL
    assert max_rel_err(ay.cpu().numpy(), oy) <= TOL


def test_kmap_multi_plane_vs_oracle(ctx, oracle_lib):
    cat = _cat(81, n_gal=90)
    rng = np.random.default_rng(5)
    cat.dlsds = np.repeat(rng.uniform(0.3, 0.9, 4), [2, 30, 30, 30])
    g = catalog.Grid.square(80., 48)
    m = ctx.hessian_maps(cat, g, ["hess_a", "hess_b", "hess_c", "mass"], kmap=True, mult=2.)
    oh = oracle_lib.hess_grid(cat, g, kmap=True)
    assert np.array_equal(m["hess_a"], oh[0])
    assert np.array_equal(m["hess_b"], oh[1])
    assert np.array_equal(m["hess_c"], oh[2])
    assert max_rel_err(m["mass"], (oh[0] + oh[2]) * 0.5 * 2.) <= 1e-12


def test_empty_and_single_halo(ctx, oracle_lib):
    g = catalog.Grid.square(10., 16)
    empty = _cat(81, n_gal=10).subset(np.array([], dtype=np.int64))
    ax, ay = ctx.gradient_grid(empty, g)
    assert not ax.any() and not ay.any()
    m = ctx.hessian_maps(empty, g, ["mu", "kappa", "ampli3"], dlsds=0.5)
    assert np.all(m["mu"] == 1.) and not m["kappa"].any() and not m["ampli3"].any()
    one = _cat(81, n_gal=10).subset(np.array([3]))
    ox, oy = oracle_lib.grad_grid(one, g)
    ax, ay = ctx.gradient_grid(one, g)
    assert max_rel_err(ax, ox) <= TOL and max_rel_err(ay, oy) <= TOL


def test_errors_are_statuses(ctx):
    g = catalog.Grid.square(10., 8)
    bad = _cat(81, n_gal=10)
    bad.type = bad.type.copy()
    bad.type[4] = 14
    with pytest.raises(lt.LensError) as e:
        ctx.upload(bad)
    assert e.value.status == 2
    nan = _cat(81, n_gal=10)
    nan.b0 = nan.b0.copy()
    nan.b0[2] = np.nan
    with pytest.raises(lt.LensError) as e:
        ctx.upload(nan)
    assert e.value.status == 3
    cut = _cat(81, n_gal=10)
    cut.rcut = cut.rcore.copy()
    with pytest.raises(lt.LensError) as e:
        ctx.upload(cut)
    assert e.value.status == 3
    with pytest.raises(lt.LensError) as e:
        ctx.hessian_maps(_cat(81, n_gal=3), g, [99])
    assert e.value.status == 1
    small = lt.Context(0, budget_bytes=4096)
    with pytest.raises(lt.LensError) as e:
        small.upload(_cat(81, n_gal=500))
    assert e.value.status == 6
    small.close()


def _c1_subsample(cat, g):
    rng = np.random.default_rng(20261204)
    idx = rng.choice(g.npix, 65536, replace=False)
    near = []
    for x0, y0, rc in zip(cat.position_x, cat.position_y, cat.rcore):
        i = int(round((x0 - g.xmin) / g.dx)); j = int(round((y0 - g.ymin) / g.dy))
        r = int(np.ceil(3 * rc / g.dx)) + 1
        for jj in range(max(0, j - r), min(g.ny, j + r + 1)):
            for ii in range(max(0, i - r), min(g.nx, i + r + 1)):
                near.append(jj * g.nx + ii)
    return np.unique(np.concatenate([idx, np.array(near, np.int64)]))


def test_c1_scale_subsample_fp64_exact(ctx, oracle_lib):
    """1000 halos on the 4096^2 grid, LT_FP64: kappa, gamma1, gamma2 equal the reference's
    FP64 arithmetic bit for bit on a pixel subsample (65536 seeded pixels plus every
    pixel within 3 rcore of a halo centre)."""
    import torch
    cat, g = catalog.workload("maps_1000h_4096")
    D = 0.6
    outs = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in ("kappa", "gamma1", "gamma2")}
    ctx.hessian_maps(ctx.upload(cat), g, list(outs), dlsds=D, out=list(outs.values()))
    ctx.synchronize()
    idx = _c1_subsample(cat, g)
    px, py = g.coords(idx)
    a, b, c, d = oracle_lib.hess_points(cat, px, py)
    for k, ref in (("kappa", (a + c) * D / 2), ("gamma1", (a - c) * D / 2), ("gamma2", b * D)):
        got = outs[k].cpu().numpy().ravel()[idx]
        assert np.array_equal(got, ref), (k, int((got != ref).sum()))


def test_c1_scale_subsample_fp64_fast(ctx, oracle_lib):
    """LT_FP64_FAST on the same subsample: within 1e-12 except where the reference formula
    is ill-conditioned (bounded by its measured conditioning)."""
    import torch
    cat, g = catalog.workload("maps_1000h_4096")
    D = 0.6
    outs = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in ("kappa", "gamma1", "gamma2")}
    ctx.hessian_maps(ctx.upload(cat), g, list(outs), precision="fp64fast", dlsds=D, out=list(outs.values()))
    ctx.synchronize()
    idx = _c1_subsample(cat, g)
    px, py = g.coords(idx)
    a, b, c, d = oracle_lib.hess_points(cat, px, py)
    # The reference formula is ill-conditioned within ~1e-3" of each halo's removable
    # singular points (0, 2 r sqrt(eps)) of the halo frame: there a 1-ulp change of the
    # pixel coordinate moves the reference's own result by up to ~1e-8, and its FP64
    # rounding error (measured against the extended-precision build of the oracle)
    # grows alike; LT_FP64_FAST rounds differently (as accurately on average), so near
    # those points each pixel is held to 1e-11 plus 64x the larger of the two.
    import oracle
    ext = oracle.Oracle(oracle.ORACLE_LD_SO).hess_points(cat, px, py)
    pert = [oracle_lib.hess_points(cat, np.nextafter(px, s * np.inf), py) for s in (1, -1)]
    pert += [oracle_lib.hess_points(cat, px, np.nextafter(py, s * np.inf)) for s in (1, -1)]
    pert.append(ext)
    for k, f in (("kappa", lambda h: (h[0] + h[2]) * D / 2), ("gamma1", lambda h: (h[0] - h[2]) * D / 2),
                 ("gamma2", lambda h: h[1] * D)):
        ref = f((a, b, c, d))
        got = outs[k].cpu().numpy().ravel()[idx]
        full = outs[k].cpu().numpy()
        rms = float(np.sqrt(np.mean(full * full)))
        den = np.maximum(np.abs(ref), rms)
        sens = np.max([np.abs(f(p) - ref) for p in pert], axis=0) / den
        err = np.abs(got - ref) / den
        bad = np.flatnonzero(err > 10 * TOL + 64 * sens)
        assert bad.size == 0, (k, [(float(err[i]), float(sens[i]), float(px[i]), float(py[i])) for i in bad[:5]])
        # away from those points: 2e-12 (the fast path's reciprocals are refined to a few
        # ulp, not correctly rounded)
        assert np.max(err[sens < 1e-14]) <= 2 * TOL, k
        print(k, "max err", float(err.max()), "pixels above 1e-12:", int((err > TOL).sum()))
