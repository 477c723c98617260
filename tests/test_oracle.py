"""The oracle (oracle/lt_oracle.c) pinned against the reference's golden vectors, the
reference's own code (oracle/_ref), and -- for the restated pieces -- finite differences.
CPU only."""
import math

import numpy as np
import pytest

from conftest import catalog_from_npz, golden, grid_from_npz, max_rel_err

from lenstool_hpc_b200 import catalog, cosmo


def test_kat_dpie95_matches_lenstool(oracle_lib):
    """Benchmarks/GradientBenchmark/setup.cpp:19-44: 95 dPIE halos, one point, Lenstool's
    deflection (-77.124413458712169, -46.092652444451353)."""
    z = golden("kat_dpie95.npz")
    cat = catalog_from_npz(z)
    ax, ay = oracle_lib.grad_points(cat, np.array([float(z["px"])]), np.array([float(z["py"])]))
    want = z["lenstool_grad"]
    assert abs(ax[0] - want[0]) <= 1e-13 * abs(want[0])
    assert abs(ay[0] - want[1]) <= 1e-13 * abs(want[1])
    # and the reference's own SoA code gave the same
    assert np.allclose([ax[0], ay[0]], z["reference_grad"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("name", ["90Pot81", "90Pot", "90PotSIS", "MarkusBenchmark"])
def test_par_fixture_gradient(oracle_lib, name):
    z = golden(f"par_{name}.npz")
    cat, g = catalog_from_npz(z), grid_from_npz(z)
    ax, ay = oracle_lib.grad_grid(cat, g)
    assert max_rel_err(ax, z["grad"][0]) <= 1e-14
    assert max_rel_err(ay, z["grad"][1]) <= 1e-14


def test_par_fixture_dpie_hessian_potential_kmap(oracle_lib):
    z = golden("par_90Pot81.npz")
    cat, g = catalog_from_npz(z), grid_from_npz(z)
    h = oracle_lib.hess_grid(cat, g)
    for k in range(4):
        assert max_rel_err(h[k], z["hess"][k]) <= 1e-14
        # reference GPU Hessian kernel, elliptical branch for every halo here (eps > 1e-4)
        assert max_rel_err(h[k], z["gpu_hess"][k]) <= 1e-13
    psi = oracle_lib.pot_grid(cat, g)
    assert max_rel_err(psi, z["pot"]) <= 1e-14
    kcat = catalog_from_npz(z)
    kcat.dlsds = np.array(z["kmap_dlsds"])
    hk = oracle_lib.hess_grid(kcat, g, kmap=True)
    for k in range(4):
        assert max_rel_err(hk[k], z["kmap"][k]) <= 1e-13
    k5 = oracle_lib.map("ampli5", *h[:3]).reshape(g.ny, g.nx)
    assert max_rel_err(k5, z["amplif5"]) <= 1e-14


def _c0_catalog(cluster_type=81, n_gal=40):
    return catalog.cluster_galaxy_catalog(2, n_gal, 20261203, cluster_type=cluster_type)


def test_reference_library_agrees_on_mixed_types(oracle_lib, ref_lib):
    """C0-like catalogue with two PIEMD (type 8) cluster halos and dPIE galaxies: two runs."""
    cat = _c0_catalog(cluster_type=8)
    g = catalog.Grid.square(100., 24)
    ax, ay = oracle_lib.grad_grid(cat, g)
    rx, ry = ref_lib.grad_grid(cat, g)
    assert max_rel_err(ax, rx) == 0. and max_rel_err(ay, ry) == 0.


def _fd_hessian(oracle_lib, cat, px, py, h):
    """Richardson-extrapolated central differences of the oracle deflection."""
    def d(step):
        axp, ayp = oracle_lib.grad_points(cat, px + step, py)
        axm, aym = oracle_lib.grad_points(cat, px - step, py)
        bxp, byp = oracle_lib.grad_points(cat, px, py + step)
        bxm, bym = oracle_lib.grad_points(cat, px, py - step)
        return ((axp - axm) / (2 * step), (byp - bym) / (2 * step), (ayp - aym) / (2 * step))
    d1, d2 = d(h), d(h / 2)
    return tuple((4 * b - a) / 3 for a, b in zip(d1, d2))


@pytest.mark.parametrize("ptype", [5, 8, 81])
def test_restated_hessian_matches_derivative_of_reference_gradient(oracle_lib, ptype):
    rng = np.random.default_rng(7)
    n = 12
    cat = catalog.make_catalog(np.full(n, ptype), rng.uniform(-20, 20, n), rng.uniform(-20, 20, n),
                               rng.uniform(150, 400, n), rng.uniform(0.05, 0.5, n), rng.uniform(0, math.pi, n),
                               rng.uniform(0.5, 2., n), rng.uniform(10., 40., n))
    px = rng.uniform(-40, 40, 64)
    py = rng.uniform(-40, 40, 64)
    a, b, c, d = oracle_lib.hess_points(cat, px, py)
    fxx, fyy, fxy = _fd_hessian(oracle_lib, cat, px, py, 1e-3)
    scale = np.max(np.abs(np.concatenate([a, c])))
    tol = 1e-6 if ptype == 5 else 1e-8   # SIS deflection starts from a float32 root
    assert np.max(np.abs(a - fxx)) <= tol * scale
    assert np.max(np.abs(c - fyy)) <= tol * scale
    assert np.max(np.abs(b - fxy)) <= tol * scale
    assert np.max(np.abs(b - d)) <= 1e-13 * scale


@pytest.mark.parametrize("ptype", [5, 8, 81])
def test_potential_gradient_is_deflection(oracle_lib, ptype):
    rng = np.random.default_rng(11)
    n = 10
    cat = catalog.make_catalog(np.full(n, ptype), rng.uniform(-20, 20, n), rng.uniform(-20, 20, n),
                               rng.uniform(150, 400, n), rng.uniform(0.05, 0.5, n), rng.uniform(0, math.pi, n),
                               rng.uniform(0.5, 2., n), rng.uniform(10., 40., n))
    px = rng.uniform(-40, 40, 48)
    py = rng.uniform(-40, 40, 48)
    ax, ay = oracle_lib.grad_points(cat, px, py)

    def dpsi(step, dx, dy):
        return (oracle_lib.pot_points(cat, px + dx * step, py + dy * step) -
                oracle_lib.pot_points(cat, px - dx * step, py - dy * step)) / (2 * step)

    for dx, dy, want in ((1, 0, ax), (0, 1, ay)):
        d1, d2 = dpsi(1e-3, dx, dy), dpsi(5e-4, dx, dy)
        fd = (4 * d2 - d1) / 3
        tol = 1e-6 if ptype == 5 else 1e-7
        assert np.max(np.abs(fd - want)) <= tol * np.max(np.abs(want))


def test_map_epilogue_identities(oracle_lib):
    rng = np.random.default_rng(3)
    a, b, c = rng.normal(0, .3, 100), rng.normal(0, .3, 100), rng.normal(0, .3, 100)
    D = 0.7
    mu = oracle_lib.map("mu", a, b, c, D)
    amp1 = oracle_lib.map("ampli1", a, b, c, D)
    assert np.allclose(mu, amp1, rtol=1e-10)
    k = oracle_lib.map("kappa", a, b, c, D)
    assert np.allclose(k, (a + c) * D / 2, rtol=0, atol=0)
    g1 = oracle_lib.map("gamma1", a, b, c, D)
    g2 = oracle_lib.map("gamma2", a, b, c, D)
    assert np.allclose(oracle_lib.map("shear3", a, b, c, D), g1, rtol=0, atol=0)
    assert np.allclose(oracle_lib.map("shear4", a, b, c, D), g2, rtol=0, atol=0)
    # shear mode 1 is |gamma| of the D-scaled matrix
    assert np.allclose(oracle_lib.map("shear1", a, b, c, D), np.hypot(g1, g2), rtol=1e-12)


def test_cosmology_closed_form_and_flat():
    c = cosmo.Cosmology(omegaX=0.)
    # the omegaX = 0 branch has a closed form; compare with the integral at tiny omegaX
    c2 = cosmo.Cosmology(omegaX=1e-12, curvature=0.3 + 1e-12 - 1.)
    d1 = cosmo.observer_object(1.5, c)
    d2 = cosmo.observer_object(1.5, c2)
    assert abs(d1 - d2) < 1e-9
    dls, dos, dol = cosmo.distances(0.35, 1.5)
    assert 0 < dls < dos and 0 < dol
    assert cosmo.object_object(1.5, 0.35, cosmo.Cosmology()) == 0.
