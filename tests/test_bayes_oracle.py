"""bayes.dat ingestion on the CPU: the reader and column layouts against a bayes.dat the
reference ships (A370 posterior, tests/golden/bayes_a370_head.dat), and the numpy statement
of a row's update (bayes.reference_state) against the reference's own
module_readParameters_setbayesmapmodels + setScalingRelations, bit for bit."""
import math

import numpy as np
import pytest

from conftest import GOLDEN, load_package

lt = load_package()
from lenstool_hpc_b200 import bayes, catalog  # noqa: E402


def test_read_a370_and_column_layout():
    names, rows = bayes.read_bayes(GOLDEN / "bayes_a370_head.dat")
    assert len(names) == 49 and rows.shape == (2, 49)
    assert names[0] == "Nsample" and names[-1] == "Chi2"
    assert rows[0, 0] == 1 and rows[0, 1] == pytest.approx(-378.928146)
    cols = bayes.columns_from_names(names)
    B = bayes
    big = {B.X, B.Y, B.EMASS, B.THETA, B.RCORE, B.VDISP}
    small = {B.VDISP, B.RCUT}
    free = [big, big, small, small, small, big, big, small, small, small]
    exp = bayes.columns_from_free(free, n_z_param=6, potfile_free=[(True, True), (True, True)])
    # the file has one more column than setbayesmapmodels reads: Chi2 (skipped)
    assert np.array_equal(cols[:-1], exp) and tuple(cols[-1]) == (B.SKIP, 0)
    assert tuple(cols[2]) == (B.X, 0) and tuple(cols[14]) == (B.VDISP, 2) and tuple(cols[15]) == (B.RCUT, 2)
    assert tuple(cols[44]) == (B.POT_CUT, 0) and tuple(cols[47]) == (B.POT_SIGMA, 1)
    with pytest.raises(ValueError):
        bayes.columns_from_names(["Nsample", "ln(Lhood)", "O1 : gamma"])


def _model(seed=3, n_pot=(30, 25)):
    """6 parameter-file halos (dPIE, PIEMD, SIS; one with emass = 0 and epot != 0, one with
    both 0) + two potfiles of dPIE galaxies (a few with mag = 0)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    types = [81, 81, 8, 8, 5, 81]
    nh = len(types)
    ng = sum(n_pot)
    t = np.array(types + [81] * ng, np.int32)
    n = t.size
    em = np.concatenate([[0.3, 0.0, 0.45, 0.0, 0.2, 0.6], rng.uniform(0., 0.5, ng)])
    ep = np.concatenate([[0.0, 0.12, 0.0, 0.0, 0.07, 0.0], np.zeros(ng)])
    mag = np.concatenate([np.zeros(nh), rng.uniform(17., 23., ng)])
    mag[nh + 3] = 0.
    mag[nh + n_pot[0] + 1] = 0.
    model = bayes.BayesModel(t, rng.uniform(-30, 30, n), rng.uniform(-30, 30, n), ep, em,
                             rng.uniform(0, math.pi, n), np.concatenate([rng.uniform(2, 10, nh), rng.uniform(.05, .2, ng)]),
                             np.concatenate([rng.uniform(600, 1100, nh), rng.uniform(80, 250, ng)]),
                             np.concatenate([rng.uniform(300, 900, nh), rng.uniform(10, 40, ng)]), mag)
    pots = [bayes.Potfile(nh, n_pot[0], mag0=19.5, sigma=180., cut=30., core=0.15, vdslope=4., slope=4.),
            bayes.Potfile(nh + n_pot[0], n_pot[1], mag0=20.1, sigma=150., cut=22., core=0.1, vdslope=3.5, slope=4.5)]
    B = bayes
    free = [{B.X, B.Y, B.EMASS, B.THETA, B.RCORE, B.VDISP, B.RCUT}, {B.EPOT, B.VDISP}, {B.THETA, B.RCORE, B.Z},
            {B.X, B.VDISP}, {B.EMASS, B.VDISP, B.THETA}, {B.RCUT}]
    pot_free = [(True, True), (False, True)]
    cols = bayes.columns_from_free(free, n_z_param=2, potfile_free=pot_free)
    flags = np.array([[1 if f in fs else 0 for f in bayes.HALO_ORDER] for fs in free], np.int32)
    return model, pots, cols, flags, pot_free, nh


def test_reference_state_equals_reference_rows(ref_lib):
    model, pots, cols, flags, pot_free, nh = _model()
    rows = bayes.synthetic_rows(model, cols, 12, np.random.Generator(np.random.PCG64(8)), potfiles=pots)
    ref = ref_lib.bayes_rows(model, nh, flags, 2, pots, pot_free, rows)
    for r in range(rows.shape[0]):
        got = bayes.reference_state(model, pots, cols, rows[r])
        for k in ref:
            assert np.array_equal(got[k], ref[k][r]), (r, k)
    # potfile galaxies follow their scaling relation; mag = 0 keeps the model's values
    g = nh + 3
    assert ref["rcore"][0][g] == model.rcore[g] and ref["rcut"][5][g] == model.rcut[g]
    assert ref["rcut"][0][nh] != ref["rcut"][1][nh]  # potfile 0's cut is free
    s = nh + pots[0].count
    assert ref["rcut"][0][s] == ref["rcut"][1][s]  # potfile 1's cut is not


def test_catalogue_from_state():
    model, pots, cols, flags, pot_free, nh = _model()
    rows = bayes.synthetic_rows(model, cols, 2, np.random.Generator(np.random.PCG64(8)), potfiles=pots)
    st = bayes.reference_state(model, pots, cols, rows[1])
    cat = bayes.catalog_from_state(model, st)
    assert cat.n == model.n and np.array_equal(cat.b0, st["b0"]) and np.array_equal(cat.anglecos, st["cos"])
    assert isinstance(cat, catalog.HaloCatalog)
