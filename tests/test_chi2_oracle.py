"""The chi2 restatement of the oracle (source barycentres, barycentric delensing, image
linking) against the reference's own delense_barycenter and chi_computation compiled
from its sources (oracle/_ref).  CPU only."""
import numpy as np
import pytest

from lenstool_hpc_b200 import catalog
from lenstool_hpc_b200.images import generate_systems

FRAME = (-100., 100., -100., 100.)


@pytest.fixture(scope="module")
def setup(oracle_lib):
    from types import SimpleNamespace
    cat = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    nfine = 512
    g = SimpleNamespace(xmin=FRAME[0], ymin=FRAME[2], dx=200. / (nfine - 1), dy=200. / (nfine - 1), nx=nfine,
                        ny=nfine, istart=0, jstart=0)
    ax, ay = oracle_lib.grad_grid(cat, g)
    ic = int(np.argmax(cat.b0))
    systems = generate_systems(lambda bx, by, dr: oracle_lib.delense(nfine, FRAME, ax, ay, bx, by, dr), 6, 11,
                               dr=0.6, centre=(cat.position_x[ic], cat.position_y[ic]), source_radius=8.)
    return cat, systems


def test_generated_systems_have_3_to_5_images(setup):
    _, s = setup
    assert s.nsys == 6 and np.all((s.nimg >= 3) & (s.nimg <= 5)) and s.x.size == s.nimg.sum()


@pytest.mark.parametrize("model", ["true", "perturbed", "far"])
def test_chi2_restatement_equals_reference(setup, oracle_lib, ref_lib, model):
    cat, s = setup
    if model == "perturbed":
        cat = catalog.perturb_catalog(cat, np.random.Generator(np.random.PCG64(5)))
    elif model == "far":  # a model far from the truth: unlinked images cost 1000 x n each
        cat = catalog.perturb_catalog(cat, np.random.Generator(np.random.PCG64(9)), rel=0.5)
    a = oracle_lib.chi2(cat, FRAME, 200, s.nimg, s.x, s.y, s.dr)
    b = ref_lib.chi2(cat, FRAME, 200, s.nimg, s.x, s.y, s.dr)
    assert np.array_equal(a["nfound"], b["nfound"])
    for k in range(s.nsys):
        m = a["nfound"][k]
        assert np.array_equal(a["fx"][k, :m], b["fx"][k, :m]) and np.array_equal(a["fy"][k, :m], b["fy"][k, :m])
    assert a["chi2"] == b["chi2"] and a["images_found"] == b["images_found"]


def test_true_model_recovers_its_images(setup, oracle_lib):
    """On the grid the images were generated on, the true model predicts every observed
    image: no 1000 penalty, chi2 of the order of the noise and the grid's resolution."""
    cat, s = setup
    a = oracle_lib.chi2(cat, FRAME, 512, s.nimg, s.x, s.y, s.dr)
    assert a["chi2"] < 1000.
    assert a["chi2"] < s.nimages * (0.05 ** 2 * 10 + (200. / 511) ** 2)


def test_chi2_penalises_missing_images(oracle_lib):
    """A system whose source has no predicted image adds 1000 x n per observed image."""
    nimg = np.array([3], np.int32)
    ix = np.array([1., 2., 3.]); iy = np.array([0., 0., 0.])
    chi, found = oracle_lib.chi2_images(nimg, ix, iy, np.zeros(1, np.int32), np.zeros(20), np.zeros(20))
    assert chi == 3 * 1000. * 3 and found == 0
