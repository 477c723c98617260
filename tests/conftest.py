"""Shared test set-up: the `gpu` marker, the package loader and common fixtures."""
import importlib.util
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    """Import the package directory `lenstool-hpc_b200/` as module `lenstool_hpc_b200`."""
    if "lenstool_hpc_b200" in sys.modules:
        return sys.modules["lenstool_hpc_b200"]
    pkg_dir = ROOT / "lenstool-hpc_b200"
    spec = importlib.util.spec_from_file_location("lenstool_hpc_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lenstool_hpc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def max_rel_err(got, ref, mask=None):
    """max |got - ref| / max(|ref|, RMS(ref)) over the (masked) pixels."""
    got = np.asarray(got, np.float64).ravel()
    ref = np.asarray(ref, np.float64).ravel()
    if mask is not None:
        m = np.asarray(mask).ravel()
        got, ref = got[m], ref[m]
    fin = np.isfinite(ref)
    if not np.array_equal(fin, np.isfinite(got)):
        return np.inf
    got, ref = got[fin], ref[fin]
    if ref.size == 0:
        return 0.
    rms = np.sqrt(np.mean(ref * ref))
    den = np.maximum(np.abs(ref), rms)
    den[den == 0] = 1.
    return float(np.max(np.abs(got - ref) / den))


def plane_close(got, exp, kind, precision):
    """A batch or serving plane against the single-grid call of the same precision.  The
    Hessian maps must be identical (same pair loops, explicitly rounded epilogues); the
    deflection and potential planes come from differently inlined code, whose FMA
    contraction the compiler chooses per kernel: 1e-13 (FP64) or 1e-7 (FP32C) of
    max(|ref|, RMS)."""
    if kind in ("potential", "deflection_x", "deflection_y"):
        return max_rel_err(got, exp) <= (1e-7 if precision == "fp32c" else 1e-13)
    return np.array_equal(got, exp, equal_nan=True)


def golden(name):
    return np.load(GOLDEN / name)


def catalog_from_npz(z):
    from lenstool_hpc_b200.catalog import HaloCatalog
    kw = {k: np.array(z[k]) for k in ("type", "position_x", "position_y", "b0", "ellipticity_angle", "anglecos",
                                       "anglesin", "ellipticity_potential", "rcore", "rcut", "dlsds")}
    return HaloCatalog(**kw).contiguous()


def grid_from_npz(z):
    from lenstool_hpc_b200.catalog import Grid
    g = z["grid"]
    return Grid(float(g[0]), float(g[1]), float(g[2]), float(g[3]), int(g[4]), int(g[5]))


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref_lib():
    import oracle
    if not oracle.REF_SO.exists():
        pytest.skip("reference library oracle/_ref/libltref.so not built")
    return oracle.RefLib()
