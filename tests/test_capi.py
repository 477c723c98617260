"""The C-ABI library loads and exports every entry point include/lt_b200.h declares; the
host-only pieces (status strings, cosmology) work without a GPU.  CPU only."""
import ctypes as C
import pathlib
import re

import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import cosmo

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    out = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        out |= set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(lt_\w+)\s*\(", text, flags=re.M))
    return out


@pytest.fixture(scope="module")
def lib():
    from lenstool_hpc_b200 import build
    build.build()
    return lt.load_library()


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert {"lt_create", "lt_hessian_maps", "lt_lens_maps"} <= syms
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(lt.EXPORTS) <= syms


def test_status_strings_and_version(lib):
    assert lib.lt_abi_version() == 1
    assert lib.lt_status_string(0) == b"ok"
    assert lib.lt_status_string(8).startswith(b"device-side wait")


def test_cosmology_matches_python_mirror(lib):
    for zl, zs in ((0.35, 1.5), (0.4, 3.0), (0.2, 0.5)):
        got = lt.cosmo_distances(zl, zs)
        want = cosmo.distances(zl, zs)
        for g, w in zip(got, want):
            assert abs(g - w) <= 1e-13 * abs(w)
    assert lt.cosmo_distances(1.5, 0.35)[0] == 0.


def test_no_device_is_reported_not_crashed(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert lib.lt_create(0, 0, C.byref(h)) == 9  # LT_ERR_NO_DEVICE
    assert lib.lt_destroy(None) == 1             # LT_ERR_INVALID_ARGUMENT
