"""The FP32 atan2 / atanh polynomial coefficients in lt_profiles32.cuh are the Remez fits
that tests/golden/fit_fast_math.py regenerates (CPU only)."""
import importlib.util
import pathlib
import re

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _fit_module():
    spec = importlib.util.spec_from_file_location("fit_fast_math", ROOT / "tests" / "golden" / "fit_fast_math.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _header_coefficients(function):
    """The float literals of `function`'s Horner chain, highest degree first."""
    text = (ROOT / "lenstool-hpc_b200" / "csrc" / "lt_profiles32.cuh").read_text()
    body = text[text.index(f"float {function}("):]
    body = body[:body.index("\n}\n")]
    lits = re.findall(r"float p = ([-0-9.e+]+)f;|fmaf?\(p, \w, ([-0-9.e+]+)f\)", body)
    return np.array([float(a or b) for a, b in lits])


def test_atan2_coefficients_are_the_remez_fit():
    c, err = _fit_module().fit_atan()
    want = np.float32(c[::-1]).astype(np.float64)
    got = _header_coefficients("fatan_unit")
    assert got.size == 8
    # equal as float32 values (the header prints them with 10 significant digits)
    assert np.all(np.abs(got - want) <= 2 * np.spacing(np.abs(want).astype(np.float32))), (got, want)
    assert err < 1e-7


def test_atanh_coefficients_are_the_remez_fit():
    c, err = _fit_module().fit_atanh_third()
    want = np.float32(c[::-1]).astype(np.float64)
    got = _header_coefficients("fatanh_third")
    assert got.size == 5 and got[-1] == 1.0
    assert np.all(np.abs(got - want) <= 2 * np.spacing(np.abs(want).astype(np.float32))), (got, want)
    assert err < 5e-9
