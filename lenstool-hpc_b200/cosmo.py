"""Angular-diameter distances in units of c/H0 (the scalars D_LS, D_OS, D_OL that scale the
lensing maps).

Restates module_cosmodistances_observerObject / _objectObject for cosmological model 1
(src/module_cosmodistances.cpp:94-151, H(z) of :226-230).  The reference integrates
H0/H(z) with GSL's QAG (epsrel 1e-6, 10 intervals, :314-338); this module uses its own
adaptive Gauss-Kronrod 7/15 rule (Piessens et al., QUADPACK, 1983) to ~1e-14, and the
same values are computed by the C++ library (lt_cosmo.cpp) for its map entry points.
"""
from __future__ import annotations

import dataclasses
import math

# Gauss-Kronrod 7/15 nodes and weights (Kronrod extension of the 7-point Gauss rule).
_XGK = (0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
        0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
        0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
        0.207784955007898467600689403773245, 0.0)
_WGK = (0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
        0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
        0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
        0.204432940075298892414161999234649, 0.209482141084727828012999174891714)
_WG = (0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
       0.381830050505118944950369775488975, 0.417959183673469387755102040816327)


@dataclasses.dataclass
class Cosmology:
    """cosmo_param of src/structure_hpc.hpp:468-478 (model 1: CPL dark energy)."""
    H0: float = 70.
    omegaM: float = 0.3
    omegaX: float = 0.7
    curvature: float = 0.
    wX: float = -1.
    wa: float = 0.
    model: int = 1

    @property
    def h(self) -> float:
        return self.H0 / 50.


def _inv_e(z: float, c: Cosmology) -> float:
    x = 1. + z
    h2 = -x * x * c.curvature + x * x * x * c.omegaM + c.omegaX * x ** (3 * (1 + c.wX + c.wa)) * math.exp(
        -3 * c.wa * z / x)
    if h2 <= 0:
        raise ValueError("H^2(z) <= 0")
    return 1. / math.sqrt(h2)


def _gk15(f, a, b):
    c = 0.5 * (a + b)
    h = 0.5 * (b - a)
    fc = f(c)
    rk = fc * _WGK[7]
    rg = fc * _WG[3]
    for j in range(7):
        fa = f(c - h * _XGK[j])
        fb = f(c + h * _XGK[j])
        rk += _WGK[j] * (fa + fb)
        if j % 2 == 1:
            rg += _WG[j // 2] * (fa + fb)
    return rk * h, abs((rk - rg) * h)


def integrate(f, a, b, tol=1e-14, depth=0):
    v, err = _gk15(f, a, b)
    if err <= tol * max(abs(v), 1e-300) or depth > 30:
        return v
    m = 0.5 * (a + b)
    return integrate(f, a, m, tol, depth + 1) + integrate(f, m, b, tol, depth + 1)


def _sk(x, k):
    return math.sin(x) if k > 0 else (math.sinh(x) if k < 0 else x)


def chi(z1: float, z2: float, c: Cosmology) -> float:
    return integrate(lambda z: _inv_e(z, c), z1, z2)


def observer_object(z: float, c: Cosmology) -> float:
    """D_A(0, z) / (c/H0), src/module_cosmodistances.cpp:94-114."""
    if c.omegaX == 0.:
        g = math.sqrt(1. + c.omegaM * z)
        return 2. * ((1. - c.omegaM - g) * (1. - g)) / c.omegaM / c.omegaM / (1. + z) / (1. + z)
    if c.curvature != 0.:
        k = math.sqrt(abs(c.curvature))
        return _sk(chi(0., z, c) * k, c.curvature) / (1 + z) / k
    return chi(0., z, c) / (1 + z)


def object_object(z1: float, z2: float, c: Cosmology) -> float:
    """D_A(z1, z2) / (c/H0), 0 when z1 >= z2, src/module_cosmodistances.cpp:128-151."""
    if z1 >= z2:
        return 0.
    if c.omegaX == 0.:
        g1 = math.sqrt(1. + c.omegaM * z1)
        g2 = math.sqrt(1. + c.omegaM * z2)
        return 2. * ((1. - c.omegaM - g1 * g2) * (g1 - g2)) / c.omegaM / c.omegaM / (1. + z1) / (1. + z2) / (1. + z2)
    if c.curvature != 0.:
        k = math.sqrt(abs(c.curvature))
        return _sk(chi(z1, z2, c) * k, c.curvature) / (1 + z2) / k
    return chi(z1, z2, c) / (1 + z2)


def distances(zl: float, zs: float, c: Cosmology | None = None):
    """(dl0s, dos, dol): the three scalars the map builders pass to their epilogues
    (src/grid_map_ampli_GPU.cu:110-112)."""
    c = c or Cosmology()
    return object_object(zl, zs, c), observer_object(zs, c), observer_object(zl, c)
