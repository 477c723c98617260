/*
 * lt_cosmo.cpp -- angular-diameter distances in units of c/H0 for the map scalars
 * D_LS, D_OS, D_OL (module_cosmodistances_observerObject/objectObject,
 * src/module_cosmodistances.cpp:94-151, H(z) of model 1 at :222-230).
 *
 * The reference integrates H0/H(z) with GSL QAG (epsrel 1e-6); GSL is not a dependency
 * here: the integral uses an adaptive Gauss-Kronrod 7/15 rule (Piessens et al.,
 * QUADPACK, 1983) refined to ~1e-14 relative.
 */
#include <cmath>

#include "../../include/lt_b200.h"

namespace {

const double kXgk[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                        0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                        0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                        0.207784955007898467600689403773245, 0.0};
const double kWgk[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                        0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                        0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                        0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
const double kWg[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                       0.381830050505118944950369775488975, 0.417959183673469387755102040816327};

struct Cosmo {
    double omegaM, omegaX, curvature, wX, wa;
};

bool inv_e(double z, const Cosmo &c, double &out)
{
    double x = 1. + z;
    double h2 = -x * x * c.curvature + x * x * x * c.omegaM +
                c.omegaX * std::pow(x, 3 * (1 + c.wX + c.wa)) * std::exp(-3 * c.wa * z / x);
    if (!(h2 > 0)) return false;
    out = 1. / std::sqrt(h2);
    return true;
}

bool gk15(const Cosmo &c, double a, double b, double &val, double &err)
{
    double m = 0.5 * (a + b), h = 0.5 * (b - a), fc;
    if (!inv_e(m, c, fc)) return false;
    double rk = fc * kWgk[7], rg = fc * kWg[3];
    for (int j = 0; j < 7; j++) {
        double fa, fb;
        if (!inv_e(m - h * kXgk[j], c, fa) || !inv_e(m + h * kXgk[j], c, fb)) return false;
        rk += kWgk[j] * (fa + fb);
        if (j % 2 == 1) rg += kWg[j / 2] * (fa + fb);
    }
    val = rk * h;
    err = std::fabs((rk - rg) * h);
    return true;
}

bool integrate(const Cosmo &c, double a, double b, int depth, double &out)
{
    double v, e;
    if (!gk15(c, a, b, v, e)) return false;
    if (e <= 1e-14 * std::fabs(v) || depth > 30) {
        out = v;
        return true;
    }
    double l, r, m = 0.5 * (a + b);
    if (!integrate(c, a, m, depth + 1, l) || !integrate(c, m, b, depth + 1, r)) return false;
    out = l + r;
    return true;
}

double sk(double x, double k) { return k > 0 ? std::sin(x) : (k < 0 ? std::sinh(x) : x); }

bool observer_object(const Cosmo &c, double z, double &out)
{
    if (c.omegaX == 0.) {
        double g = std::sqrt(1. + c.omegaM * z);
        out = 2. * ((1. - c.omegaM - g) * (1. - g)) / c.omegaM / c.omegaM / (1. + z) / (1. + z);
        return true;
    }
    double chi;
    if (!integrate(c, 0., z, 0, chi)) return false;
    if (c.curvature != 0.) {
        double k = std::sqrt(std::fabs(c.curvature));
        out = sk(chi * k, c.curvature) / (1 + z) / k;
    } else {
        out = chi / (1 + z);
    }
    return true;
}

bool object_object(const Cosmo &c, double z1, double z2, double &out)
{
    if (z1 >= z2) {
        out = 0.;
        return true;
    }
    if (c.omegaX == 0.) {
        double g1 = std::sqrt(1. + c.omegaM * z1), g2 = std::sqrt(1. + c.omegaM * z2);
        out = 2. * ((1. - c.omegaM - g1 * g2) * (g1 - g2)) / c.omegaM / c.omegaM / (1. + z1) / (1. + z2) / (1. + z2);
        return true;
    }
    double chi;
    if (!integrate(c, z1, z2, 0, chi)) return false;
    if (c.curvature != 0.) {
        double k = std::sqrt(std::fabs(c.curvature));
        out = sk(chi * k, c.curvature) / (1 + z2) / k;
    } else {
        out = chi / (1 + z2);
    }
    return true;
}

} // namespace

extern "C" lt_status lt_cosmo_distances(const lt_cosmology *cosmo, double zl, double zs, double *dls, double *dos,
                                        double *dol)
{
    if (!cosmo || !dls || !dos || !dol || cosmo->model != 1 || !std::isfinite(zl) || !std::isfinite(zs) || zl < 0 ||
        zs < 0)
        return LT_ERR_INVALID_ARGUMENT;
    Cosmo c = {cosmo->omegaM, cosmo->omegaX, cosmo->curvature, cosmo->wX, cosmo->wa};
    if (!object_object(c, zl, zs, *dls) || !observer_object(c, zs, *dos) || !observer_object(c, zl, *dol))
        return LT_ERR_INVALID_ARGUMENT;
    return LT_OK;
}
