/*
 * lt_pack.h -- per-halo records (lt_rec64, lt_rec32) from the halo parameters, shared by
 * the host upload (lt_catalog_upload) and the device re-pack (lt_catalog_update).
 *
 * Every operation goes through the pk:: helpers: plain IEEE operations on the host (the
 * host translation units are compiled without FMA contraction) and explicitly rounded
 * intrinsics on the device, so a record packed on the device equals the host's bit for
 * bit for the same parameters.
 *
 * The expressions are the reference's own per-halo sub-expressions
 * (src/gradient.cpp:764-783, src/gradient2.cpp:57-66, src/potential_GPU.cu:52-58) and the
 * potential parameters of module_readParameters_calculatePotentialparameter
 * (src/module_readParameters.cpp:2808-2871); the FP32 records carry the invariants of the
 * FP32 closed forms (lt_profiles32.cuh) and the FP64-fallback radius.
 */
#pragma once
#include <math.h>
#include <string.h>

#include "lt_halo.h"
#include "lt_profiles32.cuh"

namespace lt {
namespace pk {

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double sqr(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float f32(double a) { return __double2float_rn(a); }
#else
inline double mul(double a, double b) { return a * b; }
inline double add(double a, double b) { return a + b; }
inline double sub(double a, double b) { return a - b; }
inline double div(double a, double b) { return a / b; }
inline double sqr(double a) { return sqrt(a); }
inline float f32(double a) { return (float)a; }
#endif

/* FP64 regions of the FP32C path */
constexpr double kTau = 0.1;       /* FP64 where b0 / (2 r) > kTau                        */
constexpr double kCoreFrac = 3.0;  /* FP64 within 3 rcore of the centre                   */

/* b0 and ellipticity_potential from the velocity dispersion and the mass ellipticity
 * (src/module_readParameters.cpp:2808-2871; pi_c2 = pi / c^2 in arcsec (km/s)^-2). */
LT_HD inline void potential_parameters(int type, double vdisp, double emass, double &b0, double &eps)
{
    const double pi_c2 = 7.209970e-06;
    if (type == 5) {
        b0 = mul(mul(mul(4., pi_c2), vdisp), vdisp);
        eps = div(emass, 3.);
    } else {
        b0 = mul(mul(mul(6., pi_c2), vdisp), vdisp);
        eps = emass == 0. ? 0.00001 : div(sub(1., sqr(sub(1., mul(emass, emass)))), emass);
    }
}

/* The FP64 record (slot meaning in lt_halo.h). */
LT_HD inline void pack64(int t, double x, double y, double cs, double sn, double b0, double e, double rc,
                         double rcut, double w, lt_rec64 &r)
{
    memset(&r, 0, sizeof(r));
    r.x0 = x;
    r.y0 = y;
    r.cs = cs;
    r.sn = sn;
    r.b0 = b0;
    r.eps = e;
    r.rc = rc;
    r.rcut = rcut;
    r.w = w;
    if (t == 5) {
        r.cx1 = sub(1., e);
        r.cx1inv = add(1., e);
        r.pref_g = mul(sub(1., e), b0);
        r.pref_h = mul(add(1., e), b0);
        r.ci = mul(mul(b0, sub(1., e)), add(1., e));
        return;
    }
    const double sqe = sqr(e);
    r.sqe2 = mul(2., sqe);
    r.cx1 = div(sub(1., e), add(1., e));
    r.cx1inv = div(1., r.cx1);
    r.cxro_inv = div(1., mul(add(1., e), add(1., e)));
    r.cyro_inv = div(1., mul(sub(1., e), sub(1., e)));
    r.k4 = mul(4., e);
    r.ci = div(mul(0.5, sub(1., mul(e, e))), sqe);
    const double t05 = (t == 81) ? div(rcut, sub(rcut, rc)) : 1.0;
    r.pref_g = mul(mul(r.ci, b0), t05);
    r.pref_h = mul(mul(r.ci, b0), t05);
    r.rc2 = mul(rc, rc);
    r.rcut2 = mul(rcut, rcut);
    r.tsr_c = mul(mul(2., rc), sqe);
    r.tsr_t = mul(mul(2., rcut), sqe);
    r.e1 = div(mul(2., sqe), sub(1, e));
    r.e2 = div(mul(2., sqe), add(1, e));
    r.dr2 = mul(sub(rc, rcut), add(rc, rcut));
    r.drs = sub(rc, rcut);
    r.om2 = mul(sub(1., e), sub(1., e));
    r.e4cxi = div(mul(4., e), mul(add(1., e), add(1., e)));
    r.ok3c = mul(mul(sub(1., e), add(3., e)), rc);
    r.ok3t = mul(mul(sub(1., e), add(3., e)), rcut);
    r.i4rc2 = div(1., mul(4., mul(rc, rc)));
    r.i4rcut2 = div(1., mul(4., mul(rcut, rcut)));
}

/* module_readParameters_calculatePotentialparameter_SOA (src/module_readParameters.cpp:
 * 2873-2936) with both ellipticities as state, its branches kept: for SIS the potential
 * ellipticity drives (emass = 3 epot; emass == 0 with epot != 0 sets epot to 0), for
 * PIEMD/dPIE the mass ellipticity does (epot = (1 - sqrt(1 - e^2))/e), except emass == 0,
 * where a non-zero epot sets emass = 2 epot/(1 + epot^2) and a zero one becomes 1e-5. */
LT_HD inline void calc_potential_parameter(int type, double vdisp, double &emass, double &epot, double &b0)
{
    const double pi_c2 = 7.209970e-06;
    if (type == 5) {
        b0 = mul(mul(mul(4., pi_c2), vdisp), vdisp);
        if (emass == 0. && epot != 0.)
            epot = div(emass, 3.);
        else
            emass = mul(epot, 3.);
    } else {
        b0 = mul(mul(mul(6., pi_c2), vdisp), vdisp);
        if (emass == 0. && epot != 0.)
            emass = div(mul(2., epot), add(1., mul(epot, epot)));
        else if (emass == 0. && epot == 0.)
            epot = 0.00001;
        else
            epot = div(sub(1., sqr(sub(1., mul(emass, emass)))), emass);
    }
}

/* The domain lt_catalog_upload accepts: finite parameters, ellipticity_potential in
 * [0, 1) (SIS) or (0, 1), rcore > 0 (PIEMD, dPIE), rcut > rcore (dPIE). */
LT_HD inline bool record_ok(int t, double x, double y, double b0, double cs, double sn, double eps, double rc,
                            double rcut)
{
    if (!isfinite(x) || !isfinite(y) || !isfinite(b0) || !isfinite(cs) || !isfinite(sn) || !isfinite(eps) ||
        !isfinite(rc) || !isfinite(rcut))
        return false;
    if (t == 5 ? !(eps >= 0. && eps < 1.) : !(eps > 0. && eps < 1.)) return false;
    if (t != 5 && !(rc > 0.)) return false;
    if (t == 81 && !(rcut > rc)) return false;
    return true;
}

/* Halos summed in FP64 for every pixel by the FP32C path: cluster-scale (b0 >= 5"),
 * large cores (rcore >= 1"), nearly circular PIEMD/dPIE (ci ~ 1/(2 sqrt(e))). */
LT_HD inline bool needs_fp64_always(const lt_rec64 &r, int type)
{
    if (r.b0 >= 5.0) return true;
    if (type != 5 && r.rc >= 1.0) return true;
    if (type != 5 && r.eps < 1e-3) return true;
    return false;
}

/* The FP32 record of an FP32-class halo (the invariants of the closed forms of
 * lt_profiles32.cuh: q = (1-e)/(1+e), k = sqrt(1 - q^2) = 2 sqrt(e)/(1+e), s = (1+e) r,
 * A = b0 (1-e) t05) and its FP64 disc: the larger of the near field (b0 / 2r > kTau) and
 * kCoreFrac core radii. */
LT_HD inline void pack32(const lt_rec64 &r, int type, int idx64, lt_rec32 &o)
{
    memset(&o, 0, sizeof(o));
    o.x0 = r.x0;
    o.y0 = r.y0;
    o.cs = f32(r.cs);
    o.sn = f32(r.sn);
    o.c2t = f32(sub(mul(r.cs, r.cs), mul(r.sn, r.sn)));
    o.s2t = f32(mul(mul(2., r.cs), r.sn));
    o.w = f32(r.w);
    o.type = type;
    o.idx64 = idx64;
    const double e = r.eps;
    const double near_r = div(r.b0, mul(2., kTau));
    o.rnear2 = f32(mul(near_r, near_r));
    if (type == 5) {
        o.q2 = f32(sub(1., e));
        o.k = f32(add(1., e));
        o.K = f32(mul(mul(r.b0, sub(1., e)), add(1., e)));
        o.Ak = f32(r.b0);
        return;
    }
    const double ope = add(1., e), ome = sub(1., e);
    const double q = div(ome, ope), q2 = mul(q, q), opq2 = add(1., q2);
    const double k = div(mul(2., sqr(e)), ope);
    const double t05 = (type == 81) ? div(r.rcut, sub(r.rcut, r.rc)) : 1.0;
    const double A = mul(mul(r.b0, ome), t05), K = mul(0.5, A);
    const double sc = mul(ope, r.rc), st = mul(ope, r.rcut);
    const double sc2 = mul(sc, sc), st2 = mul(st, st), ds2 = mul(sub(sc, st), add(sc, st));
    const double c1 = sub(q2, 1.);
    o.q2 = f32(q2);
    o.k = f32(k);
    o.k2 = f32(mul(k, k));
    o.sc = f32(sc);
    o.st = f32(st);
    o.ds = f32(sub(sc, st));
    o.dsq2 = f32(mul(q2, sub(sc, st)));
    o.q2sc2 = f32(mul(q2, sc2));
    o.q2st2 = f32(mul(q2, st2));
    o.dq2s2 = f32(mul(q2, ds2));
    o.opsc2 = f32(mul(opq2, sc2));
    o.opst2 = f32(mul(opq2, st2));
    o.opds2 = f32(mul(opq2, ds2));
    o.tsc = f32(mul(2., sc));
    o.tst = f32(mul(2., st));
    o.K = f32(K);
    o.Kc1sc2 = f32(mul(mul(K, c1), sc2));
    o.Kc1st2 = f32(mul(mul(K, c1), st2));
    o.Ak = f32(div(A, k));
    o.qsc = f32(mul(q, sc));
    o.qst = f32(mul(q, st));
    o.q2sc = f32(mul(q2, sc));
    o.q2st = f32(mul(q2, st));
    o.Asc = f32(mul(0.5, mul(A, sc)));
    o.Ascl2 = f32(mul(mul(0.5, mul(A, sc)), 0.69314718055994530942));
    o.Ast = f32(mul(0.5, mul(A, st)));
    o.i4rc2 = f32(div(1., mul(4., mul(r.rc, r.rc))));
    o.i4rcut2 = f32(div(1., mul(4., mul(r.rcut, r.rcut))));
    const double core_r2 = mul(mul(kCoreFrac, r.rc), mul(kCoreFrac, r.rc));
    /* one radius for both round regions: the near field and the core */
    if (core_r2 > mul(near_r, near_r)) o.rnear2 = f32(core_r2);
}

/* The FP64 closed-form record (lt_halo.h: lt_nie64) of any halo. */
LT_HD inline void pack_nie64(const lt_rec64 &r, int type, lt_nie64 &o)
{
    memset(&o, 0, sizeof(o));
    o.x0 = r.x0;
    o.y0 = r.y0;
    o.cs = r.cs;
    o.sn = r.sn;
    o.c2t = sub(mul(r.cs, r.cs), mul(r.sn, r.sn));
    o.s2t = mul(mul(2., r.cs), r.sn);
    o.w = r.w;
    const double e = r.eps;
    if (type == 5) {
        o.q2 = sub(1., e);
        o.k = add(1., e);
        o.K = mul(mul(r.b0, sub(1., e)), add(1., e));
        return;
    }
    const double ope = add(1., e), ome = sub(1., e);
    const double q = div(ome, ope), q2 = mul(q, q), opq2 = add(1., q2);
    const double t05 = (type == 81) ? div(r.rcut, sub(r.rcut, r.rc)) : 1.0;
    const double K = mul(0.5, mul(mul(r.b0, ome), t05));
    const double sc = mul(ope, r.rc), st = mul(ope, r.rcut);
    const double sc2 = mul(sc, sc), st2 = mul(st, st), ds2 = mul(sub(sc, st), add(sc, st));
    const double c1 = sub(q2, 1.);
    o.q2 = q2;
    o.k = div(mul(2., sqr(e)), ope);
    o.sc = sc;
    o.st = st;
    o.ds = sub(sc, st);
    o.q2sc2 = mul(q2, sc2);
    o.q2st2 = mul(q2, st2);
    o.dq2s2 = mul(q2, ds2);
    o.opsc2 = mul(opq2, sc2);
    o.opst2 = mul(opq2, st2);
    o.opds2 = mul(opq2, ds2);
    o.tsc = mul(2., sc);
    o.tst = mul(2., st);
    o.K = K;
    o.Kc1sc2 = mul(mul(K, c1), sc2);
    o.Kc1st2 = mul(mul(K, c1), st2);
}

} // namespace pk
} // namespace lt
