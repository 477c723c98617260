/*
 * lt_profiles64.cuh -- FP64 per-pair profile arithmetic (one halo record, one pixel).
 *
 * Formulas follow the reference's FP64 CPU path; divisions by per-halo constants
 * become multiplications by the precomputed reciprocals of lt_rec64, and divisions by
 * per-pair denominators are done once as a reciprocal.  These changes move results by
 * a few ulp; the tests hold this path to 1e-12 of the reference.
 *
 *   deflection:  SIS src/gradient.cpp:260-299, PIEMD :548-607, dPIE :744-811,
 *                complex-log term KERNEL src/gradient.hpp:64-76
 *   Hessian:     dPIE src/gradient2.cpp:92-205 with mdci05 :54-83; PIEMD = one mdci05
 *                term; SIS = derivative of the SIS deflection (restated)
 *   potential:   dPIE src/potential_GPU.cu:47-116 (pi05 with the complex helpers of
 *                src/lt_math_GPU.cuh); PIEMD = one pi05 term; SIS = b0 R (restated)
 */
#pragma once
#include "lt_halo.h"

namespace lt {

/* Reciprocal and reciprocal square root for the per-pair denominators: the hardware
 * approximations (rcp.approx.ftz.f64, rsqrt.approx.ftz.f64; ~20 correct bits) refined by one
 * third-order step: with e = 1 - x y, 1/x = y/(1 - e) = y (1 + e + e^2 + O(e^3)); with
 * h = 1 - x y^2, 1/sqrt(x) = y (1 - h)^(-1/2) = y (1 + h/2 + 3 h^2/8 + O(h^3)).  The
 * truncation is ~e^3 (~1e-18), so the result is within a few ulp of the correctly rounded
 * value for positive normal inputs (checked against 1/x and 1/sqrt(x) by the tests).
 * Three FP64 operations for a reciprocal and five for a reciprocal square root (two
 * Newton steps take four and eight), and one approximation, instead of the IEEE division
 * and square-root sequences. */
__device__ __forceinline__ double rcp64(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

__device__ __forceinline__ double rsqrt64(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = fma(-x * y, y, 1.0);
    return fma(y * h, fma(0.375, h, 0.5), y);
}

struct Frame64 {
    double u, v;
};

/* Offset from the halo centre rotated into the halo frame (x' = x cos + y sin,
 * y' = y cos - x sin; src/gradient.hpp:29-37). */
__device__ __forceinline__ Frame64 to_frame(const lt_rec64 &h, double px, double py)
{
    double tx = px - h.x0, ty = py - h.y0;
    Frame64 f;
    f.u = tx * h.cs + ty * h.sn;
    f.v = ty * h.cs - tx * h.sn;
    return f;
}

/* ---------------------------------------------------------------- deflection ---- */

/* log|z|^2 and arg z of the PIEMD complex ratio for one radius (KERNEL macro). */
__device__ __forceinline__ void piemd_log_term(double u, double uu, double v, double nre, double vq, double sqe2,
                                               double rem2, double r2, double tsr, double &lq, double &la)
{
    const double q = r2 + rem2;
    double nim = sqe2 * (q * rsqrt64(q)) - vq;
    double dim = tsr - v;
    double inv = rcp64(uu + dim * dim);
    double zre = (nre * u + nim * dim) * inv;
    double zim = (nim * u - nre * dim) * inv;
    lq = log(zre * zre + zim * zim);
    la = atan2(zim, zre);
}

template <int TYPE>
__device__ __forceinline__ void grad_pair(const lt_rec64 &h, double px, double py, double &gx, double &gy)
{
    Frame64 f = to_frame(h, px, py);
    double u = f.u, v = f.v;
    if (TYPE == 5) {
        /* inverse radius from a single-precision root and one Newton step, as the
         * reference (src/gradient.cpp:287-288) */
        double q = u * u * h.cx1 + v * v * h.cx1inv;
        double r = 1. / (double)sqrtf((float)q);
        r = r * (1.5 - 0.5 * q * r * r);
        double fx = h.pref_g * u * r;
        double fy = h.pref_h * v * r;
        gx += fx * h.cs - fy * h.sn;
        gy += fy * h.cs + fx * h.sn;
    } else {
        double uu = u * u;
        double rem2 = uu * h.cxro_inv + v * v * h.cyro_inv;
        double vq = v * h.cx1inv;
        double nre = h.cx1 * u;
        double lq, la;
        piemd_log_term(u, uu, v, nre, vq, h.sqe2, rem2, h.rc2, h.tsr_c, lq, la);
        double re, im;
        if (TYPE == 81) {
            double lq2, la2;
            piemd_log_term(u, uu, v, nre, vq, h.sqe2, rem2, h.rcut2, h.tsr_t, lq2, la2);
            re = h.pref_g * (la - la2);
            im = -0.5 * h.pref_g * (lq - lq2);
        } else {
            re = h.pref_g * la;
            im = -0.5 * h.pref_g * lq;
        }
        gx += re * h.cs - im * h.sn;
        gy += im * h.cs + re * h.sn;
    }
}

/* ------------------------------------------------------------------- Hessian ---- */

struct Hess64 {
    double xx, yy, xy;
};

/* The three bracketed terms of mdci05 (didxre, didyre, didyim without the factor ci).
 * With t1 = 2 sqrt(e) w - v/cx1 (the small factor of den1 near the removable singular
 * point u = 0, v = 2 r sqrt(e)), the numerators factor exactly:
 *   didxre: cx1 (2 sqrt(e) u^2/((1+e)^2 w) - t1)
 *   didyre: u (2 sqrt(e) v cx1/((1-e)^2 w) - 1)
 *   didyim: t1 (1/cx1 - 2 sqrt(e) v/((1-e)^2 w))
 * (for didyim, 4e = (2 sqrt(e))^2 turns the reference's four terms into the product), so
 * numerator and denominator share one rounded t1 and the numerators cancel no digits. */
__device__ __forceinline__ void mdci05_terms(const lt_rec64 &h, double u, double uu, double v, double vv,
                                             double vq, double rem2, double r2, double tsr, double &X, double &Y,
                                             double &Z)
{
    (void)vv;
    const double q = r2 + rem2;
    double iw = rsqrt64(q);
    double wrem = q * iw;
    double t1 = h.sqe2 * wrem - vq;
    double den1 = h.cx1 * h.cx1 * uu + t1 * t1;
    double num2 = tsr - v;
    double den2 = uu + num2 * num2;
    double i1 = rcp64(den1);
    double i2 = rcp64(den2);
    double sv = h.sqe2 * v * h.cyro_inv * iw;
    X = h.cx1 * (h.sqe2 * uu * h.cxro_inv * iw - t1) * i1 + num2 * i2;
    Y = u * (sv * h.cx1 - 1.0) * i1 + u * i2;
    Z = t1 * (h.cx1inv - sv) * i1 - num2 * i2;
}

/* H = R^T H' R for the symmetric halo-frame Hessian H' = [[a, b], [b, c]]; the
 * reference applies the same rotation in two steps (src/gradient2.cpp:146-156). */
__device__ __forceinline__ void rotate_acc(const lt_rec64 &h, double a, double b, double c, double w, Hess64 &acc)
{
    double cs = h.cs, sn = h.sn;
    double cc = cs * cs, ss = sn * sn, csn = cs * sn;
    acc.xx += w * (a * cc - 2. * b * csn + c * ss);
    acc.yy += w * (a * ss + 2. * b * csn + c * cc);
    acc.xy += w * ((a - c) * csn + b * (cc - ss));
}

template <int TYPE>
__device__ __forceinline__ void hess_pair(const lt_rec64 &h, double px, double py, double w, Hess64 &acc)
{
    Frame64 f = to_frame(h, px, py);
    double u = f.u, v = f.v;
    double uu = u * u, vv = v * v;
    if (TYPE == 5) {
        double q = uu * h.cx1 + vv * h.cx1inv;
        double rs = rsqrt64(q);
        double k = h.ci * (rs * rs * rs);
        rotate_acc(h, k * vv, -k * u * v, k * uu, w, acc);
    } else {
        double rem2 = uu * h.cxro_inv + vv * h.cyro_inv;
        double vq = v * h.cx1inv;
        double X, Y, Z;
        mdci05_terms(h, u, uu, v, vv, vq, rem2, h.rc2, h.tsr_c, X, Y, Z);
        if (TYPE == 81) {
            double X2, Y2, Z2;
            mdci05_terms(h, u, uu, v, vv, vq, rem2, h.rcut2, h.tsr_t, X2, Y2, Z2);
            X -= X2;
            Y -= Y2;
            Z -= Z2;
        }
        rotate_acc(h, h.pref_h * X, h.pref_h * Y, h.pref_h * Z, w, acc);
    }
}

/* ----------------------------------------------------------------- potential ---- */

struct Cpx {
    double re, im;
};
__device__ __forceinline__ Cpx cmul(Cpx a, Cpx b) { return {a.re * b.re - a.im * b.im, a.im * b.re + b.im * a.re}; }
/* a/b, zero when |b| = 0 (dcpx_GPU, src/lt_math_GPU.cuh:224-243) */
__device__ __forceinline__ Cpx cdiv(Cpx a, Cpx b)
{
    double n = b.re * b.re + b.im * b.im;
    if (n == 0.) return {0., 0.};
    double in = 1.0 / n;
    return {(a.re * b.re + a.im * b.im) * in, (a.im * b.re - a.re * b.im) * in};
}
__device__ __forceinline__ Cpx clog(Cpx a) { return {0.5 * log(a.re * a.re + a.im * a.im), atan2(a.im, a.re)}; }

/* cosh of (re, im) given cos(im), sin(im) (coshcpx_GPU, src/lt_math_GPU.cuh:297-307). */
__device__ __forceinline__ Cpx ccosh_cs(double re, double c, double s)
{
    double ep = exp(re), em = exp(-re);
    return {0.5 * (ep + em) * c, 0.5 * (ep - em) * s};
}

/* One pi05 term without its prefactor b0 ci / sqrt(rem2): r (Im(ckk) x - Re(ckk) y).
 * eta, cosh(eta)^2 and sinh(2 eta) depend only on the pixel and are shared by the
 * core and cut radii. */
__device__ __forceinline__ double pi05_core(double u, double v, double srem, double rem2, double r, double r2,
                                            double eta_re, double ce, double se, Cpx ch2, Cpx sh2e)
{
    double zr = 0.5 * log((srem + sqrt(r2 + rem2)) / r);
    Cpx b1 = ccosh_cs(eta_re + zr, ce, se);
    Cpx b2 = ccosh_cs(eta_re - zr, ce, se);
    Cpx a1 = clog(cdiv(ch2, cmul(b1, b2)));
    Cpx a2 = clog(cdiv(b1, b2));
    double ez = exp(2. * zr), emz = exp(-2. * zr);
    Cpx sh2z = {0.5 * (ez - emz), 0.};
    Cpx c1 = cmul(sh2e, a1);
    Cpx c2 = cmul(sh2z, a2);
    double kre = c1.re + c2.re, kim = c1.im + c2.im;
    return r * (kim * u - kre * v);
}

template <int TYPE>
__device__ __forceinline__ void pot_pair(const lt_rec64 &h, double px, double py, double &psi)
{
    Frame64 f = to_frame(h, px, py);
    double u = f.u, v = f.v;
    double uu = u * u, vv = v * v;
    if (TYPE == 5) {
        psi += h.b0 * sqrt(uu * h.cx1 + vv * h.cx1inv);
        return;
    }
    double rem2 = uu * h.cxro_inv + vv * h.cyro_inv;
    double srem = sqrt(rem2);
    double z = sqrt(uu + vv);
    double eta_re = -.5 * asinh(h.e1 * v / z);
    double eta_im = .5 * asin(h.e2 * u / z);
    double se, ce;
    sincos(eta_im, &se, &ce);
    Cpx ch = ccosh_cs(eta_re, ce, se);
    Cpx ch2 = {ch.re * ch.re - ch.im * ch.im, 2. * ch.re * ch.im};
    double s2, c2;
    sincos(2. * eta_im, &s2, &c2);
    double e2p = exp(2. * eta_re), e2m = exp(-2. * eta_re);
    Cpx sh2e = {0.5 * (e2p - e2m) * c2, 0.5 * (e2p + e2m) * s2};
    double t = pi05_core(u, v, srem, rem2, h.rc, h.rc2, eta_re, ce, se, ch2, sh2e);
    if (TYPE == 81) t -= pi05_core(u, v, srem, rem2, h.rcut, h.rcut2, eta_re, ce, se, ch2, sh2e);
    psi += h.pref_h * t / srem;
}

/* pi05 in the cancellation-free N+- form (N+- = (cosh 2a + cos 2 eta_im)(1 +- tanh eta
 * tanh zeta), no complex quotient, no branch wrap), in FP64: per dPIE pair 4 log and 4 atan2
 * in place of the formula's 16 exp, 6 log, 4 atan2, asinh, asin and 2 sincos.  Against an
 * extended-precision evaluation of pi05 it is within 1e-13 of a term's scale where the
 * reference formula in FP64 is within 2e-13 (checked per term over e in [1e-5, 0.73], r in
 * [0.05, 800]).  pot_pair_fast uses it only near the points where the cheaper
 * deflection-based form below loses digits. */
struct Pi05Shared64 {
    double sh2r, sh2i, E2, iE2, sh2a, c2e, t, itd4;
};

__device__ __forceinline__ double pi05_term64(const Pi05Shared64 &p, double u, double v, double srem, double rem2,
                                              double r, double r2)
{
    const double q = sqrt(r2 + rem2);
    const double qr = q + r;
    const double dm = (srem * qr + rem2) * rcp64(r * qr); /* rho - 1 */
    const double rho = 1. + dm, rho1 = rho + 1.;
    const double inv = rcp64(rho * rho1);
    const double irho = rho1 * inv, irho1 = rho * inv;
    const double tz = dm * irho1;
    const double sh2z = 0.5 * dm * rho1 * irho;
    const double ch2z = 0.25 * rho1 * rho1 * irho;
    const double m = 2. * irho1 * p.sh2a;
    const double A = (p.E2 - m) + p.c2e, C = (p.iE2 + m) + p.c2e, B = tz * p.t, B2 = B * B;
    const double np2 = A * A + B2, nm2 = C * C + B2;
    const double a2r = 0.5 * log(np2 * rcp64(nm2));
    const double a2i = atan2(B * (A + C), A * C - B2);
    const double a1r = -0.5 * log((ch2z * ch2z) * (np2 * nm2) * p.itd4);
    const double a1i = atan2(2. * B * tz * p.sh2a, A * C + B2);
    const double kr = (p.sh2r * a1r - p.sh2i * a1i) + sh2z * a2r;
    const double ki = (p.sh2i * a1r + p.sh2r * a1i) + sh2z * a2i;
    return r * (ki * u - kr * v);
}

/* The potential through the deflection (the derivation and the record invariants are
 * those of pot32 in lt_profiles32.cuh), in FP64 with CUDA's log, log1p and atan2: per dPIE
 * pair 3 logarithms and 1 atan2.  log64 is the complex logarithm of the PIEMD ratio
 * z = N/D (TYPE 8) or of z_c/z_t (TYPE 81): as log(1 + eps) in the cancellation-free form
 * of log32, or, where `split` (near the core radius's 0/0 point, where that form loses
 * digits on the scale of rcut), as log z_c - log z_t (digits lost on the scale of rc). */
struct Log64 {
    double li, lr, wc, wt;
};

/* log z = log(N/D) of one PIEMD radius r (w = sqrt(r^2 + rho^2), tsr = 2 sqrt(e) r): |z|^2
 * straight from |N|^2/|D|^2, and arg z = arg(N conj D) with the imaginary part
 * u (2 sqrt(e) (w - cx1 r) - v (1/cx1 - cx1)) (1/cx1 - cx1 = 4e/(1-e^2) = e1 e2), free of the
 * cancellation of its two products for small e. */
__device__ __forceinline__ void piemd_log64(const lt_rec64 &h, double u, double v, double uu, double w, double r,
                                            double tsr, double &li, double &lr)
{
    const double nr = h.cx1 * u;
    const double nci = h.sqe2 * w - v * h.cx1inv;
    const double dci = tsr - v;
    lr = 0.5 * log((nr * nr + nci * nci) * rcp64(uu + dci * dci));
    li = atan2(u * (h.sqe2 * fma(-h.cx1, r, w) - v * (h.e1 * h.e2)), nr * u + nci * dci);
}

template <int TYPE>
__device__ __forceinline__ Log64 log64(const lt_rec64 &h, double u, double v, double uu, double rho2, bool split)
{
    Log64 o;
    const double xc = h.rc2 + rho2;
    o.wc = xc * rsqrt64(xc);
    if (TYPE == 8) {
        piemd_log64(h, u, v, uu, o.wc, h.rc, h.tsr_c, o.li, o.lr);
        o.wt = 0.;
        return o;
    }
    const double xt = h.rcut2 + rho2;
    o.wt = xt * rsqrt64(xt);
    if (split) {
        double li_t, lr_t;
        piemd_log64(h, u, v, uu, o.wc, h.rc, h.tsr_c, o.li, o.lr);
        piemd_log64(h, u, v, uu, o.wt, h.rcut, h.tsr_t, li_t, lr_t);
        o.li -= li_t;
        o.lr -= lr_t;
        return o;
    }
    const double nr = h.cx1 * u;
    const double dci = h.tsr_c - v;
    const double dw = h.dr2 * rcp64(o.wc + o.wt);
    const double nti = h.sqe2 * o.wt - v * h.cx1inv;
    const double dti = h.tsr_t - v;
    const double dni = h.sqe2 * dw, ddi = h.sqe2 * h.drs;
    const double numr = ddi * nti - dni * dti;
    const double numi = dni * u - ddi * nr;
    const double denr = u * nr - dci * nti;
    const double deni = u * nti + dci * nr;
    const double c = numr * denr + numi * deni;
    const double d = numi * denr - numr * deni;
    const double B = denr * denr + deni * deni;
    o.lr = 0.5 * log1p(fma(2., c, numr * numr + numi * numi) * rcp64(B));
    o.li = atan2(d, B + c);
    return o;
}

template <int TYPE>
__device__ __forceinline__ double pot64_defl(const lt_rec64 &h, double u, double v, double uu, double rho2,
                                             bool split)
{
    const Log64 z = log64<TYPE>(h, u, v, uu, rho2, split);
    const double ut = h.e4cxi * uu;
    double hs = h.rc * log1p((rho2 * rcp64(z.wc + h.rc) * fma(h.om2, z.wc, h.ok3c) + ut) * h.i4rc2);
    if (TYPE == 81)
        hs -= h.rcut * log1p((rho2 * rcp64(z.wt + h.rcut) * fma(h.om2, z.wt, h.ok3t) + ut) * h.i4rcut2);
    return h.pref_h * ((u * z.li - v * z.lr) - 0.5 * h.sqe2 * hs);
}

/* Zones of pot_pair_fast, as squared radii.  The quotients of the deflection form are 0/0
 * at u = 0, v = 2 sqrt(e) r and lose ~1e-16 s/distance near those points, s the size of
 * the terms they are built from.  Measured against an extended-precision pi05 (emulating
 * these formulas), psi stays within 1e-13 of itself outside
 *   0.0316 rc of the core point and 0.02 rcut of the cut point (dPIE): there the N+- form
 *   of pi05_term64 is used (and at the centre itself, where pi05 is 0/0 as the reference's);
 *   0.02 rcut of the core point (dPIE): there log z_c - log z_t (s = rc), elsewhere
 *   log(1 + eps) (s = rcut).
 * (Near the centre the N+- form is only good to ~1e-12 of the small psi there; the
 * deflection form is regular at the centre.) */
constexpr double kSingCut64 = 4e-4;  /* x rcut^2 */
constexpr double kSingCore64 = 1e-3; /* x rc^2 */

/* The deflection of LT_FP64_FAST: for a dPIE pair away from its two 0/0 points, the
 * cancellation-free log(1 + eps) of log64 (1 log1p + 1 atan2, in place of the reference's
 * 2 log + 2 atan2); within 0.02 rcut of either point, and for PIEMD and SIS, the reference's
 * form of grad_pair.  alpha = pref (arg, -log| |) of z_c/z_t in the halo frame, as grad_pair. */
template <int TYPE>
__device__ __forceinline__ void grad_pair_fast(const lt_rec64 &h, double px, double py, double &gx, double &gy)
{
    if (TYPE != 81) {
        grad_pair<TYPE>(h, px, py, gx, gy);
        return;
    }
    Frame64 f = to_frame(h, px, py);
    const double u = f.u, v = f.v, uu = u * u;
    const double dvc = v - h.tsr_c, dvt = v - h.tsr_t;
    if ((uu + dvc * dvc < kSingCut64 * h.rcut2) | (uu + dvt * dvt < kSingCut64 * h.rcut2)) {
        grad_pair<TYPE>(h, px, py, gx, gy);
        return;
    }
    const Log64 z = log64<81>(h, u, v, uu, uu * h.cxro_inv + v * v * h.cyro_inv, false);
    const double re = h.pref_g * z.li, im = -h.pref_g * z.lr;
    gx += re * h.cs - im * h.sn;
    gy += im * h.cs + re * h.sn;
}

template <int TYPE>
__device__ __forceinline__ void pot_pair_fast(const lt_rec64 &h, double px, double py, double &psi)
{
    Frame64 f = to_frame(h, px, py);
    const double u = f.u, v = f.v;
    const double uu = u * u, vv = v * v;
    if (TYPE == 5) {
        psi += h.b0 * sqrt(uu * h.cx1 + vv * h.cx1inv);
        return;
    }
    const double rem2 = uu * h.cxro_inv + vv * h.cyro_inv;
    const double dvc = v - h.tsr_c;
    const double dc2 = uu + dvc * dvc;
    bool sing = (uu + vv == 0.) | (dc2 < kSingCore64 * h.rc2);
    bool split = false;
    if (TYPE == 81) {
        const double dvt = v - h.tsr_t;
        sing |= uu + dvt * dvt < kSingCut64 * h.rcut2;
        split = dc2 < kSingCut64 * h.rcut2;
    }
    if (!sing) {
        psi += pot64_defl<TYPE>(h, u, v, uu, rem2, split);
        return;
    }
    const double irem = rsqrt64(rem2), srem = rem2 * irem;
    const double iz = rsqrt64(uu + vv);
    const double s = h.e1 * v * iz, t = h.e2 * u * iz;
    const double g = fabs(s) + sqrt(s * s + 1.);
    const double ig = rcp64(g);
    Pi05Shared64 p;
    p.E2 = s >= 0. ? ig : g;
    p.iE2 = s >= 0. ? g : ig;
    const double ch2a = 0.5 * (p.E2 + p.iE2);
    p.sh2a = 0.5 * (p.E2 - p.iE2);
    p.c2e = sqrt(fmax(1. - t * t, 0.));
    p.t = t;
    p.sh2r = p.sh2a * p.c2e;
    p.sh2i = ch2a * t;
    const double itd = rcp64(ch2a + p.c2e), itd2 = itd * itd;
    p.itd4 = itd2 * itd2;
    double term = pi05_term64(p, u, v, srem, rem2, h.rc, h.rc2);
    if (TYPE == 81) term -= pi05_term64(p, u, v, srem, rem2, h.rcut, h.rcut2);
    psi += h.pref_h * term * irem;
}

} // namespace lt

/* ------------------------------------------------ reference-exact Hessian ---- */
/* The reference's Hessian arithmetic with its rounding sequence: every operation is a
 * separately rounded IEEE operation (no contraction into FMA, true division and square
 * root), in C's left-to-right evaluation order.  The results are bit-identical to the
 * reference FP64 CPU path (src/gradient2.cpp:54-205), whose formula is ill-conditioned
 * near each halo's removable singular points and near small-ellipticity cores: any other
 * rounding sequence differs there by up to ~1e-12 of the map scale. */
namespace lt {
namespace ex {
__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double V(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double R(double a) { return __dsqrt_rn(a); }

struct Mat {
    double a, b, c, d;
};

/* mdci05_hpc, src/gradient2.cpp:54-83 */
__device__ __forceinline__ Mat mdci05(double x, double y, double eps, double rc, double b0)
{
    const double sqe = R(eps);
    const double cx1 = V(S(1., eps), A(1., eps));
    const double cx1inv = V(1., cx1);
    const double cxro = M(A(1., eps), A(1., eps));
    const double cyro = M(S(1., eps), S(1., eps));
    const double ci = V(M(0.5, S(1., M(eps, eps))), sqe);
    const double wrem = R(A(A(M(rc, rc), V(M(x, x), cxro)), V(M(y, y), cyro)));
    const double sq2 = M(2., sqe);
    double den1 = S(M(sq2, wrem), M(y, cx1inv));
    den1 = A(M(M(M(cx1, cx1), x), x), M(den1, den1));
    const double num2 = S(M(M(2., rc), sqe), y);
    const double den2 = A(M(x, x), M(num2, num2));
    double t = A(S(V(V(M(M(sq2, x), x), cxro), wrem), M(sq2, wrem)), M(y, cx1inv));
    const double didxre = M(ci, A(V(M(cx1, t), den1), V(num2, den2)));
    t = S(V(V(M(M(M(sq2, x), y), cx1), cyro), wrem), x);
    const double didyre = M(ci, A(V(t, den1), V(x, den2)));
    t = S(M(M(sq2, wrem), cx1inv), M(M(y, cx1inv), cx1inv));
    t = S(t, V(M(M(4., eps), y), cyro));
    t = A(t, M(V(V(M(M(sq2, y), y), cyro), wrem), cx1inv));
    const double didyim = M(ci, S(V(t, den1), V(num2, den2)));
    Mat r;
    r.a = M(b0, didxre);
    r.b = r.d = M(b0, didyre);
    r.c = M(b0, didyim);
    return r;
}

/* two-step rotation back to the sky frame, src/gradient2.cpp:146-156 */
__device__ __forceinline__ void rotate_acc(const Mat &h, double cs, double sn, Mat &acc)
{
    const double ma = A(M(h.a, cs), M(h.b, -sn));
    const double mb = A(M(h.a, sn), M(h.b, cs));
    const double mc = A(M(h.d, sn), M(h.c, cs));
    const double md = A(M(h.d, cs), M(h.c, -sn));
    acc.a = A(acc.a, S(M(cs, ma), M(sn, md)));
    acc.b = A(acc.b, S(M(cs, mb), M(sn, mc)));
    acc.c = A(acc.c, A(M(sn, mb), M(cs, mc)));
    acc.d = A(acc.d, A(M(sn, ma), M(cs, md)));
}

/* One halo's Hessian added to the run accumulator `acc`: dPIE src/gradient2.cpp:92-205;
 * PIEMD (one mdci05 term) and SIS restated with the same rounding discipline. */
template <int TYPE>
__device__ __forceinline__ void hess_pair(const lt_rec64 &h, double px, double py, Mat &acc)
{
    const double tx = S(px, h.x0), ty = S(py, h.y0);
    const double u = A(M(tx, h.cs), M(ty, h.sn));
    const double v = S(M(ty, h.cs), M(tx, h.sn));
    Mat m;
    if (TYPE == 81) {
        const double t05 = V(h.rcut, S(h.rcut, h.rc));
        Mat core = mdci05(u, v, h.eps, h.rc, h.b0);
        const Mat cut = mdci05(u, v, h.eps, h.rcut, h.b0);
        m.a = M(t05, S(core.a, cut.a));
        m.b = M(t05, S(core.b, cut.b));
        m.c = M(t05, S(core.c, cut.c));
        m.d = M(t05, S(core.d, cut.d));
    } else if (TYPE == 8) {
        m = mdci05(u, v, h.eps, h.rc, h.b0);
    } else {
        const double e = h.eps;
        const double q = A(M(M(u, u), S(1., e)), M(M(v, v), A(1., e)));
        const double r = R(q);
        const double k = V(M(M(h.b0, S(1., e)), A(1., e)), M(q, r));
        m.a = M(M(k, v), v);
        m.c = M(M(k, u), u);
        m.b = m.d = M(M(-k, u), v);
    }
    rotate_acc(m, h.cs, h.sn, acc);
}
} // namespace ex

/* Convergence and sky-frame shear of one pair, unweighted, from the real-valued closed form
 * (lt_profiles32.cuh's forms in FP64, record lt_nie64): the FP32C path's recomputation of
 * pixels near critical curves.  About 70 FP64 operations for a dPIE pair against ~95 for
 * the reference's quotient form, and no 0/0 point; equal to it within ~1e-15 of the terms.
 * Every operation's rounding is pinned (explicit round-to-nearest multiply, add and fused
 * multiply-add), so the function can be inlined into any kernel, and interleaved over
 * several pixels, and still round each pair alike everywhere. */
struct Kg64 {
    double k, g1, g2;
};

template <int TYPE>
__device__ __forceinline__ Kg64 nie_kg64(const lt_nie64 &h, double px, double py)
{
    using ex::A;
    using ex::M;
    using ex::S;
    const double tx = S(px, h.x0), ty = S(py, h.y0);
    const double u = __fma_rn(tx, h.cs, M(ty, h.sn)), v = __fma_rn(ty, h.cs, -M(tx, h.sn));
    const double uu = M(u, u), vv = M(v, v), uv = M(u, v);
    double k, g1, g2;
    if (TYPE == 5) {
        const double ir = rsqrt64(__fma_rn(h.q2, uu, M(h.k, vv)));
        const double kk = M(M(h.K, ir), M(ir, ir));
        const double hk = M(0.5, kk);
        k = M(hk, A(uu, vv));
        g1 = M(hk, S(vv, uu));
        g2 = M(-kk, uv);
    } else {
        const double B = __fma_rn(h.q2, uu, vv), r2 = A(uu, vv);
        const double pc2 = A(B, h.q2sc2);
        const double ipc = rsqrt64(pc2), pc = M(pc2, ipc);
        const double Dc = __fma_rn(h.tsc, pc, A(h.opsc2, r2));
        if (TYPE == 8) {
            const double E = M(ipc, rcp64(Dc));
            k = M(h.K, ipc);
            g1 = __fma_rn(h.Kc1sc2, E, M(M(h.K, S(vv, uu)), E));
            g2 = M(M(-2. * h.K, uv), E);
        } else {
            const double pt2 = A(B, h.q2st2);
            const double ipt = rsqrt64(pt2), pt = M(pt2, ipt);
            const double Dt = __fma_rn(h.tst, pt, A(h.opst2, r2));
            const double dpsi = M(h.dq2s2, rcp64(A(pc, pt)));
            const double dD = __fma_rn(2., __fma_rn(pt, h.ds, M(h.sc, dpsi)), h.opds2);
            const double dpD = __fma_rn(dpsi, Dc, M(pt, dD));
            const double Ec = M(ipc, rcp64(Dc)), Et = M(ipt, rcp64(Dt));
            const double dEK = M(M(-h.K, M(dpD, Ec)), Et);
            k = M(M(-h.K, dpsi), M(ipc, ipt));
            g1 = __fma_rn(h.Kc1sc2, Ec, __fma_rn(-h.Kc1st2, Et, M(S(vv, uu), dEK)));
            g2 = M(-2., M(uv, dEK));
        }
    }
    return {k, __fma_rn(g1, h.c2t, -M(g2, h.s2t)), __fma_rn(g1, h.s2t, M(g2, h.c2t))};
}

/* The FP64 terms of one pair as out-of-line functions, for the FP32C path's FP64 work (its
 * cluster-scale halos, the near field of its galaxies, the recomputation near critical
 * curves).  Compiled once per profile type, they round alike in every kernel that calls
 * them, whatever else that kernel computes, so a map is the same from the grid kernels
 * and the work-queue tiles bit for bit; and their registers are not the calling pair
 * loop's. */
template <int TYPE>
__device__ __noinline__ Hess64 hess_term(const lt_rec64 &h, double px, double py, double w)
{
    Hess64 a = {0., 0., 0.};
    hess_pair<TYPE>(h, px, py, w, a);
    return a;
}

template <int TYPE>
__device__ __noinline__ double pot_term(const lt_rec64 &h, double px, double py)
{
    double p = 0.;
    pot_pair_fast<TYPE>(h, px, py, p);
    return p;
}

template <int TYPE>
__device__ __noinline__ double2 grad_term(const lt_rec64 &h, double px, double py)
{
    double gx = 0., gy = 0.;
    grad_pair_fast<TYPE>(h, px, py, gx, gy);
    return make_double2(gx, gy);
}
} // namespace lt
