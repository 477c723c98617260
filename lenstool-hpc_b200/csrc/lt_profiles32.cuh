/*
 * lt_profiles32.cuh -- FP32 per-pair Hessian arithmetic of the compensated path.
 *
 * The reference's mdci05 (src/gradient2.cpp:54-83) loses ~5 digits in FP32: the dPIE
 * term is the difference of two PIEMD terms (core and cut radius) that nearly cancel
 * far from the halo, and each PIEMD term is itself a difference of two fractions.  The
 * FP32 path therefore evaluates the same Hessian through forms without those
 * cancellations (derived here; they equal mdci05 to rounding in FP64, checked by the
 * tests):
 *
 *   w(s)  = sqrt(s^2 + rho^2),  rho^2 = u^2/(1+e)^2 + v^2/(1-e)^2
 *   kappa = b0/(2 w(s))                             (PIEMD convergence, core s)
 *   kappa_dPIE = b0 t05 (rc^2 - rcut^2)/(2 w_c w_t (w_c + w_t)) * (-1)
 *   gamma1 + i gamma2 = (ci b0/2) (Im q, -Re q),  q = F/G,
 *     N = cx1 u + i(2 sqrt(e) w - v/cx1),  D = u + i(2 s sqrt(e) - v),  G = N D,
 *     F = M D - 2 N with M = dN/dx + i dN/dy (simplified to avoid cancellation):
 *     Re F = 4e u [1/(1-e^2) - 2 sqrt(e) v/(w (1-e^2)^2) - s/(w (1+e)^2)]
 *     Im F = 2 s sqrt(e)(cx1 + 1/cx1) - 2 sqrt(e)(s^2/w + w) + 4e v/(1-e^2)
 *            - 4e s v/(w (1-e)^2)
 *   dPIE:  q_c - q_t = (dF G_c - F_c dG)/(G_c G_t), with dF, dG built from
 *     w_c - w_t = (rc^2 - rcut^2)/(w_c + w_t) and the other exact core-cut differences.
 *
 * The forms are still singular (0/0) at the point u = 0, v = 2 s sqrt(e) of each radius;
 * the kernel evaluates pairs near those points, near the core, close to a galaxy
 * (b0/2r > tau) and every cluster-scale halo in FP64 instead.
 */
#pragma once
#include <stdint.h>

struct alignas(16) lt_rec32 {
    double x0, y0;
    float cs, sn, c2t, s2t;       /* cos, sin of the angle; cos 2 angle, sin 2 angle        */
    float s2, cx1, icx1, cxi;     /* 2 sqrt(e), (1-e)/(1+e), 1/cx1, 1/(1+e)^2                */
    float cyi, ome2, e4, kpre;    /* 1/(1-e)^2, 1/(1-e^2), 4e, kappa prefactor               */
    float gpre, rc, rcut, drs;    /* gamma prefactor, rc, rcut, rc - rcut                    */
    float dr2, rc2, rcut2, w;     /* rc^2 - rcut^2, rc^2, rcut^2, Kmap weight                */
    float rnear2, singv, sing_r2, core_r2; /* FP64 fallback regions (squared radii)          */
    float cpi, s2rc, s2rcut, irc; /* cx1 + 1/cx1, 2 sqrt(e) rc, 2 sqrt(e) rcut, 1/rc           */
    float e1, e2, ppre, ircut;    /* potential: 2 sqrt(e)/(1-e), 2 sqrt(e)/(1+e), prefactor, 1/rcut */
    int32_t type, idx64, pad0, pad1;
};
static_assert(sizeof(lt_rec32) == 160, "record size");

namespace lt {
/* rnear2 of an FP64 proxy record: a halo of the FP32 class whose parameters, after an
 * in-place update, need FP64 everywhere.  Every pixel then falls in its fallback region,
 * and its potential terms are taken in FP64 as well. */
constexpr float kProxy64 = __builtin_huge_valf();
} // namespace lt

#ifdef __CUDACC__
namespace lt {

__device__ __forceinline__ float frcp(float x) { return __fdividef(1.0f, x); }

/* Square root to the approximate instruction's accuracy (relative error ~2^-23), for
 * operands whose rounding the compensated path tolerates; zero and denormals give 0. */
__device__ __forceinline__ float fsqrt(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* atan2 in FP32.  a = min(|x|,|y|)/max(|x|,|y|) in [0, 1]; atan a = a P(a^2) with P of
 * degree 7, fitted to atan(a)/a on [0, 1] by a Remez exchange on the relative error
 * (max 9.9e-8 in exact arithmetic); then atan2 = pi/2 - atan a where |y| > |x|,
 * pi - that where x < 0, with the sign of y.  Against FP64 atan2: <= 3.8e-7 absolute,
 * 3e-7 relative (checked over |x|, |y| in [1e-6, 1e3]).  Needs (x, y) != (0, 0). */
__device__ __forceinline__ float fatan2(float y, float x)
{
    const float ax = fabsf(x), ay = fabsf(y);
    const float a = fminf(ax, ay) * frcp(fmaxf(ax, ay));
    const float s = a * a;
    float p = -4.693276249e-03f;
    p = fmaf(p, s, 2.425240353e-02f);
    p = fmaf(p, s, -5.948639289e-02f);
    p = fmaf(p, s, 9.914293140e-02f);
    p = fmaf(p, s, -1.401948035e-01f);
    p = fmaf(p, s, 1.996972412e-01f);
    p = fmaf(p, s, -3.333199024e-01f);
    p = fmaf(p, s, 9.999998808e-01f);
    float r = a * p;
    r = ay > ax ? 1.57079637f - r : r;
    r = x < 0.f ? 3.14159274f - r : r;
    return copysignf(r, y);
}

struct KG32 {
    float k, g1, g2; /* halo-frame convergence and shear */
};

/* F(s) of the header comment. */
__device__ __forceinline__ void f_num(const lt_rec32 &h, float u, float v, float s, float s2s, float ss, float w,
                                      float iw, float &fr, float &fi)
{
    fr = h.e4 * u * (h.ome2 - h.s2 * v * iw * h.ome2 * h.ome2 - s * iw * h.cxi);
    fi = s2s * h.cpi - h.s2 * (ss * iw + w) + h.e4 * v * h.ome2 - h.e4 * s * v * iw * h.cyi;
}

template <int TYPE>
__device__ __forceinline__ KG32 hess32(const lt_rec32 &h, float u, float v)
{
    KG32 r;
    if (TYPE == 5) {
        /* SIS: psi = b0 R, R^2 = (1-e)u^2 + (1+e)v^2; kpre = b0 (1-e)(1+e) */
        const float q = u * u * h.cx1 + v * v * h.icx1;
        const float ir = rsqrtf(q);
        const float k = h.kpre * ir * ir * ir;
        r.k = 0.5f * k * (u * u + v * v);
        r.g1 = 0.5f * k * (v * v - u * u);
        r.g2 = -k * u * v;
        return r;
    }
    const float rho2 = u * u * h.cxi + v * v * h.cyi;
    const float xc = h.rc2 + rho2;
    const float iwc = rsqrtf(xc);
    const float wc = xc * iwc;
    const float nr = h.cx1 * u;
    const float nci = h.s2 * wc - v * h.icx1;
    const float dci = h.s2rc - v;
    /* G_c = N_c D_c */
    const float gcr = nr * u - nci * dci, gci = nr * dci + nci * u;
    float fcr, fci;
    f_num(h, u, v, h.rc, h.s2rc, h.rc2, wc, iwc, fcr, fci);
    if (TYPE == 8) {
        r.k = h.kpre * iwc;
        const float inv = frcp(gcr * gcr + gci * gci);
        const float qr = (fcr * gcr + fci * gci) * inv;
        const float qi = (fci * gcr - fcr * gci) * inv;
        r.g1 = h.gpre * qi;
        r.g2 = -h.gpre * qr;
        return r;
    }
    /* TYPE 81: core minus cut, differences taken analytically */
    const float xt = h.rcut2 + rho2;
    const float iwt = rsqrtf(xt);
    const float wt = xt * iwt;
    const float ssum = frcp(wc + wt);
    const float iww = iwc * iwt;
    const float dw = h.dr2 * ssum;   /* w_c - w_t */
    const float diw = -dw * iww;     /* 1/w_c - 1/w_t */
    r.k = h.kpre * h.dr2 * iww * ssum;
    const float nti = h.s2 * wt - v * h.icx1;
    const float dti = h.s2rcut - v;
    const float gtr = nr * u - nti * dti, gti = nr * dti + nti * u;
    const float dni = h.s2 * dw;     /* N_c - N_t = i dni */
    const float ddi = h.s2 * h.drs;  /* D_c - D_t = i ddi */
    /* dG = dN D_c + N_t dD */
    const float dgr = -dni * dci - nti * ddi;
    const float dgi = dni * u + nr * ddi;
    const float dsw = (h.rc * wt - h.rcut * wc) * iww;        /* rc/w_c - rcut/w_t */
    const float ds2w = (h.rc2 * wt - h.rcut2 * wc) * iww;     /* rc^2/w_c - rcut^2/w_t */
    const float dfr = h.e4 * u * (-h.s2 * v * diw * h.ome2 * h.ome2 - dsw * h.cxi);
    const float dfi = ddi * h.cpi - h.s2 * (ds2w + dw) - h.e4 * v * dsw * h.cyi;
    /* numerator dF G_c - F_c dG, denominator G_c G_t */
    const float n_r = (dfr * gcr - dfi * gci) - (fcr * dgr - fci * dgi);
    const float n_i = (dfr * gci + dfi * gcr) - (fcr * dgi + fci * dgr);
    const float d_r = gcr * gtr - gci * gti;
    const float d_i = gcr * gti + gci * gtr;
    const float inv = frcp(d_r * d_r + d_i * d_i);
    const float qr = (n_r * d_r + n_i * d_i) * inv;
    const float qi = (n_i * d_r - n_r * d_i) * inv;
    r.g1 = h.gpre * qi;
    r.g2 = -h.gpre * qr;
    return r;
}

struct G32 {
    float x, y; /* halo-frame deflection */
};

/* Deflection, FP32.  The reference writes the PIEMD deflection as
 * pref (arg z, -log|z|) with z = N/D, N = cx1 u + i(2 sqrt(e) w - v/cx1),
 * D = u + i(2 r sqrt(e) - v), w = sqrt(r^2 + rho^2) (the KERNEL of src/gradient.cpp:
 * 548-607, 744-811; pref = ci b0 [rcut/(rcut - rc)]), and the cut dPIE as the difference
 * of the core and cut terms, which cancel far from the halo.  Here that difference is
 * log(z_c/z_t) = log(1 + eps) with eps = (dN D_t - dD N_t)/(D_c N_t), built from the exact
 * differences dN = N_c - N_t = i 2 sqrt(e) (w_c - w_t), w_c - w_t = (rc^2 - rcut^2)/(w_c + w_t),
 * and dD = i 2 sqrt(e) (rc - rcut): no digit is lost to the cancellation, and
 * Re log(1 + eps) = log1p(2 eps_r + |eps|^2)/2, Im = atan2(eps_i, 1 + eps_r).  (The
 * reference's two arguments never straddle the branch cut here: arg z_c - arg z_t equals
 * arg(z_c/z_t), checked over the workload catalogues.)  SIS (src/gradient.cpp:260-299):
 * b0 ((1-e) u, (1+e) v)/sqrt((1-e) u^2 + (1+e) v^2). */
template <int TYPE>
__device__ __forceinline__ G32 grad32(const lt_rec32 &h, float u, float v)
{
    if (TYPE == 5) {
        const float ir = rsqrtf(u * u * h.cx1 + v * v * h.icx1);
        return {h.ppre * h.cx1 * u * ir, h.ppre * h.icx1 * v * ir};
    }
    const float rho2 = u * u * h.cxi + v * v * h.cyi;
    const float xc = h.rc2 + rho2;
    const float wc = xc * rsqrtf(xc);
    const float nr = h.cx1 * u;
    const float dci = h.s2rc - v;
    if (TYPE == 8) {
        const float nci = h.s2 * wc - v * h.icx1;
        /* z = N/D: log|z| = (log|N|^2 - log|D|^2)/2, arg z = arg(N conj(D)) */
        const float lr = 0.5f * __logf((nr * nr + nci * nci) * frcp(u * u + dci * dci));
        const float li = fatan2(nci * u - nr * dci, nr * u + nci * dci);
        return {h.ppre * li, -h.ppre * lr};
    }
    const float xt = h.rcut2 + rho2;
    const float wt = xt * rsqrtf(xt);
    const float dw = h.dr2 * frcp(wc + wt);
    const float nti = h.s2 * wt - v * h.icx1;
    const float dti = h.s2rcut - v;
    const float dni = h.s2 * dw, ddi = h.s2 * h.drs;
    /* num = i dni D_t - i ddi N_t,  den = D_c N_t */
    const float numr = ddi * nti - dni * dti;
    const float numi = dni * u - ddi * nr;
    const float denr = u * nr - dci * nti;
    const float deni = u * nti + dci * nr;
    const float inv = frcp(denr * denr + deni * deni);
    const float er = (numr * denr + numi * deni) * inv;
    const float ei = (numi * denr - numr * deni) * inv;
    const float lr = 0.5f * log1pf(er * (2.f + er) + ei * ei);
    const float li = fatan2(ei, 1.f + er);
    return {h.ppre * li, -h.ppre * lr};
}

/* Potential, FP32.  pi05 of src/potential_GPU.cu:47-72 is, with b1 = cosh(eta + zeta),
 * b2 = cosh(eta - zeta) (zeta real), r (Im k u - Re k v) b0 ci/rho_e with
 *   k = sinh(2 eta) log(cosh^2 eta/(b1 b2)) + sinh(2 zeta) log(b1/b2).
 * Writing w = tanh eta tanh zeta and a = eta_re,
 *   b1 b2 = cosh^2 eta cosh^2 zeta (1 - w)(1 + w),   b1/b2 = (1 + w)/(1 - w),
 *   1 +- w = N+- / (cosh 2a + cos 2 eta_im),
 *   N+  = (e^{2a}  - 2 sinh 2a/(rho + 1) + cos 2 eta_im) + i B,
 *   N-  = (e^{-2a} + 2 sinh 2a/(rho + 1) + cos 2 eta_im) - i B,   B = tanh zeta sin 2 eta_im,
 * whose real parts are sums of positive terms or lose at most half (no cancellation, also
 * where tanh eta -> +-1 at high ellipticity), so
 *   log(b1/b2) = log|N+|^2/|N-|^2 / 2 + i arg(N+ conj N-),
 *   log(cosh^2 eta/(b1 b2)) = -log(cosh^4 zeta |N+|^2 |N-|^2/(cosh 2a + cos 2 eta_im)^4)/2
 *                             - i arg(N+ N-),
 * with Re(N+ N-) = Re N+ Re N- + B^2 > 0 and Im(N+ N-) = -2 B tanh zeta sinh 2a exactly;
 * the arguments are those of the reference's principal logarithms (both |arg| < pi), and no
 * complex quotient is formed.  With s = e1 v/z and t = e2 u/z:
 *   e^{2a} = exp(-asinh s) = (|s| + sqrt(s^2 + 1))^(-sign s),
 *   sin 2 eta_im = t, cos 2 eta_im = sqrt(1 - t^2),
 *   e^{2 zeta} = rho = (rho_e + sqrt(r^2 + rho_e^2))/r, with rho - 1 taken without
 *   cancellation as (rho_e + rho_e^2/(sqrt(r^2 + rho_e^2) + r))/r,
 *   tanh zeta = (rho - 1)/(rho + 1), cosh^2 zeta = (rho + 1)^2/(4 rho),
 *   sinh 2 zeta = (rho - 1)(rho + 1)/(2 rho).
 * Returns the halo's potential without the FP64 cluster terms; far from the halo the
 * core - cut difference loses ~1e-5 of the term, small against the map's scale. */
struct Pi05Shared {
    float sh2r, sh2i;      /* sinh(2 eta) */
    float E2, iE2, sh2a;   /* e^{2a}, e^{-2a}, sinh 2a */
    float c2e, t;          /* cos, sin of 2 eta_im */
    float itd4;            /* (cosh 2a + cos 2 eta_im)^-4 */
};

__device__ __forceinline__ float pi05_term32(const Pi05Shared &p, float u, float v, float srem, float rem2, float r,
                                             float r2, float ir)
{
    const float q = fsqrt(r2 + rem2);
    const float dm = (srem + rem2 * frcp(q + r)) * ir; /* rho - 1 */
    const float rho = 1.f + dm, rho1 = rho + 1.f;
    const float inv = frcp(rho * rho1);
    const float irho = rho1 * inv, irho1 = rho * inv;
    const float tz = dm * irho1;                        /* tanh zeta */
    const float sh2z = 0.5f * dm * rho1 * irho;         /* sinh 2 zeta */
    const float ch2z = 0.25f * rho1 * rho1 * irho;      /* cosh^2 zeta */
    const float m = 2.f * irho1 * p.sh2a;
    const float A = (p.E2 - m) + p.c2e, C = (p.iE2 + m) + p.c2e, B = tz * p.t, B2 = B * B;
    const float np2 = A * A + B2, nm2 = C * C + B2;
    const float a2r = 0.5f * __logf(np2 * frcp(nm2));
    const float a2i = fatan2(B * (A + C), A * C - B2);
    const float a1r = -0.5f * __logf((ch2z * ch2z) * (np2 * nm2) * p.itd4);
    const float a1i = fatan2(2.f * B * tz * p.sh2a, A * C + B2);
    const float kr = (p.sh2r * a1r - p.sh2i * a1i) + sh2z * a2r;
    const float ki = (p.sh2i * a1r + p.sh2r * a1i) + sh2z * a2i;
    return r * (ki * u - kr * v);
}

template <int TYPE>
__device__ __forceinline__ float pot32(const lt_rec32 &h, float u, float v)
{
    if (TYPE == 5) return h.ppre * fsqrt(u * u * h.cx1 + v * v * h.icx1);
    const float uu = u * u, vv = v * v;
    const float rem2 = uu * h.cxi + vv * h.cyi;
    const float irem = rsqrtf(rem2);
    const float srem = rem2 * irem;
    const float iz = rsqrtf(uu + vv);
    const float s = h.e1 * v * iz;
    const float t = h.e2 * u * iz;
    const float g = fabsf(s) + fsqrt(s * s + 1.f);
    const float ig = frcp(g);
    const float E2 = s >= 0.f ? ig : g, iE2 = s >= 0.f ? g : ig; /* exp(+-2 eta_re) */
    const float ch2a = 0.5f * (E2 + iE2), sh2a = 0.5f * (E2 - iE2);
    const float c2e = fsqrt(fmaxf(1.f - t * t, 0.f));
    Pi05Shared p;
    p.sh2r = sh2a * c2e;
    p.sh2i = ch2a * t;
    p.E2 = E2;
    p.iE2 = iE2;
    p.sh2a = sh2a;
    p.c2e = c2e;
    p.t = t;
    const float itd = frcp(ch2a + c2e), itd2 = itd * itd;
    p.itd4 = itd2 * itd2;
    float term = pi05_term32(p, u, v, srem, rem2, h.rc, h.rc2, h.irc);
    if (TYPE == 81) term -= pi05_term32(p, u, v, srem, rem2, h.rcut, h.rcut2, h.ircut);
    return h.ppre * term * irem;
}

/* Kahan compensated accumulation of one FP32 component. */
__device__ __forceinline__ void kahan_add(float &s, float &c, float x)
{
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

} // namespace lt
#endif
