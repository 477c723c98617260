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
    float cpi, s2rc, s2rcut, pad; /* cx1 + 1/cx1, 2 sqrt(e) rc, 2 sqrt(e) rcut                */
    float e1, e2, ppre, pad2;     /* potential: 2 sqrt(e)/(1-e), 2 sqrt(e)/(1+e), prefactor   */
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
        const float lr = 0.5f * (logf(nr * nr + nci * nci) - logf(u * u + dci * dci));
        const float li = atan2f(nci * u - nr * dci, nr * u + nci * dci);
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
    const float li = atan2f(ei, 1.f + er);
    return {h.ppre * li, -h.ppre * lr};
}

/* Potential, FP32.  pi05 of src/potential_GPU.cu:47-72 evaluated through identities that
 * remove its transcendental functions except the two complex logarithms per radius:
 *   exp(eta_re) = exp(-asinh(s)/2) = (|s| + sqrt(s^2 + 1))^(-sign(s)/2),  s = e1 v/z,
 *   eta_im = asin(t)/2, t = e2 u/z:  sin 2eta_im = t, cos 2eta_im = sqrt(1 - t^2),
 *     cos eta_im = sqrt((1 + cos 2eta_im)/2), sin eta_im = t/(2 cos eta_im),
 *   exp(zeta) = sqrt(ratio), ratio = (sqrt(rho^2) + sqrt(r^2 + rho^2))/r,
 *   sinh(2 zeta) = (ratio - 1/ratio)/2.
 * Returns the halo's potential without the FP64 cluster terms; far from the halo the
 * core - cut difference loses ~1e-5 of the term, small against the map's scale. */
struct Pi05Shared {
    float E, iE, ce, se, c2e, t;  /* exp(eta_re)^{+-1}, cos/sin eta_im, cos/sin 2 eta_im */
    float ch2r, ch2i;             /* cosh(eta)^2 */
    float sh2r, sh2i;             /* sinh(2 eta) */
};

__device__ __forceinline__ float clog_re2(float a, float b) { return 0.5f * __logf(a * a + b * b); }

__device__ __forceinline__ float pi05_term32(const Pi05Shared &p, float u, float v, float srem, float rem2, float r,
                                             float r2)
{
    const float ratio = (srem + sqrtf(r2 + rem2)) * frcp(r);
    const float Z = sqrtf(ratio);
    const float iZ = frcp(Z);
    const float ez = p.E * Z, iez = p.iE * iZ, ezm = p.E * iZ, iezm = p.iE * Z;
    const float b1r = 0.5f * (ez + iez) * p.ce, b1i = 0.5f * (ez - iez) * p.se;
    const float b2r = 0.5f * (ezm + iezm) * p.ce, b2i = 0.5f * (ezm - iezm) * p.se;
    /* b1 b2 and the two quotients */
    const float pr = b1r * b2r - b1i * b2i, pi = b1r * b2i + b1i * b2r;
    const float ip = frcp(pr * pr + pi * pi);
    const float q1r = (p.ch2r * pr + p.ch2i * pi) * ip, q1i = (p.ch2i * pr - p.ch2r * pi) * ip;
    const float ib2 = frcp(b2r * b2r + b2i * b2i);
    const float q2r = (b1r * b2r + b1i * b2i) * ib2, q2i = (b1i * b2r - b1r * b2i) * ib2;
    const float a1r = clog_re2(q1r, q1i), a1i = atan2f(q1i, q1r);
    const float a2r = clog_re2(q2r, q2i), a2i = atan2f(q2i, q2r);
    const float sh2z = 0.5f * (ratio - frcp(ratio));
    const float kr = (p.sh2r * a1r - p.sh2i * a1i) + sh2z * a2r;
    const float ki = (p.sh2i * a1r + p.sh2r * a1i) + sh2z * a2i;
    return r * (ki * u - kr * v);
}

template <int TYPE>
__device__ __forceinline__ float pot32(const lt_rec32 &h, float u, float v)
{
    if (TYPE == 5) return h.ppre * sqrtf(u * u * h.cx1 + v * v * h.icx1);
    const float uu = u * u, vv = v * v;
    const float rem2 = uu * h.cxi + vv * h.cyi;
    const float srem = sqrtf(rem2);
    const float iz = rsqrtf(uu + vv);
    Pi05Shared p;
    const float s = h.e1 * v * iz;
    const float t = fabsf(s) + sqrtf(s * s + 1.f);
    const float rt = rsqrtf(t), st = t * rt;
    p.E = s >= 0.f ? rt : st;
    p.iE = s >= 0.f ? st : rt;
    p.t = h.e2 * u * iz;
    p.c2e = sqrtf(fmaxf(1.f - p.t * p.t, 0.f));
    p.ce = sqrtf(0.5f * (1.f + p.c2e));
    p.se = 0.5f * p.t * frcp(p.ce);
    const float chr = 0.5f * (p.E + p.iE) * p.ce, chi = 0.5f * (p.E - p.iE) * p.se;
    p.ch2r = chr * chr - chi * chi;
    p.ch2i = 2.f * chr * chi;
    const float E2 = p.E * p.E, iE2 = p.iE * p.iE;
    p.sh2r = 0.5f * (E2 - iE2) * p.c2e;
    p.sh2i = 0.5f * (E2 + iE2) * p.t;
    float term = pi05_term32(p, u, v, srem, rem2, h.rc, h.rc2);
    if (TYPE == 81) term -= pi05_term32(p, u, v, srem, rem2, h.rcut, h.rcut2);
    return h.ppre * term * frcp(srem);
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
