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
    float rnear2, singv, sing_r2, pad2;    /* FP64 fallback regions: squared radius of the near
                                              field or core (larger of the two), the cut
                                              radius's singular point and its squared radius */
    float cpi, s2rc, s2rcut, ok3c; /* cx1 + 1/cx1, 2 sqrt(e) rc, 2 sqrt(e) rcut, (1-e)(3+e) rc */
    float om2, e4cxi, ppre, i4rc2; /* potential: (1-e)^2, 4e/(1+e)^2, prefactor, 1/(4 rc^2)    */
    int32_t type, idx64;
    float ok3t, i4rcut2;           /* (1-e)(3+e) rcut, 1/(4 rcut^2)                             */
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

/* atanh s for |s| <= 1/3: s P(s^2), P = 1 + c1 x + ... + c4 x^4 fitted to atanh(sqrt x)/sqrt x
 * on [0, 1/9] by a Remez exchange on the relative error (4.5e-9 in exact arithmetic; 1.2e-7
 * relative evaluated in FP32).  log1p(t)/2 = atanh(t/(2 + t)). */
__device__ __forceinline__ float fatanh_third(float s)
{
    const float x = s * s;
    float p = 1.400599331e-01f;
    p = fmaf(p, x, 1.400090307e-01f);
    p = fmaf(p, x, 2.001076341e-01f);
    p = fmaf(p, x, 3.333320916e-01f);
    p = fmaf(p, x, 1.0f);
    return s * p;
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
 * and dD = i 2 sqrt(e) (rc - rcut): no digit is lost to the cancellation.  With
 * eps = num/den, A = |den + num|^2 and B = |den|^2 (A - B = 2 Re(num conj den) + |num|^2
 * taken directly), Re log(1 + eps) = log(A/B)/2 = atanh((A - B)/(A + B)) (fatanh_third
 * where |s| <= 1/3, i.e. A/B in [1/2, 2]; __logf(A/B)/2 outside, where it is good to a
 * few ulp), and Im log(1 + eps) = atan2(Im(num conj den), B + Re(num conj den)), the
 * scale |den|^-2 dropped from both arguments.  (The reference's two arguments never
 * straddle the branch cut here: arg z_c - arg z_t equals arg(z_c/z_t), checked over
 * random halos down to 1e-3 rc from the centre.)  SIS (src/gradient.cpp:260-299):
 * b0 ((1-e) u, (1+e) v)/sqrt((1-e) u^2 + (1+e) v^2). */
struct Log32 {
    float li, lr;       /* arg and log| | of z (PIEMD) or z_c/z_t (dPIE) */
    float rho2, wc, wt; /* rho^2, w_c, w_t (w_t: dPIE only) */
};

template <int TYPE>
__device__ __forceinline__ Log32 log32(const lt_rec32 &h, float u, float v)
{
    Log32 o;
    o.rho2 = u * u * h.cxi + v * v * h.cyi;
    const float xc = h.rc2 + o.rho2;
    o.wc = xc * rsqrtf(xc);
    const float nr = h.cx1 * u;
    const float dci = h.s2rc - v;
    if (TYPE == 8) {
        /* A PIEMD has no cut: its potential grows like b0 |x| with nothing to cancel the
         * few-ulp error of the approximate instructions, so this branch (rare in the FP32
         * class: galaxies are cut dPIEs) uses CUDA's accurate sqrtf, division, logf and
         * atan2f.  z = N/D, A = |N|^2, B = |D|^2: log|z| = atanh((A - B)/(A + B)), where
         * (with w_c^2 - rc^2 = rho^2) A - B = 2 v (4e v/(1-e)^2 - 2 sqrt(e) (w_c/cx1 - rc)) is
         * taken without the cancellation of |N|^2 - |D|^2 near |z| = 1 (small e); arg z =
         * arg(N conj(D)), whose imaginary part u (2 sqrt(e) (w_c - cx1 rc) - v (1/cx1 - cx1))
         * avoids the same cancellation (1/cx1 - cx1 = 4e/(1-e^2)) */
        o.wc = sqrtf(xc);
        const float nci = h.s2 * o.wc - v * h.icx1;
        const float A = nr * nr + nci * nci, B = u * u + dci * dci;
        const float amb = 2.f * v * (h.e4 * h.cyi * v - h.s2 * fmaf(o.wc, h.icx1, -h.rc));
        const float s = amb / (A + B);
        o.lr = fabsf(s) <= (1.f / 3.f) ? fatanh_third(s) : 0.5f * logf(A / B);
        o.li = atan2f(u * (h.s2 * fmaf(-h.cx1, h.rc, o.wc) - v * (h.e4 * h.ome2)), nr * u + nci * dci);
        o.wt = 0.f;
        return o;
    }
    const float xt = h.rcut2 + o.rho2;
    o.wt = xt * rsqrtf(xt);
    const float dw = h.dr2 * frcp(o.wc + o.wt);
    const float nti = h.s2 * o.wt - v * h.icx1;
    const float dti = h.s2rcut - v;
    const float dni = h.s2 * dw, ddi = h.s2 * h.drs;
    /* num = i dni D_t - i ddi N_t,  den = D_c N_t */
    const float numr = ddi * nti - dni * dti;
    const float numi = dni * u - ddi * nr;
    const float denr = u * nr - dci * nti;
    const float deni = u * nti + dci * nr;
    /* 1 + eps = (den + num)/den; c + i d = num conj(den), B = |den|^2, A = |den + num|^2 */
    const float c = numr * denr + numi * deni;
    const float d = numi * denr - numr * deni;
    const float B = denr * denr + deni * deni;
    const float amb = fmaf(2.f, c, numr * numr + numi * numi); /* A - B */
    const float apb = fmaf(2.f, B, amb);                       /* A + B */
    const float s = amb * frcp(apb); /* (A - B)/(A + B) */
    o.lr = fabsf(s) <= (1.f / 3.f) ? fatanh_third(s) : 0.5f * __logf((B + amb) * frcp(B));
    o.li = fatan2(d, B + c);
    return o;
}

template <int TYPE>
__device__ __forceinline__ G32 grad32(const lt_rec32 &h, float u, float v)
{
    if (TYPE == 5) {
        const float ir = rsqrtf(u * u * h.cx1 + v * v * h.icx1);
        return {h.ppre * h.cx1 * u * ir, h.ppre * h.icx1 * v * ir};
    }
    const Log32 z = log32<TYPE>(h, u, v);
    return {h.ppre * z.li, -h.ppre * z.lr};
}

/* log(1 + t)/2 for t >= 0: atanh(t/(2 + t)) by fatanh_third for t <= 1, __logf above
 * (1 + t >= 2, where it is good to a few ulp). */
__device__ __forceinline__ float half_log1p_pos(float t)
{
    const float s = t * frcp(2.f + t);
    return t <= 1.f ? fatanh_third(s) : 0.5f * __logf(1.f + t);
}

/* Potential, FP32, through the deflection.  For a core-softened isothermal ellipsoid the
 * potential is x . alpha plus one logarithm per core radius, and the reference's pi05
 * (src/potential_GPU.cu:47-72, PIEMD; the cut dPIE is pref (pi05(rc) - pi05(rcut)),
 * src/potential_GPU.cu:137-187) is that form with the constant that makes it vanish at the
 * centre.  In the halo frame, with alpha = ppre (li, -lr) of log32 and w_r = sqrt(r^2 + rho^2):
 *   psi = ppre [ (u li - v lr) - 2 sqrt(e) (rc H(t_c) - rcut H(t_t)) ],  H(t) = log(1 + t)/2,
 *   1 + t_r = (((1-e) w_r + (1+e) r)^2 + 4e u^2/(1+e)^2)/(4 r^2),
 * (PIEMD: the rc term alone), and t_r is taken without cancellation as
 *   t_r = [(1-e)^2 A_r w_r + (1-e)(3+e) r A_r + 4e u^2/(1+e)^2]/(4 r^2),
 *   A_r = w_r - r = rho^2/(w_r + r),
 * a sum of non-negative terms.  (In FP64 the identity holds to rounding against pi05 over
 * e_pot up to 0.33 and rc/rcut down to 1/150; the tests compare the two paths.)  The form
 * shares the deflection's singular points, so the kernels take the potential in FP64 in the
 * same fallback regions as the deflection. */
__device__ __forceinline__ float tpot32(float rho2, float uterm, float w, float r, float ok3, float i4r2, float om2)
{
    const float a = rho2 * frcp(w + r);
    return (a * fmaf(om2, w, ok3) + uterm) * i4r2;
}

template <int TYPE>
__device__ __forceinline__ float pot32(const lt_rec32 &h, float u, float v)
{
    if (TYPE == 5) return h.ppre * fsqrt(u * u * h.cx1 + v * v * h.icx1);
    const Log32 z = log32<TYPE>(h, u, v);
    const float ut = h.e4cxi * u * u;
    if (TYPE == 8) { /* accurate operations, as in log32's PIEMD branch */
        const float t = (z.rho2 / (z.wc + h.rc) * fmaf(h.om2, z.wc, h.ok3c) + ut) * h.i4rc2;
        return h.ppre * ((u * z.li - v * z.lr) - h.s2 * h.rc * 0.5f * log1pf(t));
    }
    /* core term: outside the FP64 regions (3 rc and more from the centre) t_c > 0.44, where
     * __logf(1 + t) is within 1.8e-7 absolute, on a term that carries rc << rcut */
    float hs = h.rc * 0.5f * __logf(1.f + tpot32(z.rho2, ut, z.wc, h.rc, h.ok3c, h.i4rc2, h.om2));
    hs -= h.rcut * half_log1p_pos(tpot32(z.rho2, ut, z.wt, h.rcut, h.ok3t, h.i4rcut2, h.om2));
    return h.ppre * ((u * z.li - v * z.lr) - h.s2 * hs);
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
