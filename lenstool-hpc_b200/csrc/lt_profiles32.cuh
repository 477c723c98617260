/*
 * lt_profiles32.cuh -- FP32 per-pair arithmetic of the compensated path (LT_FP32C).
 *
 * The reference writes the PIEMD Hessian, deflection and potential with complex
 * quotients of N = cx1 u + i(2 sqrt(e) w - v/cx1) and D = u + i(2 s sqrt(e) - v)
 * (mdci05, src/gradient2.cpp:54-83; the deflection of src/gradient.cpp:548-607, 744-811;
 * pi05, src/potential_GPU.cu:47-72), and the cut dPIE as the difference of a core and a
 * cut term (src/gradient2.cpp:92-167).  In FP32 those forms lose ~5 digits: the two terms
 * nearly cancel far from a galaxy, each quotient is itself a difference of fractions, and
 * N, D vanish together at u = 0, v = 2 s sqrt(e).
 *
 * The same model has a real-valued closed form.  Its density is elliptical, isodensity
 * axes (1 + e) and (1 - e): the non-singular isothermal ellipse with axis ratio
 * q = (1 - e)/(1 + e) and core s = (1 + e) r_core.  With psi_s = sqrt(q^2 (s^2 + u^2) + v^2)
 * and D_s = (1 + q^2) s^2 + 2 s psi_s + u^2 + v^2 (halo frame, u along the major axis),
 * and A = b0 (1 - e) t05 (t05 = rcut/(rcut - rc) for the dPIE, 1 for the PIEMD):
 *   kappa   = (A/2) / psi_s,
 *   gamma1  = (A/2) ((q^2 - 1) s^2 + v^2 - u^2) / (psi_s D_s),
 *   gamma2  = -A u v / (psi_s D_s),
 *   alpha_u = (A/k) atan(k u / (psi_s + s)),  alpha_v = (A/k) atanh(k v / (psi_s + q^2 s)),
 *   potential = u alpha_u + v alpha_v - (A s/2) log(1 + t_s),
 *     t_s = (u^2 + v^2 + 2 s B/(psi_s + q s)) / (4 r_core^2),  B = q^2 u^2 + v^2,
 * with k = sqrt(1 - q^2).  (They equal the reference's forms to FP64 rounding: Hessian and
 * deflection within 1e-14, the potential within the reference pi05's own error, checked
 * against the oracle by the tests; the potential's constant makes it vanish at the centre,
 * as pi05 does.)  None of them has a 0/0 point.  For the cut dPIE (core c minus cut t) the
 * differences are taken without cancellation through the exact differences
 *   psi_c - psi_t = q^2 (s_c^2 - s_t^2)/(psi_c + psi_t),
 *   D_c - D_t = (1 + q^2)(s_c^2 - s_t^2) + 2 (s_c (psi_c - psi_t) + psi_t (s_c - s_t)),
 *   psi_c D_c - psi_t D_t = (psi_c - psi_t) D_c + psi_t (D_c - D_t),
 * whose terms share one sign, and atan a_c - atan a_t = atan((a_c - a_t)/(1 + a_c a_t)),
 * atanh b_c - atanh b_t = atanh((b_c - b_t)/(1 - b_c b_t)) with a_c - a_t and b_c - b_t
 * formed from psi_c - psi_t and s_c - s_t.  Emulated in FP32 over random galaxy-scale
 * halos the per-term relative errors are below 1e-6 (kappa 6e-7, gamma 8e-7 of
 * |gamma1| + |gamma2|, deflection 1.1e-6, potential 6.5e-7).
 *
 * The kernels still evaluate in FP64 every cluster-scale halo, and the pairs within the
 * near field of a galaxy (b0/2r > tau) or 3 rcore of its centre, where one term is large.
 */
#pragma once
#include <stdint.h>

/* FP32 record of a PIEMD / cut dPIE (type 8 / 81) of the FP32 class.  Core c, cut t
 * (type 8: the core fields only).  A type-5 (SIS) record uses q2 = 1 - e, k = 1 + e,
 * K = b0 (1 - e)(1 + e) and Ak = b0. */
struct alignas(16) lt_rec32 {
    double x0, y0;
    float cs, sn, c2t, s2t;          /* cos, sin of the angle; cos, sin of twice the angle  */
    float q2, k, k2, w;              /* q^2, k = sqrt(1 - q^2), k^2, Kmap weight             */
    float sc, st, ds, dsq2;          /* s_c = (1+e) rc, s_t = (1+e) rcut, s_c - s_t, q^2 (s_c - s_t) */
    float q2sc2, q2st2, dq2s2, rnear2; /* q^2 s_c^2, q^2 s_t^2, q^2 (s_c^2 - s_t^2); FP64 disc
                                          (squared radius of the near field or the core)     */
    float opsc2, opst2, opds2, tsc;  /* (1+q^2) s_c^2, (1+q^2) s_t^2, (1+q^2)(s_c^2 - s_t^2), 2 s_c */
    float tst, K, Kc1sc2, Kc1st2;    /* 2 s_t, K = A/2, K (q^2-1) s_c^2, K (q^2-1) s_t^2       */
    float Ak, qsc, qst, q2sc;        /* A/k, q s_c, q s_t, q^2 s_c                            */
    float q2st, Asc, Ast, i4rc2;     /* q^2 s_t, A s_c/2, A s_t/2, 1/(4 rc^2)                 */
    float i4rcut2;                   /* 1/(4 rcut^2)                                          */
    int32_t type, idx64;
    float Ascl2;                     /* A s_c ln(2)/2                                         */
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

/* FP32 operations with their rounding pinned: the compiler never fuses or reorders them,
 * so every kernel that evaluates a pair (grid kernels of any shape, the work-queue tiles,
 * a call with or without the potential) rounds it alike, bit for bit. */
namespace f32 {
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
} // namespace f32

/* Reciprocal, reciprocal square root and log2 by the approximate instructions alone
 * (rcp/rsqrt/lg2.approx, relative error ~2^-23, log2 absolute ~2^-22).  The .ftz forms
 * flush subnormal operands to zero, which skips the operand scaling the default forms
 * wrap around the instruction; every operand here is a normal number (a squared radius,
 * a denominator, a log argument of 2 or more), where both forms return the same value. */
__device__ __forceinline__ float frcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float frsqrt(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
/* log2 by the approximate instruction; the natural logarithm as ln 2 log2(x) and half of it
 * as (ln 2 / 2) log2(x), for x >= 2 (where the log2 instruction's absolute error is a few
 * ulp of the result).  ln 2 / 2 in FP32 is exactly half of ln 2 in FP32, so the half
 * logarithm is exactly half of flog's value (one multiply instead of two). */
__device__ __forceinline__ float flog2(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
constexpr float kLn2f = 0.693147182f, kHalfLn2f = 0.346573591f;
__device__ __forceinline__ float flog(float x) { return __fmul_rn(flog2(x), kLn2f); }
__device__ __forceinline__ float fhalf_log(float x) { return __fmul_rn(flog2(x), kHalfLn2f); }

/* Square root to the approximate instruction's accuracy (relative error ~2^-23), for
 * operands whose rounding the compensated path tolerates; zero and denormals give 0. */
__device__ __forceinline__ float fsqrt(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* atan(a) for a in [0, 1]: a P(a^2) with P of degree 7, fitted to atan(a)/a on [0, 1] by a
 * Remez exchange on the relative error (max 9.9e-8 in exact arithmetic;
 * tests/golden/fit_fast_math.py regenerates the coefficients). */
__device__ __forceinline__ float fatan_unit(float a)
{
    using namespace f32;
    const float s = mul(a, a);
    float p = -4.693276249e-03f;
    p = fma(p, s, 2.425240353e-02f);
    p = fma(p, s, -5.948639289e-02f);
    p = fma(p, s, 9.914293140e-02f);
    p = fma(p, s, -1.401948035e-01f);
    p = fma(p, s, 1.996972412e-01f);
    p = fma(p, s, -3.333199024e-01f);
    p = fma(p, s, 9.999998808e-01f);
    return mul(a, p);
}

/* atan2 in FP32: a = min(|x|,|y|)/max(|x|,|y|), atan a by fatan_unit, then
 * pi/2 - atan a where |y| > |x|, pi - that where x < 0, with the sign of y.  Against FP64
 * atan2: <= 3.8e-7 absolute, 3e-7 relative (checked over |x|, |y| in [1e-6, 1e3]).
 * Needs (x, y) != (0, 0). */
__device__ __forceinline__ float fatan2(float y, float x)
{
    const float ax = fabsf(x), ay = fabsf(y);
    float r = fatan_unit(f32::mul(fminf(ax, ay), frcp(fmaxf(ax, ay))));
    r = ay > ax ? f32::sub(1.57079637f, r) : r;
    r = x < 0.f ? f32::sub(3.14159274f, r) : r;
    return copysignf(r, y);
}

/* atan(y/x) for x > 0 (fatan2 without its fold for x < 0). */
__device__ __forceinline__ float fatan_pos(float y, float x)
{
    const float ay = fabsf(y);
    float r = fatan_unit(f32::mul(fminf(x, ay), frcp(fmaxf(x, ay))));
    r = ay > x ? f32::sub(1.57079637f, r) : r;
    return copysignf(r, y);
}

/* atanh s for |s| <= 1/3: s P(s^2), P = 1 + c1 x + ... + c4 x^4 fitted to atanh(sqrt x)/sqrt x
 * on [0, 1/9] by a Remez exchange on the relative error (4.5e-9 in exact arithmetic; 1.2e-7
 * relative evaluated in FP32; regenerated by tests/golden/fit_fast_math.py).
 * log1p(t)/2 = atanh(t/(2 + t)). */
__device__ __forceinline__ float fatanh_third(float s)
{
    using namespace f32;
    const float x = mul(s, s);
    float p = 1.400599331e-01f;
    p = fma(p, x, 1.400090307e-01f);
    p = fma(p, x, 2.001076341e-01f);
    p = fma(p, x, 3.333320916e-01f);
    p = fma(p, x, 1.0f);
    return mul(s, p);
}

/* atanh y for |y| < 1: fatanh_third where |y| <= 1/3, log((1 + y)/(1 - y))/2 above (an
 * argument of 2 or more, where flog is good to a few ulp). */
__device__ __forceinline__ float fatanh_any(float y)
{
    using namespace f32;
    return fabsf(y) <= (1.f / 3.f) ? fatanh_third(y) : fhalf_log(mul(add(1.f, y), frcp(sub(1.f, y))));
}

/* log(1 + t)/2 for t >= 0: atanh(t/(2 + t)) by fatanh_third for t <= 1, flog above
 * (1 + t >= 2, where flog is good to a few ulp). */
__device__ __forceinline__ float half_log1p_pos(float t)
{
    using namespace f32;
    return t <= 1.f ? fatanh_third(mul(t, frcp(add(2.f, t)))) : fhalf_log(add(1.f, t));
}

struct KG32 {
    float k, g1, g2; /* halo-frame convergence and shear */
};

struct G32 {
    float x, y; /* halo-frame deflection */
};

/* The radius-dependent quantities shared by the Hessian, deflection and potential of one
 * pair: u^2, v^2, B = q^2 u^2 + v^2, psi and 1/psi of the core (and cut) radius, and
 * psi_c - psi_t. */
struct Nie32 {
    float uu, vv, B, pc, ipc, pt, ipt, dpsi;
};

template <int TYPE>
__device__ __forceinline__ Nie32 nie32(const lt_rec32 &h, float u, float v)
{
    using namespace f32;
    Nie32 n;
    n.uu = mul(u, u);
    n.vv = mul(v, v);
    if (TYPE == 5) {
        n.B = fma(h.q2, n.uu, mul(h.k, n.vv)); /* R^2 = (1-e) u^2 + (1+e) v^2 */
        n.ipc = frsqrt(n.B);
        n.pc = mul(n.B, n.ipc);
        n.pt = n.ipt = n.dpsi = 0.f;
        return n;
    }
    n.B = fma(h.q2, n.uu, n.vv);
    if (TYPE == 8) {
        /* a PIEMD has no cut: its potential grows like b0 |x| with nothing to dilute the
         * few-ulp errors of approximate instructions, so this branch (rare in the FP32
         * class: galaxies are cut dPIEs) takes CUDA's accurate square root and divisions */
        n.pc = __fsqrt_rn(add(n.B, h.q2sc2));
        n.ipc = __fdiv_rn(1.f, n.pc);
        n.pt = n.ipt = n.dpsi = 0.f;
        return n;
    }
    const float pc2 = add(n.B, h.q2sc2), pt2 = add(n.B, h.q2st2);
    n.ipc = frsqrt(pc2);
    n.ipt = frsqrt(pt2);
    n.pc = mul(pc2, n.ipc);
    n.pt = mul(pt2, n.ipt);
    n.dpsi = mul(h.dq2s2, frcp(add(n.pc, n.pt)));
    return n;
}

/* Halo-frame Hessian (convergence, shear) of one pair. */
template <int TYPE>
__device__ __forceinline__ KG32 hess32(const lt_rec32 &h, float u, float v, const Nie32 &n)
{
    using namespace f32;
    KG32 r;
    if (TYPE == 5) {
        /* SIS: psi = b0 R; K = b0 (1-e)(1+e) */
        const float kk = mul(mul(h.K, n.ipc), mul(n.ipc, n.ipc));
        r.k = mul(mul(0.5f, kk), add(n.uu, n.vv));
        r.g1 = mul(mul(0.5f, kk), sub(n.vv, n.uu));
        r.g2 = mul(-kk, mul(u, v));
        return r;
    }
    const float r2 = add(n.uu, n.vv);
    const float Dc = fma(h.tsc, n.pc, add(h.opsc2, r2));
    if (TYPE == 8) {
        const float E = __fdiv_rn(n.ipc, Dc);
        r.k = mul(h.K, n.ipc);
        r.g1 = fma(h.Kc1sc2, E, mul(mul(h.K, sub(n.vv, n.uu)), E));
        r.g2 = mul(mul(-2.f * h.K, mul(u, v)), E);
        return r;
    }
    const float Dt = fma(h.tst, n.pt, add(h.opst2, r2));
    /* D_c - D_t and psi_c D_c - psi_t D_t (every term negative) */
    const float dD = fma(2.f, fma(n.pt, h.ds, mul(h.sc, n.dpsi)), h.opds2);
    const float dpD = fma(n.dpsi, Dc, mul(n.pt, dD));
    const float Ec = mul(n.ipc, frcp(Dc)), Et = mul(n.ipt, frcp(Dt)); /* 1/(psi D) */
    const float dEK = mul(mul(-h.K, mul(dpD, Ec)), Et);               /* K (E_c - E_t) */
    r.k = mul(mul(-h.K, n.dpsi), mul(n.ipc, n.ipt));
    r.g1 = fma(h.Kc1sc2, Ec, fma(-h.Kc1st2, Et, mul(sub(n.vv, n.uu), dEK)));
    r.g2 = mul(-2.f, mul(mul(u, v), dEK));
    return r;
}

/* Halo-frame deflection of one pair. */
template <int TYPE>
__device__ __forceinline__ G32 grad32(const lt_rec32 &h, float u, float v, const Nie32 &n)
{
    using namespace f32;
    if (TYPE == 5) /* SIS: b0 ((1-e) u, (1+e) v)/R; Ak = b0 */
        return {mul(mul(h.Ak, h.q2), mul(u, n.ipc)), mul(mul(h.Ak, h.k), mul(v, n.ipc))};
    if (TYPE == 8) { /* accurate operations, as in nie32's PIEMD branch */
        const float y = __fdiv_rn(mul(h.k, v), add(n.pc, h.q2sc));
        return {mul(h.Ak, atan2f(mul(h.k, u), add(n.pc, h.sc))),
                mul(mul(h.Ak, 0.5f), log1pf(__fdiv_rn(mul(2.f, y), sub(1.f, y))))};
    }
    /* atan a_c - atan a_t, a = k u/(psi + s):  (a_c - a_t)/(1 + a_c a_t) =
     *   -k u (dpsi + ds) / ((psi_c + s_c)(psi_t + s_t) + k^2 u^2)  (numerator terms of one sign) */
    const float nu = mul(mul(-h.k, u), add(n.dpsi, h.ds));
    const float du = fma(h.k2, n.uu, mul(add(n.pc, h.sc), add(n.pt, h.st)));
    /* atanh b_c - atanh b_t, b = k v/(psi + q^2 s):  (b_c - b_t)/(1 - b_c b_t) =
     *   -k v (dpsi + q^2 ds) / ((psi_c + q^2 s_c)(psi_t + q^2 s_t) - k^2 v^2)  (> q^2 v^2 > 0) */
    const float nv = mul(mul(-h.k, v), add(n.dpsi, h.dsq2));
    const float dv = fma(-h.k2, n.vv, mul(add(n.pc, h.q2sc), add(n.pt, h.q2st)));
    return {mul(h.Ak, fatan_pos(nu, du)), mul(h.Ak, fatanh_any(mul(nv, frcp(dv))))};
}

/* Potential of one pair from its deflection g (halo frame):
 *   u g_x + v g_y - (A s_c/2) log(1 + t_c) [+ (A s_t/2) log(1 + t_t) for the dPIE],
 *   t_s = (u^2 + v^2 + 2 s B/(psi_s + q s)) / (4 r^2), a sum of non-negative terms,
 *   1 + t_s = ((psi_s + s)^2 + k^2 u^2) / (4 r^2). */
template <int TYPE>
__device__ __forceinline__ float pot32(const lt_rec32 &h, float u, float v, const Nie32 &n, const G32 &g)
{
    using namespace f32;
    if (TYPE == 5) return mul(h.Ak, fsqrt(n.B)); /* SIS: b0 R */
    const float r2 = add(n.uu, n.vv);
    const float xa = fma(u, g.x, mul(v, g.y));
    if (TYPE == 8) { /* accurate operations */
        const float tc = mul(add(r2, __fdiv_rn(mul(h.tsc, n.B), add(n.pc, h.qsc))), h.i4rc2);
        return sub(xa, mul(h.Asc, log1pf(tc)));
    }
    /* core term: outside the FP64 disc (3 rc and more from the centre) t_c > 2, so 1 + t_c
     * is taken directly as ((psi_c + s_c)^2 + k^2 u^2) / (4 rc^2), a sum of non-negative
     * terms with psi_c + s_c shared with the deflection, and log2 of it is good to a few
     * ulp; on a term that carries rc << rcut */
    const float pcs = add(n.pc, h.sc);
    const float opt_c = mul(fma(h.k2, n.uu, mul(pcs, pcs)), h.i4rc2);
    const float tt = mul(fma(mul(h.tst, n.B), frcp(add(n.pt, h.qst)), r2), h.i4rcut2);
    return sub(xa, fma(h.Ascl2, flog2(opt_c), mul(-2.f * h.Ast, half_log1p_pos(tt))));
}

} // namespace lt
#endif
