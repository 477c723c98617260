/*
 * lt_eval.cuh -- per-chunk pair loops shared by the grid kernels (lt_grid64.cu,
 * lt_grid32.cu) and the work-queue kernel (lt_queue.cu).
 *
 * A chunk is a run of at most LT_CHUNK halo records of one profile type, staged in
 * shared memory; every thread walks the same records (shared-memory broadcast) and adds
 * their terms to the sums of its P pixels.
 */
#pragma once
#include "lt_bulk.cuh"
#include "lt_profiles32.cuh"
#include "lt_profiles64.cuh"

namespace lt {

/* ---- FP64 sums (LT_FP64 / LT_FP64_FAST) ---------------------------------------------- */

template <int OP, int P>
struct Acc64 {
    double gx[P], gy[P], hxx[P], hyy[P], hxy[P], psi[P];
    ex::Mat run[P], tot[P]; /* OP_HEX: the reference's per-run and total sums */
};

template <int OP, int P, int TYPE>
__device__ __forceinline__ void eval_chunk64(const lt_rec64 *recs, int count, const double (&px)[P], double py,
                                             int kmap, Acc64<OP, P> &acc)
{
#pragma unroll 1
    for (int h = 0; h < count; h++) {
        const lt_rec64 &r = recs[h];
        const double w = kmap ? r.w : 1.0;
#pragma unroll
        for (int k = 0; k < P; k++) {
            if ((OP & OP_GRAD) && (OP & OP_GFX)) grad_pair_fast<TYPE>(r, px[k], py, acc.gx[k], acc.gy[k]);
            if ((OP & OP_GRAD) && !(OP & OP_GFX)) grad_pair<TYPE>(r, px[k], py, acc.gx[k], acc.gy[k]);
            if (OP & OP_HESS) {
                Hess64 hh = {acc.hxx[k], acc.hyy[k], acc.hxy[k]};
                hess_pair<TYPE>(r, px[k], py, w, hh);
                acc.hxx[k] = hh.xx;
                acc.hyy[k] = hh.yy;
                acc.hxy[k] = hh.xy;
            }
            if (OP & OP_HEX) ex::hess_pair<TYPE>(r, px[k], py, acc.run[k]);
            if ((OP & OP_POT) && (OP & OP_PEX)) pot_pair<TYPE>(r, px[k], py, acc.psi[k]);
            if ((OP & OP_POT) && !(OP & OP_PEX)) pot_pair_fast<TYPE>(r, px[k], py, acc.psi[k]);
        }
    }
}

/* The FP64 recomputation's sums: convergence and sky-frame shear from the closed form
 * (nie_kg64) of one chunk of lt_nie64 records at Q pixels of arbitrary positions
 * (px[k], py[k]), added to (kap, g1, g2)[k] (by one fused multiply-add with the record's
 * weight for a Kmap).  The Q pixels' dependent chains are independent of one another, so
 * the compiler interleaves them; nie_kg64's pinned rounding keeps each pair's value the
 * same for any Q and in every kernel. */
template <int Q, int TYPE>
__device__ __forceinline__ void eval_nie_q(const lt_nie64 *recs, int count, const double (&px)[Q],
                                           const double (&py)[Q], int kmap, double (&kap)[Q], double (&g1)[Q],
                                           double (&g2)[Q])
{
#pragma unroll 1
    for (int h = 0; h < count; h++) {
        const lt_nie64 &r = recs[h];
#pragma unroll
        for (int k = 0; k < Q; k++) {
            const Kg64 t = nie_kg64<TYPE>(r, px[k], py[k]);
            if (kmap) {
                kap[k] = __fma_rn(r.w, t.k, kap[k]);
                g1[k] = __fma_rn(r.w, t.g1, g1[k]);
                g2[k] = __fma_rn(r.w, t.g2, g2[k]);
            } else {
                kap[k] = __dadd_rn(kap[k], t.k);
                g1[k] = __dadd_rn(g1[k], t.g1);
                g2[k] = __dadd_rn(g2[k], t.g2);
            }
        }
    }
}

/* eval_nie_q over one staged chunk of any profile type. */
template <int Q>
__device__ __forceinline__ void eval_nie_chunk(const lt_chunk &c, const lt_nie64 *recs, const double (&px)[Q],
                                               const double (&py)[Q], int kmap, double (&kap)[Q], double (&g1)[Q],
                                               double (&g2)[Q])
{
    switch (c.type) {
    case 81: eval_nie_q<Q, 81>(recs, c.count, px, py, kmap, kap, g1, g2); break;
    case 8: eval_nie_q<Q, 8>(recs, c.count, px, py, kmap, kap, g1, g2); break;
    case 5: eval_nie_q<Q, 5>(recs, c.count, px, py, kmap, kap, g1, g2); break;
    default: break;
    }
}

/* The recomputed pixel's Hessian from its convergence and shear sums. */
__device__ __forceinline__ void nie_hessian(double kap, double g1, double g2, double &hxx, double &hyy, double &hxy)
{
    hxx = __dadd_rn(kap, g1);
    hyy = __dsub_rn(kap, g1);
    hxy = g2;
}

/* End of a run of the reference's dispatch (src/gradient2.cpp:240-251): the run's sum
 * joins the total, weighted by the run's dlsds for the Kmap
 * (src/gradient2_GPU.cu:503-507). */
template <int OP, int P>
__device__ __forceinline__ void close_run64(Acc64<OP, P> &acc, int kmap, double w)
{
#pragma unroll
    for (int k = 0; k < P; k++) {
        ex::Mat &t = acc.tot[k];
        const ex::Mat &r = acc.run[k];
        if (kmap) {
            t.a = ex::A(t.a, ex::M(r.a, w));
            t.b = ex::A(t.b, ex::M(r.b, w));
            t.c = ex::A(t.c, ex::M(r.c, w));
            t.d = ex::A(t.d, ex::M(r.d, w));
        } else {
            t.a = ex::A(t.a, r.a);
            t.b = ex::A(t.b, r.b);
            t.c = ex::A(t.c, r.c);
            t.d = ex::A(t.d, r.d);
        }
        acc.run[k].a = acc.run[k].b = acc.run[k].c = acc.run[k].d = 0.;
    }
}

/* ---- FP32-compensated sums (LT_FP32C) ------------------------------------------------ */

/* FP32 terms are summed in FP32 over blocks of at most kBlock32 halos; each block sum then
 * joins an FP64 sum.  A block adds at most (kBlock32 - 1) u sum|t| of rounding error
 * (u = 2^-24), the order of the terms' own evaluation error, and the FP64 sums add nothing
 * further: this replaces a per-term compensated (Kahan) update at a quarter of its cost. */
constexpr int kBlock32 = 8;

/* Sums of one pixel.  FP64: convergence, shear and potential (halo-frame Hessians are
 * rotated to the sky frame before they are added) and the deflection.  FP32: the running
 * block sums, and the magnitudes of the FP32 terms from which the error of the FP32 part
 * is estimated (fp32c_total): sum kappa_i^2 and sum (|gamma1_i| + |gamma2_i|)^2 (halo
 * frame) for the terms' own errors, sum kappa_i for the rounding of the block sums. */
template <int P>
struct Acc32 {
    double kap[P], g1[P], g2[P], psi[P], gx[P], gy[P];
    float bk[P], bg1[P], bg2[P], bp[P], bgx[P], bgy[P];
    float mk[P], mg[P], ml[P];
};

/* Zero the sums of pixel k. */
template <int P>
__device__ __forceinline__ void acc32_zero(Acc32<P> &acc, int k)
{
    acc.kap[k] = acc.g1[k] = acc.g2[k] = acc.psi[k] = acc.gx[k] = acc.gy[k] = 0.;
    acc.bk[k] = acc.bg1[k] = acc.bg2[k] = acc.bp[k] = acc.bgx[k] = acc.bgy[k] = 0.f;
    acc.mk[k] = acc.mg[k] = acc.ml[k] = 0.f;
}

/* Join the FP32 block sums to the FP64 sums, with the chunk's Kmap weight w (1 outside
 * the Kmap; an FP32C chunk never mixes weights), and start new blocks. */
template <int OP, int P>
__device__ __forceinline__ void fold32(Acc32<P> &acc, double w)
{
#pragma unroll
    for (int k = 0; k < P; k++) {
        if (OP & OP_HESS) {
            acc.kap[k] = __fma_rn(w, (double)acc.bk[k], acc.kap[k]);
            acc.g1[k] = __fma_rn(w, (double)acc.bg1[k], acc.g1[k]);
            acc.g2[k] = __fma_rn(w, (double)acc.bg2[k], acc.g2[k]);
            acc.ml[k] = __fmaf_rn((float)w, acc.bk[k], acc.ml[k]);
            acc.bk[k] = acc.bg1[k] = acc.bg2[k] = 0.f;
        }
        if (OP & OP_POT) {
            acc.psi[k] = __dadd_rn(acc.psi[k], (double)acc.bp[k]);
            acc.bp[k] = 0.f;
        }
        if (OP & OP_GRAD) {
            acc.gx[k] = __dadd_rn(acc.gx[k], (double)acc.bgx[k]);
            acc.gy[k] = __dadd_rn(acc.gy[k], (double)acc.bgy[k]);
            acc.bgx[k] = acc.bgy[k] = 0.f;
        }
    }
}

/* Add one FP64 pair's Hessian (sky frame, weight included) as convergence and shear. */
template <int P>
__device__ __forceinline__ void add_hess64(Acc32<P> &acc, int k, const Hess64 &h)
{
    acc.kap[k] = __fma_rn(0.5, __dadd_rn(h.xx, h.yy), acc.kap[k]);
    acc.g1[k] = __fma_rn(0.5, __dsub_rn(h.xx, h.yy), acc.g1[k]);
    acc.g2[k] = __dadd_rn(acc.g2[k], h.xy);
}

/* The pixel box of one warp: centre (FP64) and half sizes.  Every pixel the warp's
 * lanes evaluate (the clamped ones at the grid's edges included) lies inside it. */
struct WarpBox {
    double cx, cy, hx, hy;
};

/* Box of the warp whose lane evaluates columns ix .. ix + P - 1 of row iy, with the
 * tile layout of the grid kernels (8 lanes x P columns, 4 rows per warp). */
template <int P>
__device__ __forceinline__ WarpBox warp_box(const GridArgs &a, int ix, int iy)
{
    const int lane = threadIdx.x & 31;
    const int c0 = ix - (lane & 7) * P, r0 = iy - (lane >> 3);
    const int c1 = c0 + 8 * P - 1, r1 = r0 + 3;
    const double x0 = pixel_x(a, c0 < a.nx ? c0 : a.nx - 1), x1 = pixel_x(a, c1 < a.nx ? c1 : a.nx - 1);
    const double y0 = pixel_y(a, r0 < a.ny ? r0 : a.ny - 1), y1 = pixel_y(a, r1 < a.ny ? r1 : a.ny - 1);
    return {0.5 * (x0 + x1), 0.5 * (y0 + y1), 0.5 * fabs(x1 - x0), 0.5 * fabs(y1 - y0)};
}

/* Squared distance from the box to the point (px, py) (0 inside). */
__device__ __forceinline__ double box_dist2(const WarpBox &b, double px, double py)
{
    const double dx = fmax(fabs(px - b.cx) - b.hx, 0.), dy = fmax(fabs(py - b.cy) - b.hy, 0.);
    return dx * dx + dy * dy;
}

/* Mask of the records of a chunk whose FP64 disc (near field or core) reaches the warp's
 * box: bit h for record h (count <= 64).  Lane l tests records l and l + 32 in FP64 with
 * the disc's squared radius enlarged by 1e-4 relative, beyond the FP32 rounding of the
 * per-pixel test (a few 1e-7 of a squared distance), so that a record outside the mask
 * has no pixel of the warp in its disc and the per-pixel test can be skipped for it. */
__device__ __forceinline__ uint64_t near_mask(const lt_rec32 *recs, int count, const WarpBox &b)
{
    const int lane = threadIdx.x & 31;
    uint32_t m[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int h = lane + 32 * j;
        bool hit = false;
        if (h < count) {
            const lt_rec32 &r = recs[h];
            hit = box_dist2(b, r.x0, r.y0) <= (double)r.rnear2 * (1. + 1e-4);
        }
        m[j] = __ballot_sync(0xffffffffu, hit);
    }
    return (uint64_t)m[0] | ((uint64_t)m[1] << 32);
}

template <int OP, int P, int TYPE>
__device__ __forceinline__ void eval64_chunk(const lt_rec64 *recs, int count, const double (&px)[P], double py, int kmap,
                                             Acc32<P> &acc)
{
#pragma unroll 1
    for (int h = 0; h < count; h++) {
        const lt_rec64 &r = recs[h];
        const double w = kmap ? r.w : 1.0;
#pragma unroll
        for (int k = 0; k < P; k++) {
            if (OP & OP_HESS) add_hess64(acc, k, hess_term<TYPE>(r, px[k], py, w));
            if (OP & OP_POT) acc.psi[k] = __dadd_rn(acc.psi[k], pot_term<TYPE>(r, px[k], py));
            if (OP & OP_GRAD) {
                const double2 t = grad_term<TYPE>(r, px[k], py);
                acc.gx[k] = __dadd_rn(acc.gx[k], t.x);
                acc.gy[k] = __dadd_rn(acc.gy[k], t.y);
            }
        }
    }
}

/* One chunk of FP32 records (at most 128) for the pixels px[0..P) of row py, the lane's
 * pixels (ix .. ix + P - 1, iy) of grid `a`.  Every record of an FP32C chunk has the same
 * Kmap weight. */
template <int OP, int P, int TYPE>
__device__ __forceinline__ void eval32_chunk(const lt_rec32 *recs, const lt_rec64 *recs64, int count,
                                             const double (&px)[P], double py, const GridArgs &a, int ix, int iy,
                                             Acc32<P> &acc)
{
    const int kmap = a.kmap;
    const double wchunk = kmap ? (double)recs[0].w : 1.0;
    const WarpBox box = warp_box<P>(a, ix, iy);
#pragma unroll 1
    for (int h0 = 0; h0 < count; h0 += 64) {
        const int n = count - h0 < 64 ? count - h0 : 64;
        const uint64_t mask = near_mask(recs + h0, n, box);
#pragma unroll 1
        for (int h = h0; h < h0 + n; h++) {
            const lt_rec32 &r = recs[h];
            float u[P], v[P];
            const float ty = __double2float_rn(__dsub_rn(py, r.y0));
#pragma unroll
            for (int k = 0; k < P; k++) {
                const float tx = __double2float_rn(__dsub_rn(px[k], r.x0));
                u[k] = __fmaf_rn(tx, r.cs, __fmul_rn(ty, r.sn));
                v[k] = __fmaf_rn(ty, r.cs, -__fmul_rn(tx, r.sn));
            }
            bool near = false;
            if ((mask >> (h - h0)) & 1ull) {
                /* the FP64 disc (an FP64 proxy record has rnear2 = +inf: every pixel) */
#pragma unroll
                for (int k = 0; k < P; k++) near |= __fmaf_rn(u[k], u[k], __fmul_rn(v[k], v[k])) < r.rnear2;
                near = __any_sync(0xffffffffu, near);
            }
            if (near) {
                const lt_rec64 &r64 = recs64[r.idx64];
                const double w = kmap ? r64.w : 1.0;
#pragma unroll
                for (int k = 0; k < P; k++) {
                    if (OP & OP_HESS) add_hess64(acc, k, hess_term<TYPE>(r64, px[k], py, w));
                    if (OP & OP_GRAD) {
                        const double2 t = grad_term<TYPE>(r64, px[k], py);
                        acc.gx[k] = __dadd_rn(acc.gx[k], t.x);
                        acc.gy[k] = __dadd_rn(acc.gy[k], t.y);
                    }
                    if (OP & OP_POT) acc.psi[k] = __dadd_rn(acc.psi[k], pot_term<TYPE>(r64, px[k], py));
                }
            } else {
#pragma unroll
                for (int k = 0; k < P; k++) {
                    const Nie32 n = nie32<TYPE>(r, u[k], v[k]);
                    if (OP & OP_HESS) {
                        const KG32 t = hess32<TYPE>(r, u[k], v[k], n);
                        acc.bk[k] = __fadd_rn(acc.bk[k], t.k);
                        acc.bg1[k] = __fmaf_rn(t.g1, r.c2t, __fmaf_rn(-t.g2, r.s2t, acc.bg1[k]));
                        acc.bg2[k] = __fmaf_rn(t.g1, r.s2t, __fmaf_rn(t.g2, r.c2t, acc.bg2[k]));
                        const float ag = __fadd_rn(fabsf(t.g1), fabsf(t.g2));
                        acc.mk[k] = __fmaf_rn(t.k, t.k, acc.mk[k]);
                        acc.mg[k] = __fmaf_rn(ag, ag, acc.mg[k]);
                    }
                    if (OP & (OP_GRAD | OP_POT)) {
                        const G32 t = grad32<TYPE>(r, u[k], v[k], n);
                        if (OP & OP_GRAD) {
                            acc.bgx[k] = __fmaf_rn(t.x, r.cs, __fmaf_rn(-t.y, r.sn, acc.bgx[k]));
                            acc.bgy[k] = __fmaf_rn(t.y, r.cs, __fmaf_rn(t.x, r.sn, acc.bgy[k]));
                        }
                        if (OP & OP_POT) acc.bp[k] = __fadd_rn(acc.bp[k], pot32<TYPE>(r, u[k], v[k], n, t));
                    }
                }
            }
            if ((h & (kBlock32 - 1)) == kBlock32 - 1) fold32<OP, P>(acc, wchunk);
        }
    }
    if (count & (kBlock32 - 1)) fold32<OP, P>(acc, wchunk);
}

/* Pixel totals of the FP32C sums as the sky-frame Hessian and potential, the Jacobian
 * determinant (1 - kappa D)^2 - (gamma1 D)^2 - (gamma2 D)^2 (explicitly rounded FP64, the
 * same rounding in every kernel that uses it) and an estimate of the determinant's error
 * from the FP32 terms.  The FP32 terms' relative errors (their evaluation, and their share
 * of the rounding of a block sum) have an RMS of about kEpsTerm32 (1.2e-7 for the closed
 * forms emulated with correctly rounded operations; the approximate reciprocal and square
 * roots add a little), are of either sign and independent from halo to halo, and stay
 * below 9e-7 each (measured on B200 over random galaxy-scale halos).  So the FP32 part of
 * kappa and of each shear component is held to kSpread32 standard deviations of that sum
 * of independent errors, kEpsTerm32 kSpread32 times the root sum of squares of the terms;
 * the convergence adds kEpsBlock32 of the (one-signed) sum of its terms for the coherent
 * part of the blocks' rounding.  The two shear components' errors being independent too,
 *   |d det| <= 2 D (|1 - kappa D| dk + |gamma D| dg).
 * Three standard deviations, because the tolerance a pixel is held to (mu_tol, 5e-7) is
 * half of the maps' 1e-6 target: a pixel dominated by one term at its worst measured error
 * (kappa 7.9e-7 against the estimate's 7.2e-7 of the term, shear 8.7e-7 of |g1| + |g2|
 * against 6e-7) still stays below 1e-6 (7.3e-7 at most), and a sum of many terms exceeds
 * twice its estimate only at six standard deviations.  (Five, the earlier setting, sent 87%
 * of the posterior field's pixels and 16.7% of the benchmark field's to the FP64
 * recomputation; three sends 65% and 13%, by an FP64 emulation of the estimate.) */
constexpr float kEpsTerm32 = 2.0e-7f;
constexpr float kSpread32 = 3.f;
constexpr float kEpsBlock32 = 1.2e-7f;

template <int P>
__device__ __forceinline__ void fp32c_total(const Acc32<P> &acc, int k, double D, double &hxx, double &hyy,
                                            double &hxy, double &psi, double &det, double &det_err)
{
    using namespace rn;
    const double kap = acc.kap[k], g1 = acc.g1[k], g2 = acc.g2[k];
    hxx = add(kap, g1);
    hyy = sub(kap, g1);
    hxy = g2;
    psi = acc.psi[k];
    const double omk = sub(1., mul(kap, D)), g1d = mul(g1, D), g2d = mul(g2, D);
    det = sub(sub(mul(omk, omk), mul(g1d, g1d)), mul(g2d, g2d));
    const float dk = __fmaf_rn(kEpsTerm32 * kSpread32, __fsqrt_rn(acc.mk[k]), __fmul_rn(kEpsBlock32, acc.ml[k]));
    const float dg = __fmul_rn(kEpsTerm32 * kSpread32, __fsqrt_rn(acc.mg[k]));
    const double gd = sqr(add(mul(g1d, g1d), mul(g2d, g2d)));
    det_err = mul(mul(2., D), add(mul(fabs(omk), (double)dk), mul(gd, (double)dg)));
}

/* Pixel total of the FP32C deflection sums. */
template <int P>
__device__ __forceinline__ void fp32c_grad_total(const Acc32<P> &acc, int k, double &gx, double &gy)
{
    gx = acc.gx[k];
    gy = acc.gy[k];
}

/* True when the FP32 part's error bound on the magnification exceeds mu_tol of
 * max(|mu|, 1) (near a critical curve the determinant amplifies the error of the sums):
 * |d mu| = mu^2 |d det| <= mu_tol max(|mu|, 1), i.e. |d det| <= mu_tol |det| max(1, |det|).
 * (A map of mu is measured against max(|mu|, its RMS), and its RMS is at least about 1, the
 * magnification far from any lens.)  The pixel is then recomputed in FP64. */
__device__ __forceinline__ bool fp32c_flag(double det, double det_err, double mu_tol)
{
    const double ad = fabs(det);
    return !(det_err <= mu_tol * ad * fmax(1., ad));
}

} // namespace lt
