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
        double w = kmap ? r.w : 1.0;
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

template <int P>
struct Acc32 {
    double hxx[P], hyy[P], hxy[P], psi[P], gx[P], gy[P]; /* FP64 terms, sky frame */
    float ks[P], kc[P], g1s[P], g1c[P], g2s[P], g2c[P], ps[P], pc[P]; /* Kahan sums of FP32 terms */
    float gxs[P], gxc[P], gys[P], gyc[P];
};

/* Zero the sums of pixel k. */
template <int P>
__device__ __forceinline__ void acc32_zero(Acc32<P> &acc, int k)
{
    acc.hxx[k] = acc.hyy[k] = acc.hxy[k] = acc.psi[k] = acc.gx[k] = acc.gy[k] = 0.;
    acc.ks[k] = acc.kc[k] = acc.g1s[k] = acc.g1c[k] = acc.g2s[k] = acc.g2c[k] = 0.f;
    acc.ps[k] = acc.pc[k] = acc.gxs[k] = acc.gxc[k] = acc.gys[k] = acc.gyc[k] = 0.f;
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
            if (OP & OP_HESS) {
                Hess64 hh = {acc.hxx[k], acc.hyy[k], acc.hxy[k]};
                hess_pair<TYPE>(r, px[k], py, w, hh);
                acc.hxx[k] = hh.xx;
                acc.hyy[k] = hh.yy;
                acc.hxy[k] = hh.xy;
            }
            if (OP & OP_POT) pot_pair_fast<TYPE>(r, px[k], py, acc.psi[k]);
            if (OP & OP_GRAD) grad_pair_fast<TYPE>(r, px[k], py, acc.gx[k], acc.gy[k]);
        }
    }
}

template <int OP, int P, int TYPE>
__device__ __forceinline__ void eval32_chunk(const lt_rec32 *recs, const lt_rec64 *recs64, int count,
                                             const double (&px)[P], double py, int kmap, Acc32<P> &acc)
{
#pragma unroll 1
    for (int h = 0; h < count; h++) {
        const lt_rec32 &r = recs[h];
        float u[P], v[P];
        bool near = false;
        const float ty = (float)(py - r.y0);
#pragma unroll
        for (int k = 0; k < P; k++) {
            const float tx = (float)(px[k] - r.x0);
            u[k] = tx * r.cs + ty * r.sn;
            v[k] = ty * r.cs - tx * r.sn;
            const float rr = u[k] * u[k] + v[k] * v[k];
            const float dv = v[k] - r.singv;
            near |= (rr < r.rnear2) | (u[k] * u[k] + dv * dv < r.sing_r2);
        }
        /* the FP64 fallback regions (an FP64 proxy record has rnear2 = +inf: every pixel) */
        if (__any_sync(0xffffffffu, near)) {
            const lt_rec64 &r64 = recs64[r.idx64];
            const double w = kmap ? r64.w : 1.0;
#pragma unroll
            for (int k = 0; k < P; k++) {
                if (OP & OP_HESS) {
                    Hess64 hh = {acc.hxx[k], acc.hyy[k], acc.hxy[k]};
                    hess_pair<TYPE>(r64, px[k], py, w, hh);
                    acc.hxx[k] = hh.xx;
                    acc.hyy[k] = hh.yy;
                    acc.hxy[k] = hh.xy;
                }
                if (OP & OP_GRAD) grad_pair_fast<TYPE>(r64, px[k], py, acc.gx[k], acc.gy[k]);
                if (OP & OP_POT) pot_pair_fast<TYPE>(r64, px[k], py, acc.psi[k]);
            }
        } else {
            const float w = kmap ? r.w : 1.0f;
#pragma unroll
            for (int k = 0; k < P; k++) {
                if (OP & OP_HESS) {
                    KG32 t = hess32<TYPE>(r, u[k], v[k]);
                    const float g1 = t.g1 * r.c2t - t.g2 * r.s2t;
                    const float g2 = t.g1 * r.s2t + t.g2 * r.c2t;
                    kahan_add(acc.ks[k], acc.kc[k], w * t.k);
                    kahan_add(acc.g1s[k], acc.g1c[k], w * g1);
                    kahan_add(acc.g2s[k], acc.g2c[k], w * g2);
                }
                if (OP & OP_GRAD) {
                    const G32 t = grad32<TYPE>(r, u[k], v[k]);
                    kahan_add(acc.gxs[k], acc.gxc[k], t.x * r.cs - t.y * r.sn);
                    kahan_add(acc.gys[k], acc.gyc[k], t.y * r.cs + t.x * r.sn);
                }
                if (OP & OP_POT) kahan_add(acc.ps[k], acc.pc[k], pot32<TYPE>(r, u[k], v[k]));
            }
        }
    }
}

/* Pixel totals of the FP32C sums: the FP64 terms plus the compensated FP32 sums (s - c)
 * as the sky-frame Hessian and potential, and the Jacobian determinant
 * (1 - kappa D)^2 - (gamma1 D)^2 - (gamma2 D)^2, in explicitly rounded FP64 (the same
 * rounding in every kernel that uses it). */
template <int P>
__device__ __forceinline__ void fp32c_total(const Acc32<P> &acc, int k, double D, double &hxx, double &hyy,
                                            double &hxy, double &psi, double &det)
{
    using namespace rn;
    const double kap = add(mul(0.5, add(acc.hxx[k], acc.hyy[k])), sub((double)acc.ks[k], (double)acc.kc[k]));
    const double g1 = add(mul(0.5, sub(acc.hxx[k], acc.hyy[k])), sub((double)acc.g1s[k], (double)acc.g1c[k]));
    const double g2 = add(acc.hxy[k], sub((double)acc.g2s[k], (double)acc.g2c[k]));
    hxx = add(kap, g1);
    hyy = sub(kap, g1);
    hxy = g2;
    psi = add(acc.psi[k], sub((double)acc.ps[k], (double)acc.pc[k]));
    const double omk = sub(1., mul(kap, D)), g1d = mul(g1, D), g2d = mul(g2, D);
    det = sub(sub(mul(omk, omk), mul(g1d, g1d)), mul(g2d, g2d));
}

/* Pixel total of the FP32C deflection sums. */
template <int P>
__device__ __forceinline__ void fp32c_grad_total(const Acc32<P> &acc, int k, double &gx, double &gy)
{
    gx = rn::add(acc.gx[k], rn::sub((double)acc.gxs[k], (double)acc.gxc[k]));
    gy = rn::add(acc.gy[k], rn::sub((double)acc.gys[k], (double)acc.gyc[k]));
}

} // namespace lt
