/*
 * lt_chi2.cu -- strong-lensing chi2 by barycentric delensing (lt_delense, lt_chi2,
 * lt_chi2_batch).
 *
 * The reference's chi2 (mychi_bruteforce_SOA_CPU_grid_gradient_barycentersource,
 * src/chi_CPU_barycenter.cpp:58-287) per model:
 *   1. the deflection grid over the frame, n x n, dx = (xmax - xmin)/(n - 1);
 *   2. each system's source: the barycentre of its observed images mapped to the source
 *      plane with the deflection evaluated at each image (:180-214);
 *   3. delensing (delense_barycenter, src/delense_CPU.cpp:6-140): every grid cell is split
 *      into an upper and a lower triangle; a cell whose upper (else lower) triangle,
 *      mapped to the source plane with the grid's deflection, contains the source adds
 *      the image-plane triangle's barycentre as a predicted image;
 *   4. chi_computation (src/chi_computation.cpp:11-195): predicted images are linked to
 *      observed ones and chi2 = sum |observed - predicted|^2, plus 1000 x (images of the
 *      system) per observed image left unlinked.
 * Here: step 1 is the FP64 grid kernel (deflection sums); step 2 one block per system;
 * step 3 one thread per cell testing every system, with the inclusion determinant, the
 * source-plane mapping and the barycentre in explicitly rounded FP64 in the reference's
 * operation order (so a cell tests inside exactly when the reference's test does for the
 * same deflections); the hits are appended per system with atomics and sorted back into
 * the reference's serial (row, column) order; step 4 one thread per system with the
 * reference's linking rules, and the chi2 summed in the reference's order.  All FP64.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "lt_chi2.h"
#include "lt_eval.cuh"
#include "lt_internal.h"

namespace lt {

constexpr int kMaxImg = LT_MAX_IMAGES;  /* predicted images kept per source */
constexpr int kHitCap = 64;             /* delensing hits recorded per source */

/* ---- step 2: sources ------------------------------------------------------------- */

template <int TYPE>
__device__ __forceinline__ void grad_run(const lt_rec64 *recs, int start, int count, double x, double y, double &gx,
                                         double &gy)
{
    for (int h = start; h < start + count; h++) grad_pair<TYPE>(recs[h], x, y, gx, gy);
}

/* One block per system, one thread per image: the deflection at the image over every
 * halo (chunk order, as the grid kernel), then thread 0 forms the barycentre. */
__global__ void chi2_sources_kernel(Chi2Dev c, const lt_rec64 *recs, const lt_chunk *chunks, int nchunks)
{
    __shared__ double sx[kMaxImg * 2], sy[kMaxImg * 2];
    const int s = blockIdx.x;
    if (s >= c.nsys) return;
    const int n = c.nimg[s], i0 = c.first[s];
    const double d = c.dr[s];
    for (int i = threadIdx.x; i < n && i < 2 * kMaxImg; i += blockDim.x) {
        const double x = c.ix[i0 + i], y = c.iy[i0 + i];
        double gx = 0., gy = 0.;
        for (int k = 0; k < nchunks; k++) {
            const lt_chunk ch = chunks[k];
            switch (ch.type) {
            case 81: grad_run<81>(recs, ch.start, ch.count, x, y, gx, gy); break;
            case 8: grad_run<8>(recs, ch.start, ch.count, x, y, gx, gy); break;
            case 5: grad_run<5>(recs, ch.start, ch.count, x, y, gx, gy); break;
            default: break;
            }
        }
        sx[i] = rn::sub(x, rn::mul(d, gx));
        sy[i] = rn::sub(y, rn::mul(d, gy));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bx = 0., by = 0.;
        const int m = n < 2 * kMaxImg ? n : 2 * kMaxImg;
        for (int i = 0; i < m; i++) {
            bx = rn::add(bx, sx[i]);
            by = rn::add(by, sy[i]);
        }
        c.bx[s] = rn::div(bx, (double)n);
        c.by[s] = rn::div(by, (double)n);
        c.hits[s] = 0;
    }
}

/* ---- step 3: delensing ------------------------------------------------------------ */

struct P2 {
    double x, y;
};

/* mychi_determinant, src/delense_CPU_utils.hpp:127-136, left to right */
__device__ __forceinline__ double det3(P2 A, P2 B, P2 C)
{
    using namespace rn;
    double t = sub(mul(B.x, C.y), mul(B.y, C.x));
    t = add(t, mul(A.x, B.y));
    t = sub(t, mul(A.y, B.x));
    t = add(t, mul(A.y, C.x));
    return sub(t, mul(A.x, C.y));
}

/* mychi_inside, src/delense_CPU_utils.hpp:146-160 */
__device__ __forceinline__ bool inside(P2 P, P2 a, P2 b, P2 c)
{
    const double d = det3(a, b, c);
    if (rn::mul(det3(a, b, P), d) < 0.) return false;
    if (rn::mul(det3(b, c, P), d) < 0.) return false;
    if (rn::mul(det3(c, a, P), d) < 0.) return false;
    return true;
}

__device__ __forceinline__ P2 to_source(P2 I, double d, double ax, double ay)
{
    return {rn::sub(I.x, rn::mul(d, ax)), rn::sub(I.y, rn::mul(d, ay))};
}

/* One thread per cell (grid-stride), every system per cell. */
__global__ void chi2_delense_kernel(Chi2Dev c)
{
    extern __shared__ double ssrc[]; /* bx, by, dr per system */
    for (int s = threadIdx.x; s < c.nsys; s += blockDim.x) {
        ssrc[3 * s] = c.bx[s];
        ssrc[3 * s + 1] = c.by[s];
        ssrc[3 * s + 2] = c.dr[s];
    }
    __syncthreads();
    const int m = c.n - 1;
    const long cells = (long)m * m;
    for (long cell = blockIdx.x * (long)blockDim.x + threadIdx.x; cell < cells; cell += (long)gridDim.x * blockDim.x) {
        const int y = (int)(cell / m), x = (int)(cell % m);
        const long g = (long)y * c.n + x;
        const double xp = rn::add(c.xmin, rn::mul((double)x, c.dx));
        const double yp = rn::add(c.ymin, rn::mul((double)y, c.dy));
        const double xq = rn::add(xp, c.dx), yq = rn::add(yp, c.dy);
        const double a00x = c.ax[g], a00y = c.ay[g];
        const double a01x = c.ax[g + c.n], a01y = c.ay[g + c.n];
        const double a10x = c.ax[g + 1], a10y = c.ay[g + 1];
        const double a11x = c.ax[g + c.n + 1], a11y = c.ay[g + c.n + 1];
        for (int s = 0; s < c.nsys; s++) {
            const P2 P = {ssrc[3 * s], ssrc[3 * s + 1]};
            const double d = ssrc[3 * s + 2];
            /* upper: a = (x, y), b = (x, y + dy), c = (x + dx, y) */
            bool lower = false;
            bool hit = inside(P, to_source({xp, yp}, d, a00x, a00y), to_source({xp, yq}, d, a01x, a01y),
                              to_source({xq, yp}, d, a10x, a10y));
            if (!hit) {
                /* lower: a = (x + dx, y + dy), b = (x + dx, y), c = (x, y + dy) */
                hit = inside(P, to_source({xq, yq}, d, a11x, a11y), to_source({xq, yp}, d, a10x, a10y),
                             to_source({xp, yq}, d, a01x, a01y));
                lower = true;
            }
            if (hit) {
                const int slot = atomicAdd(&c.hits[s], 1);
                if (slot < kHitCap) c.keys[s * kHitCap + slot] = (int32_t)(2 * cell + (lower ? 1 : 0));
            }
        }
    }
}

/* ---- step 4: linking and chi2 ------------------------------------------------------ */

__device__ __forceinline__ double dist2d(double ax, double ay, double bx, double by)
{
    const double x = rn::sub(ax, bx), y = rn::sub(ay, by);
    return rn::sqr(rn::add(rn::mul(x, x), rn::mul(y, y)));
}

/* One thread per system: hits back in serial order, predicted positions, the reference's
 * linking, per-image chi2 terms; then thread 0 sums them in the reference's order. */
__global__ void chi2_link_kernel(Chi2Dev c)
{
    for (int s = threadIdx.x; s < c.nsys; s += blockDim.x) {
        int nh = c.hits[s];
        const bool overflow = nh > kMaxImg;
        if (nh > kHitCap) nh = kHitCap;
        int32_t *key = c.keys + s * kHitCap;
        for (int i = 1; i < nh; i++) { /* insertion sort: (row, column) order */
            const int32_t k = key[i];
            int j = i - 1;
            while (j >= 0 && key[j] > k) {
                key[j + 1] = key[j];
                j--;
            }
            key[j + 1] = k;
        }
        const int nf = nh < kMaxImg ? nh : kMaxImg;
        const int m = c.n - 1;
        double px[kMaxImg], py[kMaxImg];
        for (int i = 0; i < nf; i++) {
            const long cell = key[i] >> 1;
            const bool lower = key[i] & 1;
            const int y = (int)(cell / m), x = (int)(cell % m);
            const double xp = rn::add(c.xmin, rn::mul((double)x, c.dx));
            const double yp = rn::add(c.ymin, rn::mul((double)y, c.dy));
            const double xq = rn::add(xp, c.dx), yq = rn::add(yp, c.dy);
            /* mychi_barycenter of the image-plane triangle (a + b + c)/3 */
            if (!lower) {
                px[i] = rn::div(rn::add(rn::add(xp, xp), xq), 3.);
                py[i] = rn::div(rn::add(rn::add(yp, yq), yp), 3.);
            } else {
                px[i] = rn::div(rn::add(rn::add(xq, xq), xp), 3.);
                py[i] = rn::div(rn::add(rn::add(yq, yp), yq), 3.);
            }
            c.fx[s * kMaxImg + i] = px[i];
            c.fy[s * kMaxImg + i] = py[i];
        }
        c.nfound[s] = nf;
        if (overflow) c.found[1] = 1;
        /* chi_computation for system s */
        const int n = c.nimg[s], i0 = c.first[s];
        int linked[kMaxImg * 2];
        double tx[kMaxImg * 2], ty[kMaxImg * 2], dist[kMaxImg * 2];
        for (int i = 0; i < n; i++) linked[i] = 0;
        for (int ii = 0; ii < nf; ii++) {
            int im = 0;
            dist[0] = dist2d(px[ii], py[ii], c.ix[i0], c.iy[i0]);
            for (int i = 1; i < n; i++) {
                dist[i] = dist2d(px[ii], py[ii], c.ix[i0 + i], c.iy[i0 + i]);
                if (dist[i] < dist[im]) im = i;
            }
            if (linked[im] == 0) {
                tx[im] = px[ii];
                ty[im] = py[ii];
                linked[im]++;
            } else {
                double qx, qy;
                if (dist[im] < dist2d(c.ix[i0 + im], c.iy[i0 + im], tx[im], ty[im])) {
                    qx = tx[im];
                    qy = ty[im];
                    tx[im] = px[ii];
                    ty[im] = py[ii];
                } else {
                    qx = px[ii];
                    qy = py[ii];
                }
                int second = 0;
                for (int i = 1; i < n && (i != im); i++)
                    if (dist[i] > dist[second]) second = i;
                for (int i = 0; i < n && linked[i] == 0; i++)
                    if (dist[i] < dist[second]) {
                        second = i;
                        im = i;
                        tx[im] = qx;
                        ty[im] = qy;
                    }
                linked[im]++;
            }
        }
        for (int i = 0; i < n; i++) {
            if (linked[i] > 0) {
                const double p1 = rn::sub(c.ix[i0 + i], tx[i]), p2 = rn::sub(c.iy[i0 + i], ty[i]);
                c.chi_terms[i0 + i] = rn::add(rn::mul(p1, p1), rn::mul(p2, p2));
            } else {
                c.chi_terms[i0 + i] = rn::mul(1000., (double)n);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double chi = 0.;
        int found = 0;
        for (int i = 0; i < c.nimages; i++) chi = rn::add(chi, c.chi_terms[i]);
        for (int s = 0; s < c.nsys; s++) found += c.nfound[s];
        c.chi2[0] = chi;
        c.found[0] = found;
    }
}

} // namespace lt

using namespace lt;

namespace {

bool frame_ok(const lt_frame *f, int n)
{
    return f && n >= 2 && std::isfinite(f->xmin) && std::isfinite(f->xmax) && std::isfinite(f->ymin) &&
           std::isfinite(f->ymax) && f->xmax > f->xmin && f->ymax > f->ymin && (long)n * n <= (1L << 31);
}

/* Device layout of one chi2 evaluation: systems, sources, hits, results. */
struct Chi2Buf {
    void *mem = nullptr;
    size_t bytes = 0;
    Chi2Dev dev;
};

} // namespace

namespace lt {

size_t chi2_layout(int nsys, int nimages, const lt_frame *f, int n, char *m, Chi2Dev &c)
{
    memset(&c, 0, sizeof(c));
    const size_t ns = (size_t)nsys, ni = (size_t)(nimages > 0 ? nimages : 1);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_nimg = take(4 * ns), o_first = take(4 * ns), o_ix = take(8 * ni), o_iy = take(8 * ni),
                 o_dr = take(8 * ns), o_bx = take(8 * ns), o_by = take(8 * ns), o_hits = take(4 * ns),
                 o_keys = take(4 * ns * kHitCap), o_terms = take(8 * ni), o_chi = take(8), o_found = take(8),
                 o_nf = take(4 * ns), o_fx = take(8 * ns * kMaxImg), o_fy = take(8 * ns * kMaxImg),
                 o_ax = take(8 * (size_t)n * n), o_ay = take(8 * (size_t)n * n);
    if (!m) return off;
    c.nsys = nsys;
    c.nimages = nimages;
    c.nimg = (const int32_t *)(m + o_nimg);
    c.first = (const int32_t *)(m + o_first);
    c.ix = (const double *)(m + o_ix);
    c.iy = (const double *)(m + o_iy);
    c.dr = (const double *)(m + o_dr);
    c.bx = (double *)(m + o_bx);
    c.by = (double *)(m + o_by);
    c.hits = (int32_t *)(m + o_hits);
    c.keys = (int32_t *)(m + o_keys);
    c.chi_terms = (double *)(m + o_terms);
    c.chi2 = (double *)(m + o_chi);
    c.found = (int32_t *)(m + o_found);
    c.nfound = (int32_t *)(m + o_nf);
    c.fx = (double *)(m + o_fx);
    c.fy = (double *)(m + o_fy);
    c.ax = (const double *)(m + o_ax);
    c.ay = (const double *)(m + o_ay);
    c.n = n;
    c.xmin = f->xmin;
    c.ymin = f->ymin;
    c.dx = (f->xmax - f->xmin) / (n - 1); /* src/chi_CPU_barycenter.cpp:104-105 */
    c.dy = (f->ymax - f->ymin) / (n - 1);
    return off;
}

lt_status chi2_buffers(lt_context *ctx, int nsys, int nimages, const lt_frame *f, int n, Chi2Buf &b)
{
    b.bytes = chi2_layout(nsys, nimages, f, n, nullptr, b.dev);
    lt_status st = dev_alloc(ctx, &b.mem, b.bytes);
    if (st != LT_OK) return st;
    chi2_layout(nsys, nimages, f, n, (char *)b.mem, b.dev);
    return LT_OK;
}

cudaError_t chi2_upload_systems_async(const Chi2Dev &c, const int32_t *nimg, const int32_t *first, const double *x,
                                      const double *y, const double *dr, cudaStream_t s)
{
    cudaError_t e = cudaMemcpyAsync((void *)c.nimg, nimg, 4 * (size_t)c.nsys, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void *)c.first, first, 4 * (size_t)c.nsys, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && c.nimages)
        e = cudaMemcpyAsync((void *)c.ix, x, 8 * (size_t)c.nimages, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && c.nimages)
        e = cudaMemcpyAsync((void *)c.iy, y, 8 * (size_t)c.nimages, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void *)c.dr, dr, 8 * (size_t)c.nsys, cudaMemcpyHostToDevice, s);
    return e;
}

lt_status upload_systems(lt_context *ctx, const lt_image_systems *sys, Chi2Buf &b, cudaStream_t s)
{
    std::vector<int32_t> first((size_t)sys->nsystems);
    int total = 0;
    for (int i = 0; i < sys->nsystems; i++) {
        first[i] = total;
        total += sys->nimages[i];
    }
    cudaError_t e = chi2_upload_systems_async(b.dev, sys->nimages, first.data(), sys->x, sys->y, sys->dlsds, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s); /* `first` is a local vector */
    if (e != cudaSuccess) return cuda_fail(ctx, e, "image systems upload");
    return LT_OK;
}

lt_status check_systems(lt_context *ctx, const lt_image_systems *sys)
{
    if (!sys || sys->nsystems < 1 || !sys->nimages || !sys->x || !sys->y || !sys->dlsds) {
        set_error(ctx, "invalid image systems");
        return LT_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < sys->nsystems; i++)
        if (sys->nimages[i] < 1 || sys->nimages[i] > 2 * kMaxImg) {
            set_error(ctx, "system %d: %d images (1..%d supported)", i, sys->nimages[i], 2 * kMaxImg);
            return LT_ERR_INVALID_ARGUMENT;
        }
    return LT_OK;
}

/* Steps 2-4 on a layout whose deflection planes hold the grid (stream-ordered). */
static int chi2_steps(lt_context *ctx, const lt_catalog *cat, const Chi2Dev &c, bool sources_given, cudaStream_t s)
{
    if (!sources_given) {
        chi2_sources_kernel<<<c.nsys, 64, 0, s>>>(c, cat->recs, cat->chunks, cat->nhalos ? cat->nchunks : 0);
        count_launch(1);
    } else {
        cudaMemsetAsync(c.hits, 0, 4 * (size_t)c.nsys, s);
    }
    const size_t smem = 24 * (size_t)c.nsys;
    chi2_delense_kernel<<<ctx->num_sms * 8, 256, smem, s>>>(c);
    count_launch(1);
    cudaMemsetAsync(c.found, 0, 8, s);
    chi2_link_kernel<<<1, 256, 0, s>>>(c);
    count_launch(1);
    return (int)cudaGetLastError();
}

/* Steps 1-4 for one catalogue on the prepared buffers (stream-ordered).  The deflection
 * grid of step 1 is FP64, or FP32C with precision LT_FP32C; the sources, the delensing and
 * the chi2 are FP64 either way. */
int chi2_launch(lt_context *ctx, const lt_catalog *cat, Chi2Buf &b, bool sources_given, bool link, cudaStream_t s,
                int precision = LT_FP64)
{
    Chi2Dev &c = b.dev;
    GridArgs a;
    memset(&a, 0, sizeof(a));
    a.recs = cat->recs;
    a.chunks = cat->chunks;
    a.nchunks = cat->nchunks;
    a.xmin = c.xmin;
    a.ymin = c.ymin;
    a.dx = c.dx;
    a.dy = c.dy;
    a.nx = c.n;
    a.ny = c.n;
    a.nout = 2;
    a.kinds[0] = KIND_GRAD_X;
    a.kinds[1] = KIND_GRAD_Y;
    a.out[0] = (double *)c.ax;
    a.out[1] = (double *)c.ay;
    a.vec_ok = (c.n % 2 == 0);
    a.scale = 1.0;
    a.D = 1.0;
    a.mult = 1.0;
    a.status = ctx->status;
    int err;
    if (cat->nhalos == 0) {
        err = (int)cudaMemsetAsync((void *)c.ax, 0, 8 * (size_t)c.n * c.n, s);
        if (err == cudaSuccess) err = (int)cudaMemsetAsync((void *)c.ay, 0, 8 * (size_t)c.n * c.n, s);
    } else if (precision == LT_FP32C) {
        err = launch_fp32c(ctx, cat, OP_GRAD, a, s);
    } else if (precision == LT_FP64_FAST) {
        /* the dPIE deflection as log(1 + eps), as the LT_FP64_FAST grid calls take it */
        err = launch_grid64_tiled(OP_GRAD | OP_GFX, a, ctx->num_sms, s, ctx->shape[LT_FP64_FAST][OP_GRAD]);
    } else {
        err = launch_grid64_tiled(OP_GRAD, a, ctx->num_sms, s, ctx->shape[LT_FP64][OP_GRAD]);
    }
    if (err != cudaSuccess) return err;
    (void)link;
    return chi2_steps(ctx, cat, c, sources_given, s);
}

int chi2_tail(lt_context *ctx, const lt_catalog *cat, const Chi2Dev &c, cudaStream_t s)
{
    return chi2_steps(ctx, cat, c, false, s);
}

} // namespace lt

extern "C" {

lt_status lt_delense(lt_context *ctx, const lt_catalog *cat, const lt_frame *frame, int32_t n, int32_t nsources,
                     const double *bx, const double *by, const double *dlsds, int32_t *nfound, double *fx,
                     double *fy)
{
    if (!ctx || !cat || !frame_ok(frame, n) || nsources < 1 || !bx || !by || !dlsds || !nfound || !fx || !fy) {
        if (ctx) set_error(ctx, "invalid delensing arguments");
        return LT_ERR_INVALID_ARGUMENT;
    }
    if ((size_t)24 * nsources > 48 * 1024) {
        set_error(ctx, "at most %d sources per call", 48 * 1024 / 24);
        return LT_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Chi2Buf b;
    lt_status st = chi2_buffers(ctx, nsources, nsources, frame, n, b);
    if (st != LT_OK) return st;
    cudaStream_t s = nullptr;
    Chi2Dev &c = b.dev;
    /* the sources are given: no images, one "image" per system only to size the link step */
    std::vector<int32_t> ones((size_t)nsources, 1), first((size_t)nsources);
    for (int i = 0; i < nsources; i++) first[i] = i;
    cudaMemcpy((void *)c.bx, bx, 8 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.by, by, 8 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.dr, dlsds, 8 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.nimg, ones.data(), 4 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.first, first.data(), 4 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.ix, bx, 8 * (size_t)nsources, cudaMemcpyHostToDevice);
    cudaMemcpy((void *)c.iy, by, 8 * (size_t)nsources, cudaMemcpyHostToDevice);
    c.nimages = nsources;
    int err = chi2_launch(ctx, cat, b, true, false, s);
    if (err == cudaSuccess) err = (int)cudaMemcpy(nfound, c.nfound, 4 * (size_t)nsources, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = (int)cudaMemcpy(fx, c.fx, 8 * (size_t)nsources * kMaxImg, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = (int)cudaMemcpy(fy, c.fy, 8 * (size_t)nsources * kMaxImg, cudaMemcpyDeviceToHost);
    int32_t flags[2] = {0, 0};
    if (err == cudaSuccess) err = (int)cudaMemcpy(flags, c.found, 8, cudaMemcpyDeviceToHost);
    dev_free(ctx, b.mem, b.bytes);
    if (err != cudaSuccess) return cuda_fail(ctx, (cudaError_t)err, "delensing");
    if (flags[1]) {
        set_error(ctx, "a source has more than %d predicted images (the first %d are returned)", kMaxImg, kMaxImg);
        return LT_ERR_QUEUE_FULL;
    }
    return LT_OK;
}

lt_status lt_chi2_batch_precision(lt_context *ctx, const lt_catalog *const *cats, int32_t nmodels,
                                  const lt_frame *frame, int32_t n, const lt_image_systems *sys, int32_t precision,
                                  double *chi2, int32_t *images_found)
{
    if (!ctx || !cats || nmodels < 1 || !frame_ok(frame, n) || !chi2) {
        if (ctx) set_error(ctx, "invalid chi2 arguments");
        return LT_ERR_INVALID_ARGUMENT;
    }
    if (precision != LT_FP64 && precision != LT_FP64_FAST && precision != LT_FP32C) {
        set_error(ctx, "chi2: unknown precision %d", precision);
        return LT_ERR_INVALID_ARGUMENT;
    }
    for (int m = 0; m < nmodels; m++)
        if (!cats[m]) {
            set_error(ctx, "model %d: NULL catalogue", m);
            return LT_ERR_INVALID_ARGUMENT;
        }
    lt_status st = check_systems(ctx, sys);
    if (st != LT_OK) return st;
    if ((size_t)24 * sys->nsystems > 48 * 1024) {
        set_error(ctx, "at most %d systems", 48 * 1024 / 24);
        return LT_ERR_INVALID_ARGUMENT;
    }
    int total = 0;
    for (int i = 0; i < sys->nsystems; i++) total += sys->nimages[i];
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Chi2Buf b;
    st = chi2_buffers(ctx, sys->nsystems, total, frame, n, b);
    if (st != LT_OK) return st;
    cudaStream_t s = nullptr;
    st = upload_systems(ctx, sys, b, s);
    /* per model: 4 launches; the chi2 and the found count go to a device array read once */
    double *d_res = nullptr;
    if (st == LT_OK) st = dev_alloc(ctx, (void **)&d_res, 16 * (size_t)nmodels);
    int err = cudaSuccess;
    for (int m = 0; st == LT_OK && m < nmodels && err == cudaSuccess; m++) {
        err = chi2_launch(ctx, cats[m], b, false, true, s, precision);
        if (err == cudaSuccess) err = (int)cudaMemcpyAsync(d_res + 2 * m, b.dev.chi2, 8, cudaMemcpyDeviceToDevice, s);
        if (err == cudaSuccess)
            err = (int)cudaMemcpyAsync(d_res + 2 * m + 1, b.dev.found, 8, cudaMemcpyDeviceToDevice, s);
    }
    std::vector<double> res(2 * (size_t)nmodels);
    if (st == LT_OK && err == cudaSuccess)
        err = (int)cudaMemcpy(res.data(), d_res, 16 * (size_t)nmodels, cudaMemcpyDeviceToHost);
    if (d_res) dev_free(ctx, d_res, 16 * (size_t)nmodels);
    dev_free(ctx, b.mem, b.bytes);
    if (st != LT_OK) return st;
    if (err != cudaSuccess) return cuda_fail(ctx, (cudaError_t)err, "chi2");
    bool overflow = false;
    for (int m = 0; m < nmodels; m++) {
        chi2[m] = res[2 * m];
        int32_t f[2];
        memcpy(f, &res[2 * m + 1], 8);
        if (images_found) images_found[m] = f[0];
        overflow |= f[1] != 0;
    }
    int32_t kst = 0;
    cudaMemcpy(&kst, ctx->status, 4, cudaMemcpyDeviceToHost);
    if (kst) return (lt_status)kst;
    if (overflow) {
        set_error(ctx, "a source had more than %d predicted images (the first %d were used)", kMaxImg, kMaxImg);
        return LT_ERR_QUEUE_FULL;
    }
    return LT_OK;
}

lt_status lt_chi2_batch(lt_context *ctx, const lt_catalog *const *cats, int32_t nmodels, const lt_frame *frame,
                        int32_t n, const lt_image_systems *sys, double *chi2, int32_t *images_found)
{
    return lt_chi2_batch_precision(ctx, cats, nmodels, frame, n, sys, LT_FP64, chi2, images_found);
}

lt_status lt_chi2(lt_context *ctx, const lt_catalog *cat, const lt_frame *frame, int32_t n,
                  const lt_image_systems *sys, double *chi2, int32_t *images_found)
{
    return lt_chi2_batch(ctx, &cat, 1, frame, n, sys, chi2, images_found);
}

} /* extern "C" */
