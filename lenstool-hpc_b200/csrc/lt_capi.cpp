/*
 * lt_capi.cpp -- the extern "C" entry points of include/lt_b200.h: contexts, catalogue
 * validation/packing/upload, and the grid calls (argument checks, host staging, launch).
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"
#include "lt_grid.cuh"
#include "lt_halo.h"
#include "lt_internal.h"
#include "lt_pack.h"

using namespace lt;

static std::atomic<uint64_t> g_launches{0};
static std::mutex g_ctx_mu;
static int g_contexts[64] = {}; /* live contexts per device (devices 0..63) */

namespace lt {
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void pass_mark(lt_context *ctx, cudaStream_t stream, int which)
{
    (void)which;
    if (!ctx->timing) return;
    cudaEvent_t e;
    if (ctx->ev_pool.empty()) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
    } else {
        e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
    }
    cudaEventRecord(e, stream);
    ctx->ev_marks.push_back(e);
}
} // namespace lt

/* ------------------------------------------------------------------ helpers ---- */

void lt::set_error(lt_context *ctx, const char *fmt, ...)
{
    if (!ctx) return;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
}

lt_status lt::cuda_fail(lt_context *ctx, cudaError_t e, const char *what)
{
    set_error(ctx, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return LT_ERR_OUT_OF_MEMORY;
    return LT_ERR_CUDA;
}

lt_status lt::dev_alloc(lt_context *ctx, void **p, size_t bytes)
{
    if (ctx->used + bytes > ctx->budget) {
        set_error(ctx, "HBM budget exceeded: %zu in use + %zu requested > %zu", ctx->used, bytes, ctx->budget);
        return LT_ERR_BUDGET;
    }
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    ctx->used += bytes;
    return LT_OK;
}

void lt::dev_free(lt_context *ctx, void *p, size_t bytes)
{
    if (!p) return;
    cudaFree(p);
    ctx->used -= bytes;
}

/* Device staging planes for host-pointer outputs, grown on demand. */
lt_status lt::scratch_planes(lt_context *ctx, int n, size_t plane_bytes, double **planes)
{
    size_t need = (size_t)n * plane_bytes;
    if (need > ctx->scratch_bytes) {
        dev_free(ctx, ctx->scratch, ctx->scratch_bytes);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
        lt_status st = dev_alloc(ctx, &ctx->scratch, need);
        if (st != LT_OK) return st;
        ctx->scratch_bytes = need;
    }
    for (int i = 0; i < n; i++) planes[i] = (double *)((char *)ctx->scratch + (size_t)i * plane_bytes);
    return LT_OK;
}

/* Pixel list (and its counter, in the first 16 bytes) of the recomputation pass. */
lt_status lt::list_buffer(lt_context *ctx, long npix, int32_t **list, int32_t **count)
{
    size_t need = 16 + sizeof(int32_t) * (size_t)npix;
    if (need > ctx->list_bytes) {
        dev_free(ctx, ctx->list, ctx->list_bytes);
        ctx->list = nullptr;
        ctx->list_bytes = 0;
        lt_status st = dev_alloc(ctx, &ctx->list, need);
        if (st != LT_OK) return st;
        ctx->list_bytes = need;
    }
    *count = (int32_t *)ctx->list;
    *list = (int32_t *)((char *)ctx->list + 16);
    return LT_OK;
}

bool lt::is_device_pointer(const void *p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

/* ---------------------------------------------------------------- packing ---- */

/* Per-halo invariants (lt_halo.h, packed by lt_pack.h). */
static void pack_one(const lt_halo_soa *s, int i, lt_rec64 &r)
{
    pk::pack64(s->type[i], s->position_x[i], s->position_y[i], s->anglecos[i], s->anglesin[i], s->b0[i],
               s->ellipticity_potential[i], s->rcore[i], s->rcut[i], s->dlsds ? s->dlsds[i] : 1.0, r);
}

/* Domain checks: the reference would divide by zero or take sqrt of a negative value
 * (and silently produce NaN maps); here the upload fails with a status instead. */
static lt_status validate(lt_context *ctx, const lt_halo_soa *s)
{
    for (int i = 0; i < s->nhalos; i++) {
        const int t = s->type[i];
        if (t != 5 && t != 8 && t != 81) {
            set_error(ctx, "halo %d: unknown profile type %d (supported: 5, 8, 81)", i, t);
            return LT_ERR_UNKNOWN_PROFILE;
        }
        const double v[] = {s->position_x[i], s->position_y[i], s->b0[i], s->anglecos[i], s->anglesin[i],
                            s->ellipticity_potential[i], s->rcore[i], s->rcut[i], s->dlsds ? s->dlsds[i] : 1.0};
        for (double x : v)
            if (!std::isfinite(x)) {
                set_error(ctx, "halo %d: non-finite parameter", i);
                return LT_ERR_NONFINITE;
            }
        const double e = s->ellipticity_potential[i];
        if (t == 5 ? !(e >= 0. && e < 1.) : !(e > 0. && e < 1.)) {
            set_error(ctx, "halo %d: ellipticity_potential %g outside the profile's domain", i, e);
            return LT_ERR_NONFINITE;
        }
        if (t != 5 && !(s->rcore[i] > 0.)) {
            set_error(ctx, "halo %d: rcore must be > 0", i);
            return LT_ERR_NONFINITE;
        }
        if (t == 81 && !(s->rcut[i] > s->rcore[i])) {
            set_error(ctx, "halo %d: rcut must exceed rcore for the cut dPIE", i);
            return LT_ERR_NONFINITE;
        }
    }
    return LT_OK;
}

/* Runs of equal type (and, with `dlsds`, equal D_LS/D_OS: the Kmap's runs,
 * src/gradient2_GPU.cu:484-512) split into chunks of at most max_chunk halos; the last
 * chunk of each run carries CHUNK_RUN_END. */
std::vector<lt_chunk> lt::make_chunks(const int32_t *type, int n, int max_chunk, const double *dlsds)
{
    std::vector<lt_chunk> ch;
    int s = 0;
    while (s < n) {
        int e = s + 1;
        while (e < n && type[e] == type[s] && (!dlsds || dlsds[e] == dlsds[s])) e++;
        for (int c = s; c < e; c += max_chunk) {
            lt_chunk k;
            k.start = c;
            k.count = (e - c) < max_chunk ? (e - c) : max_chunk;
            k.type = type[s];
            k.pad = (c + k.count == e) ? CHUNK_RUN_END : 0;
            ch.push_back(k);
        }
        s = e;
    }
    return ch;
}

/* (called with or without ctx->mu held: lt_catalog_upload releases a half-built
 * catalogue under the lock) */
void lt::free_catalog(lt_context *ctx, lt_catalog *cat)
{
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    dev_free(ctx, cat->recs, sizeof(lt_rec64) * (size_t)cat->nhalos);
    dev_free(ctx, cat->chunks, sizeof(lt_chunk) * (size_t)(cat->nchunks + cat->nchunks_k));
    dev_free(ctx, cat->aux, cat->aux_bytes);
    dev_free(ctx, cat->stage, cat->stage_bytes);
    delete cat;
}

/* ------------------------------------------------------------------- API ---- */

extern "C" {

int32_t lt_abi_version(void) { return LT_B200_ABI_VERSION; }

uint64_t lt_kernel_launch_count(void) { return g_launches.load(); }

const char *lt_status_string(lt_status s)
{
    switch (s) {
    case LT_OK: return "ok";
    case LT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LT_ERR_UNKNOWN_PROFILE: return "unknown profile type";
    case LT_ERR_NONFINITE: return "non-finite or out-of-domain halo parameter";
    case LT_ERR_CUDA: return "CUDA error";
    case LT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case LT_ERR_BUDGET: return "HBM budget exceeded";
    case LT_ERR_QUEUE_FULL: return "queue full";
    case LT_ERR_TIMEOUT: return "device-side wait timed out";
    case LT_ERR_NO_DEVICE: return "no usable CUDA device";
    case LT_ERR_NOT_READY: return "not ready";
    }
    return "unknown status";
}

const char *lt_last_error(const lt_context *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

lt_status lt_create(int device, size_t budget, lt_context **out)
{
    if (!out) return LT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return LT_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return LT_ERR_NO_DEVICE;
    if (prop.major < 10) return LT_ERR_NO_DEVICE; /* built for sm_100a only */
    lt_context *ctx = new (std::nothrow) lt_context();
    if (!ctx) return LT_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    /* default kernel shapes (pixels per thread, CTAs per SM, threads, records per stage),
     * from sweeps on B200 of the 1000-halo workload; lt_autotune refines them for a given
     * catalogue */
    for (int p = 0; p < 3; p++)
        for (int o = 0; o < 8; o++) ctx->shape[p][o] = LT_SHAPE(2, 1);
    ctx->shape[LT_FP64][OP_HESS] = LT_SHAPE(2, 2);
    ctx->shape[LT_FP64][OP_POT] = LT_SHAPE(1, 2);
    ctx->shape[LT_FP64][OP_HESS | OP_POT] = LT_SHAPE(1, 2);
    ctx->shape[LT_FP64][OP_GRAD] = LT_SHAPE(2, 2);
    ctx->shape[LT_FP64_FAST][OP_HESS] = LT_SHAPE(2, 2);
    ctx->shape[LT_FP64_FAST][OP_POT] = LT_SHAPE(1, 2);
    ctx->shape[LT_FP64_FAST][OP_HESS | OP_POT] = LT_SHAPE(1, 2);
    ctx->shape[LT_FP64_FAST][OP_GRAD] = LT_SHAPE(2, 2);
    ctx->shape[LT_FP32C][OP_HESS] = LT_SHAPE4(2, 2, 256, 128);
    ctx->shape[LT_FP32C][OP_POT] = LT_SHAPE4(2, 2, 256, 128);
    ctx->shape[LT_FP32C][OP_HESS | OP_POT] = LT_SHAPE4(2, 2, 256, 128);
    ctx->shape[LT_FP32C][OP_GRAD] = LT_SHAPE4(2, 2, 256, 128);
    cudaSetDevice(device);
    if (configure_kernels32() != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return LT_ERR_CUDA;
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    ctx->budget = budget ? budget : (size_t)(0.9 * (double)free_b);
    ctx->used = 0;
    lt_status st = dev_alloc(ctx, (void **)&ctx->status, 64);
    if (st != LT_OK) {
        delete ctx;
        return st;
    }
    cudaMemset(ctx->status, 0, 64);
    if (device < 64) {
        std::lock_guard<std::mutex> lock(g_ctx_mu);
        g_contexts[device]++;
    }
    *out = ctx;
    return LT_OK;
}

lt_status lt_destroy(lt_context *ctx)
{
    if (!ctx) return LT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    dev_free(ctx, ctx->scratch, ctx->scratch_bytes);
    dev_free(ctx, ctx->list, ctx->list_bytes);
    dev_free(ctx, ctx->status, 64);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    destroy_extensions(ctx);
    for (cudaEvent_t e : ctx->ev_marks) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->device < 64) {
        std::lock_guard<std::mutex> lock(g_ctx_mu);
        if (--g_contexts[ctx->device] == 0) noalloc_forget(ctx->device);
    }
    delete ctx;
    return LT_OK;
}

lt_status lt_set_pass_timing(lt_context *ctx, int32_t on)
{
    if (!ctx) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ctx->timing = on != 0;
    if (!ctx->timing) {
        for (cudaEvent_t e : ctx->ev_marks) ctx->ev_pool.push_back(e);
        ctx->ev_marks.clear();
    }
    return LT_OK;
}

lt_status lt_pass_times(lt_context *ctx, double *pass1_ms, double *pass2_ms, int32_t *calls)
{
    if (!ctx || !pass1_ms || !pass2_ms || !calls) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    *pass1_ms = *pass2_ms = 0.;
    *calls = 0;
    const size_t n = ctx->ev_marks.size() / 3 * 3;
    lt_status st = LT_OK;
    if (n) {
        cudaError_t e = cudaEventSynchronize(ctx->ev_marks[n - 1]);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "pass timing");
    }
    for (size_t i = 0; st == LT_OK && i < n; i += 3) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ctx->ev_marks[i], ctx->ev_marks[i + 1]);
        cudaEventElapsedTime(&b, ctx->ev_marks[i + 1], ctx->ev_marks[i + 2]);
        *pass1_ms += a;
        *pass2_ms += b;
        ++*calls;
    }
    for (cudaEvent_t e : ctx->ev_marks) ctx->ev_pool.push_back(e);
    ctx->ev_marks.clear();
    return st;
}

lt_status lt_recompute_count(lt_context *ctx, uint64_t *pixels)
{
    if (!ctx || !pixels) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    uint64_t c = 0;
    /* words 2..3 of the status block: the 64-bit count that the recomputation kernels add to */
    cudaError_t e = cudaMemcpy(&c, ctx->status + 2, sizeof(c), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(ctx->status + 2, 0, sizeof(c));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "recompute count");
    *pixels = c;
    return LT_OK;
}

lt_status lt_catalog_upload(lt_context *ctx, const lt_halo_soa *s, lt_catalog **out)
{
    if (!ctx || !s || !out || s->nhalos < 0) return LT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (s->nhalos > 0 && (!s->type || !s->position_x || !s->position_y || !s->b0 || !s->anglecos ||
                          !s->anglesin || !s->ellipticity_potential || !s->rcore || !s->rcut)) {
        set_error(ctx, "catalogue field pointer is NULL");
        return LT_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    lt_status st = validate(ctx, s);
    if (st != LT_OK) return st;
    lt_catalog *cat = new (std::nothrow) lt_catalog();
    if (!cat) return LT_ERR_OUT_OF_MEMORY;
    cat->nhalos = s->nhalos;
    cat->host_recs.resize(s->nhalos);
    cat->host_types.assign(s->type, s->type + s->nhalos);
    for (int i = 0; i < s->nhalos; i++) pack_one(s, i, cat->host_recs[i]);
    std::vector<lt_chunk> ch = make_chunks(s->type, s->nhalos, LT_CHUNK);
    std::vector<double> w(s->nhalos);
    for (int i = 0; i < s->nhalos; i++) w[i] = cat->host_recs[i].w;
    std::vector<lt_chunk> chk = make_chunks(s->type, s->nhalos, LT_CHUNK, w.data());
    cat->nchunks = (int32_t)ch.size();
    cat->nchunks_k = (int32_t)chk.size();
    size_t rb = sizeof(lt_rec64) * (size_t)s->nhalos, cb = sizeof(lt_chunk) * (ch.size() + chk.size());
    cat->bytes = rb + cb;
    st = dev_alloc(ctx, (void **)&cat->recs, rb);
    if (st == LT_OK) st = dev_alloc(ctx, (void **)&cat->chunks, cb);
    cat->chunks_k = cat->chunks + ch.size();
    if (st == LT_OK && rb) {
        cudaError_t e = cudaMemcpy(cat->recs, cat->host_recs.data(), rb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(cat->chunks, ch.data(), sizeof(lt_chunk) * ch.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(cat->chunks_k, chk.data(), sizeof(lt_chunk) * chk.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "catalogue upload");
    }
    if (st == LT_OK) st = prepare_catalog_extensions(ctx, cat);
    if (st != LT_OK) {
        lt_catalog_release(ctx, cat);
        return st;
    }
    *out = cat;
    return LT_OK;
}

lt_status lt_catalog_release(lt_context *ctx, lt_catalog *cat)
{
    if (!ctx || !cat) return LT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (defer_release(ctx, cat)) return LT_OK;
    free_catalog(ctx, cat);
    return LT_OK;
}

int32_t lt_catalog_nhalos(const lt_catalog *cat) { return cat ? cat->nhalos : -1; }

lt_status lt_synchronize(lt_context *ctx, void *stream)
{
    if (!ctx) return LT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stream synchronize");
    int32_t st = 0;
    e = cudaMemcpy(&st, ctx->status, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "status read");
    if (st != 0) {
        cudaMemset(ctx->status, 0, sizeof(int32_t));
        set_error(ctx, "kernel reported status %d", st);
        return (lt_status)st;
    }
    return LT_OK;
}

} // extern "C"

/* ------------------------------------------------------------- grid calls ---- */

/* host-output calls: the grid in about this many bands of rows, of at least this many rows */
static const int kHostBands = 8;
static const int kMinBandRows = 64;

bool lt::grid_ok(const lt_grid *g)
{
    return g && g->nx > 0 && g->ny > 0 && std::isfinite(g->xmin) && std::isfinite(g->ymin) &&
           std::isfinite(g->dx) && std::isfinite(g->dy) && (long)g->nx * g->ny <= (1L << 31);
}

/* Run one grid evaluation: `kinds`/`outs` are the requested planes (host or device). */
lt_status lt::run_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *g, int precision, int op, int kmap,
                       double D, double mult, double scale, int nout, const int *kinds, double *const *outs,
                       void *stream)
{
    if (!ctx || !cat || !grid_ok(g) || nout < 1 || nout > LT_MAX_MAPS) {
        if (ctx) set_error(ctx, "invalid grid-call arguments");
        return LT_ERR_INVALID_ARGUMENT;
    }
    if (precision != LT_FP64 && precision != LT_FP32C && precision != LT_FP64_FAST) {
        set_error(ctx, "unknown precision %d", precision);
        return LT_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < nout; i++)
        if (!outs[i]) {
            set_error(ctx, "output %d is NULL", i);
            return LT_ERR_INVALID_ARGUMENT;
        }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    const size_t npix = (size_t)g->nx * g->ny;
    const size_t plane = npix * sizeof(double);
    bool host = false;
    for (int i = 0; i < nout; i++) host |= !is_device_pointer(outs[i]);
    double *dev_out[LT_MAX_MAPS];
    if (host) {
        lt_status st = scratch_planes(ctx, nout, plane, dev_out);
        if (st != LT_OK) return st;
    } else {
        for (int i = 0; i < nout; i++) dev_out[i] = outs[i];
    }
    GridArgs a;
    memset(&a, 0, sizeof(a));
    a.recs = cat->recs;
    a.chunks = kmap ? cat->chunks_k : cat->chunks;
    a.nchunks = kmap ? cat->nchunks_k : cat->nchunks;
    a.kmap = kmap;
    a.xmin = g->xmin;
    a.ymin = g->ymin;
    a.dx = g->dx;
    a.dy = g->dy;
    a.nx = g->nx;
    a.ny = g->ny;
    a.istart = g->istart;
    a.jstart = g->jstart;
    a.nout = nout;
    a.vec_ok = (g->nx % 2 == 0);
    for (int i = 0; i < nout; i++) {
        a.kinds[i] = kinds[i];
        a.out[i] = dev_out[i];
        if (((uintptr_t)dev_out[i]) % 16) a.vec_ok = 0;
    }
    a.D = D;
    a.mult = mult;
    a.scale = scale;
    a.status = ctx->status;
    cudaStream_t s = (cudaStream_t)stream;
    /* the kernels of one band of rows (the whole grid for device outputs) */
    auto launch = [&](GridArgs &b) -> int {
        if (cat->nhalos == 0) {
            for (int i = 0; i < nout; i++) cudaMemsetAsync(b.out[i], 0, sizeof(double) * (size_t)b.nx * b.ny, s);
            if (kinds[0] == KIND_GRAD_X) return (int)cudaSuccess;
            /* maps of an empty catalogue: evaluate the epilogue on zero sums */
            count_launch(1);
            return launch_epilogue_zero(b, ctx->num_sms, s);
        }
        if (precision == LT_FP64) {
            /* the Hessian with the reference's rounding sequence, the potential through its
             * pi05 formula */
            const int xop = ((op & OP_HESS) ? ((op & ~OP_HESS) | OP_HEX) : op) | ((op & OP_POT) ? OP_PEX : 0);
            return launch_grid64_tiled(xop, b, ctx->num_sms, s, ctx->shape[LT_FP64][op & 7]);
        }
        if (precision == LT_FP64_FAST) {
            /* the dPIE deflection as log(1 + eps) (a deflection-only call: no kernel combines it) */
            const int fop = op == OP_GRAD ? (OP_GRAD | OP_GFX) : op;
            return launch_grid64_tiled(fop, b, ctx->num_sms, s, ctx->shape[LT_FP64_FAST][op & 7]);
        }
        return launch_fp32c(ctx, cat, op, b, s);
    };
    if (!host) {
        const int err = launch(a);
        if (err != cudaSuccess) return cuda_fail(ctx, (cudaError_t)err, "grid kernel launch");
        return LT_OK;
    }
    /* Host outputs: the grid in bands of rows, each band's planes copied to the host on a
     * second stream while the next bands compute.  Every band is launched before the first
     * copy is issued, since a copy into pageable memory returns only once it is done.
     * Bands start on multiples of 8 rows, the kernels' tile height, so every warp covers
     * the pixels it covers in one launch over the whole grid and the maps are the same
     * bit for bit. */
    int band = (int)(((long)g->ny + kHostBands - 1) / kHostBands);
    band = (band + 7) / 8 * 8;
    if (band < kMinBandRows) band = kMinBandRows;
    if (!ctx->copy_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "copy stream");
    }
    std::vector<cudaEvent_t> done;
    int err = cudaSuccess;
    for (int j0 = 0; j0 < g->ny; j0 += band) {
        GridArgs b = a;
        b.ny = std::min(band, g->ny - j0);
        b.jstart = g->jstart + j0;
        for (int i = 0; i < nout; i++) b.out[i] = dev_out[i] + (size_t)j0 * g->nx;
        err = launch(b);
        cudaEvent_t ev;
        if (err == cudaSuccess) err = (int)cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (err != cudaSuccess) break;
        done.push_back(ev);
        cudaEventRecord(ev, s);
    }
    for (size_t k = 0; k < done.size() && err == cudaSuccess; k++) {
        const int j0 = (int)k * band;
        const size_t off = (size_t)j0 * g->nx, n = (size_t)std::min(band, g->ny - j0) * g->nx;
        cudaStreamWaitEvent(ctx->copy_stream, done[k], 0);
        for (int i = 0; i < nout && err == cudaSuccess; i++)
            err = (int)cudaMemcpyAsync(outs[i] + off, dev_out[i] + off, n * sizeof(double), cudaMemcpyDeviceToHost,
                                       ctx->copy_stream);
    }
    const cudaError_t se = cudaStreamSynchronize(ctx->copy_stream);
    for (cudaEvent_t ev : done) cudaEventDestroy(ev);
    if (err != cudaSuccess) return cuda_fail(ctx, (cudaError_t)err, "grid kernel launch or result copy");
    if (se != cudaSuccess) return cuda_fail(ctx, se, "result copy");
    return lt_synchronize(ctx, stream);
}

/* Tile bookkeeping shared by the launchers. */
int lt::launch_grid64_tiled(int op, GridArgs &a, int num_sms, void *stream, int shape)
{
    int err = launch_grid64(op, a, num_sms, stream, false, shape);
    count_launch(1);
    return err;
}

extern "C" {

lt_status lt_gradient_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                           double scale, double *ax, double *ay, void *stream)
{
    const int kinds[2] = {KIND_GRAD_X, KIND_GRAD_Y};
    double *outs[2] = {ax, ay};
    return run_grid(ctx, cat, grid, precision, OP_GRAD, 0, 1.0, 1.0, scale, 2, kinds, outs, stream);
}

} /* extern "C" */

bool lt::hess_kind_ok(int k)
{
    return (k >= LT_MAP_HESS_A && k <= LT_MAP_HESS_D) || (k >= LT_MAP_AMPLI1 && k <= LT_MAP_AMPLI6) ||
           (k >= LT_MAP_SHEAR1 && k <= LT_MAP_SHEAR4) || (k >= LT_MAP_KAPPA && k <= LT_MAP_MU) || k == LT_MAP_MASS;
}

extern "C" {

lt_status lt_hessian_maps(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                          int32_t kmap, double dlsds, double mult, const lt_map_request *maps, int32_t nmaps,
                          void *stream)
{
    if (!maps || nmaps < 1 || nmaps > LT_MAX_MAPS) {
        if (ctx) set_error(ctx, "between 1 and %d maps must be requested", LT_MAX_MAPS);
        return LT_ERR_INVALID_ARGUMENT;
    }
    int kinds[LT_MAX_MAPS];
    double *outs[LT_MAX_MAPS];
    for (int i = 0; i < nmaps; i++) {
        if (!hess_kind_ok(maps[i].kind)) {
            if (ctx) set_error(ctx, "unknown map kind %d", maps[i].kind);
            return LT_ERR_INVALID_ARGUMENT;
        }
        kinds[i] = maps[i].kind;
        outs[i] = maps[i].out;
    }
    return run_grid(ctx, cat, grid, precision, OP_HESS, kmap ? 1 : 0, dlsds, mult, 1.0, nmaps, kinds, outs, stream);
}

lt_status lt_potential_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                            double scale, double *psi, void *stream)
{
    const int kinds[1] = {KIND_POT};
    double *outs[1] = {psi};
    return run_grid(ctx, cat, grid, precision, OP_POT, 0, 1.0, 1.0, scale, 1, kinds, outs, stream);
}

lt_status lt_lens_maps(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision, double dlsds,
                       double *kappa, double *gamma1, double *gamma2, double *mu, double *psi, void *stream)
{
    int kinds[5];
    double *outs[5];
    int n = 0, op = 0;
    const int ks[4] = {LT_MAP_KAPPA, LT_MAP_GAMMA1, LT_MAP_GAMMA2, LT_MAP_MU};
    double *os[4] = {kappa, gamma1, gamma2, mu};
    for (int i = 0; i < 4; i++)
        if (os[i]) {
            kinds[n] = ks[i];
            outs[n++] = os[i];
            op |= OP_HESS;
        }
    if (psi) {
        kinds[n] = KIND_POT;
        outs[n++] = psi;
        op |= OP_POT;
    }
    if (n == 0) {
        if (ctx) set_error(ctx, "no output requested");
        return LT_ERR_INVALID_ARGUMENT;
    }
    return run_grid(ctx, cat, grid, precision, op, 0, dlsds, 1.0, dlsds, n, kinds, outs, stream);
}

} // extern "C"

/* ------------------------------------------------------- shapes and autotuning ---- */

static bool sums_ok(int precision, int sums)
{
    if (precision != LT_FP64 && precision != LT_FP32C && precision != LT_FP64_FAST) return false;
    return sums == OP_GRAD || sums == OP_HESS || sums == OP_POT || sums == (OP_HESS | OP_POT);
}

extern "C" {

lt_status lt_set_kernel_shape(lt_context *ctx, int32_t precision, int32_t sums, int32_t ppt, int32_t cps)
{
    if (!ctx || !sums_ok(precision, sums) || (ppt != 1 && ppt != 2) || (cps != 1 && cps != 2))
        return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->shape[precision][sums] = LT_SHAPE(ppt, cps);
    return LT_OK;
}

lt_status lt_get_kernel_shape(const lt_context *ctx, int32_t precision, int32_t sums, int32_t *ppt, int32_t *cps)
{
    if (!ctx || !ppt || !cps || !sums_ok(precision, sums)) return LT_ERR_INVALID_ARGUMENT;
    const int s = ctx->shape[precision][sums];
    *ppt = shape_ppt(s);
    *cps = shape_cps(s);
    return LT_OK;
}

static bool config_ok(int precision, const lt_kernel_config *c)
{
    if (!c) return false;
    const int s = LT_SHAPE4(c->pixels_per_thread, c->ctas_per_sm, c->threads, c->chunk);
    if (c->pixels_per_thread < 1 || c->pixels_per_thread > 2 || c->ctas_per_sm < 1 || c->ctas_per_sm > 4 ||
        (c->threads != 128 && c->threads != 256) || (c->chunk != 32 && c->chunk != 64 && c->chunk != 128))
        return false;
    if (precision == LT_FP32C) return shape32_ok(s);
    /* the FP64 kernels come in the four (pixels, CTAs) shapes at 256 threads, 64-record stages */
    return c->threads == 256 && c->chunk == 64 && c->ctas_per_sm <= 2;
}

lt_status lt_set_kernel_config(lt_context *ctx, int32_t precision, int32_t sums, const lt_kernel_config *c)
{
    if (!ctx || !sums_ok(precision, sums) || !config_ok(precision, c)) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->shape[precision][sums] = LT_SHAPE4(c->pixels_per_thread, c->ctas_per_sm, c->threads, c->chunk);
    return LT_OK;
}

lt_status lt_get_kernel_config(const lt_context *ctx, int32_t precision, int32_t sums, lt_kernel_config *c)
{
    if (!ctx || !c || !sums_ok(precision, sums)) return LT_ERR_INVALID_ARGUMENT;
    const int s = ctx->shape[precision][sums];
    c->pixels_per_thread = shape_ppt(s);
    c->ctas_per_sm = shape_cps(s);
    c->threads = shape_threads(s);
    c->chunk = shape_cap(s);
    return LT_OK;
}

lt_status lt_autotune(lt_context *ctx, const lt_catalog *cat, int32_t precision, int32_t sums, int32_t grid_n,
                      double *best_ms)
{
    if (!ctx || !cat || !sums_ok(precision, sums) || grid_n < 8 || grid_n > 8192) return LT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    /* a grid over the catalogue's extent (10% margin) */
    double lo = -1., hi = 1.;
    for (const lt_rec64 &r : cat->host_recs) {
        lo = std::fmin(lo, std::fmin(r.x0, r.y0));
        hi = std::fmax(hi, std::fmax(r.x0, r.y0));
    }
    const double pad = 0.1 * (hi - lo);
    lt_grid g;
    g.xmin = g.ymin = lo - pad;
    g.dx = g.dy = (hi - lo + 2 * pad) / (grid_n - 1);
    g.nx = g.ny = grid_n;
    g.istart = g.jstart = 0;
    int kinds[2];
    int nout = 0;
    if (sums & OP_GRAD) {
        kinds[nout++] = KIND_GRAD_X;
        kinds[nout++] = KIND_GRAD_Y;
    }
    if (sums & OP_HESS) kinds[nout++] = LT_MAP_KAPPA;
    if (sums & OP_POT) kinds[nout++] = KIND_POT;
    double *planes = nullptr;
    const size_t plane = sizeof(double) * (size_t)grid_n * grid_n;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        lt_status st = dev_alloc(ctx, (void **)&planes, nout * plane);
        if (st != LT_OK) return st;
    }
    double *outs[2] = {planes, planes + (size_t)grid_n * grid_n};
    /* the search space: FP32C every built shape (pixels per thread, CTAs per SM, threads
     * per CTA) with every stage size; the FP64 kernels their four (pixels, CTAs) shapes */
    std::vector<int> shapes;
    if (precision == LT_FP32C) {
        for (int k = 0; k < kNumShapes32; k++)
            for (int cap : {32, 64, 128}) shapes.push_back((kShapes32[k] & 0xffff) | ((cap / 32) << 16));
    } else {
        shapes = {LT_SHAPE(1, 1), LT_SHAPE(1, 2), LT_SHAPE(2, 1), LT_SHAPE(2, 2)};
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int best_shape = ctx->shape[precision][sums];
    lt_status st = LT_OK;
    for (size_t k = 0; k < shapes.size() && st == LT_OK; k++) {
        ctx->shape[precision][sums] = shapes[k];
        st = run_grid(ctx, cat, &g, precision, sums, 0, 1.0, 1.0, 1.0, nout, kinds, outs, nullptr);
        if (st != LT_OK) break;
        cudaEventRecord(e0, nullptr);
        for (int rep = 0; rep < 2 && st == LT_OK; rep++)
            st = run_grid(ctx, cat, &g, precision, sums, 0, 1.0, 1.0, 1.0, nout, kinds, outs, nullptr);
        cudaEventRecord(e1, nullptr);
        if (st == LT_OK) st = lt_synchronize(ctx, nullptr);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (st == LT_OK && ms / 2 < best) {
            best = ms / 2;
            best_shape = shapes[k];
        }
    }
    ctx->shape[precision][sums] = best_shape;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        dev_free(ctx, planes, nout * plane);
    }
    if (best_ms) *best_ms = best;
    return st;
}

} // extern "C"
