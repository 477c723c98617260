/*
 * lt_noalloc.cu -- lt_hessian_maps_noalloc: the LT_FP32C Hessian-map call with device
 * outputs, allocating no memory during the call.
 *
 * lt_hessian_maps in LT_FP32C grows a context-owned buffer (cudaMalloc) for the list of
 * pixels it recomputes in FP64 near critical curves.  This variant keeps that list in a
 * file-scope static device array of fixed size instead, so the call itself performs no
 * allocation: no cudaMalloc/cudaFree, no allocating library routine.  Limits that follow:
 *   - a grid has at most LT_NOALLOC_MAX_PIXELS pixels (the list holds one entry per
 *     pixel in the worst case); larger grids are rejected with LT_ERR_INVALID_ARGUMENT;
 *   - outputs must be device pointers (host outputs would need staging memory);
 *   - the array is one per process and device: calls that overlap in time (two threads,
 *     or two streams of one device) race on it and must be serialised by the caller.
 * The list's length word must start at zero; the call zeroes it on its stream before
 * pass 1.  The array's address is looked up once per device (cudaGetSymbolAddress with
 * that device current); that first call also loads the module's data on the device, so
 * it should come before any stream capture that includes this call.  The address is
 * forgotten when the last context of the device is destroyed.
 */
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "lt_internal.h"

#define LT_NOALLOC_MAX_PIXELS (1 << 22) /* 2048 x 2048; the array is 16 MiB + 256 B */

namespace lt {
int launch_fp32c_with_list(lt_context *ctx, const lt_catalog *cat, GridArgs &a, int32_t *list, int32_t *count,
                           int32_t cap, void *stream);
}

using namespace lt;

/* [0]: length word of the list (entries 1..63 unused, keeping the list 256-byte aligned),
 * [64 ..]: pixel indices */
static __device__ __align__(256) int32_t g_noalloc_list[64 + LT_NOALLOC_MAX_PIXELS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_lookup_mu;
int32_t *g_list_addr[kMaxDevices] = {};

/* Device address of g_noalloc_list on ctx's device (looked up once per device). */
lt_status list_address(lt_context *ctx, int32_t **out)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices) {
        set_error(ctx, "device %d: the no-allocation call supports devices 0..%d", ctx->device, kMaxDevices - 1);
        return LT_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_lookup_mu);
    if (!g_list_addr[ctx->device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_list); /* ctx's device is current */
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress of the static list");
        g_list_addr[ctx->device] = (int32_t *)p;
    }
    *out = g_list_addr[ctx->device];
    return LT_OK;
}
} // namespace

namespace lt {
/* Called by lt_destroy for the last context of a device: the next call looks the array
 * up again (after a device reset its module, and so its address, is new). */
void noalloc_forget(int device)
{
    if (device < 0 || device >= kMaxDevices) return;
    std::lock_guard<std::mutex> lock(g_lookup_mu);
    g_list_addr[device] = nullptr;
}
} // namespace lt

extern "C" lt_status lt_hessian_maps_noalloc(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid,
                                              int32_t kmap, double dlsds, double mult, const lt_map_request *maps,
                                              int32_t nmaps, void *stream)
{
    if (!ctx || !cat || !maps || !grid_ok(grid) || nmaps < 1 || nmaps > LT_MAX_MAPS) {
        if (ctx) set_error(ctx, "invalid arguments");
        return LT_ERR_INVALID_ARGUMENT;
    }
    const long npix = (long)grid->nx * grid->ny;
    if (npix > LT_NOALLOC_MAX_PIXELS) {
        set_error(ctx, "grid of %ld pixels exceeds the no-allocation call's limit of %d pixels", npix,
                  LT_NOALLOC_MAX_PIXELS);
        return LT_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < nmaps; i++) {
        if (!hess_kind_ok(maps[i].kind)) {
            set_error(ctx, "unknown map kind %d", maps[i].kind);
            return LT_ERR_INVALID_ARGUMENT;
        }
        if (!maps[i].out || !is_device_pointer(maps[i].out)) {
            set_error(ctx, "output %d must be a device pointer (the call stages nothing through host memory)", i);
            return LT_ERR_INVALID_ARGUMENT;
        }
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    int32_t *base = nullptr;
    lt_status st = list_address(ctx, &base);
    if (st != LT_OK) return st;
    GridArgs a;
    memset(&a, 0, sizeof(a));
    a.recs = cat->recs;
    a.chunks = kmap ? cat->chunks_k : cat->chunks;
    a.nchunks = kmap ? cat->nchunks_k : cat->nchunks;
    a.kmap = kmap ? 1 : 0;
    a.xmin = grid->xmin;
    a.ymin = grid->ymin;
    a.dx = grid->dx;
    a.dy = grid->dy;
    a.nx = grid->nx;
    a.ny = grid->ny;
    a.istart = grid->istart;
    a.jstart = grid->jstart;
    a.nout = nmaps;
    a.vec_ok = (grid->nx % 2 == 0);
    for (int i = 0; i < nmaps; i++) {
        a.kinds[i] = maps[i].kind;
        a.out[i] = maps[i].out;
        if (((uintptr_t)maps[i].out) % 16) a.vec_ok = 0;
    }
    a.D = dlsds;
    a.mult = mult;
    a.scale = 1.0;
    a.status = ctx->status;
    cudaStream_t s = (cudaStream_t)stream;
    int err;
    if (cat->nhalos == 0) {
        /* maps of an empty catalogue: the epilogue evaluated on zero sums */
        err = launch_epilogue_zero(a, ctx->num_sms, s);
        count_launch(1);
    } else {
        err = launch_fp32c_with_list(ctx, cat, a, base + 64, base, LT_NOALLOC_MAX_PIXELS, s);
    }
    if (err != cudaSuccess) return cuda_fail(ctx, (cudaError_t)err, "no-allocation Hessian maps");
    return LT_OK;
}
