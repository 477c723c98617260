/*
 * lt_batch.cpp -- lt_request validation and packing into queue descriptors, and the
 * graph-captured batch (lt_batch_*).
 *
 * The reference's posterior driver evaluates one map per call, each call allocating,
 * copying, launching, synchronising and freeing (utils/maps/main.cpp:432-587 over
 * map_grid_ampli_GPU, src/grid_map_ampli_GPU.cu:93-192).  A batch packs all requests
 * once; every lt_batch_launch then replays one CUDA graph of two kernels (queue reset +
 * the persistent work-queue kernel) that evaluates every request's tiles.
 */
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"
#include "lt_internal.h"
#include "lt_queue.h"

using namespace lt;

struct lt_batch {
    int mode = 0;
    int variant = 0; /* queue kernel variant (FP32C: pixels per thread, CTAs per SM) */
    int n = 0;
    QSlot *slots = nullptr;
    QState *state = nullptr;
    size_t bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace lt {

static int public_kind(int k, int &op)
{
    switch (k) {
    case LT_MAP_POTENTIAL: op |= OP_POT; return KIND_POT;
    case LT_MAP_DEFLECTION_X: op |= OP_GRAD; return KIND_GRAD_X;
    case LT_MAP_DEFLECTION_Y: op |= OP_GRAD; return KIND_GRAD_Y;
    default:
        if (!hess_kind_ok(k)) return -1;
        op |= OP_HESS;
        return k;
    }
}

/* Validate a request and fill its queue descriptor.  `outs` (may be NULL) replaces the
 * request's output pointers (the serving loop's staging planes for host outputs);
 * otherwise the request's outputs must be device pointers.  FP32C tiles have `ppt32`
 * pixels per thread (the queue kernel variant's). */
lt_status make_queue_item(lt_context *ctx, const lt_request *r, int precision, double *const *outs, QItem *it,
                          int ppt32)
{
    if (!r || !r->cat || !grid_ok(&r->grid) || r->nmaps < 1 || r->nmaps > LT_MAX_MAPS) {
        set_error(ctx, "invalid request (catalogue, grid or map count)");
        return LT_ERR_INVALID_ARGUMENT;
    }
    if (precision != LT_FP32C && precision != LT_FP64) {
        set_error(ctx, "batches and the serving loop run LT_FP32C or LT_FP64 (precision %d)", precision);
        return LT_ERR_INVALID_ARGUMENT;
    }
    const lt_catalog *cat = r->cat;
    memset(it, 0, sizeof(*it));
    GridArgs &a = it->g;
    int op = 0;
    bool det = false;
    a.vec_ok = (r->grid.nx % 2 == 0);
    for (int i = 0; i < r->nmaps; i++) {
        const int k = public_kind(r->maps[i].kind, op);
        if (k < 0) {
            set_error(ctx, "request map %d: unknown kind %d", i, r->maps[i].kind);
            return LT_ERR_INVALID_ARGUMENT;
        }
        double *o = outs ? outs[i] : r->maps[i].out;
        if (!o) {
            set_error(ctx, "request map %d: output is NULL", i);
            return LT_ERR_INVALID_ARGUMENT;
        }
        if (!outs && !is_device_pointer(o)) {
            set_error(ctx, "request map %d: batch outputs must be device pointers", i);
            return LT_ERR_INVALID_ARGUMENT;
        }
        a.kinds[i] = k;
        a.out[i] = o;
        if (((uintptr_t)o) % 16) a.vec_ok = 0;
        det |= det_sensitive(k);
    }
    const bool c32 = precision == LT_FP32C;
    a.recs = cat->recs;
    a.chunks = r->kmap ? cat->chunks_k : cat->chunks;
    a.nchunks = r->kmap ? cat->nchunks_k : cat->nchunks;
    a.kmap = r->kmap ? 1 : 0;
    a.xmin = r->grid.xmin;
    a.ymin = r->grid.ymin;
    a.dx = r->grid.dx;
    a.dy = r->grid.dy;
    a.nx = r->grid.nx;
    a.ny = r->grid.ny;
    a.istart = r->grid.istart;
    a.jstart = r->grid.jstart;
    a.nout = r->nmaps;
    a.D = r->dlsds;
    a.mult = r->mult;
    a.scale = r->scale;
    a.status = ctx->status;
    it->op = op;
    it->ppt = c32 ? (ppt32 == 1 ? 1 : 2) : ((op & OP_POT) ? 1 : 2);
    const int P = it->ppt;
    a.tiles_x = (a.nx + 32 * P - 1) / (32 * P);
    a.ntiles = a.tiles_x * ((a.ny + 7) / 8);
    it->ntiles = a.ntiles;
    if (c32) {
        const Fp32cCatalog &fc = *reinterpret_cast<const Fp32cCatalog *>(&cat->aux_desc);
        it->recs32 = fc.recs32;
        it->chunks32 = fc.chunks;
        it->nchunks32 = cat->nhalos ? fc.nchunks : 0;
        it->nie64 = fc.nie;
        it->mu_tol = det ? kMuTol32 : 0.0;
    }
    if (cat->nhalos == 0) a.nchunks = 0;
    return LT_OK;
}

} // namespace lt

extern "C" {

lt_status lt_batch_create(lt_context *ctx, const lt_request *reqs, int32_t nreqs, int32_t precision,
                          lt_batch **out)
{
    if (!ctx || !out || !reqs || nreqs < 1) return LT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    /* the queue kernel variant nearest to the context's (tuned) FP32C Hessian shape */
    const int variant = queue_variant(ctx->shape[LT_FP32C][OP_HESS]);
    std::vector<QSlot> host((size_t)nreqs);
    std::vector<double> cost((size_t)nreqs);
    for (int i = 0; i < nreqs; i++) {
        QSlot &s = host[i];
        memset(&s, 0, sizeof(s));
        lt_status st = make_queue_item(ctx, &reqs[i], precision, nullptr, &s.item, shape_ppt(variant));
        if (st != LT_OK) {
            set_error(ctx, "request %d: %s", i, lt_last_error(ctx));
            return st;
        }
        cost[i] = (double)s.item.ntiles * (double)(reqs[i].cat->nhalos + 1);
    }
    /* costliest requests first: the queue runs them in order, so the cheap ones fill the
     * tail (longest-processing-time-first) */
    std::vector<int> order((size_t)nreqs);
    for (int i = 0; i < nreqs; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<QSlot> slots((size_t)nreqs);
    for (int i = 0; i < nreqs; i++) {
        slots[i] = host[order[i]];
        slots[i].item.seq = (uint32_t)i;
    }
    lt_batch *b = new (std::nothrow) lt_batch();
    if (!b) return LT_ERR_OUT_OF_MEMORY;
    b->mode = precision == LT_FP32C ? QMODE_C32 : QMODE_EXACT;
    b->variant = variant;
    b->n = nreqs;
    b->bytes = sizeof(QSlot) * (size_t)nreqs + sizeof(QState);
    void *mem = nullptr;
    lt_status st = dev_alloc(ctx, &mem, b->bytes);
    if (st != LT_OK) {
        delete b;
        return st;
    }
    b->state = (QState *)mem;
    b->slots = (QSlot *)((char *)mem + sizeof(QState));
    cudaError_t e = cudaMemcpy(b->slots, slots.data(), sizeof(QSlot) * (size_t)nreqs, cudaMemcpyHostToDevice);
    const int blocks = queue_blocks(b->mode, b->variant, ctx->num_sms);
    cudaStream_t cs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        QArgs q;
        q.slots = b->slots;
        q.state = b->state;
        q.nslots = nreqs;
        q.window = 1;
        q.idle_polls = 0;
        q.desc_polls = 1 << 30; /* every descriptor is in place before the graph runs */
        q.status = ctx->status;
        launch_queue_reset(b->slots, b->state, nreqs, cs);
        launch_queue(b->mode, b->variant, q, blocks, cs);
        e = cudaStreamEndCapture(cs, &b->graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        if (b->graph) cudaGraphDestroy(b->graph);
        dev_free(ctx, mem, b->bytes);
        delete b;
        return cuda_fail(ctx, e, "batch graph");
    }
    *out = b;
    return LT_OK;
}

lt_status lt_batch_launch(lt_context *ctx, lt_batch *b, void *stream)
{
    if (!ctx || !b) return LT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph launch");
    count_launch(2);
    return LT_OK;
}

int32_t lt_batch_size(const lt_batch *b) { return b ? b->n : -1; }

lt_status lt_batch_config(const lt_batch *b, lt_kernel_config *c)
{
    if (!b || !c) return LT_ERR_INVALID_ARGUMENT;
    c->pixels_per_thread = b->mode == QMODE_C32 ? shape_ppt(b->variant) : 0;
    c->ctas_per_sm = b->mode == QMODE_C32 ? shape_cps(b->variant) : 2;
    c->threads = 256;
    c->chunk = LT_CHUNK;
    return LT_OK;
}

lt_status lt_batch_destroy(lt_context *ctx, lt_batch *b)
{
    if (!ctx || !b) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    dev_free(ctx, b->state, b->bytes);
    delete b;
    return LT_OK;
}

} /* extern "C" */
