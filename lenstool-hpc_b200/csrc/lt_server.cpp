/*
 * lt_server.cpp -- the continuous-batching serving loop (lt_server_*).
 *
 * Requests (lt_request: catalogue handle, grid, output planes) are submitted from any
 * thread and complete asynchronously.  A scheduler thread per server:
 *   1. admits queued requests in arrival order while a ring slot is free and, for
 *      host-pointer outputs, their planes fit in the server's HBM arena (free-memory
 *      accounting: a request that does not fit waits until earlier results free space);
 *   2. publishes an admitted request to the running persistent kernel: the slot
 *      descriptor, then the published count, copied on the publish stream in that order;
 *   3. keeps the persistent kernel (lt_queue.cu) running while requests are in flight,
 *      relaunching it after it left idle;
 *   4. sees completions in a mapped host word per slot, copies host-pointer results out
 *      on the copy stream, returns their arena bytes and frees the slot.
 * Requests admitted while others are on the GPU share it tile by tile (the kernel serves
 * the oldest `window` requests round-robin), so a result is the same alone and in a mix:
 * each pixel's sums are evaluated by one thread with the same arithmetic either way.
 *
 * The reference has no serving mode: each map is one blocking call that allocates and
 * frees its buffers (src/grid_map_ampli_GPU.cu:93-192).
 */
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"
#include "lt_arena.h"
#include "lt_chi2.h"
#include "lt_internal.h"
#include "lt_queue.h"

using namespace lt;

namespace lt {
lt_status make_queue_item(lt_context *ctx, const lt_request *r, int precision, double *const *outs, QItem *it,
                          int ppt32);
void free_catalog(lt_context *ctx, lt_catalog *cat);

/* Context-level state of the serving extension: catalogues released while a server
 * runs are freed when the last server of the context is destroyed (a cudaFree would
 * wait for the persistent kernel, and its memory must not be reused under it). */
struct Extensions {
    std::mutex mu;
    int servers = 0;
    std::vector<lt_catalog *> deferred;
};

static Extensions *ext_of(lt_context *ctx)
{
    if (!ctx->ext) ctx->ext = new Extensions();
    return (Extensions *)ctx->ext;
}

bool defer_release(lt_context *ctx, lt_catalog *cat)
{
    if (!ctx->ext) return false;
    Extensions *x = (Extensions *)ctx->ext;
    std::lock_guard<std::mutex> lock(x->mu);
    if (x->servers == 0) return false;
    x->deferred.push_back(cat);
    return true;
}

void destroy_extensions(lt_context *ctx)
{
    if (!ctx->ext) return;
    Extensions *x = (Extensions *)ctx->ext;
    for (lt_catalog *c : x->deferred) free_catalog(ctx, c);
    delete x;
    ctx->ext = nullptr;
}

} // namespace lt

namespace {

/* R_TAIL: a chi2 request whose deflection grid is done, waiting for its delensing */
enum { R_QUEUED = 0, R_RUNNING = 1, R_COPYING = 2, R_DONE = 3, R_FAILED = 4, R_TAIL = 5 };
enum { K_MAPS = 0, K_CHI2 = 1 };

using Clock = std::chrono::steady_clock;

struct SrvReq {
    uint64_t ticket = 0;
    int kind = K_MAPS;
    lt_request req;
    bool host_out = false;
    size_t plane = 0;          /* bytes per output plane */
    size_t arena_off = Arena::kFail;
    int slot = -1;
    uint64_t seq = 0;
    int state = R_QUEUED;
    lt_status status = LT_OK;
    Clock::time_point t_submit, t_admit, t_gpu, t_done;
    cudaEvent_t copied = nullptr;
    /* chi2 requests: the systems (host copies), the device layout in the arena, results */
    lt_frame frame{};
    int n = 0;
    std::vector<int32_t> nimg, first;
    std::vector<double> ix, iy, dr;
    size_t chi_bytes = 0;
    Chi2Dev dev{};
    double chi2 = 0.;
    int32_t found = 0;
    bool overflow = false;
};

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

} // namespace

struct lt_server {
    lt_context *ctx = nullptr;
    int precision = LT_FP32C, mode = QMODE_C32;
    int nslots = 64, window = 8, idle_polls = 20000, desc_polls = 2000000, blocks = 0;
    int variant = LT_SHAPE(2, 2);        /* queue kernel variant (FP32C: pixels, CTAs per SM) */
    bool drop_next = false;              /* fault injection: publish the next request without its descriptor */
    QSlot *slots = nullptr;
    QState *state = nullptr;
    size_t dev_bytes = 0, arena_bytes = 0;
    char *arena_mem = nullptr;
    Arena arena;
    QSlot *h_slots = nullptr;            /* pinned staging of slot descriptors */
    unsigned long long *h_pub = nullptr; /* pinned staging of published counts */
    uint32_t *h_flags = nullptr;         /* mapped completion words */
    uint32_t *d_flags = nullptr;
    int32_t *h_status = nullptr;         /* pinned copy of the device status word */
    double *h_chi = nullptr;             /* pinned chi2 results, two words per slot */
    int32_t *h_yield = nullptr;          /* pinned {1, 0}: the values written to QState::yield */
    cudaStream_t loop_stream = nullptr, pub_stream = nullptr, copy_stream = nullptr;
    cudaEvent_t loop_done = nullptr;
    bool loop_launched = false;
    bool yielding = false;               /* QState::yield was set and not yet cleared */
    std::thread thr;
    std::mutex mu;
    std::condition_variable cv_done, cv_work;
    std::deque<SrvReq *> pending;
    std::vector<SrvReq *> ring;
    std::map<uint64_t, SrvReq *> reqs;
    uint64_t next_ticket = 1, next_seq = 0;
    bool stopping = false;
    lt_status broken = LT_OK;
    lt_server_stats stats{};
    int inflight = 0;
};

namespace {

void finish(lt_server *s, SrvReq *r, lt_status st)
{
    r->status = st;
    r->state = st == LT_OK ? R_DONE : R_FAILED;
    r->t_done = Clock::now();
    if (r->arena_off != Arena::kFail) {
        s->arena.release(r->arena_off);
        r->arena_off = Arena::kFail;
    }
    if (r->slot >= 0) {
        s->ring[r->slot] = nullptr;
        r->slot = -1;
        s->inflight--;
    }
    if (st == LT_OK)
        s->stats.completed++;
    else
        s->stats.failed++;
}

/* Admit the oldest queued requests that fit (scheduler thread, lock held). */
void admit(lt_server *s)
{
    while (!s->pending.empty()) {
        SrvReq *r = s->pending.front();
        const int slot = (int)(s->next_seq % (uint64_t)s->nslots);
        if (s->ring[slot]) return; /* the slot's previous request is still running */
        double *outs[LT_MAX_MAPS] = {};
        if (r->kind == K_CHI2) {
            /* the chi2 buffers and the deflection planes in the arena; the systems are
             * copied on the publish stream ahead of the grid's descriptor */
            const size_t off = s->arena.alloc(r->chi_bytes);
            if (off == Arena::kFail) return;
            r->arena_off = off;
            chi2_layout((int)r->nimg.size(), (int)r->ix.size(), &r->frame, r->n, s->arena_mem + off, r->dev);
            const cudaError_t e = chi2_upload_systems_async(r->dev, r->nimg.data(), r->first.data(), r->ix.data(),
                                                            r->iy.data(), r->dr.data(), s->pub_stream);
            if (e != cudaSuccess) {
                s->pending.pop_front();
                set_error(s->ctx, "chi2 systems upload: %s", cudaGetErrorString(e));
                finish(s, r, LT_ERR_CUDA);
                s->cv_done.notify_all();
                continue;
            }
            r->req.grid = {r->dev.xmin, r->dev.ymin, r->dev.dx, r->dev.dy, r->n, r->n, 0, 0};
            outs[0] = (double *)r->dev.ax;
            outs[1] = (double *)r->dev.ay;
        } else if (r->host_out) {
            const size_t off = s->arena.alloc(r->plane * (size_t)r->req.nmaps);
            if (off == Arena::kFail) return; /* waits for results to free arena space */
            r->arena_off = off;
            for (int i = 0; i < r->req.nmaps; i++) outs[i] = (double *)(s->arena_mem + off + (size_t)i * r->plane);
        } else {
            for (int i = 0; i < r->req.nmaps; i++) outs[i] = r->req.maps[i].out;
        }
        QSlot &hs = s->h_slots[slot];
        memset(&hs, 0, sizeof(hs));
        lt_status st = make_queue_item(s->ctx, &r->req, s->precision, outs, &hs.item, shape_ppt(s->variant));
        s->pending.pop_front();
        if (st != LT_OK) {
            finish(s, r, st);
            s->cv_done.notify_all();
            continue;
        }
        const uint64_t seq = s->next_seq++;
        hs.item.seq = (uint32_t)seq;
        hs.item.host_flag = s->d_flags + slot;
        hs.ctr = (unsigned long long)(uint32_t)seq << 32;
        hs.done = 0u;
        __atomic_store_n(&s->h_flags[slot], 0u, __ATOMIC_RELEASE);
        s->h_pub[slot] = seq + 1;
        if (s->drop_next) /* injected fault: the descriptor is lost, the request still published */
            s->drop_next = false;
        else
            cudaMemcpyAsync(&s->slots[slot], &hs, sizeof(QSlot), cudaMemcpyHostToDevice, s->pub_stream);
        cudaMemcpyAsync(&s->state->published, &s->h_pub[slot], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                        s->pub_stream);
        r->slot = slot;
        r->seq = seq;
        r->state = R_RUNNING;
        r->t_admit = Clock::now();
        s->ring[slot] = r;
        s->inflight++;
        s->stats.admitted++;
        if (s->inflight > s->stats.max_inflight) s->stats.max_inflight = s->inflight;
    }
}

/* Completions seen in the mapped words; host-pointer results are copied out. */
bool collect(lt_server *s)
{
    bool any = false;
    for (int slot = 0; slot < s->nslots; slot++) {
        SrvReq *r = s->ring[slot];
        if (!r) continue;
        if (r->state == R_RUNNING) {
            const uint32_t f = __atomic_load_n(&s->h_flags[slot], __ATOMIC_ACQUIRE);
            if (f != (uint32_t)r->seq + 1u) continue;
            r->t_gpu = Clock::now();
            any = true;
            if (r->kind == K_CHI2) { /* the grid is done: delensing next (run_tails) */
                r->state = R_TAIL;
                continue;
            }
            if (!r->host_out) {
                finish(s, r, LT_OK);
                continue;
            }
            const size_t npix = (size_t)r->req.grid.nx * r->req.grid.ny;
            cudaError_t e = cudaSuccess;
            for (int i = 0; i < r->req.nmaps && e == cudaSuccess; i++)
                e = cudaMemcpyAsync(r->req.maps[i].out, s->arena_mem + r->arena_off + (size_t)i * r->plane,
                                    npix * sizeof(double), cudaMemcpyDefault, s->copy_stream);
            if (e == cudaSuccess && !r->copied) e = cudaEventCreateWithFlags(&r->copied, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventRecord(r->copied, s->copy_stream);
            if (e != cudaSuccess) {
                set_error(s->ctx, "result copy: %s", cudaGetErrorString(e));
                finish(s, r, LT_ERR_CUDA);
                continue;
            }
            r->state = R_COPYING;
        }
        if (r->state == R_COPYING) {
            const cudaError_t e = cudaEventQuery(r->copied);
            if (e == cudaErrorNotReady) continue;
            any = true;
            if (e == cudaSuccess && r->kind == K_CHI2) {
                r->chi2 = s->h_chi[2 * slot];
                int32_t f[2];
                memcpy(f, &s->h_chi[2 * slot + 1], sizeof(f));
                r->found = f[0];
                r->overflow = f[1] != 0;
            }
            finish(s, r, e == cudaSuccess ? LT_OK : LT_ERR_CUDA);
        }
    }
    return any;
}

/* Delensing and chi2 of the chi2 requests whose grids are done.  They run on the loop
 * stream between two launches of the persistent kernel, which otherwise holds every SM:
 * the kernel is asked to leave at its next claim (QState::yield; unclaimed tiles stay in
 * their slots), the tails run with the whole GPU, and the loop is relaunched after them. */
void run_tails(lt_server *s)
{
    bool waiting = false;
    for (SrvReq *r : s->ring)
        if (r && r->state == R_TAIL) waiting = true;
    const bool busy = s->loop_launched && cudaEventQuery(s->loop_done) == cudaErrorNotReady;
    if (waiting && busy) {
        if (!s->yielding) {
            cudaMemcpyAsync(&s->state->yield, &s->h_yield[0], sizeof(int32_t), cudaMemcpyHostToDevice, s->pub_stream);
            s->yielding = true;
        }
        return;
    }
    if (waiting) {
        cudaEvent_t pub;
        cudaEventCreateWithFlags(&pub, cudaEventDisableTiming);
        cudaEventRecord(pub, s->pub_stream);
        cudaStreamWaitEvent(s->loop_stream, pub, 0);
        cudaEventDestroy(pub);
        for (int slot = 0; slot < s->nslots; slot++) {
            SrvReq *r = s->ring[slot];
            if (!r || r->state != R_TAIL) continue;
            cudaError_t e = (cudaError_t)chi2_tail(s->ctx, r->req.cat, r->dev, s->loop_stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&s->h_chi[2 * slot], r->dev.chi2, sizeof(double), cudaMemcpyDeviceToHost,
                                    s->loop_stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&s->h_chi[2 * slot + 1], r->dev.found, 2 * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, s->loop_stream);
            if (e == cudaSuccess && !r->copied) e = cudaEventCreateWithFlags(&r->copied, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventRecord(r->copied, s->loop_stream);
            if (e != cudaSuccess) {
                set_error(s->ctx, "chi2 delensing: %s", cudaGetErrorString(e));
                finish(s, r, LT_ERR_CUDA);
                continue;
            }
            r->state = R_COPYING;
        }
    }
    if (!busy && s->yielding) {
        cudaMemcpyAsync(&s->state->yield, &s->h_yield[1], sizeof(int32_t), cudaMemcpyHostToDevice, s->pub_stream);
        s->yielding = false;
    }
}

/* The loop reported a published request whose descriptor never reached the device
 * (QState::stuck = its seq + 1): fail that request with LT_ERR_TIMEOUT, put an empty
 * descriptor of its seq in its slot so the device's head moves past it, and clear the
 * report.  Returns false when no running request has that seq. */
bool drop_stuck(lt_server *s)
{
    const uint32_t seq = (uint32_t)s->h_status[1] - 1u;
    for (int slot = 0; slot < s->nslots; slot++) {
        SrvReq *r = s->ring[slot];
        if (!r || r->state != R_RUNNING || (uint32_t)r->seq != seq) continue;
        QSlot &hs = s->h_slots[slot];
        memset(&hs, 0, sizeof(hs));
        hs.item.seq = seq;
        hs.item.ntiles = 0;
        hs.ctr = (unsigned long long)seq << 32;
        cudaMemcpyAsync(&s->slots[slot], &hs, sizeof(QSlot), cudaMemcpyHostToDevice, s->pub_stream);
        cudaMemsetAsync(&s->state->stuck, 0, sizeof(uint32_t), s->pub_stream);
        cudaMemsetAsync(s->ctx->status, 0, sizeof(int32_t), s->pub_stream);
        set_error(s->ctx, "request %llu: its descriptor did not reach the device within the wait limit",
                  (unsigned long long)r->ticket);
        finish(s, r, LT_ERR_TIMEOUT);
        s->stats.timed_out++;
        s->cv_done.notify_all();
        return true;
    }
    return false;
}

/* Keep the persistent kernel running while requests are in flight. */
void keep_loop(lt_server *s)
{
    bool running_req = false;
    for (SrvReq *r : s->ring)
        if (r && r->state == R_RUNNING) running_req = true;
    if (!running_req || s->yielding) return; /* a yield is cleared by run_tails first */
    if (s->loop_launched) {
        const cudaError_t e = cudaEventQuery(s->loop_done);
        if (e == cudaErrorNotReady) return;
        /* the kernel has left: was it a bounded wait that gave up? */
        cudaMemcpyAsync(s->h_status, s->ctx->status, sizeof(int32_t), cudaMemcpyDeviceToHost, s->pub_stream);
        cudaMemcpyAsync(s->h_status + 1, &s->state->stuck, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->pub_stream);
        cudaStreamSynchronize(s->pub_stream);
        if (e == cudaSuccess && *s->h_status == LT_ERR_TIMEOUT && s->h_status[1] != 0 && drop_stuck(s))
            return; /* relaunched at the next pass, without the request */
        if (e != cudaSuccess || *s->h_status != 0) {
            const lt_status st = e != cudaSuccess ? LT_ERR_CUDA : (lt_status)*s->h_status;
            set_error(s->ctx, "serving loop kernel stopped: %s",
                      e != cudaSuccess ? cudaGetErrorString(e) : lt_status_string(st));
            s->broken = st;
            for (SrvReq *r : s->ring)
                if (r && r->state == R_RUNNING) finish(s, r, st);
            while (!s->pending.empty()) {
                finish(s, s->pending.front(), st);
                s->pending.pop_front();
            }
            s->cv_done.notify_all();
            return;
        }
    }
    QArgs q;
    q.slots = s->slots;
    q.state = s->state;
    q.nslots = s->nslots;
    q.window = s->window;
    q.idle_polls = s->idle_polls;
    q.desc_polls = s->desc_polls;
    q.status = s->ctx->status;
    /* a new launch starts with no CTA idle and no yield pending (the last launch may have
     * left together on idle, setting yield from the device) */
    cudaMemsetAsync(&s->state->yield, 0, 2 * sizeof(int32_t), s->pub_stream);
    /* the published count and descriptors reach the device before the kernel starts */
    cudaEvent_t pub;
    cudaEventCreateWithFlags(&pub, cudaEventDisableTiming);
    cudaEventRecord(pub, s->pub_stream);
    cudaStreamWaitEvent(s->loop_stream, pub, 0);
    cudaEventDestroy(pub);
    const int err = launch_queue(s->mode, s->variant, q, s->blocks, s->loop_stream);
    count_launch(1);
    cudaEventRecord(s->loop_done, s->loop_stream);
    s->loop_launched = true;
    s->stats.loop_launches++;
    if (err != cudaSuccess) {
        set_error(s->ctx, "serving loop launch: %s", cudaGetErrorString((cudaError_t)err));
        s->broken = LT_ERR_CUDA;
    }
}

/* Requests still unfinished this long after lt_server_destroy began are failed. */
constexpr double kStopGraceS = 120.0;

void scheduler(lt_server *s)
{
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lock(s->mu);
    Clock::time_point stop_seen{};
    for (;;) {
        if (s->stopping && s->pending.empty() && s->inflight == 0) break;
        if (s->stopping) {
            if (stop_seen == Clock::time_point{}) stop_seen = Clock::now();
            if (std::chrono::duration<double>(Clock::now() - stop_seen).count() > kStopGraceS) {
                set_error(s->ctx, "server stopped with unfinished requests");
                for (SrvReq *r : s->ring)
                    if (r) finish(s, r, LT_ERR_TIMEOUT);
                while (!s->pending.empty()) {
                    finish(s, s->pending.front(), LT_ERR_TIMEOUT);
                    s->pending.pop_front();
                }
                s->cv_done.notify_all();
                break;
            }
        }
        const bool done = collect(s);
        if (s->broken == LT_OK) admit(s);
        if (s->broken == LT_OK) run_tails(s);
        if (s->broken == LT_OK) keep_loop(s);
        if (done) s->cv_done.notify_all();
        const bool busy = s->inflight > 0 || !s->pending.empty();
        s->cv_work.wait_for(lock, std::chrono::microseconds(busy ? 20 : 2000));
    }
}

} // namespace

extern "C" {

lt_status lt_server_create(lt_context *ctx, const lt_server_config *cfg, lt_server **out)
{
    if (!ctx || !out) return LT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    lt_server_config c{};
    if (cfg) c = *cfg;
    if (c.precision != LT_FP32C && c.precision != LT_FP64) {
        set_error(ctx, "the serving loop runs LT_FP32C or LT_FP64");
        return LT_ERR_INVALID_ARGUMENT;
    }
    if (c.slots < 0 || c.window < 0 || c.idle_us < 0 || c.descriptor_wait_us < 0) return LT_ERR_INVALID_ARGUMENT;
    lt_server *s = new (std::nothrow) lt_server();
    if (!s) return LT_ERR_OUT_OF_MEMORY;
    s->ctx = ctx;
    s->precision = c.precision;
    s->mode = c.precision == LT_FP32C ? QMODE_C32 : QMODE_EXACT;
    s->nslots = c.slots ? c.slots : 64;
    s->window = std::min(c.window ? c.window : 8, s->nslots);
    s->idle_polls = c.idle_us ? c.idle_us : 20000;
    s->desc_polls = c.descriptor_wait_us > 0 ? c.descriptor_wait_us : 2000000;
    const size_t arena_bytes = c.output_bytes ? c.output_bytes : ((size_t)4 << 30);
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    s->dev_bytes = sizeof(QState) + sizeof(QSlot) * (size_t)s->nslots;
    void *mem = nullptr;
    lt_status st = dev_alloc(ctx, &mem, s->dev_bytes);
    if (st != LT_OK) {
        delete s;
        return st;
    }
    s->state = (QState *)mem;
    s->slots = (QSlot *)((char *)mem + sizeof(QState));
    st = dev_alloc(ctx, (void **)&s->arena_mem, arena_bytes);
    if (st != LT_OK) {
        dev_free(ctx, mem, s->dev_bytes);
        delete s;
        return st;
    }
    s->arena.reset(arena_bytes);
    s->arena_bytes = arena_bytes;
    cudaError_t e = cudaMemset(mem, 0, s->dev_bytes);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_slots, sizeof(QSlot) * (size_t)s->nslots, 0);
    if (e == cudaSuccess)
        e = cudaHostAlloc((void **)&s->h_pub, sizeof(unsigned long long) * (size_t)s->nslots, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_status, 16 + sizeof(QState), 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_chi, 2 * sizeof(double) * (size_t)s->nslots, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_yield, 2 * sizeof(int32_t), 0);
    if (e == cudaSuccess)
        e = cudaHostAlloc((void **)&s->h_flags, sizeof(uint32_t) * (size_t)s->nslots, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&s->d_flags, s->h_flags, 0);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->loop_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->pub_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->loop_done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (s->h_slots) cudaFreeHost(s->h_slots);
        if (s->h_pub) cudaFreeHost(s->h_pub);
        if (s->h_status) cudaFreeHost(s->h_status);
        if (s->h_chi) cudaFreeHost(s->h_chi);
        if (s->h_yield) cudaFreeHost(s->h_yield);
        if (s->h_flags) cudaFreeHost(s->h_flags);
        dev_free(ctx, s->arena_mem, arena_bytes);
        dev_free(ctx, mem, s->dev_bytes);
        delete s;
        return cuda_fail(ctx, e, "server setup");
    }
    /* every slot starts out showing request seq 2^32 - 1 (an "earlier" request for the
     * first ones), so a slot whose descriptor has not arrived never reads as request 0 */
    memset(s->h_slots, 0, sizeof(QSlot) * (size_t)s->nslots);
    for (int i = 0; i < s->nslots; i++) {
        s->h_slots[i].item.seq = 0xffffffffu;
        s->h_slots[i].ctr = 0xffffffffull << 32;
    }
    e = cudaMemcpy(s->slots, s->h_slots, sizeof(QSlot) * (size_t)s->nslots, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        /* the same clean-up as above, after which every buffer is allocated */
        cudaFreeHost(s->h_slots);
        cudaFreeHost(s->h_pub);
        cudaFreeHost(s->h_status);
        cudaFreeHost(s->h_chi);
        cudaFreeHost(s->h_yield);
        cudaFreeHost(s->h_flags);
        cudaStreamDestroy(s->loop_stream);
        cudaStreamDestroy(s->pub_stream);
        cudaStreamDestroy(s->copy_stream);
        cudaEventDestroy(s->loop_done);
        dev_free(ctx, s->arena_mem, arena_bytes);
        dev_free(ctx, mem, s->dev_bytes);
        delete s;
        return cuda_fail(ctx, e, "server setup");
    }
    memset(s->h_flags, 0, sizeof(uint32_t) * (size_t)s->nslots);
    memset(s->h_chi, 0, 2 * sizeof(double) * (size_t)s->nslots);
    s->h_yield[0] = 1;
    s->h_yield[1] = 0;
    s->ring.assign((size_t)s->nslots, nullptr);
    s->variant = queue_variant(ctx->shape[LT_FP32C][OP_HESS]);
    s->blocks = queue_blocks(s->mode, s->variant, ctx->num_sms);
    {
        Extensions *x = ext_of(ctx);
        std::lock_guard<std::mutex> xl(x->mu);
        x->servers++;
    }
    s->thr = std::thread(scheduler, s);
    *out = s;
    return LT_OK;
}

lt_status lt_server_submit(lt_server *s, const lt_request *req, uint64_t *ticket)
{
    if (!s || !req || !ticket) return LT_ERR_INVALID_ARGUMENT;
    *ticket = 0;
    SrvReq *r = new (std::nothrow) SrvReq();
    if (!r) return LT_ERR_OUT_OF_MEMORY;
    r->req = *req;
    r->t_submit = Clock::now();
    /* validate now (errors are the caller's), with placeholder planes for host outputs */
    bool host = false;
    for (int i = 0; i < req->nmaps && i < LT_MAX_MAPS; i++)
        if (req->maps[i].out && !is_device_pointer(req->maps[i].out)) host = true;
    double *probe[LT_MAX_MAPS];
    for (int i = 0; i < LT_MAX_MAPS; i++) probe[i] = (double *)s->arena_mem;
    QItem tmp;
    lt_status st = make_queue_item(s->ctx, req, s->precision, host ? probe : nullptr, &tmp, shape_ppt(s->variant));
    if (st == LT_OK && host)
        for (int i = 0; i < req->nmaps; i++)
            if (!req->maps[i].out) st = LT_ERR_INVALID_ARGUMENT;
    if (st != LT_OK) {
        delete r;
        return st;
    }
    r->host_out = host;
    r->plane = Arena::round((size_t)req->grid.nx * req->grid.ny * sizeof(double));
    if (host && r->plane * (size_t)req->nmaps > s->arena.size()) {
        set_error(s->ctx, "request needs %zu bytes of output planes; the server's arena holds %zu",
                  r->plane * (size_t)req->nmaps, s->arena.size());
        delete r;
        return LT_ERR_BUDGET;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->broken != LT_OK || s->stopping) {
        delete r;
        return s->broken != LT_OK ? s->broken : LT_ERR_INVALID_ARGUMENT;
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->pending.push_back(r);
    s->stats.submitted++;
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return LT_OK;
}

lt_status lt_server_submit_chi2(lt_server *s, const lt_catalog *cat, const lt_frame *frame, int32_t n,
                                const lt_image_systems *sys, uint64_t *ticket)
{
    if (!s || !cat || !frame || !ticket) return LT_ERR_INVALID_ARGUMENT;
    *ticket = 0;
    lt_context *ctx = s->ctx;
    if (!(n >= 2 && std::isfinite(frame->xmin) && std::isfinite(frame->xmax) && std::isfinite(frame->ymin) &&
          std::isfinite(frame->ymax) && frame->xmax > frame->xmin && frame->ymax > frame->ymin &&
          (long)n * n <= (1L << 31))) {
        set_error(ctx, "chi2 request: invalid frame or grid size");
        return LT_ERR_INVALID_ARGUMENT;
    }
    lt_status st = check_systems(ctx, sys);
    if (st != LT_OK) return st;
    if ((size_t)24 * sys->nsystems > 48 * 1024) {
        set_error(ctx, "chi2 request: at most %d systems", 48 * 1024 / 24);
        return LT_ERR_INVALID_ARGUMENT;
    }
    SrvReq *r = new (std::nothrow) SrvReq();
    if (!r) return LT_ERR_OUT_OF_MEMORY;
    r->kind = K_CHI2;
    r->t_submit = Clock::now();
    r->frame = *frame;
    r->n = n;
    r->nimg.assign(sys->nimages, sys->nimages + sys->nsystems);
    r->first.resize((size_t)sys->nsystems);
    int total = 0;
    for (int i = 0; i < sys->nsystems; i++) {
        r->first[i] = total;
        total += sys->nimages[i];
    }
    r->ix.assign(sys->x, sys->x + total);
    r->iy.assign(sys->y, sys->y + total);
    r->dr.assign(sys->dlsds, sys->dlsds + sys->nsystems);
    r->chi_bytes = chi2_layout(sys->nsystems, total, frame, n, nullptr, r->dev);
    /* the deflection grid of the chi2, served by the loop like a map request */
    lt_request &g = r->req;
    memset(&g, 0, sizeof(g));
    g.cat = cat;
    g.dlsds = 1.0;
    g.mult = 1.0;
    g.scale = 1.0;
    g.nmaps = 2;
    g.maps[0].kind = LT_MAP_DEFLECTION_X;
    g.maps[1].kind = LT_MAP_DEFLECTION_Y;
    g.grid = {frame->xmin, frame->ymin, (frame->xmax - frame->xmin) / (n - 1), (frame->ymax - frame->ymin) / (n - 1),
              n, n, 0, 0};
    double *probe[LT_MAX_MAPS];
    for (int i = 0; i < LT_MAX_MAPS; i++) probe[i] = (double *)s->arena_mem;
    QItem tmp;
    st = make_queue_item(ctx, &g, s->precision, probe, &tmp, shape_ppt(s->variant));
    if (st == LT_OK && r->chi_bytes > s->arena.size()) {
        set_error(ctx, "chi2 request needs %zu bytes; the server's arena holds %zu", r->chi_bytes, s->arena.size());
        st = LT_ERR_BUDGET;
    }
    if (st != LT_OK) {
        delete r;
        return st;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->broken != LT_OK || s->stopping) {
        delete r;
        return s->broken != LT_OK ? s->broken : LT_ERR_INVALID_ARGUMENT;
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->pending.push_back(r);
    s->stats.submitted++;
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return LT_OK;
}

lt_status lt_server_chi2_result(lt_server *s, uint64_t ticket, double *chi2, int32_t *images_found)
{
    if (!s || !chi2) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || it->second->kind != K_CHI2) return LT_ERR_INVALID_ARGUMENT;
    const SrvReq *r = it->second;
    if (r->state == R_FAILED) return r->status;
    if (r->state != R_DONE) return LT_ERR_NOT_READY;
    *chi2 = r->chi2;
    if (images_found) *images_found = r->found;
    if (r->overflow) {
        set_error(s->ctx, "a source had more than %d predicted images (the first %d were used)", LT_MAX_IMAGES,
                  LT_MAX_IMAGES);
        return LT_ERR_QUEUE_FULL;
    }
    return LT_OK;
}

lt_status lt_server_poll(lt_server *s, uint64_t ticket)
{
    if (!s) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return LT_ERR_INVALID_ARGUMENT;
    const SrvReq *r = it->second;
    if (r->state == R_DONE) return LT_OK;
    if (r->state == R_FAILED) return r->status;
    return LT_ERR_NOT_READY;
}

lt_status lt_server_wait(lt_server *s, uint64_t ticket, double timeout_s)
{
    if (!s) return LT_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return LT_ERR_INVALID_ARGUMENT;
    SrvReq *r = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0));
    while (r->state != R_DONE && r->state != R_FAILED) {
        if (s->cv_done.wait_until(lock, until) == std::cv_status::timeout && r->state != R_DONE &&
            r->state != R_FAILED)
            return LT_ERR_NOT_READY;
    }
    return r->state == R_DONE ? LT_OK : r->status;
}

lt_status lt_server_request_times(lt_server *s, uint64_t ticket, double *queued_ms, double *gpu_ms,
                                  double *total_ms)
{
    if (!s) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return LT_ERR_INVALID_ARGUMENT;
    const SrvReq *r = it->second;
    if (r->state != R_DONE) return r->state == R_FAILED ? r->status : LT_ERR_NOT_READY;
    if (queued_ms) *queued_ms = ms_between(r->t_submit, r->t_admit);
    if (gpu_ms) *gpu_ms = ms_between(r->t_admit, r->t_gpu);
    if (total_ms) *total_ms = ms_between(r->t_submit, r->t_done);
    return LT_OK;
}

lt_status lt_server_release(lt_server *s, uint64_t ticket)
{
    if (!s) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return LT_ERR_INVALID_ARGUMENT;
    SrvReq *r = it->second;
    if (r->state != R_DONE && r->state != R_FAILED) return LT_ERR_NOT_READY;
    if (r->copied) cudaEventDestroy(r->copied);
    delete r;
    s->reqs.erase(it);
    return LT_OK;
}

lt_status lt_server_get_stats(lt_server *s, lt_server_stats *out)
{
    if (!s || !out) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->arena_bytes = s->arena.size();
    out->arena_peak = s->arena.peak();
    out->inflight = s->inflight;
    out->queued = (int32_t)s->pending.size();
    out->loop_running = s->loop_launched && cudaEventQuery(s->loop_done) == cudaErrorNotReady;
    /* the device's view of the queue (a copy on the publish stream, after every
     * publication issued so far) */
    QState *hq = (QState *)((char *)s->h_status + 16);
    cudaMemcpyAsync(hq, s->state, sizeof(QState), cudaMemcpyDeviceToHost, s->pub_stream);
    if (cudaStreamSynchronize(s->pub_stream) == cudaSuccess) {
        out->device_published = hq->published;
        out->device_head = hq->head;
    }
    return LT_OK;
}

lt_status lt_server_inject_fault(lt_server *s, int32_t fault)
{
    if (!s || fault != LT_FAULT_DROP_DESCRIPTOR) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    s->drop_next = true;
    return LT_OK;
}

lt_status lt_server_destroy(lt_server *s)
{
    if (!s) return LT_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->cv_work.notify_one();
    }
    s->thr.join(); /* every submitted request has completed or failed */
    lt_context *ctx = s->ctx;
    cudaSetDevice(ctx->device);
    int32_t one = 1;
    cudaMemcpyAsync(&s->state->stop, &one, sizeof(one), cudaMemcpyHostToDevice, s->pub_stream);
    cudaStreamSynchronize(s->pub_stream);
    if (s->loop_launched) cudaEventSynchronize(s->loop_done);
    cudaStreamSynchronize(s->copy_stream);
    for (auto &kv : s->reqs) {
        if (kv.second->copied) cudaEventDestroy(kv.second->copied);
        delete kv.second;
    }
    cudaEventDestroy(s->loop_done);
    cudaStreamDestroy(s->loop_stream);
    cudaStreamDestroy(s->pub_stream);
    cudaStreamDestroy(s->copy_stream);
    cudaFreeHost(s->h_slots);
    cudaFreeHost(s->h_pub);
    cudaFreeHost(s->h_status);
    cudaFreeHost(s->h_chi);
    cudaFreeHost(s->h_yield);
    cudaFreeHost(s->h_flags);
    std::vector<lt_catalog *> deferred;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        dev_free(ctx, s->arena_mem, s->arena_bytes);
        dev_free(ctx, s->state, s->dev_bytes);
        Extensions *x = ext_of(ctx);
        std::lock_guard<std::mutex> xl(x->mu);
        if (--x->servers == 0) deferred.swap(x->deferred);
    }
    for (lt_catalog *c : deferred) free_catalog(ctx, c);
    delete s;
    return LT_OK;
}

} /* extern "C" */
