/*
 * lt_queue.cu -- the work-queue kernel: many (catalogue, grid) requests evaluated by one
 * persistent launch.  It serves two entry points:
 *   - batches (lt_batch_*): a fixed list of requests, run as a CUDA graph of two nodes
 *     (queue reset + the persistent kernel) that the caller replays;
 *   - the serving loop (lt_server_*): requests submitted at any time are admitted into a
 *     ring of device slots while earlier ones are still on the GPU (continuous batching).
 *
 * Device side
 *   - A request occupies one slot of a ring: its descriptor (QItem), a claim word
 *     ctr = (seq << 32) | next_tile and a completion counter.  The reference evaluates
 *     one map per call and synchronises (utils/maps/main.cpp:432-587 calling
 *     map_grid_ampli_GPU, src/grid_map_ampli_GPU.cu:93-192); here the unit of work is a
 *     (request, pixel tile) pair and the tiles of every admitted request share the GPU.
 *   - Thread 0 of each CTA claims a tile by compare-and-swap on ctr, round-robin over the
 *     `window` oldest requests (processor sharing: a small request admitted behind a
 *     large one does not wait for all of it).  A CAS only succeeds while the slot still
 *     holds request `seq` with tiles left, so a slot is never claimed from while it is
 *     being rewritten for a later request.
 *   - The tile is evaluated with the same per-chunk pair loops as the single-grid
 *     kernels (lt_eval.cuh), halo chunks staged into shared memory by cp.async.bulk.
 *     FP32C tiles recompute in FP64, inside the tile, the pixels whose FP32 error bound
 *     on mu exceeds the tolerance, so a request needs no second pass and no pixel list.
 *   - The CTA that completes the last tile of a request publishes the completion: for
 *     the serving loop a word in mapped host memory set to seq + 1.
 *   - Idle CTAs poll for new requests with __nanosleep for a bounded number of polls and
 *     then leave; the host relaunches the loop when new work arrives.  Every mbarrier wait
 *     is bounded (lt_bulk.cuh).
 *   - Descriptors and claim words are read with ld.global.cg (L2), never through L1,
 *     because the host rewrites slots while the kernel runs.
 */
#include <algorithm>
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

#include "lt_eval.cuh"
#include "lt_internal.h"
#include "lt_queue.h"

namespace lt {

constexpr int kQThreads = 256;

/* ------------------------------------------------------------------ device ---- */

__device__ __forceinline__ lt_chunk ldcg_chunk(const lt_chunk *p)
{
    const int4 v = __ldcg(reinterpret_cast<const int4 *>(p));
    lt_chunk c;
    c.start = v.x;
    c.count = v.y;
    c.type = v.z;
    c.pad = v.w;
    return c;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

/* Double-buffered staging of halo chunks into shared memory (see lt_bulk.cuh). */
struct Stage {
    unsigned char *buf[2];
    uint64_t *bar;
    uint32_t phase[2];
    int next;
};

/* Walk `n` chunks of `chunks`: chunk i + 1 is copied while chunk i is evaluated by
 * fn(chunk, staged records).  Every thread of the block calls it; it returns false
 * (block-uniformly) when a bounded wait gave up. */
template <class Fn>
__device__ __forceinline__ bool walk_chunks(Stage &st, const lt_chunk *chunks, int n, const lt_rec64 *r64,
                                            const lt_rec32 *r32, int32_t *status, Fn &&fn)
{
    if (n <= 0) return true;
    auto issue = [&](int i, int b) {
        const lt_chunk c = ldcg_chunk(chunks + i);
        const void *src;
        uint32_t bytes;
        if (c.pad & CHUNK_FP32) {
            src = r32 + c.start;
            bytes = (uint32_t)c.count * (uint32_t)sizeof(lt_rec32);
        } else {
            src = r64 + c.start;
            bytes = (uint32_t)c.count * (uint32_t)sizeof(lt_rec64);
        }
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&st.bar[b], bytes);
        bulk_g2s(st.buf[b], src, bytes, &st.bar[b]);
    };
    int b = st.next;
    if (threadIdx.x == 0) issue(0, b);
    for (int i = 0; i < n; i++) {
        if (threadIdx.x == 0 && i + 1 < n) issue(i + 1, b ^ 1);
        if (!wait_tile(&st.bar[b], st.phase[b], status)) {
            if (threadIdx.x == 0 && i + 1 < n) drain_tile(&st.bar[b ^ 1], st.phase[b ^ 1]);
            return false;
        }
        st.phase[b] ^= 1;
        fn(ldcg_chunk(chunks + i), st.buf[b]);
        __syncthreads(); /* buffer b is refilled by the copy issued in the next iteration */
        b ^= 1;
    }
    st.next = b;
    return true;
}

__device__ __forceinline__ bool is_grad_kind(int k) { return k == KIND_GRAD_X || k == KIND_GRAD_Y; }

/* Pixel of this thread in tile `tile` (same layout as the single-grid kernels). */
template <int P>
__device__ __forceinline__ void tile_pixel(const GridArgs &a, int tile, int &ix, int &iy)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ox = (warp & 3) * (8 * P) + (lane & 7) * P;
    const int oy = (warp >> 2) * 4 + (lane >> 3);
    const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    ix = tx * 32 * P + ox;
    iy = ty * 8 + oy;
}

/* FP64 sums of one tile (grid64_kernel's per-tile work): deflection, the reference-order
 * Hessian (OP_HEX) or the fast one (OP_HESS), potential.  Writes the output planes of
 * the deflection kinds when OP is OP_GRAD, the others otherwise. */
template <int OP, int P>
__device__ __noinline__ bool tile64(const QItem &it, int tile, Stage &st, int32_t *status)
{
    const GridArgs &a = it.g;
    int ix, iy;
    tile_pixel<P>(a, tile, ix, iy);
    const double py = pixel_y(a, iy < a.ny ? iy : a.ny - 1);
    double px[P];
    Acc64<OP, P> acc;
#pragma unroll
    for (int k = 0; k < P; k++) {
        px[k] = pixel_x(a, (ix + k) < a.nx ? ix + k : a.nx - 1);
        acc.gx[k] = acc.gy[k] = acc.hxx[k] = acc.hyy[k] = acc.hxy[k] = acc.psi[k] = 0.;
        acc.run[k].a = acc.run[k].b = acc.run[k].c = acc.run[k].d = 0.;
        acc.tot[k].a = acc.tot[k].b = acc.tot[k].c = acc.tot[k].d = 0.;
    }
    const bool ok = walk_chunks(st, a.chunks, a.nchunks, a.recs, nullptr, status,
                                [&](const lt_chunk &c, const unsigned char *buf) {
                                    const lt_rec64 *recs = reinterpret_cast<const lt_rec64 *>(buf);
                                    switch (c.type) {
                                    case 81: eval_chunk64<OP, P, 81>(recs, c.count, px, py, a.kmap, acc); break;
                                    case 8: eval_chunk64<OP, P, 8>(recs, c.count, px, py, a.kmap, acc); break;
                                    case 5: eval_chunk64<OP, P, 5>(recs, c.count, px, py, a.kmap, acc); break;
                                    default: break;
                                    }
                                    if ((OP & OP_HEX) && (c.pad & CHUNK_RUN_END))
                                        close_run64<OP, P>(acc, a.kmap, recs[c.count - 1].w);
                                });
    if (!ok) return false;
    if (iy < a.ny) {
        const long row = (long)iy * a.nx;
        const bool full = a.vec_ok && (ix + P <= a.nx);
        if (OP & OP_HEX) {
#pragma unroll
            for (int k = 0; k < P; k++) {
                acc.hxx[k] = acc.tot[k].a;
                acc.hxy[k] = acc.tot[k].b;
                acc.hyy[k] = acc.tot[k].c;
            }
        }
        for (int o = 0; o < a.nout; o++) {
            const int kind = a.kinds[o];
            if (is_grad_kind(kind) != (OP == OP_GRAD)) continue;
            double v[P];
#pragma unroll
            for (int k = 0; k < P; k++)
                v[k] = map_value4(kind, acc.gx[k], acc.gy[k], acc.hxx[k], acc.hyy[k], acc.hxy[k],
                                  (OP & OP_HEX) ? acc.tot[k].d : acc.hxy[k], acc.psi[k], a.D, a.mult, a.scale);
            double *dst = a.out[o] + row + ix;
            if (P == 2 && full) {
                *reinterpret_cast<double2 *>(dst) = make_double2(v[0], v[1 % P]);
            } else {
#pragma unroll
                for (int k = 0; k < P; k++)
                    if (ix + k < a.nx) dst[k] = v[k];
            }
        }
    }
    return true;
}

/* FP32C (or, with an all-FP64 chunk list, fast FP64) Hessian/potential sums of one tile:
 * grid32c_kernel's per-tile work followed by the FP64 recomputation of the tile's
 * pixels whose FP32 error bound on mu exceeds mu_tol (the single-grid path's second pass,
 * same arithmetic). */
template <int OP, int P>
__device__ __noinline__ bool tile32(const QItem &it, int tile, Stage &st, int32_t *status, int16_t *s_list, int *s_count)
{
    const GridArgs &a = it.g;
    int ix, iy;
    tile_pixel<P>(a, tile, ix, iy);
    const double py = pixel_y(a, iy < a.ny ? iy : a.ny - 1);
    double px[P];
    Acc32<P> acc;
#pragma unroll
    for (int k = 0; k < P; k++) {
        px[k] = pixel_x(a, (ix + k) < a.nx ? ix + k : a.nx - 1);
        acc32_zero(acc, k);
    }
    bool ok = walk_chunks(st, it.chunks32, it.nchunks32, a.recs, it.recs32, status,
                          [&](const lt_chunk &c, const unsigned char *buf) {
                              if (c.pad & CHUNK_FP32) {
                                  const lt_rec32 *recs = reinterpret_cast<const lt_rec32 *>(buf);
                                  switch (c.type) {
                                  case 81:
                                      eval32_chunk<OP, P, 81>(recs, a.recs, c.count, px, py, a, ix, iy, acc);
                                      break;
                                  case 8:
                                      eval32_chunk<OP, P, 8>(recs, a.recs, c.count, px, py, a, ix, iy, acc);
                                      break;
                                  case 5:
                                      eval32_chunk<OP, P, 5>(recs, a.recs, c.count, px, py, a, ix, iy, acc);
                                      break;
                                  default: break;
                                  }
                              } else {
                                  const lt_rec64 *recs = reinterpret_cast<const lt_rec64 *>(buf);
                                  switch (c.type) {
                                  case 81: eval64_chunk<OP, P, 81>(recs, c.count, px, py, a.kmap, acc); break;
                                  case 8: eval64_chunk<OP, P, 8>(recs, c.count, px, py, a.kmap, acc); break;
                                  case 5: eval64_chunk<OP, P, 5>(recs, c.count, px, py, a.kmap, acc); break;
                                  default: break;
                                  }
                              }
                          });
    if (!ok) return false;
    const bool recompute = (OP & OP_HESS) && it.mu_tol > 0.;
    if (recompute && threadIdx.x == 0) *s_count = 0;
    if (recompute) __syncthreads();
    if (iy < a.ny) {
        const long row = (long)iy * a.nx;
        double hxx[P], hyy[P], hxy[P], psi[P], gx[P], gy[P];
        bool flag[P];
#pragma unroll
        for (int k = 0; k < P; k++) {
            double det, det_err;
            fp32c_total(acc, k, a.D, hxx[k], hyy[k], hxy[k], psi[k], det, det_err);
            fp32c_grad_total(acc, k, gx[k], gy[k]);
            flag[k] = recompute && fp32c_flag(det, det_err, it.mu_tol);
        }
        const bool full = a.vec_ok && (ix + P <= a.nx);
        for (int o = 0; o < a.nout; o++) {
            const int kind = a.kinds[o];
            if (is_grad_kind(kind) != (OP == OP_GRAD)) continue;
            double v[P];
#pragma unroll
            for (int k = 0; k < P; k++)
                v[k] = map_value(kind, gx[k], gy[k], hxx[k], hyy[k], hxy[k], psi[k], a.D, a.mult, a.scale);
            double *dst = a.out[o] + row + ix;
            if (P == 2 && full) {
                *reinterpret_cast<double2 *>(dst) = make_double2(v[0], v[1 % P]);
            } else {
#pragma unroll
                for (int k = 0; k < P; k++)
                    if (ix + k < a.nx) dst[k] = v[k];
            }
        }
        if (recompute) {
            const int tile_x0 = (tile % a.tiles_x) * 32 * P, tile_y0 = (tile / a.tiles_x) * 8;
#pragma unroll
            for (int k = 0; k < P; k++)
                if (flag[k] && ix + k < a.nx) {
                    const int slot = atomicAdd(s_count, 1);
                    s_list[slot] = (int16_t)((iy - tile_y0) * 32 * P + (ix + k - tile_x0));
                }
        }
    }
    if (!recompute) return true;
    __syncthreads();
    /* the flagged pixels (at most the tile's 32 P x 8 = P kQThreads), in one walk of the
     * catalogue's FP64 closed-form records: thread t takes entries t and t + kQThreads; a warp
     * with no second entry evaluates one pixel a thread (an empty second pixel would double
     * its work) */
    const int n = *s_count;
    const int tile_x0 = (tile % a.tiles_x) * 32 * P, tile_y0 = (tile / a.tiles_x) * 8;
    if (n == 0) return true;
    /* the count of recomputed pixels (lt_recompute_count): word 2 of the status block */
    if (threadIdx.x == 0 && status)
        atomicAdd(reinterpret_cast<unsigned long long *>(status + 2), (unsigned long long)n);
    bool have[P];
    int qx[P], qy[P];
    double qpx[P], qpy[P], kap[P], g1[P], g2[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
        const int e = k * kQThreads + (int)threadIdx.x;
        have[k] = e < n;
        const int l = have[k] ? s_list[e] : 0;
        qx[k] = tile_x0 + l % (32 * P);
        qy[k] = tile_y0 + l / (32 * P);
        qpx[k] = pixel_x(a, qx[k]);
        qpy[k] = pixel_y(a, qy[k]);
        kap[k] = g1[k] = g2[k] = 0.;
    }
    const bool one = !__any_sync(0xffffffffu, P == 2 && have[P - 1]); /* warp-uniform */
    double px1[1] = {qpx[0]}, py1[1] = {qpy[0]}, kap1[1] = {0.}, g11[1] = {0.}, g21[1] = {0.};
    const bool ok2 = walk_chunks(st, a.chunks, a.nchunks, reinterpret_cast<const lt_rec64 *>(it.nie64), nullptr,
                                 status, [&](const lt_chunk &c, const unsigned char *buf) {
                                     if (!have[0]) return;
                                     const lt_nie64 *recs = reinterpret_cast<const lt_nie64 *>(buf);
                                     if (one)
                                         eval_nie_chunk<1>(c, recs, px1, py1, a.kmap, kap1, g11, g21);
                                     else
                                         eval_nie_chunk<P>(c, recs, qpx, qpy, a.kmap, kap, g1, g2);
                                 });
    if (!ok2) return false;
    if (one) {
        kap[0] = kap1[0];
        g1[0] = g11[0];
        g2[0] = g21[0];
    }
#pragma unroll
    for (int k = 0; k < P; k++) {
        if (!have[k]) continue;
        const long p = (long)qy[k] * a.nx + qx[k];
        double hxx, hyy, hxy;
        nie_hessian(kap[k], g1[k], g2[k], hxx, hyy, hxy);
        for (int o = 0; o < a.nout; o++) {
            const int kind = a.kinds[o];
            if (is_grad_kind(kind) || kind == KIND_POT) continue;
            a.out[o][p] = map_value(kind, 0., 0., hxx, hyy, hxy, 0., a.D, a.mult, a.scale);
        }
    }
    return true;
}

/* Claim one tile (thread 0).  Returns 1 with (slot, tile) set, 0 when no published
 * request has tiles left, 2 when none has and the oldest published request's descriptor
 * has not arrived (its seq in *missing).  Every attempt either claims a tile or finds the
 * head request exhausted and moves the head on (here or in another CTA), so the attempts
 * are bounded by the published requests; the limit below is only a safety net. */
__device__ int claim_tile(const QArgs &q, int &slot_out, int &tile_out, uint32_t *missing)
{
    QState *st = q.state;
    for (int attempt = 0; attempt < (1 << 20); attempt++) {
        const unsigned long long h = ld_acquire_u64(&st->head);
        const unsigned long long p = ld_acquire_u64(&st->published);
        if (h >= p) return 0;
        unsigned long long span = p - h;
        if (span > (unsigned long long)q.window) span = (unsigned long long)q.window;
        const unsigned long long r0 = atomicAdd(&st->rotor, 1ull);
        bool head_exhausted = false, head_missing = false;
        for (unsigned long long k = 0; k < span; k++) {
            const unsigned long long r = h + (r0 + k) % span;
            QSlot *s = q.slots + (r % (unsigned long long)q.nslots);
            unsigned long long c = __ldcg(&s->ctr);
            const int nt = __ldcg(&s->item.ntiles);
            const uint32_t seq = (uint32_t)__ldcg(reinterpret_cast<const int *>(&s->item.seq));
            while ((uint32_t)(c >> 32) == (uint32_t)r && seq == (uint32_t)r && (int)(c & 0xffffffffu) < nt) {
                const unsigned long long prev = atomicCAS(&s->ctr, c, c + 1ull);
                if (prev == c) {
                    slot_out = (int)(r % (unsigned long long)q.nslots);
                    tile_out = (int)(c & 0xffffffffu);
                    return 1;
                }
                c = prev;
            }
            /* exhausted: the slot shows request r with every tile claimed, or a later
             * request (r has completed).  A slot still showing an earlier request has
             * not received r's descriptor yet: r is not exhausted. */
            const int32_t age = (int32_t)((uint32_t)(c >> 32) - (uint32_t)r);
            if (r == h && age >= 0) head_exhausted = true;
            if (r == h && (age < 0 || seq != (uint32_t)r)) head_missing = true;
        }
        /* the head request has no tiles left (or its slot already holds a later
         * request): move the head on */
        if (head_exhausted) {
            atomicCAS(&st->head, h, h + 1ull);
        } else if (head_missing) {
            *missing = (uint32_t)h;
            return 2;
        }
    }
    return 0;
}

template <int MODE, int P32, int MINB>
__global__ void __launch_bounds__(kQThreads, MINB) queue_kernel(const QArgs q)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ __align__(16) QItem item;
    __shared__ int s_slot, s_tile, s_count;
    __shared__ int16_t s_list[kQThreads * 2];
    const int tid = threadIdx.x;
    Stage st;
    st.buf[0] = smem;
    st.buf[1] = smem + LT_CHUNK * sizeof(lt_rec64);
    st.bar = bars;
    st.phase[0] = st.phase[1] = 0;
    st.next = 0;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    for (;;) {
        if (tid == 0) {
            int slot = -1, tile = 0;
            bool counted = false; /* this CTA is in QState::idle */
            int missing_polls = 0;
            for (int polls = 0;; polls++) {
                if (*(volatile int32_t *)&q.state->yield) break;
                uint32_t missing = 0;
                const int got = claim_tile(q, slot, tile, &missing);
                if (got == 1) {
                    if (counted) atomicSub(&q.state->idle, 1);
                    break;
                }
                slot = -1;
                /* a published request whose descriptor does not arrive: a bounded wait (not
                 * an idle poll: the launch does not leave on idle meanwhile), then the
                 * request is reported (its seq + 1 in QState::stuck, the status word
                 * LT_ERR_TIMEOUT) and the launch leaves */
                if (got == 2) {
                    if (++missing_polls > q.desc_polls) {
                        atomicExch(&q.state->stuck, missing + 1u);
                        if (q.status) atomicExch(q.status, (int32_t)LT_ERR_TIMEOUT);
                        atomicExch(&q.state->yield, 1);
                        break;
                    }
                    __nanosleep(1000);
                    continue;
                }
                missing_polls = 0;
                if (*(volatile int32_t *)&q.state->stop) break;
                if (!counted) {
                    atomicAdd(&q.state->idle, 1);
                    counted = true;
                }
                /* leave on idle only together: a CTA that left alone would leave work that
                 * arrives later to fewer CTAs until the whole launch ends */
                if (polls >= q.idle_polls && *(volatile int32_t *)&q.state->idle >= (int32_t)gridDim.x) {
                    atomicExch(&q.state->yield, 1);
                    break;
                }
                __nanosleep(1000);
            }
            s_slot = slot;
            s_tile = tile;
        }
        __syncthreads();
        const int slot = s_slot, tile = s_tile;
        if (slot < 0) break;
        {
            const int4 *src = reinterpret_cast<const int4 *>(&q.slots[slot].item);
            int4 *dst = reinterpret_cast<int4 *>(&item);
            for (int i = tid; i < (int)(sizeof(QItem) / 16); i += kQThreads) dst[i] = __ldcg(src + i);
        }
        __syncthreads();
        bool ok = true;
        const int hp = item.op & (OP_HESS | OP_POT);
        if (MODE == QMODE_C32) {
            if (item.op & OP_GRAD) ok = tile32<OP_GRAD, P32>(item, tile, st, q.status, s_list, &s_count);
            if (ok && hp == OP_HESS) ok = tile32<OP_HESS, P32>(item, tile, st, q.status, s_list, &s_count);
            if (ok && hp == OP_POT) ok = tile32<OP_POT, P32>(item, tile, st, q.status, s_list, &s_count);
            if (ok && hp == (OP_HESS | OP_POT))
                ok = tile32<OP_HESS | OP_POT, P32>(item, tile, st, q.status, s_list, &s_count);
        } else if (item.ppt == 2) { /* requests without the potential */
            if (item.op & OP_GRAD) ok = tile64<OP_GRAD, 2>(item, tile, st, q.status);
            if (ok && hp == OP_HESS) ok = tile64<OP_HEX, 2>(item, tile, st, q.status);
        } else {
            if (item.op & OP_GRAD) ok = tile64<OP_GRAD, 1>(item, tile, st, q.status);
            if (ok && hp == OP_HESS) ok = tile64<OP_HEX, 1>(item, tile, st, q.status);
            if (ok && hp == OP_POT) ok = tile64<OP_POT | OP_PEX, 1>(item, tile, st, q.status);
            if (ok && hp == (OP_HESS | OP_POT))
                ok = tile64<OP_HEX | OP_POT | OP_PEX, 1>(item, tile, st, q.status);
        }
        __syncthreads();
        if (!ok) break; /* a bounded wait gave up; the status word says so */
        if (tid == 0) {
            __threadfence(); /* this CTA's output stores before its completion count */
            const unsigned int d = atomicAdd(&q.slots[slot].done, 1u) + 1u;
            if (d == (unsigned int)item.ntiles && item.host_flag) {
                __threadfence_system();
                *(volatile uint32_t *)item.host_flag = item.seq + 1u;
            }
        }
    }
}

/* Batch reset: every request published, claim words and counters zeroed, stop set so
 * that the persistent kernel leaves when the queue is drained. */
__global__ void queue_reset_kernel(QSlot *slots, QState *state, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        slots[i].ctr = (unsigned long long)(uint32_t)i << 32;
        slots[i].done = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        state->published = (unsigned long long)n;
        state->head = 0ull;
        state->rotor = 0ull;
        state->stop = 1;
        state->yield = 0;
        state->idle = 0;
    }
}

/* ------------------------------------------------------------------- host ---- */

using QKern = void (*)(const QArgs);

static QKern queue_kernel_for(int mode, int variant)
{
    if (mode != QMODE_C32) return queue_kernel<QMODE_EXACT, 2, 2>;
    switch (variant) {
    case LT_SHAPE(1, 1): return queue_kernel<QMODE_C32, 1, 1>;
    case LT_SHAPE(1, 2): return queue_kernel<QMODE_C32, 1, 2>;
    case LT_SHAPE(2, 1): return queue_kernel<QMODE_C32, 2, 1>;
    default: return queue_kernel<QMODE_C32, 2, 2>;
    }
}

/* The built variant nearest to an FP32C grid-kernel shape: its pixels per thread, and its
 * resident threads per SM rounded to 256 or 512. */
int queue_variant(int shape32)
{
    const int ppt = shape_ppt(shape32) == 1 ? 1 : 2;
    const int threads = shape_cps(shape32) * shape_threads(shape32);
    return LT_SHAPE(ppt, threads > 384 ? 2 : 1);
}

int queue_blocks(int mode, int variant, int num_sms)
{
    const size_t smem = 2 * LT_CHUNK * sizeof(lt_rec64);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, queue_kernel_for(mode, variant), kQThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

int launch_queue(int mode, int variant, const QArgs &q, int blocks, cudaStream_t s)
{
    const size_t smem = 2 * LT_CHUNK * sizeof(lt_rec64);
    queue_kernel_for(mode, variant)<<<blocks, kQThreads, smem, s>>>(q);
    return (int)cudaGetLastError();
}

int launch_queue_reset(QSlot *slots, QState *state, int n, cudaStream_t s)
{
    int blocks = (n + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 1024) blocks = 1024;
    queue_reset_kernel<<<blocks, 256, 0, s>>>(slots, state, n);
    return (int)cudaGetLastError();
}

} // namespace lt
