/*
 * lt_queue.h -- device layout of the work queue shared by the batch and serving entry
 * points (lt_batch.cpp, lt_server.cpp) and the persistent kernel (lt_queue.cu).
 */
#pragma once
#include <stdint.h>

#include <cuda_runtime.h>

#include "lt_grid.cuh"

struct lt_rec32;

namespace lt {

/* kernel modes: FP32C tiles (P = 2), or the LT_FP64 tiles with the reference-order
 * Hessian (P per request) */
enum { QMODE_C32 = 0, QMODE_EXACT = 1 };

/* One request: one grid of output planes over one catalogue. */
struct alignas(16) QItem {
    GridArgs g;                 /* FP64 records and chunk list (the Kmap list when kmap),
                                   geometry (tiles_x, ntiles for this request's P),
                                   outputs, D, mult, scale, status */
    const lt_rec32 *recs32;     /* FP32C records */
    const lt_chunk *chunks32;   /* FP32C chunk list (FP32 and FP64-class chunks) */
    int32_t nchunks32;
    int32_t op;                 /* OP_GRAD | OP_HESS | OP_POT */
    int32_t ntiles;
    uint32_t seq;               /* request sequence number (low 32 bits) */
    int32_t ppt;                /* pixels per thread of the tiles (QMODE_EXACT) */
    int32_t pad0;
    double mu_tol;              /* FP32C: recompute pixels whose FP32 error bound on mu exceeds
                                   this in FP64 (0: none) */
    uint32_t *host_flag;        /* mapped host word set to seq + 1 on completion, or null */
    const lt_nie64 *nie64;      /* FP32C: the closed-form FP64 records of the recomputation */
};
static_assert(sizeof(QItem) % 16 == 0, "QItem is copied in 16-byte units");

struct alignas(16) QSlot {
    QItem item;
    unsigned long long ctr;     /* (seq << 32) | next tile to claim */
    unsigned int done;          /* tiles completed */
    unsigned int pad;
};

struct alignas(16) QState {
    unsigned long long published; /* requests published (host-written) */
    unsigned long long head;       /* oldest request that may have unclaimed tiles */
    unsigned long long rotor;      /* round-robin counter over the window */
    int32_t stop;                  /* leave when no published request has work */
    int32_t yield;                 /* leave at the next claim; unclaimed tiles stay for the next launch */
    int32_t idle;                  /* CTAs of the running launch without work (or gone) */
    uint32_t stuck;                /* seq + 1 of a published request whose descriptor never came */
};

struct QArgs {
    QSlot *slots;
    QState *state;
    int32_t nslots;
    int32_t window;                /* requests served round-robin (1: first come, first served) */
    int32_t idle_polls;            /* polls of ~1 us before an idle CTA leaves */
    int32_t desc_polls;            /* polls of ~1 us a CTA waits for the descriptor of the oldest
                                      published request before reporting LT_ERR_TIMEOUT */
    int32_t *status;               /* device status word (LT_ERR_TIMEOUT from a bounded wait) */
};

/* Persistent-kernel variants: the FP32C tiles come with 1 or 2 pixels per thread and
 * registers cut for 1 or 2 resident CTAs per SM (256 threads); `variant` is their
 * LT_SHAPE(pixels, CTAs).  The LT_FP64 tiles have one variant (2 CTAs per SM). */
int queue_variant(int shape32);
int queue_blocks(int mode, int variant, int num_sms);
int launch_queue(int mode, int variant, const QArgs &q, int blocks, cudaStream_t s);
int launch_queue_reset(QSlot *slots, QState *state, int n, cudaStream_t s);

} // namespace lt
