/*
 * lt_grid.cuh -- launch arguments shared by the grid kernels and the host launchers.
 */
#pragma once
#include <stdint.h>
#include "lt_halo.h"
#include "../../include/lt_b200.h"

namespace lt {

/* internal output kinds besides lt_map_kind */
enum {
    KIND_GRAD_X = 100, /* deflection x * scale */
    KIND_GRAD_Y = 101, /* deflection y * scale */
    KIND_POT = 102     /* potential * scale */
};

/* which sums a kernel evaluates; OP_HEX is the Hessian with the reference's rounding
 * sequence (LT_FP64), OP_HESS the reformulated one (LT_FP64_FAST and the FP32C path);
 * OP_PEX with OP_POT takes the potential through the reference's pi05 formula (LT_FP64),
 * OP_POT alone through the deflection (LT_FP64_FAST, FP32C's FP64 halos); OP_GFX with
 * OP_GRAD takes the dPIE deflection as log(1 + eps) (LT_FP64_FAST; FP32C's FP64 terms
 * always do), OP_GRAD alone in the reference's two-logarithm form (LT_FP64, the queue's
 * exact tiles, the chi2 points); OP_NI with OP_HESS takes the Hessian from the FP64
 * closed-form records lt_nie64 (nie_kg64: the FP32C path's FP64 recomputation) */
enum { OP_GRAD = 1, OP_HESS = 2, OP_POT = 4, OP_HEX = 8, OP_PEX = 16, OP_GFX = 32, OP_NI = 64 };

/* chunk.pad bits: FP32 records (FP32C list), last chunk of a run */
enum { CHUNK_FP32 = 1, CHUNK_RUN_END = 2 };

struct GridArgs {
    const lt_rec64 *recs;
    const lt_chunk *chunks;
    int32_t nchunks;
    int32_t kmap;
    double xmin, ymin, dx, dy;
    int32_t nx, ny, istart, jstart;
    int32_t tiles_x, ntiles;
    int32_t nout, vec_ok;
    int32_t kinds[LT_MAX_MAPS];
    double *out[LT_MAX_MAPS];
    double D, mult, scale;
    int32_t *status; /* device word: 0, or an lt_status set by a kernel */
    /* list mode: evaluate the pixels list[0 .. min(*list_count, list_cap)) */
    const int32_t *list;
    const int32_t *list_count;
    int32_t list_cap;
};

/* Kernel shape: pixels per thread (1 or 2), resident CTAs per SM the register budget is
 * cut for (1-4), threads per CTA (128 or 256) and halo records per shared-memory stage
 * (32, 64 or 128).  LT_SHAPE keeps 256 threads and 64-record stages. */
#define LT_SHAPE4(ppt, cps, nt, cap) ((ppt) | ((cps) << 4) | (((nt) / 32) << 8) | (((cap) / 32) << 16))
#define LT_SHAPE(ppt, cps) LT_SHAPE4(ppt, cps, 256, 64)

inline int shape_ppt(int s) { return s & 15; }
inline int shape_cps(int s) { return (s >> 4) & 15; }
inline int shape_threads(int s) { return ((s >> 8) & 255) * 32; }
inline int shape_cap(int s) { return ((s >> 16) & 15) * 32; }

/* Launch the FP64 grid kernel for the sums in `op` (OP_* mask).  Returns the CUDA error. */
int launch_grid64(int op, const GridArgs &args, int num_sms, void *stream, bool list_mode = false,
                  int shape = LT_SHAPE(2, 1));

} // namespace lt
