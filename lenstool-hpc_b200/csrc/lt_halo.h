/*
 * lt_halo.h -- device layout of a packed halo catalogue (shared by host and device code).
 *
 * Each halo becomes one 256-byte record of per-halo invariants, so that the per-pair
 * work of the grid kernels starts from the pixel offset.  The invariants are the
 * sub-expressions the reference recomputes for every pixel (src/gradient.cpp:744-811,
 * src/gradient2.cpp:54-83, src/potential_GPU.cu:47-72), evaluated once with the same
 * formulas.  Records are 16-byte aligned so that tiles of them can be moved into shared
 * memory with cp.async.bulk.
 *
 * Meaning of the slots by profile type
 *   type 81 (cut dPIE) and 8 (PIEMD):
 *     sqe2 = 2 sqrt(eps), cx1 = (1-eps)/(1+eps), cx1inv = 1/cx1,
 *     cxro_inv = 1/(1+eps)^2, cyro_inv = 1/(1-eps)^2, k4 = 4 eps,
 *     ci = (1-eps^2)/(2 sqrt(eps)),
 *     pref_g = ci * b0 * rcut/(rcut - rc)  (81) | ci * b0  (8)      -- deflection
 *     pref_h = ci * b0 * rcut/(rcut - rc)  (81) | ci * b0  (8)      -- Hessian, potential
 *     rc2 = rc^2, rcut2 = rcut^2, tsr_c = 2 rc sqrt(eps), tsr_t = 2 rcut sqrt(eps),
 *     e1 = 2 sqrt(eps)/(1-eps), e2 = 2 sqrt(eps)/(1+eps),
 *     dr2 = rc^2 - rcut^2, drs = rc - rcut, om2 = (1-eps)^2, e4cxi = 4 eps/(1+eps)^2,
 *     ok3c = (1-eps)(3+eps) rc, ok3t = (1-eps)(3+eps) rcut, i4rc2 = 1/(4 rc^2),
 *     i4rcut2 = 1/(4 rcut^2)  (the deflection-based potential of lt_profiles64.cuh)
 *   type 5 (SIS): cx1 = 1-eps, cx1inv = 1+eps, pref_g = (1-eps) b0,
 *     pref_h = (1+eps) b0, ci = b0 (1-eps)(1+eps)
 *   all: w = dlsds (Kmap weight), type in `type`.
 */
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LT_HD __host__ __device__
#else
#define LT_HD
#endif

struct alignas(16) lt_rec64 {
    double x0, y0, cs, sn;
    double b0, eps, rc, rcut;
    double sqe2, cx1, cx1inv, cxro_inv;
    double cyro_inv, ci, pref_g, pref_h;
    double rc2, rcut2, tsr_c, tsr_t;
    double e1, e2, w, k4;
    double dr2, drs, om2, e4cxi;
    double ok3c, ok3t, i4rc2, i4rcut2;
};
static_assert(sizeof(lt_rec64) == 256, "record size");

/* The FP64 record of the closed-form Hessian (the real-valued forms of
 * lt_profiles32.cuh in FP64: q = (1-e)/(1+e), s = (1+e) r, K = b0 (1-e) t05 / 2), used by
 * the FP32C path's FP64 recomputation.  Same size as lt_rec64 so that the FP64 chunk
 * lists and staging serve both.  A type-5 (SIS) record uses q2 = 1 - e, k = 1 + e,
 * K = b0 (1-e)(1+e). */
struct alignas(16) lt_nie64 {
    double x0, y0, cs, sn;
    double c2t, s2t, w, k;
    double q2, sc, st, ds;
    double q2sc2, q2st2, dq2s2, opsc2;
    double opst2, opds2, tsc, tst;
    double K, Kc1sc2, Kc1st2, pad0;
    double pad[8];
};
static_assert(sizeof(lt_nie64) == sizeof(lt_rec64), "record size");

/* A chunk: a run of consecutive halos of one type, at most LT_CHUNK halos long.  The
 * grid kernels walk the chunk list; runs of equal type are the reference's dispatch unit
 * (src/gradient.cpp:899-929). */
struct lt_chunk {
    int32_t start, count, type, pad;
};

#define LT_CHUNK 64
