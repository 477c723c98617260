/*
 * lt_chi2.h -- the device layout and the steps of one chi2 evaluation (lt_chi2.cu), shared
 * by the chi2 entry points and the serving loop's chi2 requests (lt_server.cpp).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"

struct lt_catalog;

namespace lt {

struct Chi2Dev {
    /* systems */
    int nsys, nimages;
    const int32_t *nimg, *first;        /* images per system, index of its first image */
    const double *ix, *iy, *dr;
    /* grid */
    int n;
    double xmin, ymin, dx, dy;
    const double *ax, *ay;              /* deflection grid, n x n */
    /* work */
    double *bx, *by;                    /* source per system */
    int32_t *hits, *keys;               /* hit count and hit keys (2 * cell + lower) per system */
    /* results */
    double *chi_terms;                  /* per observed image: its chi2 term */
    double *chi2;                       /* [0]: chi2; written by the reduction */
    int32_t *found;                     /* [0]: predicted images; [1]: 1 if a source overflowed */
    int32_t *nfound;                    /* predicted images per system (<= LT_MAX_IMAGES) */
    double *fx, *fy;                    /* predicted images, nsys x LT_MAX_IMAGES */
};

/* Bytes of one evaluation's device buffers (systems, work, results, the n x n deflection
 * planes); with `mem`, also lays them out there and fills `c` (grid from the frame:
 * dx = (xmax - xmin)/(n - 1), src/chi_CPU_barycenter.cpp:104-105). */
size_t chi2_layout(int nsys, int nimages, const lt_frame *f, int n, char *mem, Chi2Dev &c);

/* Copy the systems (host arrays; `first` = index of each system's first image) into the
 * layout, stream-ordered; the host arrays must stay valid until the copies have run. */
cudaError_t chi2_upload_systems_async(const Chi2Dev &c, const int32_t *nimg, const int32_t *first, const double *x,
                                      const double *y, const double *dr, cudaStream_t s);

/* Steps 2-4 (sources, delensing, link and chi2) on a layout whose deflection planes hold
 * the grid, stream-ordered; results in c.chi2[0] and c.found[0..1]. */
int chi2_tail(lt_context *ctx, const lt_catalog *cat, const Chi2Dev &c, cudaStream_t s);

lt_status check_systems(lt_context *ctx, const lt_image_systems *sys);

} // namespace lt
