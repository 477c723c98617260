/*
 * lt_grid64.cu -- FP64 persistent grid kernel: deflection, Hessian (+ map epilogue) and
 * potential sums over a packed halo catalogue.
 *
 * Work layout
 *   - A CTA of 256 threads owns a pixel tile of (32 P) x 8 pixels; each thread owns P
 *     adjacent pixels of one row (P = 2: one 16-byte store per output plane).
 *   - CTAs are persistent: grid = resident CTAs per SM x SMs, tiles strided by gridDim.
 *   - The halo catalogue is walked in chunks of LT_CHUNK records (each chunk holds one
 *     profile type).  Chunk k+1 is brought into shared memory by one cp.async.bulk
 *     while chunk k is evaluated; every thread then reads the same record (a shared-memory
 *     broadcast), so the per-halo invariants cost no global traffic in the pair loop.
 *   - The pair loop is specialised per profile type (no function pointers, unlike the
 *     reference's device function tables, src/gradient_GPU.cu:910-922).
 */
#include <cuda_runtime.h>
#include "lt_bulk.cuh"
#include "lt_internal.h"
#include "lt_eval.cuh"

namespace lt {

constexpr int kThreads = 256;

template <int OP, int P, bool LIST, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) grid64_kernel(const GridArgs a)
{
    static_assert(!LIST || (OP == (OP_HESS | OP_NI)), "list mode: the FP64 recomputation's Hessian");
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    lt_rec64 *buf0 = reinterpret_cast<lt_rec64 *>(smem);
    lt_rec64 *buf1 = buf0 + LT_CHUNK;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int kTileW = 32 * P;
    const int ox = (warp & 3) * (8 * P) + (lane & 7) * P; /* pixel offset in the tile */
    const int oy = (warp >> 2) * 4 + (lane >> 3);

    int ntiles = a.ntiles, nlist = 0;
    if (LIST) {
        nlist = *a.list_count;
        nlist = nlist < a.list_cap ? nlist : a.list_cap;
        ntiles = (nlist + kThreads * P - 1) / (kThreads * P);
        /* the count of recomputed pixels (lt_recompute_count): the 64-bit word 2 of the
         * context's status block */
        if (blockIdx.x == 0 && tid == 0 && a.status)
            atomicAdd(reinterpret_cast<unsigned long long *>(a.status + 2), (unsigned long long)nlist);
    }
    const int my_tiles = ((int)blockIdx.x < ntiles) ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const long steps = (long)my_tiles * a.nchunks;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (steps == 0) return;

    auto issue = [&](long s) {
        const lt_chunk c = a.chunks[s % a.nchunks];
        lt_rec64 *dst = (s & 1) ? buf1 : buf0;
        uint64_t *bar = &bars[s & 1];
        uint32_t bytes = (uint32_t)c.count * (uint32_t)sizeof(lt_rec64);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, bytes);
        bulk_g2s(dst, a.recs + c.start, bytes, bar);
    };
    if (tid == 0) issue(0);

    uint32_t phase0 = 0, phase1 = 0;
    Acc64<OP, P> acc;
    double px[P], py = 0.;
    int ix = 0, iy = 0;
    double lpy[P];     /* list mode: each pixel's own row coordinate */
    int lx[P], ly[P];  /* list mode: each pixel's column and row (ly >= ny: no pixel) */

    for (long s = 0; s < steps; s++) {
        const int ci = (int)(s % a.nchunks);
        if (ci == 0) {
            const int tile = blockIdx.x + (int)(s / a.nchunks) * gridDim.x;
            if (LIST) {
                /* P list entries a thread, kThreads apart */
#pragma unroll
                for (int k = 0; k < P; k++) {
                    const int e = (tile * P + k) * kThreads + tid;
                    const int p = a.list[e < nlist ? e : nlist - 1];
                    lx[k] = p % a.nx;
                    ly[k] = e < nlist ? p / a.nx : a.ny; /* rows >= ny are not stored */
                    px[k] = pixel_x(a, lx[k]);
                    lpy[k] = pixel_y(a, ly[k] < a.ny ? ly[k] : a.ny - 1);
                    acc.hxx[k] = acc.hyy[k] = acc.hxy[k] = 0.;
                }
            } else {
                const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
                ix = tx * kTileW + ox;
                iy = ty * 8 + oy;
                const int cy = iy < a.ny ? iy : a.ny - 1;
                py = pixel_y(a, cy);
#pragma unroll
                for (int k = 0; k < P; k++) {
                    const int cx = (ix + k) < a.nx ? ix + k : a.nx - 1;
                    px[k] = pixel_x(a, cx);
                    acc.gx[k] = acc.gy[k] = acc.hxx[k] = acc.hyy[k] = acc.hxy[k] = acc.psi[k] = 0.;
                    acc.run[k].a = acc.run[k].b = acc.run[k].c = acc.run[k].d = 0.;
                    acc.tot[k].a = acc.tot[k].b = acc.tot[k].c = acc.tot[k].d = 0.;
                }
            }
        }
        if (tid == 0 && s + 1 < steps) issue(s + 1);

        const int b = (int)(s & 1);
        uint64_t *bar = &bars[b];
        const uint32_t par = b ? phase1 : phase0;
        if (!wait_tile(bar, par, a.status)) {
            if (tid == 0 && s + 1 < steps) drain_tile(&bars[b ^ 1], b ? phase0 : phase1);
            return;
        }
        if (b) phase1 ^= 1; else phase0 ^= 1;

        const lt_chunk c = a.chunks[ci];
        const lt_rec64 *recs = b ? buf1 : buf0;
        if (LIST) {
            /* the staged records are the closed-form records lt_nie64; acc.hxx, acc.hyy and
             * acc.hxy hold the convergence and shear sums */
            eval_nie_chunk<P>(c, reinterpret_cast<const lt_nie64 *>(recs), px, lpy, a.kmap, acc.hxx, acc.hyy,
                              acc.hxy);
            if (ci == a.nchunks - 1) {
#pragma unroll
                for (int k = 0; k < P; k++) {
                    if (ly[k] >= a.ny) continue;
                    const long pix = (long)ly[k] * a.nx + lx[k];
                    double hxx, hyy, hxy;
                    nie_hessian(acc.hxx[k], acc.hyy[k], acc.hxy[k], hxx, hyy, hxy);
                    for (int o = 0; o < a.nout; o++)
                        a.out[o][pix] = map_value4(a.kinds[o], 0., 0., hxx, hyy, hxy, hxy, 0., a.D, a.mult, a.scale);
                }
            }
            __syncthreads(); /* buffer b is refilled by the copy issued at step s + 1 */
            continue;
        }
        switch (c.type) {
        case 81: eval_chunk64<OP, P, 81>(recs, c.count, px, py, a.kmap, acc); break;
        case 8: eval_chunk64<OP, P, 8>(recs, c.count, px, py, a.kmap, acc); break;
        case 5: eval_chunk64<OP, P, 5>(recs, c.count, px, py, a.kmap, acc); break;
        default: break;
        }
        if ((OP & OP_HEX) && (c.pad & CHUNK_RUN_END)) close_run64<OP, P>(acc, a.kmap, recs[c.count - 1].w);

        if (ci == a.nchunks - 1 && iy < a.ny) {
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
                double v[P];
#pragma unroll
                for (int k = 0; k < P; k++)
                    v[k] = map_value4(a.kinds[o], acc.gx[k], acc.gy[k], acc.hxx[k], acc.hyy[k], acc.hxy[k],
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
        __syncthreads(); /* buffer b is refilled by the copy issued at step s + 1 */
    }
}

/* Launch one shape: P pixels per thread, registers cut for MINB resident CTAs per SM.
 * Tiles are (32 P) x 8 pixels; persistent grid of (resident CTAs per SM) x SMs. */
template <int OP, int P, bool LIST, int MINB>
static int launch_op(const GridArgs &args, int num_sms, cudaStream_t stream)
{
    const size_t smem = 2 * LT_CHUNK * sizeof(lt_rec64);
    auto kern = grid64_kernel<OP, P, LIST, MINB>;
    GridArgs a = args;
    a.tiles_x = (a.nx + 32 * P - 1) / (32 * P);
    a.ntiles = a.tiles_x * ((a.ny + 7) / 8);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = num_sms * per_sm;
    if (!LIST && blocks > a.ntiles) blocks = a.ntiles;
    if (blocks < 1) blocks = 1;
    kern<<<blocks, kThreads, smem, stream>>>(a);
    return (int)cudaGetLastError();
}

template <int OP>
static int launch_shape(int shape, const GridArgs &a, int num_sms, cudaStream_t s)
{
    switch (shape) {
    case LT_SHAPE(1, 1): return launch_op<OP, 1, false, 1>(a, num_sms, s);
    case LT_SHAPE(1, 2): return launch_op<OP, 1, false, 2>(a, num_sms, s);
    case LT_SHAPE(2, 2): return launch_op<OP, 2, false, 2>(a, num_sms, s);
    default: return launch_op<OP, 2, false, 1>(a, num_sms, s);
    }
}

int launch_grid64(int op, const GridArgs &args, int num_sms, void *stream, bool list_mode, int shape)
{
    cudaStream_t s = (cudaStream_t)stream;
    if (list_mode) { /* the FP32C recomputation pass: the out-of-line fast Hessian */
        if (op != OP_HESS) return (int)cudaErrorInvalidValue;
        return launch_op<OP_HESS | OP_NI, 2, true, 2>(args, num_sms, s);
    }
    switch (op) {
    case OP_GRAD: return launch_shape<OP_GRAD>(shape, args, num_sms, s);
    case OP_GRAD | OP_GFX: return launch_shape<OP_GRAD | OP_GFX>(shape, args, num_sms, s);
    case OP_HESS: return launch_shape<OP_HESS>(shape, args, num_sms, s);
    case OP_POT: return launch_shape<OP_POT>(shape, args, num_sms, s);
    case OP_HESS | OP_POT: return launch_shape<OP_HESS | OP_POT>(shape, args, num_sms, s);
    case OP_HEX: return launch_shape<OP_HEX>(shape, args, num_sms, s);
    case OP_POT | OP_PEX: return launch_shape<OP_POT | OP_PEX>(shape, args, num_sms, s);
    case OP_HEX | OP_POT | OP_PEX: return launch_shape<OP_HEX | OP_POT | OP_PEX>(shape, args, num_sms, s);
    default: return (int)cudaErrorInvalidValue;
    }
}

} // namespace lt

namespace lt {

int launch_grid64_list(int op, GridArgs &a, int num_sms, void *stream)
{
    a.vec_ok = 0;
    return launch_grid64(op, a, num_sms, stream, true, LT_SHAPE(1, 2));
}

/* Maps of an empty catalogue: the epilogue evaluated on zero sums. */
__global__ void epilogue_zero_kernel(const GridArgs a)
{
    const long npix = (long)a.nx * a.ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x)
        for (int o = 0; o < a.nout; o++) a.out[o][p] = map_value(a.kinds[o], 0., 0., 0., 0., 0., 0., a.D, a.mult, a.scale);
}

__global__ void planes_epilogue_kernel(int kind, double *out, const double *a, const double *b, const double *c,
                                       double D, double mult, long npix)
{
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x)
        out[p] = map_value(kind, 0., 0., a[p], c[p], b[p], a[p], D, mult, mult);
}

int launch_planes_epilogue(int kind, double *out, const double *a, const double *b, const double *c, double D,
                           double mult, int nx, int ny, int num_sms, void *stream)
{
    planes_epilogue_kernel<<<num_sms * 4, 256, 0, (cudaStream_t)stream>>>(kind, out, a, b, c, D, mult, (long)nx * ny);
    count_launch(1);
    return (int)cudaGetLastError();
}

int launch_epilogue_zero(const GridArgs &a, int num_sms, void *stream)
{
    epilogue_zero_kernel<<<num_sms * 4, 256, 0, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

} // namespace lt
