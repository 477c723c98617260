/*
 * lt_grid32.cu -- the FP32-compensated (LT_FP32C) Hessian-map path.
 *
 * Pass 1 (grid32c_kernel), per pixel tile:
 *   - cluster-scale halos (b0 >= 5", rcore >= 1", or e < 1e-3) are summed in FP64 from
 *     the FP64 records;
 *   - every other halo is evaluated with the FP32 forms of lt_profiles32.cuh, unless any
 *     pixel of the warp lies in one of the halo's FP64 regions (near the galaxy where
 *     b0/2r > 0.1, within (0.3 + 1.5 e) rcut of the cut radius' singular point, within 3 rcore of
 *     the centre); then the warp evaluates that halo in FP64 (warp-uniform branch);
 *     A warp first tests a chunk's fallback regions against its pixel box (one ballot), so
 *     the per-pixel test runs only for the few halos whose regions reach the box;
 *   - FP32 terms are rotated to the sky frame and summed in FP32 over blocks of 8 halos,
 *     each block sum joining FP64 sums; the Jacobian determinant (1-k)^2 - g^2 is formed
 *     in FP64, with a bound on its error from the magnitudes of the FP32 terms;
 *   - pixels where that bound allows a relative error of mu above kMuTol32 (near critical
 *     curves, where the determinant amplifies any error) are appended to a device list.
 * Pass 2 (the FP64 grid kernel in list mode) recomputes the flagged pixels in FP64 and
 * overwrites them.  The pixel count of pass 2 is read on the device: no host round trip.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "lt_bulk.cuh"
#include "lt_internal.h"
#include "lt_eval.cuh"
#include "lt_pack.h"

namespace lt {


lt_status prepare_catalog_extensions(lt_context *ctx, lt_catalog *cat)
{
    const int n = cat->nhalos;
    const std::vector<int32_t> &types = cat->host_types;
    std::vector<lt_chunk> host_chunks;
    /* FP64-class halos keep their FP64 records; the others get FP32 records.  Chunks
     * never mix precision or type. */
    std::vector<lt_rec32> r32;
    std::vector<int32_t> t32;
    std::vector<double> w32;
    std::vector<int32_t> idx64_always, t64, idx32((size_t)n, -1);
    for (int i = 0; i < n; i++) {
        if (pk::needs_fp64_always(cat->host_recs[i], types[i])) {
            idx64_always.push_back(i);
            t64.push_back(types[i]);
        } else {
            lt_rec32 o;
            pk::pack32(cat->host_recs[i], types[i], i, o);
            idx32[i] = (int32_t)r32.size();
            r32.push_back(o);
            t32.push_back(types[i]);
            w32.push_back((double)o.w);
        }
    }
    /* the mixed chunk list for one stage size: FP64-class chunks (runs of consecutive
     * original indices of one type), then FP32 chunks (runs of one type and one Kmap
     * weight: the block sums take the weight once per chunk) */
    auto build_list = [&](int cap) {
        std::vector<lt_chunk> out;
        for (size_t k = 0; k < idx64_always.size();) {
            size_t e = k + 1;
            while (e < idx64_always.size() && idx64_always[e] == idx64_always[e - 1] + 1 && t64[e] == t64[k] &&
                   (int)(e - k) < cap)
                e++;
            lt_chunk c;
            c.start = idx64_always[k];
            c.count = (int32_t)(e - k);
            c.type = t64[k];
            c.pad = 0; /* FP64 records; the fast Hessian needs no run boundaries */
            out.push_back(c);
            k = e;
        }
        for (lt_chunk c : make_chunks(t32.data(), (int)t32.size(), cap, w32.data())) {
            c.pad = CHUNK_FP32;
            out.push_back(c);
        }
        return out;
    };
    const std::vector<lt_chunk> l64 = build_list(LT_CHUNK), l32 = build_list(32), l128 = build_list(128);
    host_chunks = l64;
    host_chunks.insert(host_chunks.end(), l32.begin(), l32.end());
    host_chunks.insert(host_chunks.end(), l128.begin(), l128.end());
    Fp32cCatalog h;
    h.n32 = (int32_t)r32.size();
    h.nchunks = (int32_t)l64.size();
    h.nchunks_s = (int32_t)l32.size();
    h.nchunks_l = (int32_t)l128.size();
    std::vector<lt_nie64> nie((size_t)n);
    for (int i = 0; i < n; i++) pk::pack_nie64(cat->host_recs[i], types[i], nie[i]);
    size_t rb = sizeof(lt_rec32) * r32.size(), cb = sizeof(lt_chunk) * host_chunks.size();
    const size_t ib = sizeof(int32_t) * (size_t)n, nb = sizeof(lt_nie64) * (size_t)n;
    size_t total = sizeof(Fp32cCatalog) + nb + rb + cb + 2 * ib + 64;
    void *mem = nullptr;
    lt_status st = dev_alloc(ctx, &mem, total);
    if (st != LT_OK) return st;
    char *base = (char *)mem;
    h.nie = (lt_nie64 *)(base + 64);
    base += nb;
    h.recs32 = (lt_rec32 *)(base + 64);
    h.chunks = (lt_chunk *)(base + 64 + rb);
    h.chunks_s = h.chunks + l64.size();
    h.chunks_l = h.chunks_s + l32.size();
    h.idx32 = (int32_t *)(base + 64 + rb + cb);
    h.types = h.idx32 + n;
    cudaError_t e = cudaSuccess;
    if (rb) e = cudaMemcpy(h.recs32, r32.data(), rb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && cb) e = cudaMemcpy(h.chunks, host_chunks.data(), cb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ib) e = cudaMemcpy(h.idx32, idx32.data(), ib, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ib) e = cudaMemcpy(h.types, types.data(), ib, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nb) e = cudaMemcpy(h.nie, nie.data(), nb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        dev_free(ctx, mem, total);
        return cuda_fail(ctx, e, "FP32 catalogue upload");
    }
    /* the descriptor stays on the host side of the catalogue, the data on the device */
    static_assert(sizeof(Fp32cCatalog) <= sizeof(((lt_catalog *)0)->aux_desc), "descriptor size");
    cat->aux = mem;
    cat->aux_bytes = total;
    memcpy(cat->aux_desc, &h, sizeof(h));
    return LT_OK;
}

struct C32Args {
    GridArgs g;
    const lt_rec32 *recs32;
    const lt_chunk *chunks; /* mixed list, pad & CHUNK_FP32 for FP32 records */
    int32_t nchunks;
    int32_t cap;            /* records per shared-memory stage (the chunk list's maximum) */
    int32_t *list;
    int32_t *list_count;
    int32_t list_cap;
    double mu_tol; /* recompute pixels whose FP32 error bound on mu exceeds this (0: none) */
};

/* Pass 1.  NT threads per CTA (8 lanes x P columns by 4 rows per warp, warps 4 across):
 * a tile is 32 P columns by NT / 32 rows; registers are cut for MINB resident CTAs per
 * SM.  Persistent CTAs stride over the tiles; for each tile the chunks of the catalogue
 * are staged into shared memory by cp.async.bulk, chunk k + 1 in flight while chunk k is
 * evaluated. */
template <int OP, int P, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) grid32c_kernel(const C32Args A)
{
    const GridArgs &a = A.g;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    unsigned char *buf0 = smem;
    unsigned char *buf1 = smem + (size_t)A.cap * sizeof(lt_rec64);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int kTileW = 32 * P, kTileH = NT / 32;
    const int ox = (warp & 3) * (8 * P) + (lane & 7) * P;
    const int oy = (warp >> 2) * 4 + (lane >> 3);
    const int my_tiles = (blockIdx.x < a.ntiles) ? (a.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long steps = (long)my_tiles * A.nchunks;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (steps == 0) return;

    auto issue = [&](long s) {
        const lt_chunk c = A.chunks[s % A.nchunks];
        unsigned char *dst = (s & 1) ? buf1 : buf0;
        uint64_t *bar = &bars[s & 1];
        const void *src;
        uint32_t bytes;
        if (c.pad & CHUNK_FP32) {
            src = A.recs32 + c.start;
            bytes = (uint32_t)c.count * (uint32_t)sizeof(lt_rec32);
        } else {
            src = a.recs + c.start;
            bytes = (uint32_t)c.count * (uint32_t)sizeof(lt_rec64);
        }
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, bytes);
        bulk_g2s(dst, src, bytes, bar);
    };
    if (tid == 0) issue(0);

    uint32_t phase0 = 0, phase1 = 0;
    Acc32<P> acc;
    double px[P], py = 0.;
    int ix = 0, iy = 0;

    for (long s = 0; s < steps; s++) {
        const int ci = (int)(s % A.nchunks);
        if (ci == 0) {
            const int tile = blockIdx.x + (int)(s / A.nchunks) * gridDim.x;
            const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
            ix = tx * kTileW + ox;
            iy = ty * kTileH + oy;
            py = pixel_y(a, iy < a.ny ? iy : a.ny - 1);
#pragma unroll
            for (int k = 0; k < P; k++) {
                px[k] = pixel_x(a, (ix + k) < a.nx ? ix + k : a.nx - 1);
                acc32_zero(acc, k);
            }
        }
        if (tid == 0 && s + 1 < steps) issue(s + 1);
        const int b = (int)(s & 1);
        const uint32_t par = b ? phase1 : phase0;
        if (!wait_tile(&bars[b], par, a.status)) {
            if (tid == 0 && s + 1 < steps) drain_tile(&bars[b ^ 1], b ? phase0 : phase1);
            return;
        }
        if (b) phase1 ^= 1; else phase0 ^= 1;

        const lt_chunk c = A.chunks[ci];
        const unsigned char *buf = b ? buf1 : buf0;
        if (c.pad & CHUNK_FP32) {
            const lt_rec32 *recs = reinterpret_cast<const lt_rec32 *>(buf);
            switch (c.type) {
            case 81: eval32_chunk<OP, P, 81>(recs, a.recs, c.count, px, py, a, ix, iy, acc); break;
            case 8: eval32_chunk<OP, P, 8>(recs, a.recs, c.count, px, py, a, ix, iy, acc); break;
            case 5: eval32_chunk<OP, P, 5>(recs, a.recs, c.count, px, py, a, ix, iy, acc); break;
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

        if (ci == A.nchunks - 1 && iy < a.ny) {
            const long row = (long)iy * a.nx;
            double hxx[P], hyy[P], hxy[P], psi[P], gx[P], gy[P];
            bool flag[P];
#pragma unroll
            for (int k = 0; k < P; k++) {
                double det, det_err;
                fp32c_total(acc, k, a.D, hxx[k], hyy[k], hxy[k], psi[k], det, det_err);
                fp32c_grad_total(acc, k, gx[k], gy[k]);
                flag[k] = (OP & OP_HESS) && A.mu_tol > 0. && fp32c_flag(det, det_err, A.mu_tol);
            }
            const bool full = a.vec_ok && (ix + P <= a.nx);
            for (int o = 0; o < a.nout; o++) {
                double v[P];
#pragma unroll
                for (int k = 0; k < P; k++)
                    v[k] = map_value(a.kinds[o], gx[k], gy[k], hxx[k], hyy[k], hxy[k], psi[k], a.D, a.mult, a.scale);
                double *dst = a.out[o] + row + ix;
                if (P == 2 && full) {
                    *reinterpret_cast<double2 *>(dst) = make_double2(v[0], v[1 % P]);
                } else {
#pragma unroll
                    for (int k = 0; k < P; k++)
                        if (ix + k < a.nx) dst[k] = v[k];
                }
            }
            if (A.list) {
#pragma unroll
                for (int k = 0; k < P; k++)
                    if (flag[k] && ix + k < a.nx) {
                        const int slot = atomicAdd(A.list_count, 1);
                        if (slot < A.list_cap) A.list[slot] = (int32_t)(row + ix + k);
                    }
            }
        }
        __syncthreads();
    }
}

using Kern32 = void (*)(const C32Args);

/* The FP32C kernel shapes (pixels per thread, CTAs per SM, threads per CTA); the halo
 * stage size (records per chunk: 32, 64 or 128) is a launch argument. */
template <int OP>
static Kern32 pick_shape32(int shape)
{
    switch (shape & 0xffff) {
    case LT_SHAPE(1, 1) & 0xffff: return grid32c_kernel<OP, 1, 256, 1>;
    case LT_SHAPE(1, 2) & 0xffff: return grid32c_kernel<OP, 1, 256, 2>;
    case LT_SHAPE(2, 1) & 0xffff: return grid32c_kernel<OP, 2, 256, 1>;
    case LT_SHAPE(2, 2) & 0xffff: return grid32c_kernel<OP, 2, 256, 2>;
    case LT_SHAPE4(1, 2, 128, 64) & 0xffff: return grid32c_kernel<OP, 1, 128, 2>;
    case LT_SHAPE4(1, 4, 128, 64) & 0xffff: return grid32c_kernel<OP, 1, 128, 4>;
    case LT_SHAPE4(2, 2, 128, 64) & 0xffff: return grid32c_kernel<OP, 2, 128, 2>;
    case LT_SHAPE4(2, 3, 128, 64) & 0xffff: return grid32c_kernel<OP, 2, 128, 3>;
    case LT_SHAPE4(2, 4, 128, 64) & 0xffff: return grid32c_kernel<OP, 2, 128, 4>;
    default: return nullptr;
    }
}

static Kern32 pick_kernel32(int op, int shape)
{
    switch (op) {
    case OP_HESS: return pick_shape32<OP_HESS>(shape);
    case OP_POT: return pick_shape32<OP_POT>(shape);
    case OP_HESS | OP_POT: return pick_shape32<OP_HESS | OP_POT>(shape);
    case OP_GRAD: return pick_shape32<OP_GRAD>(shape);
    default: return nullptr;
    }
}

/* Every FP32C shape the kernels are built for (the autotuner's search space with the
 * stage sizes 32, 64 and 128). */
const int kShapes32[] = {LT_SHAPE(1, 1), LT_SHAPE(1, 2), LT_SHAPE(2, 1), LT_SHAPE(2, 2),
                         LT_SHAPE4(1, 2, 128, 64), LT_SHAPE4(1, 4, 128, 64), LT_SHAPE4(2, 2, 128, 64),
                         LT_SHAPE4(2, 3, 128, 64), LT_SHAPE4(2, 4, 128, 64)};
const int kNumShapes32 = (int)(sizeof(kShapes32) / sizeof(kShapes32[0]));

/* Allow every FP32C kernel the dynamic shared memory of the largest stage (two 128-record
 * stages, 64 KB) on the current device: once per context, not per launch (the attribute
 * call is far slower than a small launch). */
int configure_kernels32()
{
    const size_t smem = 2 * (size_t)128 * sizeof(lt_rec64);
    for (int op : {(int)OP_HESS, (int)OP_POT, (int)(OP_HESS | OP_POT), (int)OP_GRAD})
        for (int k = 0; k < kNumShapes32; k++) {
            const cudaError_t e = cudaFuncSetAttribute(pick_kernel32(op, kShapes32[k]),
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return (int)e;
        }
    return (int)cudaSuccess;
}

bool shape32_ok(int shape)
{
    const int cap = shape_cap(shape);
    return pick_shape32<OP_HESS>(shape) != nullptr && (cap == 32 || cap == 64 || cap == 128);
}

/* The chunk list of the catalogue for a stage size. */
static void chunks_for_cap(const Fp32cCatalog &fc, int cap, const lt_chunk **chunks, int32_t *n)
{
    if (cap == 32) {
        *chunks = fc.chunks_s;
        *n = fc.nchunks_s;
    } else if (cap == 128) {
        *chunks = fc.chunks_l;
        *n = fc.nchunks_l;
    } else {
        *chunks = fc.chunks;
        *n = fc.nchunks;
    }
}

/* Pass 1 launch with the context's shape for (FP32C, op). */
static int launch_pass1(lt_context *ctx, const Fp32cCatalog &fc, int op, C32Args &A, cudaStream_t s)
{
    const int shape = ctx->shape[LT_FP32C][op & 7];
    Kern32 kern = pick_kernel32(op, shape);
    if (!kern) return (int)cudaErrorInvalidValue;
    const int P = shape_ppt(shape), NT = shape_threads(shape), cap = shape_cap(shape);
    A.cap = cap;
    chunks_for_cap(fc, cap, &A.chunks, &A.nchunks);
    A.recs32 = fc.recs32;
    A.g.tiles_x = (A.g.nx + 32 * P - 1) / (32 * P);
    A.g.ntiles = A.g.tiles_x * ((A.g.ny + NT / 32 - 1) / (NT / 32));
    const size_t smem = 2 * (size_t)cap * sizeof(lt_rec64); /* allowed once by configure_kernels32 */
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = ctx->num_sms * per_sm;
    if (blocks > A.g.ntiles) blocks = A.g.ntiles;
    kern<<<blocks, NT, smem, s>>>(A);
    count_launch(1);
    return (int)cudaGetLastError();
}

/* maps whose value depends on the Jacobian determinant (amplified near critical curves) */
bool det_sensitive(int kind)
{
    return kind == LT_MAP_MU || kind == LT_MAP_AMPLI1 || kind == LT_MAP_AMPLI2 || kind == LT_MAP_AMPLI3 ||
           kind == LT_MAP_AMPLI4 || kind == LT_MAP_SHEAR2;
}

int launch_fp32c(lt_context *ctx, const lt_catalog *cat, int op, GridArgs &a, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    const Fp32cCatalog &fc = *reinterpret_cast<const Fp32cCatalog *>(&cat->aux_desc);
    if ((op & OP_GRAD) && op != OP_GRAD) {
        set_error(ctx, "FP32C deflection grids are computed on their own");
        return (int)cudaErrorNotSupported;
    }
    C32Args A;
    memset(&A, 0, sizeof(A));
    A.g = a;
    bool det = false;
    for (int o = 0; o < a.nout; o++) det |= det_sensitive(a.kinds[o]);
    A.mu_tol = det ? kMuTol32 : 0.0;
    const long npix = (long)a.nx * a.ny;
    if (det) {
        lt_status st = list_buffer(ctx, npix, &A.list, &A.list_count);
        if (st != LT_OK) return (int)cudaErrorMemoryAllocation;
        A.list_cap = (int32_t)npix;
        cudaMemsetAsync(A.list_count, 0, sizeof(int32_t), s);
    }
    pass_mark(ctx, s, 0);
    int err = launch_pass1(ctx, fc, op, A, s);
    pass_mark(ctx, s, 1);
    if (err != cudaSuccess || !det) {
        pass_mark(ctx, s, 2);
        return err;
    }
    /* pass 2: FP64 recomputation of the flagged pixels' Hessian maps (the potential of
     * those pixels keeps its FP32C value) */
    GridArgs r = A.g;
    r.nout = 0;
    for (int o = 0; o < a.nout; o++)
        if (a.kinds[o] != KIND_POT) {
            r.kinds[r.nout] = a.kinds[o];
            r.out[r.nout++] = a.out[o];
        }
    r.list = A.list;
    r.list_count = A.list_count;
    r.list_cap = A.list_cap;
    r.recs = reinterpret_cast<const lt_rec64 *>(fc.nie); /* the closed-form FP64 records */
    err = launch_grid64_list(OP_HESS, r, ctx->num_sms, stream);
    count_launch(1);
    pass_mark(ctx, s, 2);
    return err;
}

/* launch_fp32c for the Hessian maps with a caller-provided recomputation list: `list`
 * holds up to `cap` pixel indices and `count` its length word, which this function
 * zeroes on `stream` before pass 1.  Nothing is allocated. */
int launch_fp32c_with_list(lt_context *ctx, const lt_catalog *cat, GridArgs &a, int32_t *list, int32_t *count,
                           int32_t cap, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    const Fp32cCatalog &fc = *reinterpret_cast<const Fp32cCatalog *>(&cat->aux_desc);
    C32Args A;
    memset(&A, 0, sizeof(A));
    A.g = a;
    bool det = false;
    for (int o = 0; o < a.nout; o++) det |= det_sensitive(a.kinds[o]);
    A.mu_tol = det ? kMuTol32 : 0.0;
    if (det) {
        if ((long)a.nx * a.ny > (long)cap) return (int)cudaErrorInvalidValue;
        A.list = list;
        A.list_count = count;
        A.list_cap = cap;
        cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return (int)e;
    }
    int err = launch_pass1(ctx, fc, OP_HESS, A, s);
    if (err != cudaSuccess || !det) return err;
    GridArgs r = A.g;
    r.list = A.list;
    r.list_count = A.list_count;
    r.list_cap = A.list_cap;
    r.recs = reinterpret_cast<const lt_rec64 *>(fc.nie); /* the closed-form FP64 records */
    err = launch_grid64_list(OP_HESS, r, ctx->num_sms, stream);
    count_launch(1);
    return err;
}


} // namespace lt
