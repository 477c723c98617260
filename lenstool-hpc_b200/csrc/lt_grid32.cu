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
 *   - FP32 terms are rotated to the sky frame and added with Kahan compensation; the
 *     pixel total combines the FP64 and compensated FP32 sums in FP64, and the Jacobian
 *     determinant (1-k)^2 - g^2 is formed in FP64.
 *   - pixels whose magnification exceeds the flag threshold (near critical curves, where
 *     the determinant amplifies any error) are appended to a device list.
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

static const double kMuFlag = LT_FP32C_MU_FLAG; /* recompute pixels with |mu| above this (error ~ mu^2) */

lt_status prepare_catalog_extensions(lt_context *ctx, lt_catalog *cat)
{
    const int n = cat->nhalos;
    const std::vector<int32_t> &types = cat->host_types;
    std::vector<lt_chunk> host_chunks;
    /* FP64-class halos keep their FP64 records; the others get FP32 records.  Chunks
     * never mix precision or type. */
    std::vector<lt_rec32> r32;
    std::vector<int32_t> t32;
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
        }
    }
    /* FP64-class chunks: runs of consecutive original indices of one type */
    for (size_t k = 0; k < idx64_always.size();) {
        size_t e = k + 1;
        while (e < idx64_always.size() && idx64_always[e] == idx64_always[e - 1] + 1 && t64[e] == t64[k] &&
               (int)(e - k) < LT_CHUNK)
            e++;
        lt_chunk c;
        c.start = idx64_always[k];
        c.count = (int32_t)(e - k);
        c.type = t64[k];
        c.pad = 0; /* FP64 records; the fast Hessian needs no run boundaries */
        host_chunks.push_back(c);
        k = e;
    }
    std::vector<lt_chunk> c32 = make_chunks(t32.data(), (int)t32.size(), LT_CHUNK);
    for (lt_chunk c : c32) {
        c.pad = CHUNK_FP32;
        host_chunks.push_back(c);
    }
    Fp32cCatalog h;
    h.n32 = (int32_t)r32.size();
    h.nchunks = (int32_t)host_chunks.size();
    size_t rb = sizeof(lt_rec32) * r32.size(), cb = sizeof(lt_chunk) * host_chunks.size();
    const size_t ib = sizeof(int32_t) * (size_t)n;
    size_t total = sizeof(Fp32cCatalog) + rb + cb + 2 * ib + 64;
    void *mem = nullptr;
    lt_status st = dev_alloc(ctx, &mem, total);
    if (st != LT_OK) return st;
    char *base = (char *)mem;
    h.recs32 = (lt_rec32 *)(base + 64);
    h.chunks = (lt_chunk *)(base + 64 + rb);
    h.idx32 = (int32_t *)(base + 64 + rb + cb);
    h.types = h.idx32 + n;
    cudaError_t e = cudaSuccess;
    if (rb) e = cudaMemcpy(h.recs32, r32.data(), rb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && cb) e = cudaMemcpy(h.chunks, host_chunks.data(), cb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ib) e = cudaMemcpy(h.idx32, idx32.data(), ib, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ib) e = cudaMemcpy(h.types, types.data(), ib, cudaMemcpyHostToDevice);
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

constexpr int kThreads32 = 256;

struct C32Args {
    GridArgs g;
    const lt_rec32 *recs32;
    const lt_chunk *chunks; /* mixed list, pad = 1 for FP32 records */
    int32_t nchunks;
    int32_t *list;
    int32_t *list_count;
    int32_t list_cap;
    double mu_flag;
};

template <int OP, int P, int MINB>
__global__ void __launch_bounds__(kThreads32, MINB) grid32c_kernel(const C32Args A)
{
    const GridArgs &a = A.g;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    unsigned char *buf0 = smem;
    unsigned char *buf1 = smem + LT_CHUNK * sizeof(lt_rec64);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int kTileW = 32 * P;
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
            iy = ty * 8 + oy;
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
            case 81: eval32_chunk<OP, P, 81>(recs, a.recs, c.count, px, py, a.kmap, acc); break;
            case 8: eval32_chunk<OP, P, 8>(recs, a.recs, c.count, px, py, a.kmap, acc); break;
            case 5: eval32_chunk<OP, P, 5>(recs, a.recs, c.count, px, py, a.kmap, acc); break;
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
                double det;
                fp32c_total(acc, k, a.D, hxx[k], hyy[k], hxy[k], psi[k], det);
                fp32c_grad_total(acc, k, gx[k], gy[k]);
                flag[k] = (OP & OP_HESS) && !(fabs(det) * A.mu_flag >= 1.0);
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

template <int OP>
static void (*pick_shape32(int shape))(const C32Args)
{
    switch (shape) {
    case LT_SHAPE(1, 1): return grid32c_kernel<OP, 1, 1>;
    case LT_SHAPE(1, 2): return grid32c_kernel<OP, 1, 2>;
    case LT_SHAPE(2, 2): return grid32c_kernel<OP, 2, 2>;
    default: return grid32c_kernel<OP, 2, 1>;
    }
}

static void (*pick_kernel32(int op, int shape))(const C32Args)
{
    switch (op) {
    case OP_HESS: return pick_shape32<OP_HESS>(shape);
    case OP_POT: return pick_shape32<OP_POT>(shape);
    case OP_HESS | OP_POT: return pick_shape32<OP_HESS | OP_POT>(shape);
    case OP_GRAD: return pick_shape32<OP_GRAD>(shape);
    default: return nullptr;
    }
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
    int err = cudaSuccess;
    C32Args A;
    memset(&A, 0, sizeof(A));
    A.g = a;
    bool det = false;
    for (int o = 0; o < a.nout; o++) det |= det_sensitive(a.kinds[o]);
    const int shape = ctx->shape[LT_FP32C][op & 7];
    const int ppt = (shape & 15) == 1 ? 1 : 2;
    A.g.tiles_x = (a.nx + 32 * ppt - 1) / (32 * ppt);
    A.g.ntiles = A.g.tiles_x * ((a.ny + 7) / 8);
    A.recs32 = fc.recs32;
    A.chunks = fc.chunks;
    A.nchunks = fc.nchunks;
    A.mu_flag = det ? kMuFlag : 0.0;
    const long npix = (long)a.nx * a.ny;
    if (det) {
        lt_status st = list_buffer(ctx, npix, &A.list, &A.list_count);
        if (st != LT_OK) return (int)cudaErrorMemoryAllocation;
        A.list_cap = (int32_t)npix;
        cudaMemsetAsync(A.list_count, 0, sizeof(int32_t), s);
    }
    const size_t smem = 2 * LT_CHUNK * sizeof(lt_rec64);
    void (*kern)(const C32Args) = pick_kernel32(op, shape);
    if (!kern) return (int)cudaErrorInvalidValue;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads32, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = ctx->num_sms * per_sm;
    if (blocks > A.g.ntiles) blocks = A.g.ntiles;
    kern<<<blocks, kThreads32, smem, s>>>(A);
    count_launch(1);
    err = (int)cudaGetLastError();
    if (err != cudaSuccess || !det) return err;
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
    err = launch_grid64_list(OP_HESS, r, ctx->num_sms, stream);
    count_launch(1);
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
    const int shape = ctx->shape[LT_FP32C][OP_HESS];
    const int ppt = (shape & 15) == 1 ? 1 : 2;
    A.g.tiles_x = (a.nx + 32 * ppt - 1) / (32 * ppt);
    A.g.ntiles = A.g.tiles_x * ((a.ny + 7) / 8);
    A.recs32 = fc.recs32;
    A.chunks = fc.chunks;
    A.nchunks = fc.nchunks;
    A.mu_flag = det ? kMuFlag : 0.0;
    if (det) {
        if ((long)a.nx * a.ny > (long)cap) return (int)cudaErrorInvalidValue;
        A.list = list;
        A.list_count = count;
        A.list_cap = cap;
        cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return (int)e;
    }
    const size_t smem = 2 * LT_CHUNK * sizeof(lt_rec64);
    void (*kern)(const C32Args) = pick_kernel32(OP_HESS, shape);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads32, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = ctx->num_sms * per_sm;
    if (blocks > A.g.ntiles) blocks = A.g.ntiles;
    kern<<<blocks, kThreads32, smem, s>>>(A);
    count_launch(1);
    int err = (int)cudaGetLastError();
    if (err != cudaSuccess || !det) return err;
    GridArgs r = A.g;
    r.list = A.list;
    r.list_count = A.list_count;
    r.list_cap = A.list_cap;
    err = launch_grid64_list(OP_HESS, r, ctx->num_sms, stream);
    count_launch(1);
    return err;
}


} // namespace lt
