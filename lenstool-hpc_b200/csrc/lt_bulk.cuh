/*
 * lt_bulk.cuh -- shared-memory staging of halo tiles with the Blackwell bulk-copy
 * engine (cp.async.bulk, global -> shared, completion on an mbarrier), and the map
 * epilogue shared by the grid kernels.
 *
 * Every wait on an mbarrier is bounded: after LT_WAIT_LIMIT polls the kernel records
 * LT_ERR_TIMEOUT in its status word and the block leaves together (see wait_tile).
 */
#pragma once
#include <stdint.h>
#include "lt_grid.cuh"

#define LT_WAIT_LIMIT (1u << 24)

namespace lt {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* Arrive once and announce `bytes` of incoming transactions. */
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

/* Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from global to
 * this CTA's shared memory, completing on `bar`.  No multicast. */
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

/* Bounded wait of the whole block for phase `parity` of `bar`.  Returns false (after
 * recording LT_ERR_TIMEOUT) when any thread gave up; every thread of the block takes
 * the same branch because the outcome is reduced with __syncthreads_or. */
__device__ __forceinline__ bool wait_tile(uint64_t *bar, uint32_t parity, int32_t *status)
{
    int gave_up = 0;
    uint32_t tries = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++tries > LT_WAIT_LIMIT) {
            gave_up = 1;
            break;
        }
    }
    if (__syncthreads_or(gave_up)) {
        if (threadIdx.x == 0 && status) atomicExch(status, (int32_t)LT_ERR_TIMEOUT);
        return false;
    }
    return true;
}

/* Before leaving after a timeout, let a copy still in flight land (bounded). */
__device__ __forceinline__ void drain_tile(uint64_t *bar, uint32_t parity)
{
    uint32_t tries = 0;
    while (!mbar_try_wait(bar, parity) && ++tries < LT_WAIT_LIMIT) {
    }
}

/* Coordinates of pixel column i / row j without a fused multiply-add, so that they equal
 * the reference's xmin + (i + istart) dx bit for bit. */
__device__ __forceinline__ double pixel_x(const GridArgs &a, int i)
{
    return __dadd_rn(a.xmin, __dmul_rn((double)(i + a.istart), a.dx));
}
__device__ __forceinline__ double pixel_y(const GridArgs &a, int j)
{
    return __dadd_rn(a.ymin, __dmul_rn((double)(j + a.jstart), a.dy));
}

/* Round-to-nearest operations that the compiler may not fuse into FMAs: the map
 * epilogues use them so that every kernel rounds a map exactly alike (and in the
 * reference's C operation order), whatever the surrounding code. */
namespace rn {
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double sqr(double a) { return __dsqrt_rn(a); }
} // namespace rn

/* Eigenvalues of [[A, B], [B, C]] (formeli_ampli, src/grid_map_ampli_GPU.cu:549-572). */
__device__ __forceinline__ void eigen2(double A, double B, double C, double &lam, double &mu)
{
    const double amc = rn::sub(A, C);
    const double delta = rn::add(rn::mul(amc, amc), rn::mul(rn::mul(4., B), B));
    const double e = rn::sqr(delta);
    lam = rn::mul(.5, rn::add(rn::add(A, C), e));
    mu = rn::mul(.5, rn::sub(rn::add(A, C), e));
}

/* Value of one output plane at one pixel from the pixel's sums (hyx: the Hessian's d
 * entry, equal to hxy up to rounding).  Formulas and operation order of the reference's
 * map kernels: ampli src/grid_map_ampli_GPU.cu:329-547, shear src/grid_map_shear_GPU.cu:
 * 208-369, mass src/grid_map_mass_GPU.cu:307-322. */
__device__ __forceinline__ double map_value4(int kind, double gx, double gy, double hxx, double hyy, double hxy,
                                             double hyx, double psi, double D, double mult, double scale)
{
    using namespace rn;
    const double a = hxx, b = hxy, c = hyy;
    double lam, mu;
    switch (kind) {
    case LT_MAP_HESS_A: return a;
    case LT_MAP_HESS_B: return b;
    case LT_MAP_HESS_C: return c;
    case LT_MAP_HESS_D: return hyx;
    case LT_MAP_AMPLI1:
        eigen2(sub(1., mul(a, D)), -mul(b, D), sub(1., mul(c, D)), lam, mu);
        return div(1., mul(lam, mu));
    case LT_MAP_AMPLI2:
        eigen2(sub(1., mul(a, D)), -mul(b, D), sub(1., mul(c, D)), lam, mu);
        return div(1., fabs(mul(lam, mu)));
    case LT_MAP_AMPLI3:
        eigen2(sub(1., mul(a, D)), -mul(b, D), sub(1., mul(c, D)), lam, mu);
        return mul(-2.5, log10(fabs(mul(lam, mu))));
    case LT_MAP_AMPLI4: {
        const double k = div(mul(add(a, c), D), 2.);
        const double g1 = div(mul(sub(a, c), D), 2.);
        const double g2 = mul(b, D);
        const double g = sqr(add(mul(g1, g1), mul(g2, g2)));
        const double gp = div(g, sub(1., k));
        const double gp2 = mul(gp, gp);
        return div(mul(sub(1., k), add(1., gp2)), sub(1., gp2));
    }
    case LT_MAP_AMPLI5: return div(add(a, c), 2.);
    case LT_MAP_AMPLI6: {
        const double g1 = div(sub(a, c), 2.);
        return sqr(add(mul(g1, g1), mul(b, b)));
    }
    case LT_MAP_SHEAR1:
        eigen2(sub(1., mul(a, D)), -mul(b, D), sub(1., mul(c, D)), lam, mu);
        return div(sub(lam, mu), 2.);
    case LT_MAP_SHEAR2: {
        eigen2(sub(1., mul(a, D)), -mul(b, D), sub(1., mul(c, D)), lam, mu);
        const double q = div(lam, mu);
        const double q2 = mul(q, q);
        return fabs(div(sub(q2, 1.), add(q2, 1.)));
    }
    case LT_MAP_SHEAR3:
    case LT_MAP_GAMMA1: return div(mul(sub(a, c), D), 2.);
    case LT_MAP_SHEAR4:
    case LT_MAP_GAMMA2: return mul(b, D);
    case LT_MAP_KAPPA: return div(mul(add(a, c), D), 2.);
    case LT_MAP_MU: {
        const double k = div(mul(add(a, c), D), 2.);
        const double g1 = div(mul(sub(a, c), D), 2.);
        const double g2 = mul(b, D);
        const double omk = sub(1., k);
        return div(1., sub(sub(mul(omk, omk), mul(g1, g1)), mul(g2, g2)));
    }
    case LT_MAP_MASS: return mul(mul(add(a, c), 0.5), mult);
    case KIND_GRAD_X: return mul(gx, scale);
    case KIND_GRAD_Y: return mul(gy, scale);
    case KIND_POT: return mul(psi, scale);
    default: return 0.;
    }
}

__device__ __forceinline__ double map_value(int kind, double gx, double gy, double hxx, double hyy, double hxy,
                                            double psi, double D, double mult, double scale)
{
    return map_value4(kind, gx, gy, hxx, hyy, hxy, hxy, psi, D, mult, scale);
}

} // namespace lt
