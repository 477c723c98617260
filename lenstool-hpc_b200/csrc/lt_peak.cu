/*
 * lt_peak.cu -- FMA-pipe throughput of the current GPU, measured with independent FMA
 * chains.  The grid kernels here are bound by the FP64 or FP32 pipe rather than by HBM
 * or the tensor cores; this number is the denominator of their roofline fraction.
 */
#include <cuda_runtime.h>

#include "lt_internal.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

template <typename T>
__global__ void fma_chain_kernel(T seed, T *sink)
{
    T a = seed + (T)threadIdx.x * (T)1e-7, b = (T)0.999999;
    T acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) acc[c] = a + (T)c;
#pragma unroll 4
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) acc[c] = fma(acc[c], b, a);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += acc[c];
    if (s == (T)-12345.) sink[0] = s; /* keeps the chains live; never true */
}

template <typename T>
double measure(int device)
{
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 0.;
    cudaSetDevice(device);
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T)) != cudaSuccess) return 0.;
    const int threads = 256, blocks = prop.multiProcessorCount * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        fma_chain_kernel<T><<<blocks, threads>>>((T)1.0, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * kChains * (double)kIters * threads * blocks;
        if (rep > 0 && ms > 0.f) best = flops / (ms * 1e-3) / 1e12 > best ? flops / (ms * 1e-3) / 1e12 : best;
    }
    lt::count_launch(4);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return best;
}

} // namespace

extern "C" double lt_measure_fma_peak(int fp32, int device)
{
    return fp32 ? measure<float>(device) : measure<double>(device);
}

/* ---- the per-pair reciprocal and reciprocal square root (lt_profiles64.cuh) ---- */

#include "lt_profiles64.cuh"

namespace {
__global__ void fast_math_kernel(const double *x, double *rcp, double *rsq, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        rcp[i] = lt::rcp64(x[i]);
        rsq[i] = lt::rsqrt64(x[i]);
    }
}

int eval_fast_math(int device, int n, const double *x, double *rcp, double *rsqrt)
{
    if (n < 1 || !x || !rcp || !rsqrt) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 4;
    double *d = nullptr;
    const size_t b = sizeof(double) * (size_t)n;
    if (cudaMalloc(&d, 3 * b) != cudaSuccess) return 5;
    cudaError_t e = cudaMemcpy(d, x, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        fast_math_kernel<<<256, 256>>>(d, d + n, d + 2 * n, n);
        lt::count_launch(1);
        e = cudaMemcpy(rcp, d + n, b, cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = cudaMemcpy(rsqrt, d + 2 * n, b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 4;
}
} // namespace

extern "C" int lt_eval_fast_math(int device, int n, const double *x, double *rcp, double *rsqrt)
{
    return eval_fast_math(device, n, x, rcp, rsqrt);
}

/* ---- the FP32 atan2 and square root of the compensated pair loops (lt_profiles32.cuh) ---- */

#include "lt_profiles32.cuh"

namespace {
__global__ void fast_math32_kernel(const float *y, const float *x, float *own, float *cuda, float *sq, float *th,
                                   int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        own[i] = lt::fatan2(y[i], x[i]);
        cuda[i] = atan2f(y[i], x[i]);
        sq[i] = lt::fsqrt(x[i]);
        th[i] = lt::fatanh_third(y[i]);
    }
}
} // namespace

extern "C" int lt_eval_fast_math32(int device, int n, const float *y, const float *x, float *atan2_own,
                                   float *atan2_cuda, float *sqrt_own, float *atanh_own)
{
    if (n < 1 || !y || !x || !atan2_own || !atan2_cuda || !sqrt_own || !atanh_own) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 4;
    float *d = nullptr;
    const size_t b = sizeof(float) * (size_t)n;
    if (cudaMalloc(&d, 6 * b) != cudaSuccess) return 5;
    cudaError_t e = cudaMemcpy(d, y, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, x, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        fast_math32_kernel<<<256, 256>>>(d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, d + 4 * (size_t)n,
                                         d + 5 * (size_t)n, n);
        lt::count_launch(1);
        e = cudaMemcpy(atan2_own, d + 2 * (size_t)n, b, cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = cudaMemcpy(atan2_cuda, d + 3 * (size_t)n, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sqrt_own, d + 4 * (size_t)n, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(atanh_own, d + 5 * (size_t)n, b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 4;
}

/* ---- the approximate reciprocal, reciprocal square root and logarithm of the pair loops ---- */

namespace {
__global__ void approx32_kernel(const float *x, float *rcp, float *rsq, float *lg, float *lg_cuda, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        rcp[i] = lt::frcp(x[i]);
        rsq[i] = lt::frsqrt(x[i]);
        lg[i] = lt::flog(x[i]);
        lg_cuda[i] = logf(x[i]);
    }
}
} // namespace

extern "C" int lt_eval_approx32(int device, int n, const float *x, float *rcp, float *rsqrt, float *log_own,
                                float *log_cuda)
{
    if (n < 1 || !x || !rcp || !rsqrt || !log_own || !log_cuda) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 4;
    float *d = nullptr;
    const size_t b = sizeof(float) * (size_t)n;
    if (cudaMalloc(&d, 5 * b) != cudaSuccess) return 5;
    cudaError_t e = cudaMemcpy(d, x, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        approx32_kernel<<<256, 256>>>(d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, d + 4 * (size_t)n, n);
        lt::count_launch(1);
        e = cudaMemcpy(rcp, d + n, b, cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = cudaMemcpy(rsqrt, d + 2 * (size_t)n, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(log_own, d + 3 * (size_t)n, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(log_cuda, d + 4 * (size_t)n, b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 4;
}
