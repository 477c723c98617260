/*
 * cuda_host_stubs.h -- force-included when the reference's GPU profile sources are
 * compiled as plain host C++ into the checker library oracle/_ref/libltref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA qualifiers become empty, and the launch indices
 * become per-thread host variables, so that a reference __global__ function can be run
 * on the CPU one pixel at a time by setting blockIdx/threadIdx before each call.
 */
#pragma once
#include <math.h>
#include <stdio.h>

struct lt_dim3_stub { unsigned x, y, z; };
extern thread_local lt_dim3_stub threadIdx, blockIdx, blockDim, gridDim;

#define __device__
#define __global__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline
