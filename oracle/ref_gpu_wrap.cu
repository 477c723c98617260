/*
 * ref_gpu_wrap.cu -- extern "C" doors into the reference's own GPU kernels, compiled from
 * its sources for sm_100a by oracle/Makefile into oracle/_ref/libltref_gpu.so (type_t =
 * double, the reference's FP64 build) and oracle/_ref/libltref_gpu32.so (type_t = float,
 * its default build).
 *
 * TEST INFRASTRUCTURE ONLY: parity of the product's FP64 maps against the reference GPU
 * kernels, and the reference-GPU timing reported beside the reference CPU arm of bench.py.
 * Nothing in the product links it.
 *
 * The kernels are the reference's, unmodified, launched as its wrappers launch them
 * (32 x 16 threads per block, one thread per pixel; src/grid_gradient2_GPU.cu:27-29,
 * 196-207, src/grid_potential_GPU.cu:166-181):
 *   module_potentialDerivatives_totalGradient2_SOA_GPU (src/gradient2_GPU.cu:335-398)
 *   module_potential_totalPotential_SOA_GPU            (src/potential_GPU.cu:139-187)
 * Both dispatch type 81 only, so the door accepts dPIE catalogues only, and both read the
 * type of halo nhalos (src/gradient2_GPU.cu:366), so the device type array carries a
 * sentinel slot.
 */
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "structure_hpc.hpp"
#include "gradient2_GPU.cuh"

/* src/potential_GPU.cuh:36-38 (that header also defines lt_math_GPU.cuh's functions,
 * which potential_GPU.cu already holds) */
__global__ void module_potential_totalPotential_SOA_GPU(type_t *potential_GPU, const struct Potential_SOA *lens,
                                                        const struct grid_param *frame, int nhalos, type_t dx,
                                                        type_t dy, int nbgridcells_x, int nbgridcells_y, int istart,
                                                        int jstart);

namespace {

#define BLOCK_X 32
#define BLOCK_Y 16

struct Dev {
    std::vector<void *> ptrs;
    ~Dev()
    {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    T *alloc(size_t n)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (T *)p;
    }
};

template <class T>
T *upload(Dev &d, const double *src, int n)
{
    std::vector<T> h((size_t)n);
    for (int i = 0; i < n; i++) h[i] = (T)src[i];
    T *p = d.alloc<T>((size_t)(n > 0 ? n : 1));
    if (p && n) cudaMemcpy(p, h.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
    return p;
}

} // namespace

extern "C" {

/* which = 0: the Hessian grid (4 planes a, b, c, d), 1: the potential grid.  Catalogue
 * arrays in lenstool order (x, y, cos, sin, epot, rcore, rcut, b0); grid xmin + i dx,
 * ymin + j dy.  One untimed launch, then `reps` launches timed with CUDA events; *ms =
 * mean milliseconds per launch.  out (optional): the planes of the last launch, nx*ny
 * doubles each.  Returns 0, -1 (a type other than 81, or bad sizes), or a CUDA error. */
int ltrefgpu_grid(int which, int n, const int *type, const double *x, const double *y, const double *cs,
                  const double *sn, const double *eps, const double *rc, const double *rcut, const double *b0,
                  double xmin, double ymin, double dx, double dy, int nx, int ny, int reps, double *ms, double *out)
{
    if (n < 1 || nx < 1 || ny < 1 || reps < 1 || (which != 0 && which != 1)) return -1;
    for (int i = 0; i < n; i++)
        if (type[i] != 81) return -1;
    Dev d;
    std::vector<int> t(type, type + n);
    t.push_back(-1); /* the sentinel the run loop reads */
    int *type_d = d.alloc<int>((size_t)n + 1);
    if (!type_d) return (int)cudaErrorMemoryAllocation;
    cudaMemcpy(type_d, t.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    Potential_SOA h;
    memset(&h, 0, sizeof(h));
    h.type = type_d;
    h.position_x = upload<type_t>(d, x, n);
    h.position_y = upload<type_t>(d, y, n);
    h.anglecos = upload<type_t>(d, cs, n);
    h.anglesin = upload<type_t>(d, sn, n);
    h.ellipticity_potential = upload<type_t>(d, eps, n);
    h.rcore = upload<type_t>(d, rc, n);
    h.rcut = upload<type_t>(d, rcut, n);
    h.b0 = upload<type_t>(d, b0, n);
    Potential_SOA *lens_d = d.alloc<Potential_SOA>(1);
    grid_param f;
    memset(&f, 0, sizeof(f));
    f.xmin = (type_t)xmin;
    f.ymin = (type_t)ymin;
    f.xmax = (type_t)(xmin + (nx - 1) * dx);
    f.ymax = (type_t)(ymin + (ny - 1) * dy);
    grid_param *frame_d = d.alloc<grid_param>(1);
    const size_t np = (size_t)nx * ny;
    const int nplanes = which == 0 ? 4 : 1;
    type_t *planes = d.alloc<type_t>(np * nplanes);
    if (!h.position_x || !h.position_y || !h.anglecos || !h.anglesin || !h.ellipticity_potential || !h.rcore ||
        !h.rcut || !h.b0 || !lens_d || !frame_d || !planes)
        return (int)cudaErrorMemoryAllocation;
    cudaMemcpy(lens_d, &h, sizeof(h), cudaMemcpyHostToDevice);
    cudaMemcpy(frame_d, &f, sizeof(f), cudaMemcpyHostToDevice);
    dim3 threads(BLOCK_X, BLOCK_Y);
    dim3 grid((nx + BLOCK_X - 1) / BLOCK_X, (ny + BLOCK_Y - 1) / BLOCK_Y);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.f;
    for (int r = 0; r <= reps; r++) {
        if (r == 1) cudaEventRecord(e0);
        if (which == 0)
            module_potentialDerivatives_totalGradient2_SOA_GPU<<<grid, threads>>>(
                planes, planes + np, planes + 2 * np, planes + 3 * np, lens_d, frame_d, n, (type_t)dx, (type_t)dy, nx,
                ny, 0, 0);
        else
            module_potential_totalPotential_SOA_GPU<<<grid, threads>>>(planes, lens_d, frame_d, n, (type_t)dx,
                                                                       (type_t)dy, nx, ny, 0, 0);
    }
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventElapsedTime(&total, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return (int)e;
    *ms = (double)total / reps;
    if (out) {
        std::vector<type_t> hbuf(np);
        for (int k = 0; k < nplanes; k++) {
            cudaMemcpy(hbuf.data(), planes + k * np, sizeof(type_t) * np, cudaMemcpyDeviceToHost);
            for (size_t i = 0; i < np; i++) out[k * np + i] = (double)hbuf[i];
        }
    }
    return 0;
}

int ltrefgpu_type_bytes(void) { return (int)sizeof(type_t); }

} // extern "C"
