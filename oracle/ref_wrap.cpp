/*
 * ref_wrap.cpp -- extern "C" doors into the reference's own hot-path code, linked with
 * the unmodified Lenstool-HPC sources into oracle/_ref/libltref.so by oracle/Makefile.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that pins the restatement in lt_oracle.c, and
 * the timed CPU baseline ("kind": "reference").  Nothing in the product links it.
 *
 * What runs here is the reference's code itself:
 *   - gradient_grid_CPU (src/grid_gradient_CPU.cpp:56-100) and
 *     module_potentialDerivatives_totalGradient_SOA (src/gradient.cpp:899-929);
 *   - gradient2_grid_CPU (src/grid_gradient2_CPU.cpp:54-83) and
 *     module_potentialDerivatives_totalGradient2_SOA (src/gradient2.cpp:226-254);
 *   - amplif_grid_CPU mode 5 (src/grid_amplif_CPU.cpp:38-84);
 *   - delense_barycenter (src/delense_CPU.cpp:6-140) and chi_computation
 *     (src/chi_computation.cpp:11-195), the strong-lensing chi2 by barycentric delensing;
 *   - the GPU kernels module_potential_totalPotential_SOA_GPU (src/potential_GPU.cu:139-187),
 *     module_potentialDerivatives_totalGradient2_SOA_GPU (src/gradient2_GPU.cu:337-398) and
 *     module_potentialDerivatives_Kmap_SOA_GPU (src/gradient2_GPU.cu:455-522), compiled as
 *     host C++ (oracle/cuda_host_stubs.h) and called once per pixel.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include <omp.h>

#include "structure_hpc.hpp"

thread_local lt_dim3_stub threadIdx, blockIdx, blockDim, gridDim;

/* reference entry points (C++ linkage, type_t = double) */
void gradient_grid_CPU(type_t *gx, type_t *gy, const struct grid_param *frame, const struct Potential_SOA *lens,
                       int nhalos, type_t dx, type_t dy, int nx, int ny, int istart, int jstart);
void gradient2_grid_CPU(matrix *g2, const struct grid_param *frame, const struct Potential_SOA *lens, int nhalos,
                        double dx, double dy, int nx, int ny, int istart, int jstart);
void amplif_grid_CPU(type_t *amplif, const struct cosmo_param *cosmo, const struct grid_param *frame,
                     const struct Potential_SOA *lens, int nhalos, int nbgridcells, int mode_amp, type_t z,
                     int istart, int jstart);
struct point module_potentialDerivatives_totalGradient_SOA(const struct point *p, const struct Potential_SOA *lens,
                                                           int nhalos);
struct matrix module_potentialDerivatives_totalGradient2_SOA(const struct point *p, const struct Potential_SOA *lens,
                                                             int nhalos);
void module_potential_totalPotential_SOA_GPU(type_t *pot, const struct Potential_SOA *lens,
                                             const struct grid_param *frame, int nhalos, type_t dx, type_t dy,
                                             int nx, int ny, int istart, int jstart);
void module_potentialDerivatives_totalGradient2_SOA_GPU(type_t *a, type_t *b, type_t *c, type_t *d,
                                                        const struct Potential_SOA *lens,
                                                        const struct grid_param *frame, int nhalos, type_t dx,
                                                        type_t dy, int nx, int ny, int istart, int jstart);
void module_potentialDerivatives_Kmap_SOA_GPU(type_t *a, type_t *b, type_t *c, type_t *d,
                                              const struct Potential_SOA *lens, const struct grid_param *frame,
                                              int nhalos, type_t dx, type_t dy, int nx, int ny, int istart,
                                              int jstart);
type_t module_potential_81_SOA_GPU(const struct point *p, const struct Potential_SOA *lens, int shalos, int nhalos);
void delense_barycenter(struct point *image_pos, int *locimagesfound, int *numimg, const runmode_param *runmode,
                        const struct Potential_SOA *lens, const struct grid_param *frame,
                        const int *nimages_strongLensing, const struct galaxy *sources, double *grid_gradient_x,
                        double *grid_gradient_y);
void chi_computation(double *chi, int *images_found, int *numimagesfound, struct point *imagesposition,
                     const int *nimages_strongLensing, const galaxy *images, const int nsets);

/* amplif_grid_CPU links against the reference's cosmology module, which needs GSL
 * (absent).  Mode 5 computes dl0s and never uses it; this stand-in returns 0. */
type_t module_cosmodistances_objectObject(type_t, type_t, cosmo_param) { return 0.; }

namespace {

/* A Potential_SOA view over caller arrays with the sentinel slot type[n] that the
 * reference's run dispatch reads (src/gradient.cpp:912). */
struct SoaView {
    Potential_SOA soa;
    std::vector<int> type;
    std::vector<double> z;
    SoaView(int n, const int *t, const double *x, const double *y, const double *cs, const double *sn,
            const double *eps, const double *rc, const double *rcut, const double *b0, const double *dlsds)
        : type(t, t + n), z(n > 0 ? n : 1, 0.4)
    {
        memset(&soa, 0, sizeof(soa));
        type.push_back(-1);
        soa.type = type.data();
        soa.position_x = const_cast<double *>(x);
        soa.position_y = const_cast<double *>(y);
        soa.anglecos = const_cast<double *>(cs);
        soa.anglesin = const_cast<double *>(sn);
        soa.ellipticity_potential = const_cast<double *>(eps);
        soa.rcore = const_cast<double *>(rc);
        soa.rcut = const_cast<double *>(rcut);
        soa.b0 = const_cast<double *>(b0);
        soa.dlsds = const_cast<double *>(dlsds);
        soa.z = z.data();
    }
};

grid_param make_frame(double xmin, double ymin)
{
    grid_param f;
    memset(&f, 0, sizeof(f));
    f.xmin = xmin;
    f.ymin = ymin;
    return f;
}

} // namespace

#define SOA_ARGS int n, const int *t, const double *x, const double *y, const double *cs, const double *sn, \
                 const double *eps, const double *rc, const double *rcut, const double *b0, const double *dlsds
#define SOA_PASS n, t, x, y, cs, sn, eps, rc, rcut, b0, dlsds

extern "C" {

int ltref_grad_grid(SOA_ARGS, double xmin, double ymin, double dx, double dy, int nx, int ny, int istart,
                    int jstart, double *ax, double *ay)
{
    SoaView v(SOA_PASS);
    grid_param f = make_frame(xmin, ymin);
    gradient_grid_CPU(ax, ay, &f, &v.soa, n, dx, dy, nx, ny, istart, jstart);
    return 0;
}

int ltref_hess_grid(SOA_ARGS, double xmin, double ymin, double dx, double dy, int nx, int ny, int istart,
                    int jstart, double *a, double *b, double *c, double *d)
{
    SoaView v(SOA_PASS);
    grid_param f = make_frame(xmin, ymin);
    std::vector<matrix> m((size_t)nx * ny);
    gradient2_grid_CPU(m.data(), &f, &v.soa, n, dx, dy, nx, ny, istart, jstart);
    for (size_t k = 0; k < m.size(); k++) {
        a[k] = m[k].a; b[k] = m[k].b; c[k] = m[k].c; d[k] = m[k].d;
    }
    return 0;
}

/* amplif_grid_CPU derives dx, dy from the frame of a square nbgridcells grid. */
int ltref_amplif5_grid(SOA_ARGS, double xmin, double xmax, double ymin, double ymax, int nbgridcells,
                       double *out)
{
    SoaView v(SOA_PASS);
    grid_param f;
    memset(&f, 0, sizeof(f));
    f.xmin = xmin; f.xmax = xmax; f.ymin = ymin; f.ymax = ymax;
    cosmo_param cosmo;
    memset(&cosmo, 0, sizeof(cosmo));
    amplif_grid_CPU(out, &cosmo, &f, &v.soa, n, nbgridcells, 5, 1.5, 0, 0);
    return 0;
}

int ltref_grad_points(SOA_ARGS, long np, const double *px, const double *py, double *ax, double *ay)
{
    SoaView v(SOA_PASS);
#pragma omp parallel for schedule(dynamic, 64)
    for (long k = 0; k < np; k++) {
        point p = {px[k], py[k]};
        point g = module_potentialDerivatives_totalGradient_SOA(&p, &v.soa, n);
        ax[k] = g.x;
        ay[k] = g.y;
    }
    return 0;
}

int ltref_hess_points(SOA_ARGS, long np, const double *px, const double *py, double *a, double *b, double *c,
                      double *d)
{
    SoaView v(SOA_PASS);
#pragma omp parallel for schedule(dynamic, 64)
    for (long k = 0; k < np; k++) {
        point p = {px[k], py[k]};
        matrix m = module_potentialDerivatives_totalGradient2_SOA(&p, &v.soa, n);
        a[k] = m.a; b[k] = m.b; c[k] = m.c; d[k] = m.d;
    }
    return 0;
}

/* dPIE potential at points: module_potential_81_SOA_GPU over the whole catalogue
 * (every halo must be type 81; the reference has no other potential). */
int ltref_pot81_points(SOA_ARGS, long np, const double *px, const double *py, double *psi)
{
    SoaView v(SOA_PASS);
    for (int i = 0; i < n; i++)
        if (t[i] != 81) return 2;
#pragma omp parallel for schedule(dynamic, 64)
    for (long k = 0; k < np; k++) {
        point p = {px[k], py[k]};
        psi[k] = module_potential_81_SOA_GPU(&p, &v.soa, 0, n);
    }
    return 0;
}

/* Run one reference GPU grid kernel on the CPU: one call per pixel, with the pixel's
 * launch indices set as blockIdx (blockDim 1x1). */
enum { KERNEL_POT = 0, KERNEL_HESS = 1, KERNEL_KMAP = 2 };

int ltref_gpu_kernel_grid(int which, SOA_ARGS, double xmin, double ymin, double dx, double dy, int nx, int ny,
                          int istart, int jstart, double *o0, double *o1, double *o2, double *o3)
{
    SoaView v(SOA_PASS);
    grid_param f = make_frame(xmin, ymin);
#pragma omp parallel for schedule(dynamic, 16)
    for (int row = 0; row < ny; row++) {
        blockDim.x = blockDim.y = blockDim.z = 1;
        threadIdx.x = threadIdx.y = threadIdx.z = 0;
        for (int col = 0; col < nx; col++) {
            blockIdx.x = col;
            blockIdx.y = row;
            blockIdx.z = 0;
            if (which == KERNEL_POT)
                module_potential_totalPotential_SOA_GPU(o0, &v.soa, &f, n, dx, dy, nx, ny, istart, jstart);
            else if (which == KERNEL_HESS)
                module_potentialDerivatives_totalGradient2_SOA_GPU(o0, o1, o2, o3, &v.soa, &f, n, dx, dy, nx, ny,
                                                                   istart, jstart);
            else
                module_potentialDerivatives_Kmap_SOA_GPU(o0, o1, o2, o3, &v.soa, &f, n, dx, dy, nx, ny, istart,
                                                         jstart);
        }
    }
    return 0;
}

/* Strong-lensing chi2 of one model as mychi_bruteforce_SOA_CPU_grid_gradient_barycentersource
 * computes it (src/chi_CPU_barycenter.cpp:58-287) on one process: the deflection grid
 * (gradient_grid_CPU over the frame, dx = (xmax - xmin)/(n - 1)), each system's source as
 * the barycentre of its images mapped with the exact deflection at the image
 * (:180-214), delense_barycenter on one thread (the reference's serial order; its OpenMP
 * critical section makes the order of predicted images thread-dependent), the
 * single-rank part of delense_comm (src/chi_comm.cpp:33-77: a copy), chi_computation.
 * That driver itself includes mpi.h unconditionally (through chi_comm.hpp) and is not
 * built here; its steps are repeated in this order. */
int ltref_chi2(SOA_ARGS, double xmin, double xmax, double ymin, double ymax, int nb, int nsys, const int *nimg,
               const double *ix, const double *iy, const double *dr, double *chi2, int *images_found, int *nfound,
               double *fx, double *fy)
{
    SoaView v(SOA_PASS);
    grid_param frame;
    memset(&frame, 0, sizeof(frame));
    frame.xmin = xmin;
    frame.xmax = xmax;
    frame.ymin = ymin;
    frame.ymax = ymax;
    const double dx = (frame.xmax - frame.xmin) / (nb - 1);
    const double dy = (frame.ymax - frame.ymin) / (nb - 1);
    std::vector<double> gx((size_t)nb * nb), gy((size_t)nb * nb);
    gradient_grid_CPU(gx.data(), gy.data(), &frame, &v.soa, n, dx, dy, nb, nb, 0, 0);
    int total = 0;
    for (int s = 0; s < nsys; s++) total += nimg[s];
    std::vector<galaxy> images((size_t)(total > 0 ? total : 1));
    memset(images.data(), 0, sizeof(galaxy) * images.size());
    int idx = 0;
    for (int s = 0; s < nsys; s++)
        for (int i = 0; i < nimg[s]; i++, idx++) {
            images[idx].center.x = ix[idx];
            images[idx].center.y = iy[idx];
            images[idx].dr = dr[s];
        }
    std::vector<galaxy> sources((size_t)nsys);
    idx = 0;
    for (int s = 0; s < nsys; s++) {
        sources[s].center.x = sources[s].center.y = 0.;
        for (int i = 0; i < nimg[s]; i++) {
            point Grad = module_potentialDerivatives_totalGradient_SOA(&images[idx + i].center, &v.soa, n);
            sources[s].center.x += images[idx + i].center.x - images[idx + i].dr * Grad.x;
            sources[s].center.y += images[idx + i].center.y - images[idx + i].dr * Grad.y;
        }
        sources[s].center.x /= nimg[s];
        sources[s].center.y /= nimg[s];
        sources[s].dr = images[idx].dr;
        idx += nimg[s];
    }
    runmode_param rm;
    memset(&rm, 0, sizeof(rm));
    rm.nsets = nsys;
    rm.nbgridcells = nb;
    rm.nhalos = n;
    std::vector<point> image_pos((size_t)nsys * MAXIMPERSOURCE);
    memset(image_pos.data(), 0, sizeof(point) * image_pos.size());
    std::vector<int> loc((size_t)nsys, 0);
    int numimg = 0;
    const int threads = omp_get_max_threads();
    omp_set_num_threads(1);
    delense_barycenter(image_pos.data(), loc.data(), &numimg, &rm, &v.soa, &frame, nimg, sources.data(), gx.data(),
                       gy.data());
    omp_set_num_threads(threads);
    std::vector<int> numfound((size_t)nsys, 0);
    std::vector<point> pos((size_t)nsys * MAXIMPERSOURCE);
    memset(pos.data(), 0, sizeof(point) * pos.size());
    if (numimg != 0)
        for (int s = 0; s < nsys; s++) {
            if (loc[s] == 0) continue;
            memcpy(&pos[(size_t)s * MAXIMPERSOURCE + numfound[s]], &image_pos[(size_t)s * MAXIMPERSOURCE],
                   loc[s] * sizeof(point));
            numfound[s] += loc[s];
        }
    double chi = 0.;
    int found = 0;
    chi_computation(&chi, &found, numfound.data(), pos.data(), nimg, images.data(), nsys);
    *chi2 = chi;
    *images_found = found;
    for (int s = 0; s < nsys; s++) {
        nfound[s] = numfound[s];
        for (int k = 0; k < numfound[s] && k < MAXIMPERSOURCE; k++) {
            fx[s * MAXIMPERSOURCE + k] = pos[(size_t)s * MAXIMPERSOURCE + k].x;
            fy[s * MAXIMPERSOURCE + k] = pos[(size_t)s * MAXIMPERSOURCE + k].y;
        }
    }
    return 0;
}

} // extern "C"
