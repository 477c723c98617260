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
 *   - module_readParameters_setbayesmapmodels (src/module_readParameters.cpp:132-227) with
 *     setScalingRelations and the potential-parameter step, a bayes.dat row's update;
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

/* ---- bayes.dat rows: module_readParameters_setbayesmapmodels ------------------------ */

#include <float.h>

#include "module_readParameters.hpp"

/* module_readParameters.cpp needs the observer distance only for potfile lengths given
 * in kpc, which these calls never pass (the GSL-based cosmology module is absent). */
type_t module_cosmodistances_observerObject(type_t, cosmo_param) { abort(); }

extern "C" {

/* The reference's own per-row update (src/module_readParameters.cpp:132-227, with
 * setScalingRelations :1539-1656 and the potential-parameter step :2873-2936) applied to
 * rows 0..nrows-1 in turn.  Halos 0..nhalos-1 are the parameter-file halos (SOA_index =
 * identity), halos nhalos..ntot-1 the potfile galaxies, potfile after potfile.  The model
 * state is first taken to the fixed point of the potential-parameter step (three passes
 * of the reference's function).  free_flags: nhalos x 9 in the order x, y, epot, emass,
 * theta, rcore, vdisp, rcut, z; pot_params: npot x 7 (count, mag0, sigma, cut, core,
 * vdslope, slope); pot_free: npot x 2 (ircut, isigma).  out: nrows x 8 x ntot (x, y, b0,
 * epot, cos, sin, rcore, rcut). */
int ltref_bayes_rows(int nhalos, int ntot, const int *type, const double *x, const double *y, const double *epot,
                     const double *emass, const double *theta, const double *rcore, const double *vdisp,
                     const double *rcut, const double *mag, const int *free_flags, int n_z_param, int npot,
                     const double *pot_params, const int *pot_free, int nparam, int nrows, const double *rows,
                     double *out)
{
    if (npot > N_MAX_POTFILE) return -1;
    std::vector<int> t(type, type + ntot), soa_index((size_t)ntot);
    std::vector<double> f[16];
    for (auto &v : f) v.assign((size_t)ntot, 0.);
    Potential_SOA L;
    memset(&L, 0, sizeof(L));
    L.type = t.data();
    L.position_x = f[0].data();
    L.position_y = f[1].data();
    L.b0 = f[2].data();
    L.vdisp = f[3].data();
    L.ellipticity_angle = f[4].data();
    L.ellipticity = f[5].data();
    L.ellipticity_potential = f[6].data();
    L.rcore = f[7].data();
    L.rcut = f[8].data();
    L.z = f[9].data();
    L.mag = f[10].data();
    L.anglecos = f[11].data();
    L.anglesin = f[12].data();
    L.dlsds = f[13].data();
    L.SOA_index = soa_index.data();
    for (int i = 0; i < ntot; i++) {
        soa_index[i] = i;
        L.position_x[i] = x[i];
        L.position_y[i] = y[i];
        L.vdisp[i] = vdisp[i];
        L.ellipticity_angle[i] = theta[i];
        L.ellipticity[i] = emass[i];
        L.ellipticity_potential[i] = epot[i];
        L.rcore[i] = rcore[i];
        L.rcut[i] = rcut[i];
        L.mag[i] = mag ? mag[i] : 0.;
        L.anglecos[i] = cos(theta[i]);
        L.anglesin[i] = sin(theta[i]);
    }
    for (int it = 0; it < 3; it++)
        for (int i = 0; i < ntot; i++) module_readParameters_calculatePotentialparameter_SOA(&L, i);
    runmode_param rm = runmode_param();
    rm.nhalos = nhalos;
    rm.n_tot_halos = ntot;
    rm.N_z_param = n_z_param;
    rm.potfile = npot > 0;
    rm.Nb_potfile = npot;
    cosmo_param cosmo;
    memset(&cosmo, 0, sizeof(cosmo));
    std::vector<potentialoptimization> lim((size_t)(nhalos > 0 ? nhalos : 1));
    memset(lim.data(), 0, sizeof(potentialoptimization) * lim.size());
    for (int i = 0; i < nhalos; i++) {
        const int *fl = free_flags + 9 * i;
        lim[i].position.x.block = fl[0];
        lim[i].position.y.block = fl[1];
        lim[i].ellipticity_potential.block = fl[2];
        lim[i].ellipticity.block = fl[3];
        lim[i].ellipticity_angle.block = fl[4];
        lim[i].rcore.block = fl[5];
        lim[i].vdisp.block = fl[6];
        lim[i].rcut.block = fl[7];
        lim[i].z.block = fl[8];
    }
    std::vector<potfile_param> pf((size_t)(npot > 0 ? npot : 1));
    memset(pf.data(), 0, sizeof(potfile_param) * pf.size());
    for (int k = 0; k < npot; k++) {
        const double *q = pot_params + 7 * k;
        potfile_param &p = pf[k];
        p.ftype = 1;
        p.npotfile = (int)q[0];
        rm.npotfile[k] = p.npotfile;
        p.mag0 = q[1];
        p.sigma1 = q[2];
        p.cut1 = q[3];
        p.cutkpc1 = DBL_MAX;
        p.core = q[4];
        p.corekpc = -1;
        p.vdslope1 = q[5];
        p.slope1 = q[6];
        p.ircut = pot_free[2 * k];
        p.isigma = pot_free[2 * k + 1];
    }
    std::vector<double> bayespot(rows, rows + (size_t)nrows * nparam);
    for (int r = 0; r < nrows; r++) {
        module_readParameters_setbayesmapmodels(&rm, &cosmo, lim.data(), pf.data(), &L, bayespot.data(), nparam, r);
        double *o = out + (size_t)r * 8 * ntot;
        for (int i = 0; i < ntot; i++) {
            o[0 * ntot + i] = L.position_x[i];
            o[1 * ntot + i] = L.position_y[i];
            o[2 * ntot + i] = L.b0[i];
            o[3 * ntot + i] = L.ellipticity_potential[i];
            o[4 * ntot + i] = L.anglecos[i];
            o[5 * ntot + i] = L.anglesin[i];
            o[6 * ntot + i] = L.rcore[i];
            o[7 * ntot + i] = L.rcut[i];
        }
    }
    return 0;
}

} // extern "C"
