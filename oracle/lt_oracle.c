/*
 * lt_oracle.c -- CPU restatement of Lenstool-HPC's lensing-map arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may call it; the product library never links it.
 *
 * Every function cites the reference lines it restates (paths relative to the
 * Lenstool-HPC source tree).  The per-pair arithmetic keeps the reference's operation
 * order so that FP64 results agree to rounding.  Three pieces have no reference
 * source and are restated from the mathematics (parity for them is pinned by finite
 * differences of the reference-backed pieces, see tests/test_oracle.py):
 *   - SIS Hessian (derivative of src/gradient.cpp:260-299),
 *   - PIEMD Hessian (one mdci05 term, src/gradient2.cpp:54-83, without the cut),
 *   - SIS and PIEMD potential (SIS: b0*R; PIEMD: one pi05 term).
 *
 * Halo catalogue: the Potential_SOA field meaning of src/structure_hpc.hpp:257-287,
 * sorted into runs of equal type (src/module_readParameters.cpp:2289-2293).  Unlike
 * the reference, no sentinel slot type[n] is read.
 */
#include <math.h>
#include <stddef.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* LTO_EXTENDED builds the same arithmetic in x87 extended precision (64-bit mantissa),
 * liblt_oracle_ld.so: the difference between the two builds measures the FP64 rounding
 * error of the reference's own formulas at each pixel. */
#ifdef LTO_EXTENDED
#include <tgmath.h>
typedef long double real;
#else
typedef double real;
#endif

typedef struct {
    int n;
    const int *type;
    const double *x, *y;     /* position_x, position_y */
    const double *cs, *sn;   /* anglecos, anglesin */
    const double *eps;       /* ellipticity_potential */
    const double *rc, *rcut; /* rcore, rcut */
    const double *b0;        /* impact parameter */
    const double *dlsds;     /* per-halo D_LS/D_OS (Kmap weights); may be NULL */
} lto_cat;

typedef struct {
    double xmin, ymin, dx, dy;
    int nx, ny, istart, jstart;
} lto_grid;

enum { LTO_OK = 0, LTO_ERR_PROFILE = 2, LTO_ERR_ARG = 1 };

/* ---------------------------------------------------------------------------------- */
/* gradient                                                                           */
/* ---------------------------------------------------------------------------------- */

/* SIS deflection of halo i, src/gradient.cpp:260-299 (the _v2 variant).  The inverse
 * radius starts from a single-precision square root followed by one Newton step
 * (src/gradient.cpp:287-288). */
static void sis_grad_acc(const lto_cat *c, int i, real px, real py, real *gx, real *gy)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real b0 = c->b0[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    real e = c->eps[i];
    real q = u * u * (1. - e) + v * v * (1. + e);
#ifdef LTO_EXTENDED
    real r = 1. / sqrt(q); /* the exact inverse radius the seed approximates */
#else
    real r = 1. / sqrtf((float)q);
    r = r * (1.5 - 0.5 * q * r * r);
#endif
    real fx = (1. - e) * b0 * u * r;
    real fy = (1. + e) * b0 * v * r;
    *gx += fx * cs - fy * sn;
    *gy += fy * cs + fx * sn;
}

/* One complex-logarithm term of the PIEMD deflection for core radius r: the KERNEL
 * macro of src/gradient.hpp:64-76 (also piemd_1derivatives_ci05, src/gradient.cpp:60-100). */
static void piemd_term(real u, real v, real r, real sqe, real cx1, real rem2,
                       real zci_im, real *re, real *im)
{
    real nre = cx1 * u;
    real nim = 2. * sqe * sqrt(r * r + rem2) - v / cx1;
    real dim = 2. * r * sqe - v;
    real nrm = (u * u + dim * dim);
    real zre = (nre * u + nim * dim) / nrm;
    real zim = (nim * u - nre * dim) / nrm;
    real m = zre;
    real lre = log(sqrt(m * m + zim * zim));
    real lim = atan2(zim, m);
    *re = -zci_im * lim;
    *im = zci_im * lre;
}

/* PIEMD deflection, src/gradient.cpp:548-607. */
static void piemd_grad_acc(const lto_cat *c, int i, real px, real py, real *gx, real *gy)
{
    real b0 = c->b0[i];
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    real e = c->eps[i];
    real rc = c->rc[i];
    real sqe = sqrt(e);
    real cx1 = (1. - e) / (1. + e);
    real cxro = (1. + e) * (1. + e);
    real cyro = (1. - e) * (1. - e);
    real rem2 = u * u / cxro + v * v / cyro;
    real zci_im = -0.5 * (1. - e * e) / sqe;
    real re, im;
    piemd_term(u, v, rc, sqe, cx1, rem2, zci_im, &re, &im);
    *gx += b0 * (re * cs - im * sn);
    *gy += b0 * (im * cs + re * sn);
}

/* Cut dPIE deflection, src/gradient.cpp:744-811: t05 * (K(rcore) - K(rcut)). */
static void dpie_grad_acc(const lto_cat *c, int i, real px, real py, real *gx, real *gy)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    real e = c->eps[i];
    real rc = c->rc[i], rcut = c->rcut[i], b0 = c->b0[i];
    real t05 = b0 * rcut / (rcut - rc);
    real sqe = sqrt(e);
    real cx1 = (1. - e) / (1. + e);
    real cxro = (1. + e) * (1. + e);
    real cyro = (1. - e) * (1. - e);
    real rem2 = u * u / cxro + v * v / cyro;
    real zci_im = -0.5 * (1. - e * e) / sqe;
    real are, aim, bre, bim;
    piemd_term(u, v, rc, sqe, cx1, rem2, zci_im, &are, &aim);
    piemd_term(u, v, rcut, sqe, cx1, rem2, zci_im, &bre, &bim);
    real zre = t05 * (are - bre);
    real zim = t05 * (aim - bim);
    *gx += (zre * cs - zim * sn);
    *gy += (zim * cs + zre * sn);
}

/* Sum over halos at one point, dispatched over runs of equal type:
 * module_potentialDerivatives_totalGradient_SOA, src/gradient.cpp:899-929.  Each run is
 * summed on its own and then added to the total, as the reference does. */
static int grad_point(const lto_cat *c, real px, real py, double *ax, double *ay)
{
    real tx = 0., ty = 0.;
    int s = 0;
    while (s < c->n) {
        int t = c->type[s];
        int e = s + 1;
        while (e < c->n && c->type[e] == t) e++;
        real rx = 0., ry = 0.;
        switch (t) {
        case 5:  for (int i = s; i < e; i++) sis_grad_acc(c, i, px, py, &rx, &ry); break;
        case 8:  for (int i = s; i < e; i++) piemd_grad_acc(c, i, px, py, &rx, &ry); break;
        case 81: for (int i = s; i < e; i++) dpie_grad_acc(c, i, px, py, &rx, &ry); break;
        default: return LTO_ERR_PROFILE;
        }
        tx += rx;
        ty += ry;
        s = e;
    }
    *ax = tx;
    *ay = ty;
    return LTO_OK;
}

/* ---------------------------------------------------------------------------------- */
/* Hessian                                                                            */
/* ---------------------------------------------------------------------------------- */

typedef struct { real a, b, c, d; } lto_mat;

/* Second derivatives of one PIEMD term I0.5 (Kassiola & Kovner 1993):
 * mdci05_hpc, src/gradient2.cpp:54-83. */
static lto_mat mdci05(real x, real y, real eps, real rc, real b0)
{
    real sqe = sqrt(eps);
    real cx1 = (1. - eps) / (1. + eps);
    real cx1inv = 1. / cx1;
    real cxro = (1. + eps) * (1. + eps);
    real cyro = (1. - eps) * (1. - eps);
    real ci = 0.5 * (1. - eps * eps) / sqe;
    real wrem = sqrt(rc * rc + x * x / cxro + y * y / cyro);
    real den1 = 2. * sqe * wrem - y * cx1inv;
    den1 = cx1 * cx1 * x * x + den1 * den1;
    real num2 = 2. * rc * sqe - y;
    real den2 = x * x + num2 * num2;
    real didxre = ci * (cx1 * (2. * sqe * x * x / cxro / wrem - 2. * sqe * wrem + y * cx1inv) / den1 + num2 / den2);
    real didyre = ci * ((2. * sqe * x * y * cx1 / cyro / wrem - x) / den1 + x / den2);
    real didyim = ci * ((2. * sqe * wrem * cx1inv - y * cx1inv * cx1inv - 4. * eps * y / cyro +
                           2. * sqe * y * y / cyro / wrem * cx1inv) / den1 - num2 / den2);
    lto_mat r;
    r.a = b0 * didxre;
    r.b = r.d = b0 * didyre;
    r.c = b0 * didyim;
    return r;
}

/* Rotate a Hessian from the halo frame back to the sky frame, H = R^T H' R, with the
 * two-step order of src/gradient2.cpp:146-156. */
static void rotate_back_acc(lto_mat h, real cs, real sn, lto_mat *acc)
{
    lto_mat m;
    m.a = h.a * cs + h.b * -sn;
    m.b = h.a * sn + h.b * cs;
    m.c = h.d * sn + h.c * cs;
    m.d = h.d * cs + h.c * -sn;
    acc->a += cs * m.a - sn * m.d;
    acc->b += cs * m.b - sn * m.c;
    acc->c += sn * m.b + cs * m.c;
    acc->d += sn * m.a + cs * m.d;
}

/* dPIE Hessian, src/gradient2.cpp:92-205 (elliptical branch, taken for every halo). */
static void dpie_hess_acc(const lto_cat *c, int i, real px, real py, lto_mat *acc)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    real t05 = c->rcut[i] / (c->rcut[i] - c->rc[i]);
    lto_mat core = mdci05(u, v, c->eps[i], c->rc[i], c->b0[i]);
    lto_mat cut = mdci05(u, v, c->eps[i], c->rcut[i], c->b0[i]);
    core.a = t05 * (core.a - cut.a);
    core.b = t05 * (core.b - cut.b);
    core.c = t05 * (core.c - cut.c);
    core.d = t05 * (core.d - cut.d);
    rotate_back_acc(core, cs, sn, acc);
}

/* PIEMD Hessian (restated; the reference has no type-8 Hessian): one mdci05 term with
 * impact parameter b0, the dPIE structure of src/gradient2.cpp:92-156 without the cut. */
static void piemd_hess_acc(const lto_cat *c, int i, real px, real py, lto_mat *acc)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    lto_mat h = mdci05(u, v, c->eps[i], c->rc[i], c->b0[i]);
    rotate_back_acc(h, cs, sn, acc);
}

/* SIS Hessian (restated): derivative of the deflection of src/gradient.cpp:260-299.
 * With R^2 = (1-e)u^2 + (1+e)v^2 in the halo frame:
 *   psi_uu = b0 (1-e)(1+e) v^2 / R^3,  psi_vv = b0 (1-e)(1+e) u^2 / R^3,
 *   psi_uv = -b0 (1-e)(1+e) u v / R^3. */
static void sis_hess_acc(const lto_cat *c, int i, real px, real py, lto_mat *acc)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    real u = tx * cs + ty * sn;
    real v = ty * cs - tx * sn;
    real e = c->eps[i];
    real q = u * u * (1. - e) + v * v * (1. + e);
    real r = sqrt(q);
    real k = c->b0[i] * (1. - e) * (1. + e) / (q * r);
    lto_mat h;
    h.a = k * v * v;
    h.c = k * u * u;
    h.b = h.d = -k * u * v;
    rotate_back_acc(h, cs, sn, acc);
}

/* Hessian at one point, run-dispatched as module_potentialDerivatives_totalGradient2_SOA
 * (src/gradient2.cpp:226-254).  With kmap != 0 the runs also break where dlsds changes
 * and each run is weighted by its dlsds: module_potentialDerivatives_Kmap_SOA_GPU,
 * src/gradient2_GPU.cu:455-522. */
static int hess_point(const lto_cat *c, real px, real py, int kmap, lto_mat *out)
{
    lto_mat tot = {0., 0., 0., 0.};
    int s = 0;
    while (s < c->n) {
        int t = c->type[s];
        real w = kmap ? c->dlsds[s] : 1.;
        int e = s + 1;
        while (e < c->n && c->type[e] == t && (!kmap || c->dlsds[e] == w)) e++;
        lto_mat r = {0., 0., 0., 0.};
        switch (t) {
        case 5:  for (int i = s; i < e; i++) sis_hess_acc(c, i, px, py, &r); break;
        case 8:  for (int i = s; i < e; i++) piemd_hess_acc(c, i, px, py, &r); break;
        case 81: for (int i = s; i < e; i++) dpie_hess_acc(c, i, px, py, &r); break;
        default: return LTO_ERR_PROFILE;
        }
        if (kmap) {
            tot.a += r.a * w; tot.b += r.b * w; tot.c += r.c * w; tot.d += r.d * w;
        } else {
            tot.a += r.a; tot.b += r.b; tot.c += r.c; tot.d += r.d;
        }
        s = e;
    }
    *out = tot;
    return LTO_OK;
}

/* ---------------------------------------------------------------------------------- */
/* potential                                                                          */
/* ---------------------------------------------------------------------------------- */

typedef struct { real re, im; } lto_cpx;

static lto_cpx cx_add(lto_cpx a, lto_cpx b) { lto_cpx r = {a.re + b.re, a.im + b.im}; return r; }
static lto_cpx cx_sub(lto_cpx a, lto_cpx b) { lto_cpx r = {a.re - b.re, a.im - b.im}; return r; }
static lto_cpx cx_mul(lto_cpx a, lto_cpx b)
{
    lto_cpx r = {a.re * b.re - a.im * b.im, a.im * b.re + b.im * a.re};
    return r;
}
static lto_cpx cx_scale(lto_cpx a, real f) { lto_cpx r = {a.re * f, a.im * f}; return r; }
static lto_cpx cx_sq(lto_cpx a) { lto_cpx r = {a.re * a.re - a.im * a.im, 2. * a.re * a.im}; return r; }
/* a/b, zero when |b| = 0 (dcpx_GPU, src/lt_math_GPU.cuh:224-243). */
static lto_cpx cx_div(lto_cpx a, lto_cpx b)
{
    real n = b.re * b.re + b.im * b.im;
    lto_cpx r = {0., 0.};
    if (n != 0.) {
        r.re = (a.re * b.re + a.im * b.im) / n;
        r.im = (a.im * b.re - a.re * b.im) / n;
    }
    return r;
}
static lto_cpx cx_cosh(lto_cpx a)
{
    real ep = exp(a.re), em = exp(-a.re);
    lto_cpx r = {0.5 * (ep + em) * cos(a.im), 0.5 * (ep - em) * sin(a.im)};
    return r;
}
static lto_cpx cx_sinh(lto_cpx a)
{
    real ep = exp(a.re), em = exp(-a.re);
    lto_cpx r = {0.5 * (ep - em) * cos(a.im), 0.5 * (ep + em) * sin(a.im)};
    return r;
}
static lto_cpx cx_log(lto_cpx a)
{
    lto_cpx r = {log(sqrt(a.re * a.re + a.im * a.im)), atan2(a.im, a.re)};
    return r;
}

/* Potential of one PIEMD term I0.5 at (x, y) in the halo frame: pi05_gpu,
 * src/potential_GPU.cu:47-72, with the complex helpers of src/lt_math_GPU.cuh. */
static real pi05(real x, real y, real eps, real rc, real b0)
{
    real sqe = sqrt(eps);
    real ci = .5 * (1. - eps * eps) / sqe;
    real cxro = (1. + eps) * (1. + eps);
    real cyro = (1. - eps) * (1. - eps);
    real rem2 = x * x / cxro + y * y / cyro;
    real e1 = 2. * sqe / (1 - eps);
    real e2 = 2. * sqe / (1 + eps);
    real z = sqrt(x * x + y * y);
    lto_cpx eta = {-.5 * asinh(e1 * y / z), .5 * asin(e2 * x / z)};
    lto_cpx zeta = {0.5 * log((sqrt(rem2) + sqrt(rc * rc + rem2)) / rc), 0.};
    lto_cpx b1 = cx_cosh(cx_add(eta, zeta));
    lto_cpx b2 = cx_cosh(cx_sub(eta, zeta));
    lto_cpx a1 = cx_log(cx_div(cx_sq(cx_cosh(eta)), cx_mul(b1, b2)));
    lto_cpx a2 = cx_log(cx_div(b1, b2));
    lto_cpx c1 = cx_mul(cx_sinh(cx_scale(eta, 2.)), a1);
    lto_cpx c2 = cx_mul(cx_sinh(cx_scale(zeta, 2.)), a2);
    lto_cpx ckk = cx_add(c1, c2);
    return b0 * ci * rc / sqrt(rem2) * (ckk.im * x - ckk.re * y);
}

static void halo_frame(const lto_cat *c, int i, real px, real py, real *u, real *v)
{
    real tx = px - c->x[i], ty = py - c->y[i];
    real cs = c->cs[i], sn = c->sn[i];
    *u = tx * cs + ty * sn;
    *v = ty * cs - tx * sn;
}

/* Potential at one point: module_potential_totalPotential_SOA_GPU and
 * module_potential_81_SOA_GPU, src/potential_GPU.cu:75-187 (dPIE); SIS (b0 R) and
 * PIEMD (one pi05 term) are restated. */
static int pot_point(const lto_cat *c, real px, real py, double *out)
{
    real tot = 0.;
    int s = 0;
    while (s < c->n) {
        int t = c->type[s];
        int e = s + 1;
        while (e < c->n && c->type[e] == t) e++;
        real r = 0.;
        for (int i = s; i < e; i++) {
            real u, v;
            halo_frame(c, i, px, py, &u, &v);
            if (t == 81) {
                real t05 = c->rcut[i] / (c->rcut[i] - c->rc[i]);
                real pa = pi05(u, v, c->eps[i], c->rc[i], c->b0[i]);
                real ps = pi05(u, v, c->eps[i], c->rcut[i], c->b0[i]);
                r += t05 * (pa - ps);
            } else if (t == 8) {
                r += pi05(u, v, c->eps[i], c->rc[i], c->b0[i]);
            } else if (t == 5) {
                real e_ = c->eps[i];
                r += c->b0[i] * sqrt(u * u * (1. - e_) + v * v * (1. + e_));
            } else {
                return LTO_ERR_PROFILE;
            }
        }
        tot += r;
        s = e;
    }
    *out = tot;
    return LTO_OK;
}

/* ---------------------------------------------------------------------------------- */
/* grids and point lists                                                              */
/* ---------------------------------------------------------------------------------- */

/* Pixel (ii, jj) sits at xmin + (ii + istart) dx, ymin + (jj + jstart) dy and is stored
 * at jj*nx + ii: gradient_grid_general_CPU, src/grid_gradient_CPU.cpp:67-100. */
static void pixel_xy(const lto_grid *g, long p, real *px, real *py)
{
    int ii = (int)(p % g->nx), jj = (int)(p / g->nx);
    *px = g->xmin + (ii + g->istart) * g->dx;
    *py = g->ymin + (jj + g->jstart) * g->dy;
}

static void set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int lto_grad_grid(const lto_cat *c, const lto_grid *g, double *ax, double *ay, int nthreads)
{
    long np = (long)g->nx * g->ny;
    int bad = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long p = 0; p < np; p++) {
        real px, py;
        pixel_xy(g, p, &px, &py);
        bad |= grad_point(c, px, py, &ax[p], &ay[p]);
    }
    return bad;
}

int lto_hess_grid(const lto_cat *c, const lto_grid *g, int kmap, double *a, double *b,
                  double *cc, double *d, int nthreads)
{
    long np = (long)g->nx * g->ny;
    int bad = 0;
    if (kmap && !c->dlsds) return LTO_ERR_ARG;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long p = 0; p < np; p++) {
        real px, py;
        lto_mat m;
        pixel_xy(g, p, &px, &py);
        bad |= hess_point(c, px, py, kmap, &m);
        a[p] = m.a; b[p] = m.b; cc[p] = m.c; d[p] = m.d;
    }
    return bad;
}

int lto_pot_grid(const lto_cat *c, const lto_grid *g, double *psi, int nthreads)
{
    long np = (long)g->nx * g->ny;
    int bad = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long p = 0; p < np; p++) {
        real px, py;
        pixel_xy(g, p, &px, &py);
        bad |= pot_point(c, px, py, &psi[p]);
    }
    return bad;
}

/* Point-list forms: the same sums at arbitrary (px[k], py[k]). */
int lto_grad_points(const lto_cat *c, long np, const double *px, const double *py,
                    double *ax, double *ay, int nthreads)
{
    int bad = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long k = 0; k < np; k++) bad |= grad_point(c, px[k], py[k], &ax[k], &ay[k]);
    return bad;
}

int lto_hess_points(const lto_cat *c, long np, const double *px, const double *py, int kmap,
                    double *a, double *b, double *cc, double *d, int nthreads)
{
    int bad = 0;
    if (kmap && !c->dlsds) return LTO_ERR_ARG;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long k = 0; k < np; k++) {
        lto_mat m;
        bad |= hess_point(c, px[k], py[k], kmap, &m);
        a[k] = m.a; b[k] = m.b; cc[k] = m.c; d[k] = m.d;
    }
    return bad;
}

int lto_pot_points(const lto_cat *c, long np, const double *px, const double *py, double *psi,
                   int nthreads)
{
    int bad = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (long k = 0; k < np; k++) bad |= pot_point(c, px[k], py[k], &psi[k]);
    return bad;
}

/* ---------------------------------------------------------------------------------- */
/* map epilogues                                                                      */
/* ---------------------------------------------------------------------------------- */

/* Eigenvalues of the symmetric 2x2 matrix [[a, b], [b, c]]: formeli_ampli,
 * src/grid_map_ampli_GPU.cu:549-572 (the orientation is not used by any map). */
static void eigen2(real a, real b, real c, real *lam, real *mu)
{
    real delta = (a - c) * (a - c) + 4 * b * b;
    real e = sqrt(delta);
    *lam = .5 * (a + c + e);
    *mu = .5 * (a + c - e);
}

/* Map kinds (one plane each). */
enum {
    LTO_MAP_AMPLI1 = 1, LTO_MAP_AMPLI2, LTO_MAP_AMPLI3, LTO_MAP_AMPLI4, LTO_MAP_AMPLI5, LTO_MAP_AMPLI6,
    LTO_MAP_SHEAR1 = 11, LTO_MAP_SHEAR2, LTO_MAP_SHEAR3, LTO_MAP_SHEAR4,
    LTO_MAP_KAPPA = 21, LTO_MAP_GAMMA1, LTO_MAP_GAMMA2, LTO_MAP_MU, LTO_MAP_SCALE
};

/* One derived map from the Hessian planes, D = dls/ds.
 *  ampli 1-6: src/grid_map_ampli_GPU.cu:329-547;  shear 1-4: src/grid_map_shear_GPU.cu:208-369;
 *  kappa/gamma1/gamma2/mu: the D-scaled convergence, shear components and
 *  magnification 1/((1-k)^2 - g1^2 - g2^2);
 *  LTO_MAP_SCALE: (a + c)/2 * scale (mass maps, src/grid_map_mass_GPU.cu:307-322). */
int lto_map(int kind, long np, const double *a, const double *b, const double *c, double D,
            double scale, double *out)
{
    for (long p = 0; p < np; p++) {
        real A = 1. - a[p] * D, B = -b[p] * D, C = 1. - c[p] * D;
        real lam, mu, r;
        switch (kind) {
        case LTO_MAP_AMPLI1: eigen2(A, B, C, &lam, &mu); r = 1. / (lam * mu); break;
        case LTO_MAP_AMPLI2: eigen2(A, B, C, &lam, &mu); r = 1. / fabs(lam * mu); break;
        case LTO_MAP_AMPLI3: eigen2(A, B, C, &lam, &mu); r = -2.5 * log10(fabs(lam * mu)); break;
        case LTO_MAP_AMPLI4: {
            real k = (a[p] + c[p]) * D / 2.;
            real g1 = (a[p] - c[p]) * D / 2.;
            real g2 = b[p] * D;
            real g = sqrt(g1 * g1 + g2 * g2);
            real gp = g / (1 - k);
            r = (1 - k) * (1 + gp * gp) / (1 - gp * gp);
            break;
        }
        case LTO_MAP_AMPLI5: r = (a[p] + c[p]) / 2.; break;
        case LTO_MAP_AMPLI6: {
            real g1 = (a[p] - c[p]) / 2.;
            real g2 = b[p];
            r = sqrt(g1 * g1 + g2 * g2);
            break;
        }
        case LTO_MAP_SHEAR1: eigen2(A, B, C, &lam, &mu); r = (lam - mu) / 2.; break;
        case LTO_MAP_SHEAR2: {
            eigen2(A, B, C, &lam, &mu);
            real q = lam / mu;
            r = fabs((q * q - 1.) / (q * q + 1.));
            break;
        }
        case LTO_MAP_SHEAR3: r = (a[p] - c[p]) * D / 2.; break;
        case LTO_MAP_SHEAR4: r = b[p] * D; break;
        case LTO_MAP_KAPPA: r = (a[p] + c[p]) * D / 2.; break;
        case LTO_MAP_GAMMA1: r = (a[p] - c[p]) * D / 2.; break;
        case LTO_MAP_GAMMA2: r = b[p] * D; break;
        case LTO_MAP_MU: {
            real k = (a[p] + c[p]) * D / 2.;
            real g1 = (a[p] - c[p]) * D / 2.;
            real g2 = b[p] * D;
            r = 1. / ((1. - k) * (1. - k) - g1 * g1 - g2 * g2);
            break;
        }
        case LTO_MAP_SCALE: r = (a[p] + c[p]) * 0.5 * scale; break;
        default: return LTO_ERR_ARG;
        }
        out[p] = r;
    }
    return LTO_OK;
}

/* ---------------------------------------------------------------------------------- */
/* strong-lensing chi2 by barycentric delensing                                       */
/* ---------------------------------------------------------------------------------- */

/* At most this many predicted images per source (MAXIMPERSOURCE,
 * src/structure_hpc.hpp:41); a source with more reports LTO_ERR_ARG. */
#define LTO_MAXIMG 20

/* Source of each multiple-image system: the mean of its images' source-plane positions
 * theta - dr alpha(theta), alpha evaluated at each observed image
 * (src/chi_CPU_barycenter.cpp:180-214). */
int lto_source_barycenters(const lto_cat *c, int nsys, const int *nimg, const double *ix, const double *iy,
                           const double *dr, double *bx, double *by)
{
    int idx = 0;
    for (int s = 0; s < nsys; s++) {
        double sx = 0., sy = 0.;
        for (int i = 0; i < nimg[s]; i++) {
            double ax, ay;
            int st = grad_point(c, ix[idx + i], iy[idx + i], &ax, &ay);
            if (st) return st;
            sx += ix[idx + i] - dr[s] * ax;
            sy += iy[idx + i] - dr[s] * ay;
        }
        bx[s] = sx / nimg[s];
        by[s] = sy / nimg[s];
        idx += nimg[s];
    }
    return LTO_OK;
}

typedef struct { double x, y; } lto_pt;

/* mychi_determinant, src/delense_CPU_utils.hpp:127-136 */
static double tri_det(lto_pt A, lto_pt B, lto_pt C)
{
    return B.x * C.y - B.y * C.x + A.x * B.y - A.y * B.x + A.y * C.x - A.x * C.y;
}

/* mychi_inside / mychi_insideborder (identical tests), src/delense_CPU_utils.hpp:146-209 */
static int tri_inside(lto_pt P, lto_pt a, lto_pt b, lto_pt cc)
{
    double d = tri_det(a, b, cc);
    if (tri_det(a, b, P) * d < 0.) return 0;
    if (tri_det(b, cc, P) * d < 0.) return 0;
    if (tri_det(cc, a, P) * d < 0.) return 0;
    return 1;
}

/* delense_barycenter, src/delense_CPU.cpp:6-140, in its serial order (rows, then
 * columns; the upper triangle of a cell is tested first): every grid cell whose upper or
 * lower triangle, mapped to the source plane with the deflection grid (ax, ay: n x n,
 * pixel (i, j) at xmin + i dx, ymin + j dy, dx = (xmax - xmin)/(n - 1)), contains a
 * system's source adds the image-plane triangle's barycentre as a predicted image
 * (src/delense_CPU_utils.hpp:81-106, 215-225). */
int lto_delense(int n, double xmin, double xmax, double ymin, double ymax, const double *ax, const double *ay,
                int nsys, const double *bx, const double *by, const double *dr, int *nfound, double *fx, double *fy)
{
    const double dx = (xmax - xmin) / (n - 1), dy = (ymax - ymin) / (n - 1);
    int overflow = 0;
    for (int s = 0; s < nsys; s++) {
        const lto_pt P = {bx[s], by[s]};
        const double d = dr[s];
        int k = 0;
        for (int y = 0; y < n - 1; y++)
            for (int x = 0; x < n - 1; x++) {
                const double xp = xmin + x * dx, yp = ymin + y * dy;
                const long g = (long)y * n + x;
                /* upper: a = (x, y), b = (x, y + dy), c = (x + dx, y) */
                lto_pt ia = {xp, yp}, ib = {xp, yp + dy}, ic = {xp + dx, yp};
                lto_pt sa = {ia.x - d * ax[g], ia.y - d * ay[g]};
                lto_pt sb = {ib.x - d * ax[g + n], ib.y - d * ay[g + n]};
                lto_pt sc = {ic.x - d * ax[g + 1], ic.y - d * ay[g + 1]};
                int found = tri_inside(P, sa, sb, sc);
                if (!found) {
                    /* lower: a = (x + dx, y + dy), b = (x + dx, y), c = (x, y + dy) */
                    ia.x = xp + dx; ia.y = yp + dy;
                    ib.x = xp + dx; ib.y = yp;
                    ic.x = xp; ic.y = yp + dy;
                    sa.x = ia.x - d * ax[g + n + 1]; sa.y = ia.y - d * ay[g + n + 1];
                    sb.x = ib.x - d * ax[g + 1]; sb.y = ib.y - d * ay[g + 1];
                    sc.x = ic.x - d * ax[g + n]; sc.y = ic.y - d * ay[g + n];
                    found = tri_inside(P, sa, sb, sc);
                }
                if (found) {
                    if (k < LTO_MAXIMG) {
                        fx[s * LTO_MAXIMG + k] = (ia.x + ib.x + ic.x) / 3.;
                        fy[s * LTO_MAXIMG + k] = (ia.y + ib.y + ic.y) / 3.;
                    } else {
                        overflow = 1;
                    }
                    k++;
                }
            }
        nfound[s] = k < LTO_MAXIMG ? k : LTO_MAXIMG;
    }
    return overflow ? LTO_ERR_ARG : LTO_OK;
}

static double pt_dist(double ax, double ay, double bx, double by)
{
    double x = ax - bx, y = ay - by;
    return sqrt(x * x + y * y);
}

/* chi_computation, src/chi_computation.cpp:11-195: each predicted image is linked to its
 * closest observed image (a second one competing for the same observed image goes to
 * the closest observed image not yet linked, with the reference's loop bounds), then
 * chi2 = sum over linked observed images of |observed - predicted|^2 plus 1000 x
 * (images of the system) for every observed image left without a predicted one.
 * Returns chi2; *images_found counts the predicted images. */
double lto_chi2_images(int nsys, const int *nimg, const double *ix, const double *iy, const int *nfound,
                       const double *fx, const double *fy, int *images_found)
{
    double chi = 0.;
    int index = 0;
    *images_found = 0;
    for (int s = 0; s < nsys; s++) {
        const int n = nimg[s];
        int linked[LTO_MAXIMG];
        double tx[LTO_MAXIMG], ty[LTO_MAXIMG], dist[LTO_MAXIMG];
        memset(linked, 0, sizeof(linked));
        for (int ii = 0; ii < nfound[s]; ii++) {
            const double px = fx[s * LTO_MAXIMG + ii], py = fy[s * LTO_MAXIMG + ii];
            int im = 0;
            dist[0] = pt_dist(px, py, ix[index], iy[index]);
            for (int i = 1; i < n; i++) {
                dist[i] = pt_dist(px, py, ix[index + i], iy[index + i]);
                if (dist[i] < dist[im]) im = i;
            }
            (*images_found)++;
            if (linked[im] == 0) {
                tx[im] = px;
                ty[im] = py;
                linked[im]++;
            } else {
                double tempx, tempy;
                if (dist[im] < pt_dist(ix[index + im], iy[index + im], tx[im], ty[im])) {
                    tempx = tx[im];
                    tempy = ty[im];
                    tx[im] = px;
                    ty[im] = py;
                } else {
                    tempx = px;
                    tempy = py;
                }
                int second = 0;
                for (int i = 1; i < n && (i != im); i++)
                    if (dist[i] > dist[second]) second = i;
                for (int i = 0; i < n && linked[i] == 0; i++)
                    if (dist[i] < dist[second]) {
                        second = i;
                        im = i;
                        tx[im] = tempx;
                        ty[im] = tempy;
                    }
                linked[im]++;
            }
        }
        for (int i = 0; i < n; i++) {
            if (linked[i] > 0) {
                const double p1 = ix[index + i] - tx[i], p2 = iy[index + i] - ty[i];
                chi += p1 * p1 + p2 * p2;
            } else {
                chi += 1000. * n;
            }
        }
        index += n;
    }
    return chi;
}
