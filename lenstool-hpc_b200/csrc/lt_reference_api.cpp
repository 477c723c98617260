/*
 * lt_reference_api.cpp -- the reference's C++ host entry points (include/lt_reference_api.hpp)
 * implemented on the C ABI.  Every call re-reads the caller's Potential_SOA (as the
 * reference re-copies it on every call, src/grid_map_ampli_GPU.cu:119-160), so a caller
 * that rewrites its host arrays between calls (the bayes loop of utils/maps/main.cpp)
 * sees its new values.
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"
#include "../../include/lt_reference_api.hpp"
#include "lt_internal.h"

/* physical constants of src/structure_hpc.hpp:62-73 (map units) */
static const double kCH2piG = 0.11585881;
static const double kCH4piG = 0.057929405;
static const double kCH0_4piG = 2.7730112e-4;
static const double kMCRIT12 = .2343165;

namespace {

std::recursive_mutex g_mu; /* a caller's map function may call back into this API */
lt_context *g_ctx = nullptr;
int g_status = 0;

lt_context *ctx()
{
    if (!g_ctx) {
        lt_status st = lt_create(0, 0, &g_ctx);
        if (st != LT_OK) {
            fprintf(stderr, "lt_reference_api: lt_create failed: %s\n", lt_status_string(st));
            g_status = st;
            g_ctx = nullptr;
        }
    }
    return g_ctx;
}

bool report(lt_status st, const char *what)
{
    g_status = st;
    if (st != LT_OK) {
        fprintf(stderr, "lt_reference_api: %s: %s (%s)\n", what, lt_status_string(st),
                g_ctx ? lt_last_error(g_ctx) : "");
        return false;
    }
    return true;
}

/* Host copy of `n` entries behind `p`, which may be a host or a device pointer. */
template <typename T>
std::vector<T> fetch(const T *p, int n)
{
    std::vector<T> v(n > 0 ? n : 0);
    if (!p || n <= 0) return v;
    if (lt::is_device_pointer(p))
        cudaMemcpy(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost);
    else
        memcpy(v.data(), p, sizeof(T) * n);
    return v;
}

struct HostSoa {
    std::vector<int32_t> type;
    std::vector<double> x, y, b0, cs, sn, eps, rc, rcut, dlsds, z;
    lt_halo_soa view;
};

/* Read a Potential_SOA (the struct itself may live in device memory for the *_CPU_GPU
 * launchers, src/grid_gradient2_GPU.cu:186-209). */
bool read_soa(const Potential_SOA *lens, int n, HostSoa &h)
{
    if (!lens || n < 0) return false;
    Potential_SOA s;
    if (lt::is_device_pointer(lens))
        cudaMemcpy(&s, lens, sizeof(s), cudaMemcpyDeviceToHost);
    else
        s = *lens;
    std::vector<int> t = fetch(s.type, n);
    h.type.assign(t.begin(), t.end());
    h.x = fetch(s.position_x, n);
    h.y = fetch(s.position_y, n);
    h.b0 = fetch(s.b0, n);
    h.cs = fetch(s.anglecos, n);
    h.sn = fetch(s.anglesin, n);
    h.eps = fetch(s.ellipticity_potential, n);
    h.rc = fetch(s.rcore, n);
    h.rcut = fetch(s.rcut, n);
    h.dlsds = fetch(s.dlsds, n);
    h.z = fetch(s.z, n > 0 ? 1 : 0);
    if (n > 0 && (!s.type || !s.position_x || !s.position_y || !s.b0 || !s.anglecos || !s.anglesin ||
                  !s.ellipticity_potential || !s.rcore || !s.rcut))
        return false;
    h.view.nhalos = n;
    h.view.type = h.type.data();
    h.view.position_x = h.x.data();
    h.view.position_y = h.y.data();
    h.view.b0 = h.b0.data();
    h.view.anglecos = h.cs.data();
    h.view.anglesin = h.sn.data();
    h.view.ellipticity_potential = h.eps.data();
    h.view.rcore = h.rc.data();
    h.view.rcut = h.rcut.data();
    h.view.dlsds = h.dlsds.empty() ? nullptr : h.dlsds.data();
    return true;
}

grid_param read_frame(const grid_param *f)
{
    grid_param g;
    memset(&g, 0, sizeof(g));
    if (!f) return g;
    if (lt::is_device_pointer(f))
        cudaMemcpy(&g, f, sizeof(g), cudaMemcpyDeviceToHost);
    else
        g = *f;
    return g;
}

lt_grid make_grid(const grid_param &f, double dx, double dy, int nx, int ny, int istart, int jstart)
{
    lt_grid g;
    g.xmin = f.xmin;
    g.ymin = f.ymin;
    g.dx = dx;
    g.dy = dy;
    g.nx = nx;
    g.ny = ny;
    g.istart = istart;
    g.jstart = jstart;
    return g;
}

/* Uploaded catalogue for the duration of one call. */
struct Cat {
    lt_catalog *c = nullptr;
    HostSoa h;
    bool ok = false;
    Cat(const Potential_SOA *lens, int n)
    {
        if (!ctx()) return;
        if (!read_soa(lens, n, h)) {
            report(LT_ERR_INVALID_ARGUMENT, "Potential_SOA");
            return;
        }
        ok = report(lt_catalog_upload(g_ctx, &h.view, &c), "catalogue upload");
    }
    ~Cat()
    {
        if (c) lt_catalog_release(g_ctx, c);
    }
};

bool distances(const cosmo_param *cosmo, double zl, double zs, double &dls, double &dos, double &dol)
{
    lt_cosmology c;
    c.model = cosmo->model;
    c.omegaM = cosmo->omegaM;
    c.omegaX = cosmo->omegaX;
    c.curvature = cosmo->curvature;
    c.wX = cosmo->wX;
    c.wa = cosmo->wa;
    c.H0 = cosmo->H0;
    return report(lt_cosmo_distances(&c, zl, zs, &dls, &dos, &dol), "cosmology");
}

void gradient_impl(double *gx, double *gy, const grid_param *frame, const Potential_SOA *lens, int nhalos, double dx,
                   double dy, int nx, int ny, int istart, int jstart, double scale)
{
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    Cat cat(lens, nhalos);
    if (!cat.ok) return;
    grid_param f = read_frame(frame);
    lt_grid g = make_grid(f, dx, dy, nx, ny, istart, jstart);
    report(lt_gradient_grid(g_ctx, cat.c, &g, LT_FP64, scale, gx, gy, nullptr), "gradient grid");
}

void hessian_impl(double *a, double *b, double *c, double *d, const grid_param *frame, const Potential_SOA *lens,
                  int nhalos, double dx, double dy, int nx, int ny, int istart, int jstart, int kmap)
{
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    Cat cat(lens, nhalos);
    if (!cat.ok) return;
    grid_param f = read_frame(frame);
    lt_grid g = make_grid(f, dx, dy, nx, ny, istart, jstart);
    lt_map_request req[4] = {{LT_MAP_HESS_A, a}, {LT_MAP_HESS_B, b}, {LT_MAP_HESS_C, c}, {LT_MAP_HESS_D, d}};
    report(lt_hessian_maps(g_ctx, cat.c, &g, LT_FP64, kmap, 1.0, 1.0, req, 4, nullptr), "Hessian grid");
}

} // namespace

extern "C" int lt_reference_api_last_status(void) { return g_status; }

/* ------------------------------------------------------------------- deflection ---- */

void gradient_grid_GPU(type_t *gx, type_t *gy, const grid_param *frame, const Potential_SOA *lens, int nhalos,
                       int nbgridcells)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    gradient_impl(gx, gy, frame, lens, nhalos, dx, dy, nbgridcells, nbgridcells, 0, 0, 1.0);
}

void gradient_grid_GPU(type_t *gx, type_t *gy, const grid_param *frame, const Potential_SOA *lens, int nhalos,
                       type_t dx, type_t dy, int nx, int ny, int istart, int jstart)
{
    gradient_impl(gx, gy, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 1.0);
}

void gradient_grid_GPU_UM(type_t *gx, type_t *gy, const grid_param *frame, const Potential_SOA *lens, int nhalos,
                          type_t dx, type_t dy, int nx, int ny, int istart, int jstart)
{
    gradient_impl(gx, gy, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 1.0);
}

void module_potentialDerivatives_totalGradient_SOA_CPU_GPU(type_t *gx, type_t *gy, const grid_param *frame,
                                                           const Potential_SOA *lens_gpu, int nbgridcells, int nhalos)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    gradient_impl(gx, gy, frame, lens_gpu, nhalos, dx, dy, nbgridcells, nbgridcells, 0, 0, 1.0);
}

void module_potentialDerivatives_totalGradient_SOA_CPU_GPU(type_t *gx, type_t *gy, const grid_param *frame,
                                                           const Potential_SOA *lens, int nhalos, type_t dx, type_t dy,
                                                           int nx, int ny, int istart, int jstart)
{
    gradient_impl(gx, gy, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 1.0);
}

/* ---------------------------------------------------------------------- Hessian ---- */

void gradient2_grid_GPU(type_t *a, type_t *b, type_t *c, type_t *d, const grid_param *frame, const Potential_SOA *lens,
                        int nhalos, int nbgridcells)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    hessian_impl(a, b, c, d, frame, lens, nhalos, dx, dy, nbgridcells, nbgridcells, 0, 0, 0);
}

void gradient2_grid_GPU(type_t *a, type_t *b, type_t *c, type_t *d, const grid_param *frame, const Potential_SOA *lens,
                        int nhalos, type_t dx, type_t dy, int nx, int ny, int istart, int jstart)
{
    hessian_impl(a, b, c, d, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 0);
}

void module_potentialDerivatives_totalGradient2_SOA_CPU_GPU(type_t *a, type_t *b, type_t *c, type_t *d,
                                                            const grid_param *frame, const Potential_SOA *lens_gpu,
                                                            int nbgridcells, int nhalos)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    hessian_impl(a, b, c, d, frame, lens_gpu, nhalos, dx, dy, nbgridcells, nbgridcells, 0, 0, 0);
}

void module_potentialDerivatives_totalGradient2_SOA_CPU_GPU(type_t *a, type_t *b, type_t *c, type_t *d,
                                                            const grid_param *frame, const Potential_SOA *lens,
                                                            int nhalos, type_t dx, type_t dy, int nx, int ny,
                                                            int istart, int jstart)
{
    hessian_impl(a, b, c, d, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 0);
}

void module_potentialDerivatives_Kmap_SOA_CPU_GPU(type_t *a, type_t *b, type_t *c, type_t *d, const grid_param *frame,
                                                  const Potential_SOA *lens_gpu, int nhalos, type_t dx, type_t dy,
                                                  int nx, int ny, int istart, int jstart)
{
    hessian_impl(a, b, c, d, frame, lens_gpu, nhalos, dx, dy, nx, ny, istart, jstart, 1);
}

/* -------------------------------------------------------------------- potential ---- */

static void potential_impl(type_t *psi, const grid_param *frame, const Potential_SOA *lens, int nhalos, double dx,
                           double dy, int nx, int ny, int istart, int jstart, double scale)
{
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    Cat cat(lens, nhalos);
    if (!cat.ok) return;
    grid_param f = read_frame(frame);
    lt_grid g = make_grid(f, dx, dy, nx, ny, istart, jstart);
    report(lt_potential_grid(g_ctx, cat.c, &g, LT_FP64, scale, psi, nullptr), "potential grid");
}

void potential_grid_GPU(type_t *potential, const grid_param *frame, const Potential_SOA *lens, int nhalos,
                        int nbgridcells)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    potential_impl(potential, frame, lens, nhalos, dx, dy, nbgridcells, nbgridcells, 0, 0, 1.0);
}

void module_potential_SOA_CPU_GPU(type_t *potential, const grid_param *frame, const Potential_SOA *lens, int nhalos,
                                  type_t dx, type_t dy, int nx, int ny, int istart, int jstart)
{
    potential_impl(potential, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, 1.0);
}

/* ------------------------------------------------------- map epilogue functions ---- */

/* Elementwise map from device Hessian planes (the reference's separate map kernels);
 * lt::KIND_POT scales plane `a` by `mult` (potential and displacement modes). */
static void plane_map(int kind, type_t *map, type_t *a, type_t *b, type_t *c, double D, double mult, int nx, int ny)
{
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    if (!ctx()) return;
    const int err = lt::launch_planes_epilogue(kind, map, a, b, c, D, mult, nx, ny, g_ctx->num_sms, nullptr);
    report(err == cudaSuccess ? LT_OK : LT_ERR_CUDA, "map epilogue");
    cudaDeviceSynchronize();
}

#define AMPLI_FN(n, kind)                                                                                           \
    void amplif_##n##_grid_CPU_GPU(type_t *map, type_t *a, type_t *b, type_t *c, type_t *, type_t dl0s, type_t ds,   \
                                   type_t, type_t, type_t, int nx, int ny, const grid_param *)                      \
    {                                                                                                               \
        plane_map(kind, map, a, b, c, dl0s / ds, 1.0, nx, ny);                                                      \
    }
AMPLI_FN(1, LT_MAP_AMPLI1)
AMPLI_FN(2, LT_MAP_AMPLI2)
AMPLI_FN(3, LT_MAP_AMPLI3)
AMPLI_FN(4, LT_MAP_AMPLI4)
AMPLI_FN(5, LT_MAP_AMPLI5)
AMPLI_FN(6, LT_MAP_AMPLI6)
#undef AMPLI_FN
#define SHEAR_FN(n, kind)                                                                                           \
    void shear_##n##_grid_CPU_GPU(type_t *map, type_t *a, type_t *b, type_t *c, type_t *, type_t dl0s, type_t ds,    \
                                  type_t, type_t, type_t, int nx, int ny, const grid_param *)                       \
    {                                                                                                               \
        plane_map(kind, map, a, b, c, dl0s / ds, 1.0, nx, ny);                                                      \
    }
SHEAR_FN(1, LT_MAP_SHEAR1)
SHEAR_FN(2, LT_MAP_SHEAR2)
SHEAR_FN(3, LT_MAP_SHEAR3)
SHEAR_FN(4, LT_MAP_SHEAR4)
#undef SHEAR_FN

/* mass modes: unit factors of src/grid_map_mass_GPU.cu:219-300 */
static double mass_mult(int mode, double dl0s, double ds, double dl, double h, const grid_param &f, int nx, int ny)
{
    switch (mode) {
    case 1: return 1.;
    case 2: return kCH4piG * h / dl / dl0s * ds;
    case 3: {
        const double dx = (f.xmax - f.xmin) / (nx - 1), dy = (f.ymax - f.ymin) / (ny - 1);
        return kMCRIT12 / h * dx * dy * dl / dl0s * ds;
    }
    case 4: return kCH0_4piG * h / dl / dl0s * ds;
    }
    return 0.;
}
#define MASS_FN(n)                                                                                                  \
    void mass_##n##_grid_CPU_GPU(type_t *map, type_t *a, type_t *b, type_t *c, type_t *, type_t dl0s, type_t ds,     \
                                 type_t dl, type_t h, type_t, int nx, int ny, const grid_param *frame)              \
    {                                                                                                               \
        grid_param f = read_frame(frame);                                                                           \
        plane_map(LT_MAP_MASS, map, a, b, c, 1.0, mass_mult(n, dl0s, ds, dl, h, f, nx, ny), nx, ny);                \
    }
MASS_FN(1)
MASS_FN(2)
MASS_FN(3)
MASS_FN(4)
#undef MASS_FN

void potential_1_grid_CPU_GPU(type_t *potential, type_t dl0s, type_t ds, type_t, type_t, type_t, int nx, int ny,
                              const grid_param *)
{
    plane_map(lt::KIND_POT, potential, potential, potential, potential, 1.0, dl0s / ds, nx, ny);
}

void potential_2_grid_CPU_GPU(type_t *potential, type_t, type_t, type_t dl, type_t h, type_t, int nx, int ny,
                              const grid_param *)
{
    plane_map(lt::KIND_POT, potential, potential, potential, potential, 1.0, kCH2piG * h / dl, nx, ny);
}

void dpl_grid_CPU_GPU(type_t *map, type_t dl0s, type_t ds, type_t, type_t, type_t, int nx, int ny, const grid_param *)
{
    plane_map(lt::KIND_POT, map, map, map, map, 1.0, dl0s / ds, nx, ny);
}

/* ------------------------------------------------------------- map selection ---- */

map_gpu_function_t select_map_ampli_function(const runmode_param *r)
{
    static const map_gpu_function_t t[] = {amplif_1_grid_CPU_GPU, amplif_2_grid_CPU_GPU, amplif_3_grid_CPU_GPU,
                                           amplif_4_grid_CPU_GPU, amplif_5_grid_CPU_GPU, amplif_6_grid_CPU_GPU};
    if (r && r->amplif >= 1 && r->amplif <= 6) return t[r->amplif - 1];
    report(LT_ERR_INVALID_ARGUMENT, "amplification mode not supported");
    return nullptr;
}

map_gpu_function_t select_map_shear_function(const runmode_param *r)
{
    static const map_gpu_function_t t[] = {shear_1_grid_CPU_GPU, shear_2_grid_CPU_GPU, shear_3_grid_CPU_GPU,
                                           shear_4_grid_CPU_GPU};
    if (r && r->shear >= 1 && r->shear <= 4) return t[r->shear - 1];
    report(LT_ERR_INVALID_ARGUMENT, "shear mode not supported");
    return nullptr;
}

map_gpu_function_t select_map_mass_function(const runmode_param *r)
{
    static const map_gpu_function_t t[] = {mass_1_grid_CPU_GPU, mass_2_grid_CPU_GPU, mass_3_grid_CPU_GPU,
                                           mass_4_grid_CPU_GPU};
    if (r && r->mass >= 1 && r->mass <= 4) return t[r->mass - 1];
    report(LT_ERR_INVALID_ARGUMENT, "mass mode not supported");
    return nullptr;
}

map_pot_function_t select_map_potential_function(const runmode_param *r)
{
    static const map_pot_function_t t[] = {potential_1_grid_CPU_GPU, potential_2_grid_CPU_GPU};
    if (r && r->potential >= 1 && r->potential <= 2) return t[r->potential - 1];
    report(LT_ERR_INVALID_ARGUMENT, "potential mode not supported (mode 3 is a stub in the reference)");
    return nullptr;
}

/* ------------------------------------------------------------------- map builders ---- */

/* Which of our epilogues `fn` is: its map kind (or -1 for a caller-supplied function). */
static int kind_of(map_gpu_function_t fn, int *mass_mode)
{
    const map_gpu_function_t a[] = {amplif_1_grid_CPU_GPU, amplif_2_grid_CPU_GPU, amplif_3_grid_CPU_GPU,
                                    amplif_4_grid_CPU_GPU, amplif_5_grid_CPU_GPU, amplif_6_grid_CPU_GPU};
    const map_gpu_function_t s[] = {shear_1_grid_CPU_GPU, shear_2_grid_CPU_GPU, shear_3_grid_CPU_GPU,
                                    shear_4_grid_CPU_GPU};
    const map_gpu_function_t m[] = {mass_1_grid_CPU_GPU, mass_2_grid_CPU_GPU, mass_3_grid_CPU_GPU, mass_4_grid_CPU_GPU};
    for (int i = 0; i < 6; i++)
        if (fn == a[i]) return LT_MAP_AMPLI1 + i;
    for (int i = 0; i < 4; i++)
        if (fn == s[i]) return LT_MAP_SHEAR1 + i;
    for (int i = 0; i < 4; i++)
        if (fn == m[i]) {
            *mass_mode = i + 1;
            return LT_MAP_MASS;
        }
    return -1;
}

/* One Hessian-derived map of the grid: our fused kernel for our own epilogues; the
 * reference's two-step structure (device Hessian planes, then `fn`) for any other. */
static void hessian_map(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                        const Potential_SOA *lens, int nhalos, double zl, double zs, double dx, double dy, int nx,
                        int ny, int istart, int jstart, int kmap)
{
    if (!fn || !cosmo) {
        report(LT_ERR_INVALID_ARGUMENT, "map function / cosmology");
        return;
    }
    std::lock_guard<std::recursive_mutex> lock(g_mu);
    Cat cat(lens, nhalos);
    if (!cat.ok) return;
    if (zl == 0 && !cat.h.z.empty()) zl = cat.h.z[0];
    double dl0s, dos, dol;
    if (!distances(cosmo, zl, zs, dl0s, dos, dol)) return;
    grid_param f = read_frame(frame);
    lt_grid g = make_grid(f, dx, dy, nx, ny, istart, jstart);
    int mass_mode = 0;
    const int kind = kind_of(fn, &mass_mode);
    if (kind >= 0) {
        const double mult = kind == LT_MAP_MASS ? mass_mult(mass_mode, dl0s, dos, dol, cosmo->h, f, nx, ny) : 1.0;
        lt_map_request req = {kind, map};
        report(lt_hessian_maps(g_ctx, cat.c, &g, LT_FP64, kmap, dl0s / dos, mult, &req, 1, nullptr), "map");
        return;
    }
    /* caller-supplied epilogue: device planes, fn, copy back */
    const size_t plane = sizeof(double) * (size_t)nx * ny;
    double *dev = nullptr;
    if (!report(lt::dev_alloc(g_ctx, (void **)&dev, 5 * plane), "plane allocation")) return;
    double *p[5] = {dev, dev + (size_t)nx * ny, dev + 2 * (size_t)nx * ny, dev + 3 * (size_t)nx * ny,
                    dev + 4 * (size_t)nx * ny};
    lt_map_request req[4] = {{LT_MAP_HESS_A, p[0]}, {LT_MAP_HESS_B, p[1]}, {LT_MAP_HESS_C, p[2]}, {LT_MAP_HESS_D, p[3]}};
    if (report(lt_hessian_maps(g_ctx, cat.c, &g, LT_FP64, kmap, 1.0, 1.0, req, 4, nullptr), "Hessian planes") &&
        report(lt_synchronize(g_ctx, nullptr), "Hessian planes")) {
        fn(p[4], p[0], p[1], p[2], p[3], dl0s, dos, dol, cosmo->h, zs, nx, ny, frame);
        cudaDeviceSynchronize();
        cudaMemcpy(map, p[4], plane, lt::is_device_pointer(map) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost);
    }
    lt::dev_free(g_ctx, dev, 5 * plane);
}

void map_grid_ampli_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                        const Potential_SOA *lens, int nhalos, int nbgridcells, int, type_t z)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    hessian_map(fn, map, cosmo, frame, lens, nhalos, 0., z, dx, dy, nbgridcells, nbgridcells, 0, 0, 0);
}

void map_grid_ampli_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                        const Potential_SOA *lens, int nhalos, int, type_t z, type_t dx, type_t dy, int nx, int ny,
                        int istart, int jstart)
{
    hessian_map(fn, map, cosmo, frame, lens, nhalos, 0., z, dx, dy, nx, ny, istart, jstart, 0);
}

void map_grid_shear_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                        const Potential_SOA *lens, int nhalos, int nbgridcells, int, type_t z)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    hessian_map(fn, map, cosmo, frame, lens, nhalos, 0., z, dx, dy, nbgridcells, nbgridcells, 0, 0, 0);
}

void map_grid_shear_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                        const Potential_SOA *lens, int nhalos, int, type_t z, type_t dx, type_t dy, int nx, int ny,
                        int istart, int jstart)
{
    hessian_map(fn, map, cosmo, frame, lens, nhalos, 0., z, dx, dy, nx, ny, istart, jstart, 0);
}

void map_grid_mass_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                       const Potential_SOA *lens, int nhalos, int nbgridcells, int, type_t zl, type_t zs)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    hessian_map(fn, map, cosmo, frame, lens, nhalos, zl, zs, dx, dy, nbgridcells, nbgridcells, 0, 0, 1);
}

void map_grid_mass_GPU(map_gpu_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                       const Potential_SOA *lens, int nhalos, int, type_t zl, type_t zs, type_t dx, type_t dy, int nx,
                       int ny, int istart, int jstart)
{
    hessian_map(fn, map, cosmo, frame, lens, nhalos, zl, zs, dx, dy, nx, ny, istart, jstart, 1);
}

static void potential_map(map_pot_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                          const Potential_SOA *lens, int nhalos, type_t z, double dx, double dy, int nx, int ny,
                          int istart, int jstart)
{
    if (!fn || !cosmo) {
        report(LT_ERR_INVALID_ARGUMENT, "map function / cosmology");
        return;
    }
    double scale = 0.;
    {
        std::lock_guard<std::recursive_mutex> lock(g_mu);
        HostSoa h;
        if (!read_soa(lens, nhalos, h)) {
            report(LT_ERR_INVALID_ARGUMENT, "Potential_SOA");
            return;
        }
        double dl0s, dos, dol;
        if (!distances(cosmo, h.z.empty() ? 0. : h.z[0], z, dl0s, dos, dol)) return;
        if (fn == potential_1_grid_CPU_GPU)
            scale = dl0s / dos;
        else if (fn == potential_2_grid_CPU_GPU)
            scale = kCH2piG * cosmo->h / dol;
        else {
            report(LT_ERR_INVALID_ARGUMENT, "unknown potential map function");
            return;
        }
    }
    potential_impl(map, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, scale);
}

void map_grid_potential_GPU(map_pot_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                            const Potential_SOA *lens, int nhalos, int nbgridcells, int, type_t z)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    potential_map(fn, map, cosmo, frame, lens, nhalos, z, dx, dy, nbgridcells, nbgridcells, 0, 0);
}

void map_grid_potential_GPU(map_pot_function_t fn, type_t *map, const cosmo_param *cosmo, const grid_param *frame,
                            const Potential_SOA *lens, int nhalos, int, type_t z, type_t dx, type_t dy, int nx, int ny,
                            int istart, int jstart)
{
    potential_map(fn, map, cosmo, frame, lens, nhalos, z, dx, dy, nx, ny, istart, jstart);
}

static void dpl_map(type_t *dplx, type_t *dply, const cosmo_param *cosmo, const grid_param *frame,
                    const Potential_SOA *lens, int nhalos, type_t z, double dx, double dy, int nx, int ny, int istart,
                    int jstart)
{
    double scale = 0.;
    {
        std::lock_guard<std::recursive_mutex> lock(g_mu);
        HostSoa h;
        if (!cosmo || !read_soa(lens, nhalos, h)) {
            report(LT_ERR_INVALID_ARGUMENT, "Potential_SOA / cosmology");
            return;
        }
        double dl0s, dos, dol;
        if (!distances(cosmo, h.z.empty() ? 0. : h.z[0], z, dl0s, dos, dol)) return;
        scale = dl0s / dos;
    }
    gradient_impl(dplx, dply, frame, lens, nhalos, dx, dy, nx, ny, istart, jstart, scale);
}

void map_grid_dpl_GPU(map_gpu_function_t, type_t *dplx, type_t *dply, const cosmo_param *cosmo, const grid_param *frame,
                      const Potential_SOA *lens, int nhalos, int nbgridcells, int, type_t z)
{
    grid_param f = read_frame(frame);
    const double dx = (f.xmax - f.xmin) / (nbgridcells - 1), dy = (f.ymax - f.ymin) / (nbgridcells - 1);
    dpl_map(dplx, dply, cosmo, frame, lens, nhalos, z, dx, dy, nbgridcells, nbgridcells, 0, 0);
}

void map_grid_dpl_GPU(map_gpu_function_t, type_t *dplx, type_t *dply, const cosmo_param *cosmo, const grid_param *frame,
                      const Potential_SOA *lens, int nhalos, int, type_t z, type_t dx, type_t dy, int nx, int ny,
                      int istart, int jstart)
{
    dpl_map(dplx, dply, cosmo, frame, lens, nhalos, z, dx, dy, nx, ny, istart, jstart);
}
