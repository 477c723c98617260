/*
 * lt_ingest.cu -- resident catalogues re-derived on the device from posterior samples, in
 * place: lt_catalog_update (every halo's physical parameters) and lt_bayes_apply (rows of
 * a bayes.dat file against a model, potfile scaling relations included).
 *
 * The reference applies a bayes.dat row on the host and recomputes the potential
 * parameters of every halo (module_readParameters_setbayesmapmodels,
 * src/module_readParameters.cpp:132-227; setScalingRelations, :1539-1656;
 * module_readParameters_calculatePotentialparameter_SOA, :2873-2936); the maps of each
 * sample then start with a host -> device copy of the whole SoA
 * (src/grid_map_ampli_GPU.cu:119-160).  Here one thread per (sample, halo) derives the
 * halo's state, b0 and ellipticity_potential, and re-packs its FP64 and FP32C records with
 * the host packer's arithmetic (lt_pack.h), so batches and graphs that hold the
 * catalogues' handles see the new samples without re-capture.
 *
 * The profile types, the halo order and the FP32C chunk lists are those of the upload: a
 * halo of the FP32 class whose new parameters need FP64 everywhere is evaluated through
 * its FP64 record (an FP64 proxy, lt_profiles32.cuh), and an FP64-class halo stays FP64.
 * A sample outside a profile's domain is reported (LT_ERR_NONFINITE in the status word,
 * read by lt_synchronize) and leaves that halo's records unchanged.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "lt_internal.h"
#include "lt_pack.h"

namespace lt {

__device__ __forceinline__ void flag(int32_t *status, int32_t code) { atomicCAS(status, 0, code); }

/* The records of one catalogue. */
struct CatRecs {
    lt_rec64 *recs;
    lt_rec32 *recs32;
    lt_nie64 *nie;
    const int32_t *idx32;
};

/* Pack halo i's records from its potential parameters; false (records untouched) outside
 * the domain lt_catalog_upload accepts. */
__device__ __forceinline__ bool store_records(const CatRecs &c, int i, int t, double x, double y, double cs,
                                              double sn, double b0, double eps, double rc, double rcut)
{
    if (!pk::record_ok(t, x, y, b0, cs, sn, eps, rc, rcut)) return false;
    lt_rec64 r;
    pk::pack64(t, x, y, cs, sn, b0, eps, rc, rcut, c.recs[i].w, r);
    c.recs[i] = r;
    lt_nie64 q;
    pk::pack_nie64(r, t, q);
    c.nie[i] = q;
    const int j = c.idx32[i];
    if (j >= 0) {
        lt_rec32 o;
        pk::pack32(r, t, i, o);
        if (pk::needs_fp64_always(r, t)) o.rnear2 = kProxy64;
        c.recs32[j] = o;
    }
    return true;
}

/* ---- lt_catalog_update ---------------------------------------------------------------- */

struct UpdateArgs {
    int n;
    const int32_t *types;
    const double *x, *y, *vdisp, *emass, *angle, *rcore, *rcut;
    const double *cs, *sn; /* optional */
    CatRecs cat;
    int32_t *status;
};

__global__ void catalog_update_kernel(const UpdateArgs a)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int t = a.types[i];
        const double em = a.emass[i];
        if (!(em >= 0. && em < 1.) || !isfinite(a.vdisp[i]) || !isfinite(a.angle[i])) {
            flag(a.status, (int32_t)LT_ERR_NONFINITE);
            continue;
        }
        double b0, eps;
        pk::potential_parameters(t, a.vdisp[i], em, b0, eps);
        double sn, cs;
        if (a.cs) {
            cs = a.cs[i];
            sn = a.sn[i];
        } else {
            sincos(a.angle[i], &sn, &cs);
        }
        if (!store_records(a.cat, i, t, a.x[i], a.y[i], cs, sn, b0, eps, a.rcore[i], a.rcut[i]))
            flag(a.status, (int32_t)LT_ERR_NONFINITE);
    }
}

/* ---- bayes.dat rows ------------------------------------------------------------------- */

/* The model on the device: the base state of every halo (after the potential-parameter
 * step reached its fixed point), the columns that address each halo (CSR), the potfile
 * factors. */
struct BayesDev {
    int n, ncols, ntheta;
    const int32_t *types;
    const double *x, *y, *epot, *emass, *cs, *sn, *rc, *vdisp, *rcut;
    const int32_t *col_off, *col_idx, *col_field; /* columns of halo h: col_off[h] .. col_off[h+1]-1 */
    const int32_t *tslot;                          /* per column: its slot among the theta columns */
    const int32_t *pf;                             /* per halo: its potfile, or -1 */
    const int32_t *hasmag;                         /* per halo: mag != 0 */
    const double *fv, *fr, *rcs;                   /* 10^(0.4 dm/vdslope), 10^(0.8 dm/slope), core 10^(0.2 dm) */
    const double *pot_sigma, *pot_cut;             /* per potfile: the model's sigma, cut */
    const int32_t *pot_sigma_col, *pot_cut_col;    /* per potfile: the row column, or -1 */
    double dtr;                                    /* degrees to radians, acos(-1)/180 */
};

struct ApplyArgs {
    BayesDev m;
    const double *rows; /* nrows x ncols */
    const double *trig; /* nrows x ntheta x (cos, sin), or NULL: cos/sin on the device */
    const CatRecs *cats;
    int nrows;
    int32_t *status;
};

__global__ void bayes_apply_kernel(const ApplyArgs a)
{
    const BayesDev &m = a.m;
    const long total = (long)a.nrows * m.n;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
        const int r = (int)(k / m.n), h = (int)(k % m.n);
        const double *row = a.rows + (size_t)r * m.ncols;
        const int t = m.types[h];
        double x = m.x[h], y = m.y[h], epot = m.epot[h], emass = m.emass[h], cs = m.cs[h], sn = m.sn[h];
        double rc = m.rc[h], vdisp = m.vdisp[h], rcut = m.rcut[h];
        const int p = m.pf[h];
        if (p < 0) {
            /* the halo's free parameters (setbayesmapmodels, :142-188) */
            for (int q = m.col_off[h]; q < m.col_off[h + 1]; q++) {
                const int c = m.col_idx[q];
                const double v = row[c];
                switch (m.col_field[q]) {
                case LT_BAYES_X: x = v; break;
                case LT_BAYES_Y: y = v; break;
                case LT_BAYES_EPOT: epot = v; break;
                case LT_BAYES_EMASS: emass = v; break;
                case LT_BAYES_THETA:
                    if (a.trig) {
                        const double *tc = a.trig + 2 * ((size_t)r * m.ntheta + m.tslot[c]);
                        cs = tc[0];
                        sn = tc[1];
                    } else {
                        sincos(pk::mul(v, m.dtr), &sn, &cs);
                    }
                    break;
                case LT_BAYES_RCORE: rc = v; break;
                case LT_BAYES_VDISP: vdisp = v; break;
                case LT_BAYES_RCUT: rcut = v; break;
                default: break; /* LT_BAYES_Z: the maps' D_LS/D_OS is set at upload */
                }
            }
        } else if (m.hasmag[h]) {
            /* potfile scaling relations (setScalingRelations, :1613-1634) */
            const double sig = m.pot_sigma_col[p] >= 0 ? row[m.pot_sigma_col[p]] : m.pot_sigma[p];
            const double cut = m.pot_cut_col[p] >= 0 ? row[m.pot_cut_col[p]] : m.pot_cut[p];
            rc = m.rcs[h];
            vdisp = pk::mul(sig, m.fv[h]);
            rcut = pk::mul(cut, m.fr[h]);
        }
        double b0;
        pk::calc_potential_parameter(t, vdisp, emass, epot, b0);
        if (!store_records(a.cats[r], h, t, x, y, cs, sn, b0, epot, rc, rcut)) flag(a.status, (int32_t)LT_ERR_NONFINITE);
    }
}

} // namespace lt

using namespace lt;

struct lt_bayes {
    int n = 0, ncols = 0, npot = 0;
    std::vector<int32_t> types;      /* host copy: catalogues must match it */
    std::vector<int32_t> theta_cols; /* the THETA columns, in slot order */
    double dtr = 0.;
    void *mem = nullptr;
    size_t bytes = 0;
    BayesDev dev;
    void *stage = nullptr;
    size_t stage_bytes = 0;
};

static lt_status grow(lt_context *ctx, void **p, size_t *have, size_t need)
{
    if (*have >= need) return LT_OK;
    dev_free(ctx, *p, *have);
    *p = nullptr;
    *have = 0;
    lt_status st = dev_alloc(ctx, p, need);
    if (st == LT_OK) *have = need;
    return st;
}

static bool same_types(const lt_catalog *cat, const std::vector<int32_t> &types)
{
    return cat && cat->nhalos == (int32_t)types.size() && cat->host_types == types;
}

static CatRecs recs_of(const lt_catalog *cat)
{
    const Fp32cCatalog &fc = *reinterpret_cast<const Fp32cCatalog *>(&cat->aux_desc);
    CatRecs c;
    c.recs = cat->recs;
    c.recs32 = fc.recs32;
    c.nie = fc.nie;
    c.idx32 = fc.idx32;
    return c;
}

static int blocks_for(long work)
{
    const long b = (work + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

extern "C" lt_status lt_catalog_update(lt_context *ctx, lt_catalog *cat, const lt_halo_params *p, void *stream)
{
    if (!ctx || !cat || !p || p->nhalos != cat->nhalos) {
        if (ctx) set_error(ctx, "lt_catalog_update: the parameters must cover the catalogue's %d halos",
                           cat ? cat->nhalos : -1);
        return LT_ERR_INVALID_ARGUMENT;
    }
    const bool trig = p->anglecos && p->anglesin;
    const double *in[9] = {p->position_x, p->position_y, p->vdisp, p->ellipticity, p->ellipticity_angle, p->rcore,
                           p->rcut, p->anglecos, p->anglesin};
    const int nin = trig ? 9 : 7;
    for (int k = 0; k < 7; k++)
        if (!in[k] && cat->nhalos > 0) {
            set_error(ctx, "lt_catalog_update: a parameter array is NULL");
            return LT_ERR_INVALID_ARGUMENT;
        }
    if (cat->nhalos == 0) return LT_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n = (size_t)cat->nhalos, plane = n * sizeof(double);
    const double *dev[9] = {};
    bool device = true;
    for (int k = 0; k < nin; k++) device &= is_device_pointer(in[k]);
    if (device) {
        for (int k = 0; k < nin; k++) dev[k] = in[k];
    } else {
        lt_status st = grow(ctx, &cat->stage, &cat->stage_bytes, 9 * plane);
        if (st != LT_OK) return st;
        for (int k = 0; k < nin; k++) {
            double *d = (double *)cat->stage + k * n;
            cudaError_t e = cudaMemcpyAsync(d, in[k], plane, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "parameter upload");
            dev[k] = d;
        }
    }
    const Fp32cCatalog &fc = *reinterpret_cast<const Fp32cCatalog *>(&cat->aux_desc);
    UpdateArgs a;
    a.n = cat->nhalos;
    a.types = fc.types;
    a.x = dev[0];
    a.y = dev[1];
    a.vdisp = dev[2];
    a.emass = dev[3];
    a.angle = dev[4];
    a.rcore = dev[5];
    a.rcut = dev[6];
    a.cs = trig ? dev[7] : nullptr;
    a.sn = trig ? dev[8] : nullptr;
    a.cat = recs_of(cat);
    a.status = ctx->status;
    catalog_update_kernel<<<blocks_for((long)n), 256, 0, s>>>(a);
    count_launch(1);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "catalogue update");
    return LT_OK;
}

extern "C" lt_status lt_bayes_create(lt_context *ctx, const lt_bayes_model *model, int32_t npotfiles,
                                     const lt_potfile *potfiles, int32_t ncolumns, const lt_bayes_column *columns,
                                     lt_bayes **out)
{
    if (!ctx || !model || !out || model->nhalos < 0 || npotfiles < 0 || ncolumns < 0 || (npotfiles && !potfiles) ||
        (ncolumns && !columns))
        return LT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const int n = model->nhalos;
    const double *planes[9] = {model->position_x, model->position_y, model->ellipticity_potential,
                               model->ellipticity, model->ellipticity_angle, model->rcore, model->vdisp,
                               model->rcut, nullptr};
    if (n > 0 && !model->type) return LT_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 8; k++)
        if (n > 0 && !planes[k]) {
            set_error(ctx, "lt_bayes_create: a model array is NULL");
            return LT_ERR_INVALID_ARGUMENT;
        }
    if (npotfiles > 0 && !model->mag) {
        set_error(ctx, "lt_bayes_create: potfiles need the galaxies' magnitudes");
        return LT_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < n; i++)
        if (model->type[i] != 5 && model->type[i] != 8 && model->type[i] != 81) {
            set_error(ctx, "lt_bayes_create: halo %d: unknown profile type %d", i, model->type[i]);
            return LT_ERR_UNKNOWN_PROFILE;
        }
    /* potfile galaxies */
    std::vector<int32_t> pf((size_t)n, -1), hasmag((size_t)n, 0);
    std::vector<double> fv((size_t)n, 0.), fr((size_t)n, 0.), rcs((size_t)n, 0.);
    for (int p = 0; p < npotfiles; p++) {
        const lt_potfile &q = potfiles[p];
        if (q.first < 0 || q.count < 0 || q.first > n - q.count || !(q.vdslope != 0.) || !(q.slope != 0.)) {
            set_error(ctx, "lt_bayes_create: potfile %d: bad galaxy range or zero slope", p);
            return LT_ERR_INVALID_ARGUMENT;
        }
        for (int i = q.first; i < q.first + q.count; i++) {
            if (pf[i] >= 0) {
                set_error(ctx, "lt_bayes_create: halo %d is in two potfiles", i);
                return LT_ERR_INVALID_ARGUMENT;
            }
            pf[i] = p;
            const double mag = model->mag[i];
            if (mag != 0.) {
                /* setScalingRelations (src/module_readParameters.cpp:1613-1631): the
                 * magnitude terms are fixed by the catalogue, so they are taken once here */
                hasmag[i] = 1;
                rcs[i] = q.core * pow(10., 0.4 * (q.mag0 - mag) / 2.);
                fv[i] = pow(10., 0.4 * (q.mag0 - mag) / q.vdslope);
                fr[i] = pow(10., 0.4 * (q.mag0 - mag) * 2. / q.slope);
            }
        }
    }
    /* columns: CSR over halos; potfile columns */
    std::vector<int32_t> count((size_t)n + 1, 0), tslot((size_t)ncolumns, -1), theta_cols;
    std::vector<int32_t> pot_sigma_col((size_t)npotfiles, -1), pot_cut_col((size_t)npotfiles, -1);
    for (int c = 0; c < ncolumns; c++) {
        const int f = columns[c].field, tg = columns[c].target;
        if (f == LT_BAYES_SKIP) continue;
        if (f >= LT_BAYES_X && f <= LT_BAYES_Z) {
            if (tg < 0 || tg >= n || pf[tg] >= 0) {
                set_error(ctx, "lt_bayes_create: column %d addresses halo %d (not a halo outside the potfiles)", c, tg);
                return LT_ERR_INVALID_ARGUMENT;
            }
            count[tg + 1]++;
            if (f == LT_BAYES_THETA) {
                tslot[c] = (int32_t)theta_cols.size();
                theta_cols.push_back(c);
            }
        } else if (f == LT_BAYES_POT_CUT || f == LT_BAYES_POT_SIGMA) {
            if (tg < 0 || tg >= npotfiles) {
                set_error(ctx, "lt_bayes_create: column %d addresses potfile %d of %d", c, tg, npotfiles);
                return LT_ERR_INVALID_ARGUMENT;
            }
            (f == LT_BAYES_POT_CUT ? pot_cut_col : pot_sigma_col)[tg] = c;
        } else {
            set_error(ctx, "lt_bayes_create: column %d: unknown field %d", c, f);
            return LT_ERR_INVALID_ARGUMENT;
        }
    }
    for (int i = 0; i < n; i++) count[i + 1] += count[i];
    const int nused = n ? count[n] : 0;
    std::vector<int32_t> col_idx((size_t)nused), col_field((size_t)nused), fill(count.begin(), count.end());
    for (int c = 0; c < ncolumns; c++) {
        const int f = columns[c].field;
        if (f < LT_BAYES_X || f > LT_BAYES_Z) continue;
        const int q = fill[columns[c].target]++;
        col_idx[q] = c;
        col_field[q] = f;
    }
    /* the base state at the fixed point of the potential-parameter step (three passes:
     * emass == epot == 0 -> epot 1e-5 -> emass from epot -> epot from emass) */
    std::vector<double> base[9];
    for (int k = 0; k < 9; k++) base[k].resize((size_t)n);
    /* planes: x, y, epot, emass, cs, sn, rc, vdisp, rcut */
    for (int i = 0; i < n; i++) {
        base[0][i] = model->position_x[i];
        base[1][i] = model->position_y[i];
        double epot = model->ellipticity_potential[i], emass = model->ellipticity[i], b0;
        for (int it = 0; it < 3; it++) pk::calc_potential_parameter(model->type[i], model->vdisp[i], emass, epot, b0);
        base[2][i] = epot;
        base[3][i] = emass;
        base[4][i] = cos(model->ellipticity_angle[i]);
        base[5][i] = sin(model->ellipticity_angle[i]);
        base[6][i] = model->rcore[i];
        base[7][i] = model->vdisp[i];
        base[8][i] = model->rcut[i];
    }
    std::vector<double> pot_sigma((size_t)npotfiles), pot_cut((size_t)npotfiles);
    for (int p = 0; p < npotfiles; p++) {
        pot_sigma[p] = potfiles[p].sigma;
        pot_cut[p] = potfiles[p].cut;
    }
    lt_bayes *b = new (std::nothrow) lt_bayes();
    if (!b) return LT_ERR_OUT_OF_MEMORY;
    b->n = n;
    b->ncols = ncolumns;
    b->npot = npotfiles;
    b->types.assign(model->type, model->type + n);
    b->theta_cols = theta_cols;
    b->dtr = acos(-1.) / 180.;
    /* one allocation: doubles, then int32 arrays */
    const size_t nd = 12 * (size_t)n + 2 * (size_t)npotfiles;
    const size_t ni = 5 * (size_t)n + 1 + 2 * (size_t)nused + (size_t)ncolumns + 2 * (size_t)npotfiles;
    b->bytes = nd * sizeof(double) + ni * sizeof(int32_t) + 16;
    std::vector<unsigned char> host(b->bytes, 0);
    double *hd = (double *)host.data();
    int32_t *hi = (int32_t *)(host.data() + nd * sizeof(double));
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    lt_status st = dev_alloc(ctx, &b->mem, b->bytes);
    if (st != LT_OK) {
        delete b;
        return st;
    }
    double *dd = (double *)b->mem;
    int32_t *di = (int32_t *)((char *)b->mem + nd * sizeof(double));
    size_t od = 0, oi = 0;
    auto put_d = [&](const double *src, size_t cnt) {
        if (cnt) memcpy(hd + od, src, cnt * sizeof(double));
        const double *d = dd + od;
        od += cnt;
        return d;
    };
    auto put_i = [&](const int32_t *src, size_t cnt) {
        if (cnt) memcpy(hi + oi, src, cnt * sizeof(int32_t));
        const int32_t *d = di + oi;
        oi += cnt;
        return d;
    };
    BayesDev &m = b->dev;
    m.n = n;
    m.ncols = ncolumns;
    m.ntheta = (int)theta_cols.size();
    m.dtr = b->dtr;
    m.x = put_d(base[0].data(), n);
    m.y = put_d(base[1].data(), n);
    m.epot = put_d(base[2].data(), n);
    m.emass = put_d(base[3].data(), n);
    m.cs = put_d(base[4].data(), n);
    m.sn = put_d(base[5].data(), n);
    m.rc = put_d(base[6].data(), n);
    m.vdisp = put_d(base[7].data(), n);
    m.rcut = put_d(base[8].data(), n);
    m.fv = put_d(fv.data(), n);
    m.fr = put_d(fr.data(), n);
    m.rcs = put_d(rcs.data(), n);
    m.pot_sigma = put_d(pot_sigma.data(), npotfiles);
    m.pot_cut = put_d(pot_cut.data(), npotfiles);
    m.types = put_i(model->type, n);
    m.pf = put_i(pf.data(), n);
    m.hasmag = put_i(hasmag.data(), n);
    m.col_off = put_i(count.data(), (size_t)n + 1);
    m.col_idx = put_i(col_idx.data(), nused);
    m.col_field = put_i(col_field.data(), nused);
    m.tslot = put_i(tslot.data(), ncolumns);
    m.pot_sigma_col = put_i(pot_sigma_col.data(), npotfiles);
    m.pot_cut_col = put_i(pot_cut_col.data(), npotfiles);
    const cudaError_t e = cudaMemcpy(b->mem, host.data(), b->bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        dev_free(ctx, b->mem, b->bytes);
        delete b;
        return cuda_fail(ctx, e, "bayes model upload");
    }
    *out = b;
    return LT_OK;
}

extern "C" lt_status lt_bayes_apply(lt_context *ctx, lt_bayes *b, const double *rows, int32_t nrows,
                                    lt_catalog *const *cats, void *stream)
{
    if (!ctx || !b || nrows < 0 || (nrows && (!rows || !cats))) return LT_ERR_INVALID_ARGUMENT;
    for (int r = 0; r < nrows; r++)
        if (!same_types(cats[r], b->types)) {
            set_error(ctx, "lt_bayes_apply: catalogue %d does not have the model's %d halos and types", r, b->n);
            return LT_ERR_INVALID_ARGUMENT;
        }
    if (nrows == 0 || b->n == 0) return LT_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const bool dev_rows = is_device_pointer(rows);
    const size_t ntheta = b->theta_cols.size();
    const size_t row_bytes = (size_t)nrows * b->ncols * sizeof(double);
    const size_t trig_bytes = dev_rows ? 0 : (size_t)nrows * ntheta * 2 * sizeof(double);
    const size_t cat_bytes = (size_t)nrows * sizeof(CatRecs);
    const size_t o_trig = (dev_rows ? 0 : (row_bytes + 255) / 256 * 256);
    const size_t o_cats = o_trig + (trig_bytes + 255) / 256 * 256;
    lt_status st = grow(ctx, &b->stage, &b->stage_bytes, o_cats + cat_bytes);
    if (st != LT_OK) return st;
    char *stage = (char *)b->stage;
    /* host rows: cos/sin of the sampled angles on the host, as the reference does
     * (src/module_readParameters.cpp:164-166) */
    std::vector<unsigned char> host(o_cats + cat_bytes);
    if (!dev_rows) {
        memcpy(host.data(), rows, row_bytes);
        double *tr = (double *)(host.data() + o_trig);
        for (int r = 0; r < nrows; r++)
            for (size_t k = 0; k < ntheta; k++) {
                const double ang = rows[(size_t)r * b->ncols + b->theta_cols[k]] * b->dtr;
                tr[2 * ((size_t)r * ntheta + k)] = cos(ang);
                tr[2 * ((size_t)r * ntheta + k) + 1] = sin(ang);
            }
    }
    CatRecs *cr = (CatRecs *)(host.data() + o_cats);
    for (int r = 0; r < nrows; r++) cr[r] = recs_of(cats[r]);
    const size_t from = dev_rows ? o_cats : 0;
    cudaError_t e = cudaMemcpyAsync(stage + from, host.data() + from, o_cats + cat_bytes - from,
                                    cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bayes rows upload");
    ApplyArgs a;
    a.m = b->dev;
    a.rows = dev_rows ? rows : (const double *)stage;
    a.trig = dev_rows ? nullptr : (const double *)(stage + o_trig);
    a.cats = (const CatRecs *)(stage + o_cats);
    a.nrows = nrows;
    a.status = ctx->status;
    bayes_apply_kernel<<<blocks_for((long)nrows * b->n), 256, 0, s>>>(a);
    count_launch(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bayes rows");
    return LT_OK;
}

extern "C" lt_status lt_bayes_destroy(lt_context *ctx, lt_bayes *b)
{
    if (!ctx || !b) return LT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize(); /* the stage may be read by an apply in flight */
    dev_free(ctx, b->stage, b->stage_bytes);
    dev_free(ctx, b->mem, b->bytes);
    delete b;
    return LT_OK;
}
