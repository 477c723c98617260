/*
 * lt_b200.h -- C ABI of the B200 lensing-map library (liblt_b200.so).
 *
 * The library evaluates Lenstool-HPC's per-pixel sum over halos of the lens-potential
 * gradient (deflection), Hessian and potential for the SIS (type 5), PIEMD (type 8) and
 * cut dPIE (type 81) profiles, and the maps built on them, on one NVIDIA B200.
 *
 * Conventions shared by every entry point
 *   - Plain C types only; every call returns an lt_status and never exits the process.
 *   - A catalogue is uploaded once (lt_catalog_upload) and stays resident in HBM; the
 *     grid calls take the handle.  The halo fields keep the meaning of the reference's
 *     struct Potential_SOA (src/structure_hpc.hpp:257-287).
 *   - Output planes are float64, row-major nx*ny, pixel (i, j) at
 *     x = xmin + (i + istart) dx, y = ymin + (j + jstart) dy and index j*nx + i
 *     (src/grid_gradient_CPU.cpp:67-100).
 *   - Output pointers may be device pointers (the call is then asynchronous on `stream`)
 *     or host pointers (the library stages through device memory, copies back and
 *     synchronises `stream` before returning, like the reference's host wrappers).
 *   - `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream.
 *   - Precision (lt_precision below): LT_FP64 reproduces the reference FP64 CPU path (the
 *     Hessian bit for bit); LT_FP32C runs the bulk halo sum in FP32 with compensated
 *     accumulation and keeps FP64 for cluster-scale halos, near-field pairs and pixels near
 *     critical curves (its error against FP64 is bounded by the tests).
 */
#ifndef LT_B200_H
#define LT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LT_B200_ABI_VERSION 1

typedef enum {
    LT_OK = 0,
    LT_ERR_INVALID_ARGUMENT = 1,   /* NULL pointer, bad size, bad grid, bad map kind */
    LT_ERR_UNKNOWN_PROFILE = 2,    /* halo type other than 5, 8, 81 */
    LT_ERR_NONFINITE = 3,          /* NaN/Inf or out-of-domain halo parameter */
    LT_ERR_CUDA = 4,               /* a CUDA runtime call failed (see lt_last_error) */
    LT_ERR_OUT_OF_MEMORY = 5,      /* device allocation failed */
    LT_ERR_BUDGET = 6,             /* the context's HBM budget would be exceeded */
    LT_ERR_QUEUE_FULL = 7,         /* serving queue has no free slot */
    LT_ERR_TIMEOUT = 8,            /* a bounded device-side wait gave up */
    LT_ERR_NO_DEVICE = 9,          /* no CUDA device / wrong architecture */
    LT_ERR_NOT_READY = 10          /* asynchronous result not yet available */
} lt_status;

/* LT_FP64: the reference's FP64 arithmetic; the Hessian sums reproduce its rounding
 *          sequence (bit-identical to the reference CPU path), deflection and potential
 *          agree to <= 1e-12.
 * LT_FP32C: FP32 bulk with compensated accumulation and FP64 where FP32 loses digits.
 * LT_FP64_FAST: FP64 with reciprocals, FMA and shared sub-expressions, the dPIE deflection
 *          as log(z_c/z_t) taken without cancellation and the potential through the
 *          deflection (x . alpha plus one logarithm per core radius); within 2e-12 of
 *          the reference except at the formula's ill-conditioned pixels (within ~1e-3"
 *          of each halo's removable singular points), where it departs by up to ~1e-11. */
typedef enum { LT_FP64 = 0, LT_FP32C = 1, LT_FP64_FAST = 2 } lt_precision;

/* Map kinds computed from the Hessian [[a, b], [d, c]] with D = dlsds (D_LS/D_OS).
 * Reference kernels: ampli src/grid_map_ampli_GPU.cu:329-547, shear
 * src/grid_map_shear_GPU.cu:208-369, mass src/grid_map_mass_GPU.cu:307-322. */
typedef enum {
    LT_MAP_HESS_A = 0, LT_MAP_HESS_B = 1, LT_MAP_HESS_C = 2, LT_MAP_HESS_D = 3, /* raw planes */
    LT_MAP_AMPLI1 = 11,  /* 1/(lambda mu) of A = 1 - aD, B = -bD, C = 1 - cD            */
    LT_MAP_AMPLI2 = 12,  /* 1/|lambda mu|                                              */
    LT_MAP_AMPLI3 = 13,  /* -2.5 log10 |lambda mu|                                     */
    LT_MAP_AMPLI4 = 14,  /* (1-k)(1+gp^2)/(1-gp^2), gp = |g|/(1-k)                      */
    LT_MAP_AMPLI5 = 15,  /* (a + c)/2, not scaled by D (as the reference)              */
    LT_MAP_AMPLI6 = 16,  /* sqrt(((a-c)/2)^2 + b^2), not scaled by D                   */
    LT_MAP_SHEAR1 = 21,  /* (lambda - mu)/2                                            */
    LT_MAP_SHEAR2 = 22,  /* |(q^2-1)/(q^2+1)|, q = lambda/mu                           */
    LT_MAP_SHEAR3 = 23,  /* gamma1 = (a - c) D/2                                       */
    LT_MAP_SHEAR4 = 24,  /* gamma2 = b D                                               */
    LT_MAP_KAPPA = 31,   /* kappa = (a + c) D/2                                        */
    LT_MAP_GAMMA1 = 32,  /* (a - c) D/2                                                */
    LT_MAP_GAMMA2 = 33,  /* b D                                                        */
    LT_MAP_MU = 34,      /* 1/((1-kappa)^2 - gamma1^2 - gamma2^2), determinant in FP64 */
    LT_MAP_MASS = 41,    /* (a + c)/2 * mult (Kmap Hessian; mult per mass mode)        */
    /* batch and serving requests only (lt_request): */
    LT_MAP_POTENTIAL = 51,    /* potential * scale                                     */
    LT_MAP_DEFLECTION_X = 61, /* deflection x * scale                                  */
    LT_MAP_DEFLECTION_Y = 62  /* deflection y * scale                                  */
} lt_map_kind;

#define LT_MAX_MAPS 8

/* Halo catalogue, host arrays of nhalos entries (Potential_SOA fields used by the path). */
typedef struct {
    int32_t nhalos;
    const int32_t *type;                  /* 5, 8 or 81                                 */
    const double *position_x, *position_y;/* arcsec                                     */
    const double *b0;                     /* impact parameter                           */
    const double *anglecos, *anglesin;    /* cos/sin of ellipticity_angle               */
    const double *ellipticity_potential;  /* in (0, 1)                                  */
    const double *rcore, *rcut;           /* arcsec (rcut > rcore for type 81)          */
    const double *dlsds;                  /* per-halo D_LS/D_OS for Kmap; NULL = all 1  */
} lt_halo_soa;

typedef struct {
    double xmin, ymin, dx, dy;
    int32_t nx, ny, istart, jstart;
} lt_grid;

typedef struct {
    int32_t kind;    /* lt_map_kind */
    double *out;     /* nx*ny float64, host or device */
} lt_map_request;

typedef struct {
    int32_t model;   /* 1 (CPL dark energy), src/module_cosmodistances.cpp:222-230 */
    double omegaM, omegaX, curvature, wX, wa, H0;
} lt_cosmology;

typedef struct lt_context lt_context;
typedef struct lt_catalog lt_catalog;

/* ---- context and catalogues ------------------------------------------------------ */

/* Create a context on CUDA device `device`.  hbm_budget_bytes caps the device memory the
 * context may hold (0 = 90% of free memory at creation).  No counterpart in the reference
 * (its wrappers allocate and free on every call, src/grid_gradient_GPU.cu:94-178). */
lt_status lt_create(int device, size_t hbm_budget_bytes, lt_context **ctx);
lt_status lt_destroy(lt_context *ctx);

/* Validate and pack a catalogue into HBM.  Replaces the per-call cudaMalloc/cudaMemcpy of
 * the reference wrappers (src/grid_map_ampli_GPU.cu:119-160). */
lt_status lt_catalog_upload(lt_context *ctx, const lt_halo_soa *soa, lt_catalog **cat);
lt_status lt_catalog_release(lt_context *ctx, lt_catalog *cat);
int32_t lt_catalog_nhalos(const lt_catalog *cat);

/* Physical halo parameters of one posterior sample, nhalos entries in the catalogue's
 * halo order (host arrays, or all device arrays). */
typedef struct {
    int32_t nhalos;
    const double *position_x, *position_y; /* arcsec                                       */
    const double *vdisp;                   /* km/s; b0 = 6 pi/c^2 vdisp^2 (SIS: 4 pi/c^2)  */
    const double *ellipticity;             /* mass ellipticity in [0, 1)                   */
    const double *ellipticity_angle;       /* radians                                      */
    const double *rcore, *rcut;            /* arcsec                                       */
    const double *anglecos, *anglesin;     /* optional (NULL: cos/sin of the angle, device) */
} lt_halo_params;

/* Re-derive a resident catalogue from a new sample on the device, in place and
 * stream-ordered: b0 and ellipticity_potential as
 * module_readParameters_calculatePotentialparameter (src/module_readParameters.cpp:
 * 2808-2871), then the records with the upload's packing arithmetic, so a device update
 * with the same parameters gives the same records bit for bit.  The types, order, dlsds
 * and the FP32C chunk lists are kept: a halo of the FP32 class whose new parameters need
 * FP64 everywhere is evaluated through its FP64 record, an FP64-class halo stays FP64.  A
 * sample outside a profile's domain makes lt_synchronize report LT_ERR_NONFINITE and
 * leaves that halo unchanged.  Batches holding the handle see the update on their next
 * launch; do not update a catalogue that in-flight serving requests use.  Host arrays are
 * staged in a per-catalogue device buffer: successive updates of one catalogue go on one
 * stream.  The reference applies a posterior row on the host
 * (module_readParameters_setbayesmapmodels, src/module_readParameters.cpp:132-227). */
lt_status lt_catalog_update(lt_context *ctx, lt_catalog *cat, const lt_halo_params *params, void *stream);

/* ---- bayes.dat rows on the device -------------------------------------------------- */

/* The model that bayes.dat rows perturb: the Potential_SOA state of every halo in
 * catalogue order (host arrays).  Both ellipticities are state, as in
 * module_readParameters_calculatePotentialparameter_SOA (src/module_readParameters.cpp:
 * 2873-2936); the state is taken to that step's fixed point before the first row. */
typedef struct {
    int32_t nhalos;
    const int32_t *type;                   /* 5, 8 or 81                                   */
    const double *position_x, *position_y; /* arcsec                                       */
    const double *ellipticity_potential;   /* epot                                         */
    const double *ellipticity;             /* emass                                        */
    const double *ellipticity_angle;       /* radians                                      */
    const double *rcore, *vdisp, *rcut;    /* arcsec, km/s, arcsec                         */
    const double *mag;                     /* magnitudes (potfile galaxies; NULL if none)  */
} lt_bayes_model;

/* One potfile (setScalingRelations, src/module_readParameters.cpp:1539-1656, ftype 1):
 * its galaxies are halos first .. first+count-1; a galaxy with mag != 0 gets
 * rcore = core 10^(0.4 (mag0 - mag)/2), vdisp = sigma 10^(0.4 (mag0 - mag)/vdslope),
 * rcut = cut 10^(0.4 (mag0 - mag) 2/slope).  Lengths in arcsec. */
typedef struct {
    int32_t first, count;
    double mag0, sigma, cut, core, vdslope, slope;
} lt_potfile;

/* What one bayes.dat column sets (module_readParameters_setbayesmapmodels,
 * src/module_readParameters.cpp:142-216). */
typedef enum {
    LT_BAYES_SKIP = 0,      /* Nsample, ln(Lhood), image redshifts, Chi2                 */
    LT_BAYES_X = 1, LT_BAYES_Y = 2, LT_BAYES_EPOT = 3, LT_BAYES_EMASS = 4,
    LT_BAYES_THETA = 5,     /* degrees                                                    */
    LT_BAYES_RCORE = 6, LT_BAYES_VDISP = 7, LT_BAYES_RCUT = 8,
    LT_BAYES_Z = 9,         /* read, no effect on the maps (D_LS/D_OS is set at upload)   */
    LT_BAYES_POT_CUT = 10,  /* potfile `target`'s cut (arcsec)                            */
    LT_BAYES_POT_SIGMA = 11 /* potfile `target`'s sigma (km/s)                            */
} lt_bayes_field;

typedef struct {
    int32_t field;  /* lt_bayes_field                                     */
    int32_t target; /* halo index (fields 1-9, not a potfile galaxy) or potfile index */
} lt_bayes_column;

typedef struct lt_bayes lt_bayes;

/* Upload a model and the meaning of each of a row's ncolumns values. */
lt_status lt_bayes_create(lt_context *ctx, const lt_bayes_model *model, int32_t npotfiles, const lt_potfile *potfiles,
                          int32_t ncolumns, const lt_bayes_column *columns, lt_bayes **bayes);
/* Row r of `rows` (nrows x ncolumns, host or device) applied to the model re-derives
 * catalogue cats[r] (same halos and types as the model) in place, stream-ordered: one
 * thread per (row, halo) sets the free parameters, applies the potfile scaling relations
 * with the row's sigma and cut, takes the potential-parameter step and packs the records
 * as lt_catalog_update does.  Rows are independent (each starts from the model's state).
 * With host rows the cos/sin of sampled angles are taken on the host, so the records
 * equal an upload of the reference's SoA bit for bit; with device rows they are taken on
 * the device.  Host rows are staged in a per-model device buffer: successive applies of
 * one model go on one stream.  Replaces the per-sample host update and SoA upload of the
 * reference's map loop (utils/maps/main.cpp:428-470). */
lt_status lt_bayes_apply(lt_context *ctx, lt_bayes *bayes, const double *rows, int32_t nrows,
                         lt_catalog *const *cats, void *stream);
lt_status lt_bayes_destroy(lt_context *ctx, lt_bayes *bayes);

/* ---- grid evaluators ------------------------------------------------------------- */

/* Deflection grid, both planes multiplied by `scale` (1 for the raw gradient, D_LS/D_OS
 * for a displacement map).  Replaces gradient_grid_CPU/GPU (src/grid_gradient_CPU.cpp:56,
 * src/grid_gradient_GPU.cu:77-179), module_potentialDerivatives_totalGradient_SOA_CPU_GPU
 * (src/grid_gradient_GPU.cuh:40-41) and map_grid_dpl_GPU (src/grid_map_dpl_GPU.cu:75-173). */
lt_status lt_gradient_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                           double scale, double *ax, double *ay, void *stream);

/* Hessian grid and up to LT_MAX_MAPS derived maps in one pass.  kmap != 0 weights every
 * halo by its dlsds (module_potentialDerivatives_Kmap_SOA_GPU, src/gradient2_GPU.cu:455-522).
 * Replaces gradient2_grid_CPU/GPU (src/grid_gradient2_CPU.cpp:54-83,
 * src/grid_gradient2_GPU.cu:77-183) and map_grid_{ampli,shear,mass}_GPU
 * (src/grid_map_ampli_GPU.cu:93-192, src/grid_map_shear_GPU.cu:87-187,
 * src/grid_map_mass_GPU.cu:82-216). */
lt_status lt_hessian_maps(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                          int32_t kmap, double dlsds, double mult, const lt_map_request *maps, int32_t nmaps,
                          void *stream);

/* Potential grid multiplied by `scale` (D_LS/D_OS for potential mode 1, cH2piG h / D_OL
 * for mode 2).  Replaces potential_grid_GPU / module_potential_SOA_CPU_GPU
 * (src/grid_potential_GPU.cu:68-184) and map_grid_potential_GPU
 * (src/grid_map_pot_GPU.cu:83-273). */
lt_status lt_potential_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                            double scale, double *psi, void *stream);

/* All configuration-1 maps of one grid in one fused pass: kappa, gamma1, gamma2, mu (as
 * LT_MAP_*), and the potential scaled by D (any output may be NULL). */
lt_status lt_lens_maps(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t precision,
                       double dlsds, double *kappa, double *gamma1, double *gamma2, double *mu, double *psi,
                       void *stream);

/* ---- kernel shapes and the autotuner ----------------------------------------------
 * A grid kernel comes in shapes: pixels per thread (1 or 2) and the resident CTAs per SM
 * its register budget is cut for (1 or 2).  `sums` is a mask: 1 deflection, 2 Hessian,
 * 4 potential (6 = the fused lens maps).  No counterpart in the reference (its launch
 * shape is fixed, src/grid_gradient2_GPU.cu:28-29). */
lt_status lt_set_kernel_shape(lt_context *ctx, int32_t precision, int32_t sums, int32_t pixels_per_thread,
                              int32_t ctas_per_sm);
lt_status lt_get_kernel_shape(const lt_context *ctx, int32_t precision, int32_t sums, int32_t *pixels_per_thread,
                              int32_t *ctas_per_sm);
/* The full kernel configuration: besides the shape, the threads per CTA (128 or 256; a
 * tile is 32 x pixels_per_thread columns by threads / 32 rows) and the halo records per
 * shared-memory stage (32, 64 or 128).  LT_FP32C kernels come in the shapes
 * (pixels, CTAs/SM, threads) = (1|2, 1|2, 256), (1, 2|4, 128), (2, 2|3|4, 128), each with
 * every stage size; the FP64 kernels in their four 256-thread, 64-record shapes.  An
 * unbuilt configuration is LT_ERR_INVALID_ARGUMENT.  lt_set_kernel_shape keeps 256 threads
 * and 64-record stages. */
typedef struct {
    int32_t pixels_per_thread, ctas_per_sm, threads, chunk;
} lt_kernel_config;
lt_status lt_set_kernel_config(lt_context *ctx, int32_t precision, int32_t sums, const lt_kernel_config *config);
lt_status lt_get_kernel_config(const lt_context *ctx, int32_t precision, int32_t sums, lt_kernel_config *config);
/* Time every configuration for (precision, sums) on a grid_n x grid_n grid covering the
 * catalogue and keep the fastest in the context; *best_ms (may be NULL) gets its time.
 * The batches built afterwards use the tuned LT_FP32C Hessian shape where their
 * persistent kernel is built for it (pixels per thread and CTAs per SM at 256 threads). */
lt_status lt_autotune(lt_context *ctx, const lt_catalog *cat, int32_t precision, int32_t sums, int32_t grid_n,
                      double *best_ms);

/* ---- pass timing --------------------------------------------------------------------
 * With timing on, every LT_FP32C grid call records CUDA events on its stream around its
 * two passes (pass 1: the FP32C kernel; pass 2: the FP64 recomputation of the pixels
 * near critical curves).  lt_pass_times waits for the last recorded call, returns the
 * summed durations (ms) and the number of launches since the previous read (a call with
 * host outputs runs the grid in bands of rows, one launch each), and starts a new count.
 * No counterpart in the reference. */
lt_status lt_set_pass_timing(lt_context *ctx, int32_t on);
lt_status lt_pass_times(lt_context *ctx, double *pass1_ms, double *pass2_ms, int32_t *calls);

/* Pixels of the LT_FP32C calls, batches and serving loops of this context recomputed in
 * FP64 (their error estimate failed after pass 1) since the previous read; resets the
 * count.  No counterpart in the reference. */
lt_status lt_recompute_count(lt_context *ctx, uint64_t *pixels);

/* ---- requests: batches and the serving loop ----------------------------------------
 * A request is one grid of output planes over one uploaded catalogue: any mix of Hessian
 * maps (lt_map_kind 0-41, with `dlsds` as D, `kmap` and `mult` as in lt_hessian_maps),
 * the potential and the deflection (both multiplied by `scale`).  Results equal those of
 * the single-grid calls in the same precision (LT_FP32C or LT_FP64) bit for bit.
 * No counterpart in the reference, whose posterior driver makes one blocking map call
 * per sample (utils/maps/main.cpp:432-587). */
typedef struct {
    const lt_catalog *cat;
    lt_grid grid;
    int32_t kmap;
    double dlsds, mult, scale;
    int32_t nmaps;
    lt_map_request maps[LT_MAX_MAPS];
} lt_request;

typedef struct lt_batch lt_batch;

/* Pack `nreqs` requests (device-pointer outputs) into a batch: one CUDA graph whose
 * persistent kernel evaluates every request's pixel tiles, costliest requests first. */
lt_status lt_batch_create(lt_context *ctx, const lt_request *reqs, int32_t nreqs, int32_t precision,
                          lt_batch **batch);
/* Replay the batch's graph on `stream` (asynchronous; lt_synchronize reports errors). */
lt_status lt_batch_launch(lt_context *ctx, lt_batch *batch, void *stream);
int32_t lt_batch_size(const lt_batch *batch);
/* The batch's kernel configuration: its persistent kernel's pixels per thread and CTAs
 * per SM for LT_FP32C tiles (taken at lt_batch_create from the context's LT_FP32C Hessian
 * shape, as lt_autotune left it), 256 threads, 64-record stages. */
lt_status lt_batch_config(const lt_batch *batch, lt_kernel_config *config);
lt_status lt_batch_destroy(lt_context *ctx, lt_batch *batch);

typedef struct lt_server lt_server;

typedef struct {
    int32_t precision;    /* LT_FP32C or LT_FP64                                          */
    int32_t slots;        /* requests on the GPU at once (0: 64)                           */
    int32_t window;       /* oldest requests served round-robin, tile by tile (0: 8)       */
    int32_t idle_us;      /* idle time after which the persistent kernel leaves (0: 20000) */
    size_t output_bytes;  /* HBM arena staging host-pointer outputs: the admission budget  */
                          /* (0: 4 GiB)                                                    */
    int32_t descriptor_wait_us; /* the loop's bounded wait for the descriptor of a published
                                   request (~1 us polls, 0: 2 s); when it runs out the request
                                   fails with LT_ERR_TIMEOUT and the loop serves the rest   */
} lt_server_config;

typedef struct {
    uint64_t submitted, admitted, completed, failed, loop_launches;
    int32_t max_inflight, inflight, queued, loop_running;
    size_t arena_bytes, arena_peak;
    uint64_t device_published, device_head; /* the queue's counters as the device sees them */
    uint64_t timed_out;   /* requests failed because their descriptor never reached the device */
} lt_server_stats;

/* Start a serving loop on the context.  While it runs, lt_catalog_release defers the
 * release of catalogues until the context's last server is destroyed, and the context's
 * other calls wait for the loop's kernel whenever it holds the SMs. */
lt_status lt_server_create(lt_context *ctx, const lt_server_config *config, lt_server **server);
/* Queue a request (host or device outputs; host outputs are staged in the arena and
 * copied back, pinned host memory recommended).  Returns at once with a ticket;
 * LT_ERR_BUDGET if the request's planes can never fit in the arena.  The server writes
 * device outputs from its own stream: work that uses them must be complete at
 * submission, and their contents are defined once the ticket completes. */
lt_status lt_server_submit(lt_server *server, const lt_request *req, uint64_t *ticket);
/* LT_OK when the ticket's results are in place, LT_ERR_NOT_READY before, or its error. */
lt_status lt_server_poll(lt_server *server, uint64_t ticket);
/* Block until the ticket completes or `timeout_s` passes (LT_ERR_NOT_READY). */
lt_status lt_server_wait(lt_server *server, uint64_t ticket, double timeout_s);
/* Milliseconds from submission to admission, admission to GPU completion, and
 * submission to results in place. */
lt_status lt_server_request_times(lt_server *server, uint64_t ticket, double *queued_ms, double *gpu_ms,
                                  double *total_ms);
/* Forget a completed ticket. */
lt_status lt_server_release(lt_server *server, uint64_t ticket);
lt_status lt_server_get_stats(lt_server *server, lt_server_stats *stats);
/* Finish every submitted request, stop the loop and free the server. */
lt_status lt_server_destroy(lt_server *server);
/* Failure injection on the host, for tests of the loop's bounded waits:
 * LT_FAULT_DROP_DESCRIPTOR publishes the next admitted request without copying its
 * descriptor to the device (a lost message), so the loop's wait for it runs out and the
 * request fails with LT_ERR_TIMEOUT while later requests are served.  No counterpart in
 * the reference (its GPU calls exit on error, src/grid_gradient_GPU.cu:48-51). */
#define LT_FAULT_DROP_DESCRIPTOR 1
lt_status lt_server_inject_fault(lt_server *server, int32_t fault);

/* ---- Hessian maps without allocation ------------------------------------------------
 * lt_hessian_maps in LT_FP32C with device outputs, for callers that must not allocate
 * device memory during a call (a process running under a fixed device-memory plan, or a
 * timed loop that must not meet cudaMalloc's implicit synchronisation): the list of
 * pixels recomputed in FP64 lives in a static 16 MiB device array instead of a context
 * buffer grown with cudaMalloc, and the call allocates nothing.  The list's length word
 * must start at zero; the call zeroes it on `stream` itself.  Limits: grids of at most
 * 2048 x 2048 pixels (larger: LT_ERR_INVALID_ARGUMENT), device outputs only, and one array
 * per process and device, so calls that overlap in time race on it and must be
 * serialised by the caller.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress, return code checked) and loads the module's data there; make
 * that first call before any stream capture that includes this call.  The address is
 * kept until the last context of the device is destroyed (lt_destroy); a device reset
 * (cudaDeviceReset) while a context lives invalidates it, so the call must not be used
 * across a reset.  No counterpart in the reference. */
lt_status lt_hessian_maps_noalloc(lt_context *ctx, const lt_catalog *cat, const lt_grid *grid, int32_t kmap,
                                  double dlsds, double mult, const lt_map_request *maps, int32_t nmaps,
                                  void *stream);

/* ---- strong-lensing chi2 by barycentric delensing -----------------------------------
 * The reference's chi2 of a model (mychi_bruteforce_SOA_CPU_grid_gradient_barycentersource,
 * src/chi_CPU_barycenter.cpp:58-287): the deflection grid over `frame` with n x n pixels
 * (dx = (xmax - xmin)/(n - 1)), each system's source as the barycentre of its images
 * mapped to the source plane, the predicted images of that source by delensing the grid's
 * triangles (src/delense_CPU.cpp:6-140), and the link of predicted to observed images
 * with chi2 = sum |observed - predicted|^2 + 1000 x (images) per unlinked observed image
 * (src/chi_computation.cpp:11-195).  FP64; the inclusion tests round exactly as the
 * reference's for the same deflections. */
#define LT_MAX_IMAGES 20 /* predicted images kept per source (MAXIMPERSOURCE) */

typedef struct {
    double xmin, xmax, ymin, ymax;     /* the reference's grid_param frame               */
} lt_frame;

typedef struct {
    int32_t nsystems;
    const int32_t *nimages;            /* observed images per system (1..40)             */
    const double *x, *y;               /* observed positions, concatenated by system     */
    const double *dlsds;               /* per system: D_LS/D_OS of its source (dr)       */
} lt_image_systems;

/* chi2 of one model (host results; synchronous).  images_found (may be NULL) gets the
 * number of predicted images.  LT_ERR_QUEUE_FULL when a source had more than
 * LT_MAX_IMAGES predicted images (the first LT_MAX_IMAGES were used). */
lt_status lt_chi2(lt_context *ctx, const lt_catalog *cat, const lt_frame *frame, int32_t n,
                  const lt_image_systems *systems, double *chi2, int32_t *images_found);
/* chi2 of `nmodels` models against the same systems (chi2[m], images_found[m]). */
lt_status lt_chi2_batch(lt_context *ctx, const lt_catalog *const *cats, int32_t nmodels, const lt_frame *frame,
                        int32_t n, const lt_image_systems *systems, double *chi2, int32_t *images_found);
/* lt_chi2_batch with the deflection grid in `precision`: LT_FP64 (as lt_chi2_batch;
 * LT_FP64_FAST is the same grid) or LT_FP32C, whose grid is within 1e-6 of the FP64 one;
 * the sources, the delensing and the chi2 reduction are FP64 in every case.  The
 * reference computes the grid in FP64 (src/chi_CPU_barycenter.cpp:127-137). */
lt_status lt_chi2_batch_precision(lt_context *ctx, const lt_catalog *const *cats, int32_t nmodels,
                                  const lt_frame *frame, int32_t n, const lt_image_systems *systems,
                                  int32_t precision, double *chi2, int32_t *images_found);
/* Write a host map (nx * ny float64, row j at image row j + 1) as a FITS primary image in
 * the reference's layout (module_writeFits_Image, src/module_writeFits.cpp:113-206):
 * float32 data, BZERO/BSCALE, a linear arcsec WCS with pixel 1 at (xmin, ymin) and
 * CDELT = (max - min)/(n - 1), ORIGIN and DATE.  No cfitsio; host only. */
lt_status lt_write_fits(const char *path, const double *map, int32_t nx, int32_t ny, const lt_frame *frame);

/* Predicted images of given source positions (bx, by, dlsds per source) by delensing the
 * n x n grid: nfound[s] images at fx/fy[s * LT_MAX_IMAGES + k], in the reference's order.
 * No counterpart as an entry point in the reference (its step 3 of the chi2). */
lt_status lt_delense(lt_context *ctx, const lt_catalog *cat, const lt_frame *frame, int32_t n, int32_t nsources,
                     const double *bx, const double *by, const double *dlsds, int32_t *nfound, double *fx,
                     double *fy);

/* A chi2 request to the serving loop: the chi2 of `cat` against `systems` on an n x n grid
 * over `frame`, as lt_chi2_batch_precision in the server's precision.  Its deflection grid
 * is served by the persistent loop tile by tile like a map request (the grid, the systems
 * and the work buffers take arena bytes until the result is in); the loop then yields the
 * GPU at its next tile boundary for the delensing and chi2 kernels and resumes the other
 * requests' remaining tiles.  The systems are copied at submission.  No counterpart in the
 * reference, whose chi2 is one blocking call per model (src/chi_CPU_barycenter.cpp:58). */
lt_status lt_server_submit_chi2(lt_server *server, const lt_catalog *cat, const lt_frame *frame, int32_t n,
                                const lt_image_systems *systems, uint64_t *ticket);
/* The chi2 and predicted-image count of a completed chi2 ticket (LT_ERR_NOT_READY before;
 * LT_ERR_QUEUE_FULL, with the values, when a source had more than LT_MAX_IMAGES images). */
lt_status lt_server_chi2_result(lt_server *server, uint64_t ticket, double *chi2, int32_t *images_found);

/* Wait for the context's work on `stream` and report any status a kernel recorded
 * (e.g. LT_ERR_TIMEOUT from a bounded device-side wait).  Asynchronous (device-pointer)
 * calls report such errors here. */
lt_status lt_synchronize(lt_context *ctx, void *stream);

/* ---- cosmology and utilities ----------------------------------------------------- */

/* D_LS, D_OS, D_OL in units of c/H0 (module_cosmodistances_objectObject/observerObject,
 * src/module_cosmodistances.cpp:94-151).  Host only; needs no GPU. */
lt_status lt_cosmo_distances(const lt_cosmology *cosmo, double zl, double zs, double *dls, double *dos,
                             double *dol);

/* Number of kernels this library has launched in the calling process (all contexts). */
uint64_t lt_kernel_launch_count(void);

/* Measured FMA-pipe throughput of `device` in TFLOP/s (an FMA counts 2 flops), FP64
 * (fp32 = 0) or FP32 (fp32 = 1); 0 on failure.  A measurement utility with no
 * counterpart in the reference: the denominator of the grid kernels' roofline. */
double lt_measure_fma_peak(int fp32, int device);

/* Evaluate, on `device`, the reciprocal and reciprocal square root that the FP64 pair
 * loops use for their per-pair denominators (hardware approximation + one third-order
 * refinement) on n host inputs: a diagnostic for the tests (0 = LT_OK).  No counterpart in the
 * reference. */
int lt_eval_fast_math(int device, int n, const double *x, double *rcp, double *rsqrt);

/* The same for the FP32 atan2, square root and atanh of the compensated pair loops:
 * atan2(y, x) by the library's own polynomial (atan2_own) and by CUDA's atan2f
 * (atan2_cuda), the approximate square root of x (sqrt_own), and atanh(y) by the
 * polynomial the deflection and potential use for |y| <= 1/3 (atanh_own), on n host
 * inputs (0 = LT_OK). */
int lt_eval_fast_math32(int device, int n, const float *y, const float *x, float *atan2_own, float *atan2_cuda,
                        float *sqrt_own, float *atanh_own);

/* The approximate FP32 reciprocal, reciprocal square root and natural logarithm of the
 * compensated pair loops (the .ftz instruction forms; the logarithm as ln 2 log2 x) and
 * CUDA's logf, on n host inputs (0 = LT_OK). */
int lt_eval_approx32(int device, int n, const float *x, float *rcp, float *rsqrt, float *log_own, float *log_cuda);

const char *lt_status_string(lt_status status);
/* Last error message recorded by the context (never NULL). */
const char *lt_last_error(const lt_context *ctx);
int32_t lt_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LT_B200_H */
