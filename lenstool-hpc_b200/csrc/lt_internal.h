/*
 * lt_internal.h -- library-internal declarations shared by the C-ABI translation units.
 */
#pragma once
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lt_b200.h"
#include "lt_grid.cuh"
#include "lt_halo.h"

struct lt_context {
    int device = 0;
    int num_sms = 0;
    size_t budget = 0, used = 0;
    std::mutex mu;
    std::string last_error;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    int32_t *status = nullptr; /* device status word written by kernels */
    void *ext = nullptr;       /* state of the batch and serving extensions */
    void *list = nullptr;      /* pixel list of the FP32C recomputation pass (+ count) */
    size_t list_bytes = 0;
    int shape[3][8] = {};      /* kernel shape per [precision][sums mask], LT_SHAPE4() */
    cudaStream_t copy_stream = nullptr; /* host-output calls: band copies overlap the next band */
    /* pass timing (lt_set_pass_timing): CUDA events around the passes of FP32C calls */
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;   /* created events, reused */
    std::vector<cudaEvent_t> ev_marks;  /* recorded marks: triples (start, pass 1 end, pass 2 end) */
};

struct lt_catalog {
    lt_rec64 *recs = nullptr;            /* FP64 records, device */
    lt_chunk *chunks = nullptr;          /* FP64 chunk list (runs of one type), device */
    lt_chunk *chunks_k = nullptr;        /* Kmap chunk list (runs of one type and dlsds) */
    int32_t nhalos = 0;
    int32_t nchunks = 0, nchunks_k = 0;
    size_t bytes = 0;
    std::vector<lt_rec64> host_recs;     /* packed records, host copy */
    std::vector<int32_t> host_types;     /* profile type per halo */
    void *aux = nullptr;                 /* FP32C records and chunks, device */
    size_t aux_bytes = 0;
    void *stage = nullptr;               /* device staging of host parameters (lt_catalog_update) */
    size_t stage_bytes = 0;
    alignas(16) unsigned char aux_desc[96]; /* FP32C descriptor (host) */
};

struct lt_rec32;


namespace lt {

/* FP32C: a pixel whose bound on the FP32 part's error of mu, relative to max(|mu|, 1),
 * exceeds this is recomputed in FP64 (near a critical curve the determinant amplifies
 * the error of the sums as |mu|); the maps are held to 1e-6 */
constexpr double kMuTol32 = 5.0e-7;

/* FP32C catalogue (lt_catalog::aux_desc): FP32 records + a chunk list over both record
 * kinds (chunk.pad & CHUNK_FP32: FP32 records of recs32, else FP64 records of recs64). */
struct Fp32cCatalog {
    lt_rec32 *recs32;
    lt_chunk *chunks;   /* chunks of at most 64 records */
    lt_chunk *chunks_s; /* the same records in chunks of at most 32 */
    lt_chunk *chunks_l; /* ... and of at most 128 */
    int32_t nchunks, nchunks_s, nchunks_l;
    int32_t n32;
    int32_t *idx32;  /* per halo: its FP32 record, or -1 for an FP64-class halo (device) */
    int32_t *types;  /* per halo profile type (device) */
    lt_nie64 *nie;   /* per halo (upload order): the FP64 closed-form record of the recomputation */
};

void count_launch(uint64_t n);
/* With pass timing on, record mark `which` (0: before pass 1, 1: after it, 2: after
 * pass 2) on `stream`; a call without pass 2 repeats mark 1 as mark 2. */
void pass_mark(lt_context *ctx, cudaStream_t stream, int which);
/* lt_hessian_maps_noalloc: forget the static list's address on `device` (its last
 * context is being destroyed) */
void noalloc_forget(int device);
/* FP32C kernel shapes the library is built for */
extern const int kShapes32[];
extern const int kNumShapes32;
bool shape32_ok(int shape);
/* allow the FP32C kernels their largest shared-memory stage on the current device */
int configure_kernels32();
void set_error(lt_context *ctx, const char *fmt, ...);
lt_status cuda_fail(lt_context *ctx, cudaError_t e, const char *what);
lt_status dev_alloc(lt_context *ctx, void **p, size_t bytes);
void dev_free(lt_context *ctx, void *p, size_t bytes);
lt_status scratch_planes(lt_context *ctx, int n, size_t plane_bytes, double **planes);
bool is_device_pointer(const void *p);
std::vector<lt_chunk> make_chunks(const int32_t *type, int n, int max_chunk, const double *dlsds = nullptr);

lt_status run_grid(lt_context *ctx, const lt_catalog *cat, const lt_grid *g, int precision, int op, int kmap, double D,
                   double mult, double scale, int nout, const int *kinds, double *const *outs, void *stream);
int launch_grid64_tiled(int op, GridArgs &a, int num_sms, void *stream, int shape);
int launch_epilogue_zero(const GridArgs &a, int num_sms, void *stream);
int launch_grid64_list(int op, GridArgs &a, int num_sms, void *stream);
/* map kind `kind` of device planes a (xx), b (xy), c (yy) into `out` (in place allowed) */
int launch_planes_epilogue(int kind, double *out, const double *a, const double *b, const double *c, double D,
                           double mult, int nx, int ny, int num_sms, void *stream);
lt_status list_buffer(lt_context *ctx, long npix, int32_t **list, int32_t **count);

/* FP32-compensated path (lt_grid32.cu) */
lt_status prepare_catalog_extensions(lt_context *ctx, lt_catalog *cat);
int launch_fp32c(lt_context *ctx, const lt_catalog *cat, int op, GridArgs &a, void *stream);
/* true for map kinds whose value depends on the Jacobian determinant */
bool det_sensitive(int kind);
bool grid_ok(const lt_grid *g);
bool hess_kind_ok(int kind);

/* batches and the serving loop (lt_queue.cu) */
void destroy_extensions(lt_context *ctx);
/* true when the catalogue's memory must outlive a running serving loop: it is then
 * released when the last server of the context is destroyed */
bool defer_release(lt_context *ctx, lt_catalog *cat);
/* free a catalogue's device memory (waits for the device) */
void free_catalog(lt_context *ctx, lt_catalog *cat);

} // namespace lt
