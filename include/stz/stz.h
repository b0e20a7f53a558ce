/*
 * stz.h — C ABI of the B200-native STZ streaming compressor (libstz_b200.so).
 *
 * STZ ("streaming" hierarchical lossy compression of 3-D fields) splits a field
 * into parity sub-blocks level by level, predicts each level's seven odd-parity
 * sub-blocks from the decoded coarser grid, quantizes the residuals under an
 * error bound, entropy-codes them per marker chunk, and finishes with zstd.
 * Every decode mode of the reference is here: full, progressive resolution
 * (1/2, 1/4, ... of each axis) and random-access box / slice.
 *
 * Reference: FabioGrosso/SC25-STZ2. The reference is a set of C++ programs
 * whose stages are free function templates in one translation unit,
 * src/zero_all_line_dynamic_random_access_optfast3_optcr_lb_fastdec5.cpp,
 * cited below as FD5:<line>. Each entry point below names the reference
 * function it replaces.
 *
 * Conventions
 *   - Plain pointers and sizes, no exceptions. Every call returns stz_status;
 *     stz_last_error() gives a thread-local message for the last failure.
 *   - Dims are (nx, ny, nz) with x fastest (row-major z, y, x), as in the
 *     reference (FD5:113).
 *   - `_dev` entry points take CUDA device pointers on the context's device
 *     and run on the context's stream; others take host pointers. The
 *     context's stream does not wait for other streams: device inputs
 *     written on another stream must be complete before the call (synchronize
 *     the producing stream). compress / decompress / box calls return with
 *     their outputs complete; the function-level boundary calls below are
 *     asynchronous on the context's stream (stz_context_sync).
 *   - The library owns stz_stream objects; callers own every output buffer.
 *   - A context is used by one host thread at a time; streams are immutable
 *     after creation and can be shared for reading.
 */
#ifndef STZ_B200_STZ_H
#define STZ_B200_STZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum stz_status {
    STZ_OK = 0,
    STZ_ERR_ARG = 1,          /* null pointer, bad option value */
    STZ_ERR_DIMS = 2,         /* dims not divisible as the format needs (FD5:1976-2006) */
    STZ_ERR_CUDA = 3,         /* CUDA runtime failure (message in stz_last_error) */
    STZ_ERR_NOMEM = 4,        /* host or device allocation failed */
    STZ_ERR_FORMAT = 5,       /* stream bytes are not a valid container */
    STZ_ERR_ZSTD = 6,         /* zstd reported an error */
    STZ_ERR_RANGE = 7,        /* level / box / block index out of range */
    STZ_ERR_UNSUPPORTED = 8   /* valid request this build does not handle */
} stz_status;

typedef enum stz_dtype { STZ_F32 = 0, STZ_F64 = 1 } stz_dtype;

/* How opts.eb is interpreted. */
typedef enum stz_eb_mode {
    STZ_EB_ABS = 0, /* absolute */
    STZ_EB_REL = 1  /* relative to the value range max - min (computeRange, FD5:92-104) */
} stz_eb_mode;

/* What the (absolute) bound E means. */
typedef enum stz_bound_mode {
    /* max |x - x'| <= E: the level multipliers are applied to E / max(mult). */
    STZ_BOUND_POINTWISE = 0,
    /* E is the reference CLI's eb: level k uses mult_k * E (FD5:2120-2129,
     * 2139, 2203, 2249), so the pointwise bound is max(mult) * E. */
    STZ_BOUND_REFERENCE = 1
} stz_bound_mode;

typedef enum stz_predictor {
    STZ_PRED_DYNAMIC = 0, /* inverse-variance blend of cubic lines (FD5:624-748) */
    STZ_PRED_CUBIC = 1,   /* fixed tricubic-family stencils (src/float.cpp:84-273) */
    /* Staged: sub-blocks 1, 2, 4 from 1-D cubics on the coarse grid, then 3, 5,
     * 6 and 7 from inverse-variance blends of 1-D cubics through the siblings
     * decoded before them (src/dependency.cpp:90-330, stage order 659-704).
     * No learned correction; boxes and slices decode the whole field (into a
     * context buffer of the field's size) and copy the box out; the request
     * server does not take these streams. Compress keeps the finest level's
     * decoded values, a device scratch of the field's size. */
    STZ_PRED_STAGED = 2,
    /* src/stz2.cpp: float.cpp's stencils with a 12-point truncated bicubic
     * (no corner taps) for sub-blocks 3, 5, 6 and the one-axis interior cubic
     * in double (stz2.cpp:82-309). No learned correction, boxes through the
     * whole field, no request server, as STZ_PRED_STAGED (no compress scratch). */
    STZ_PRED_TRUNCATED = 3
} stz_predictor;

typedef struct stz_opts {
    double eb;            /* error bound, see eb_mode / bound_mode */
    int eb_mode;          /* stz_eb_mode */
    int bound_mode;       /* stz_bound_mode */
    double mult_base;     /* level multipliers, FD5 defaults 0.7 / 2.7 / 8.2 */
    double mult_low;
    double mult_high;
    int radius;           /* quantizer radius (SZ3 default 32768, must be <= 32768) */
    int chunk_high;       /* marker chunk edge of the finest level (FD5 default 32) */
    int chunk_low;        /* marker chunk edge of the second-finest level (FD5 default 16) */
    int zstd_level;       /* final lossless stage level (SZ3 default 3); 0 stores frames raw */
    int predictor;        /* stz_predictor */
    int threads;          /* host threads for zstd; 0 = all cores */
    /* Learned correction (this library's addition; streams that use it are
     * container version 2): an int8 MLP per level adds a correction to the
     * predictions of the second-finest and finest levels. null = none. */
    const struct stz_model* model;
    /* -1: per level and block, use the correction where a sampled code-length
     * estimate says it pays; >= 0: forced blocks, bits 0-6 for the
     * second-finest level and bits 8-14 for the finest. */
    int learned_flags;
} stz_opts;

/* Reference defaults: rel eb 1e-3, pointwise, multipliers 0.7/2.7/8.2,
 * radius 32768, chunks 32/16, zstd 3, dynamic predictor, no learned model. */
void stz_default_opts(stz_opts* opts);

typedef struct stz_context stz_context;
typedef struct stz_stream stz_stream;
typedef struct stz_model stz_model;

typedef struct stz_info {
    int dtype;            /* stz_dtype */
    int predictor;
    size_t nx, ny, nz;
    int n_levels;         /* refinement levels; decode levels 0..n_levels */
    int radius;
    int chunk_high, chunk_low;
    double eb;            /* absolute eb the level multipliers were applied to */
    double mult_base, mult_low, mult_high;
    double max_error;     /* guaranteed max |x - x'| of a full decode */
    size_t stream_bytes;  /* serialized size */
    size_t raw_payload_bytes; /* entropy-coded bytes before zstd */
    int learned_flags;    /* learned-correction blocks, encoded as stz_opts.learned_flags */
} stz_info;

const char* stz_status_string(stz_status s);
/* Message of the last failing call on this thread ("" if none). */
const char* stz_last_error(void);

/* Context: one CUDA device, one CUDA stream, cached device/pinned buffers and
 * a host thread pool for zstd. */
stz_status stz_context_create(int device, stz_context** out);
void stz_context_destroy(stz_context* ctx);
/* Wait for all work queued on the context's stream. */
stz_status stz_context_sync(stz_context* ctx);

/* The CUDA stream (cudaStream_t) all of the context's work is queued on. */
stz_status stz_context_stream(stz_context* ctx, void** stream);

/* Per-kernel timing with CUDA events on the context's stream, for
 * benchmarking. While enabled, every kernel launch is bracketed by events and
 * its duration is accumulated under the kernel's name; launches are counted
 * whether or not timing is enabled. */
stz_status stz_profile_enable(stz_context* ctx, int on);
stz_status stz_profile_reset(stz_context* ctx);
/* Number of distinct kernel names recorded, and the totals of entry i. */
stz_status stz_profile_count(stz_context* ctx, int* n);
stz_status stz_profile_entry(stz_context* ctx, int i, const char** name, double* total_ms, uint64_t* launches);

/* ---- whole-field codec ------------------------------------------------ */

/* compress(field, dims, eb) -> stream. Replaces the compress phase of
 * run_typed (FD5:2093-2309): split, base, low and high levels, each level's
 * SZ_compress / SZ_compress_finish (FD5:1258-1437) and the final zstd. */
stz_status stz_compress(stz_context* ctx, const void* field, stz_dtype dtype, size_t nx, size_t ny, size_t nz,
                        const stz_opts* opts, stz_stream** out);
stz_status stz_compress_dev(stz_context* ctx, const void* field_dev, stz_dtype dtype, size_t nx, size_t ny, size_t nz,
                            const stz_opts* opts, stz_stream** out);

/* Full decompress (FD5:2338-2453: base decode, SZ_decompress_separated per
 * residual stream FD5:1466-1576, depreprocess + merge). out holds nx*ny*nz. */
stz_status stz_decompress_full(stz_context* ctx, const stz_stream* s, void* out);
stz_status stz_decompress_full_dev(stz_context* ctx, const stz_stream* s, void* out_dev);

/* Progressive decompress: level 0 = full, 1 = half resolution (the reference's
 * mid grid, FD5:2394), 2 = quarter (its decoded base, FD5:2339), ... up to
 * n_levels. out holds (nx>>level)*(ny>>level)*(nz>>level) values; the
 * resulting dims are written to out_dims when it is not null. */
stz_status stz_decompress_level(stz_context* ctx, const stz_stream* s, int level, void* out, size_t out_dims[3]);
stz_status stz_decompress_level_dev(stz_context* ctx, const stz_stream* s, int level, void* out_dev,
                                    size_t out_dims[3]);

/* Random-access box / slice (FD5:2460-2640): lo/hi are the inclusive corner
 * coordinates of the query (make_query, FD5:1637: any order, clamped to the
 * field; lo == hi on an axis makes a slice). Only the marker chunks and levels
 * the box touches are entropy-decoded (planner FD5:1578-1839). out receives
 * the box row-major (z, y, x); its dims are written to out_dims if not null. */
stz_status stz_decompress_box(stz_context* ctx, const stz_stream* s, const int64_t lo[3], const int64_t hi[3],
                              void* out, size_t out_dims[3]);
stz_status stz_decompress_box_dev(stz_context* ctx, const stz_stream* s, const int64_t lo[3], const int64_t hi[3],
                                  void* out_dev, size_t out_dims[3]);

/* ---- stream objects --------------------------------------------------- */

/* Serialized bytes (valid while the stream lives). */
stz_status stz_stream_bytes(const stz_stream* s, const void** data, size_t* size);
/* Parse serialized bytes (copied). */
stz_status stz_stream_parse(stz_context* ctx, const void* data, size_t size, stz_stream** out);
stz_status stz_stream_info(const stz_stream* s, stz_info* info);
/* Decode the zstd frames once and keep the entropy-coded streams resident on
 * the context's device, so later decodes skip zstd and the host->device copy. */
stz_status stz_stream_upload(stz_context* ctx, stz_stream* s);
void stz_stream_free(stz_stream* s);

/* ---- learned correction models ---------------------------------------- *
 * A model file holds up to two 2112-byte level records (second-finest,
 * finest): "STZLMDL1", a u32 mask (bit 0 / bit 1: record present), then the
 * present records in that order, little-endian. A record: f64 s_in, s_out;
 * int8 w1[32][16]; i32 b1[32], m1, sh1; int8 w2[32][32]; i32 b2[32], m2, sh2;
 * int8 w3[8][32]; i32 b3[8]. */
stz_status stz_model_parse(const void* data, size_t size, stz_model** out);
stz_status stz_model_bytes(const stz_model* m, const void** data, size_t* size);
void stz_model_free(stz_model* m);

/* ---- training (on the GPU) --------------------------------------------- *
 * Pairs come from the compressor itself: for the second-finest and finest
 * levels, the decoded coarse grid the level predicts from (its 14-point cell
 * stencil, minus the mean of the 8 corners, in units of the level's eb) and
 * the true fine values minus the plain prediction (in eb). Each level's MLP
 * is trained with BF16 operands and FP32 accumulation (forward, backward and
 * Adam are this library's kernels; a training run is replayed from CUDA
 * graphs), then quantization-aware trained and exported to int8. */
typedef struct stz_train_opts {
    int epochs;          /* float epochs (default 8) */
    int qat_epochs;      /* quantization-aware epochs (default 3) */
    int batch;           /* samples per Adam step, a multiple of 128 (default 4096) */
    double lr;           /* Adam step size (default 2e-3; QAT uses lr / 8), cosine decay */
    double huber_delta;  /* loss: Huber on the residual, in eb (default 2) */
    int sample_step;     /* pairs from every n-th interior coarse cell per axis (default 2) */
    size_t max_pairs;    /* pairs kept per level (default 1 << 23) */
    uint64_t seed;       /* initialisation and shuffling (default 1) */
} stz_train_opts;
void stz_default_train_opts(stz_train_opts* t);

typedef struct stz_train_stats {
    size_t pairs[2];       /* (second-finest, finest) */
    double loss_zero[2];   /* mean Huber loss per residual without a correction, eb^2 */
    double loss_float[2];  /* after the float epochs */
    double loss_qat[2];    /* after quantization-aware training (fake-quantized forward) */
    double loss_int8[2];   /* exported int8 model, integer inference on the stored features */
    double s_in[2], s_t[2];/* input and target scales */
    double train_ms;       /* device time of the fit */
} stz_train_stats;

typedef struct stz_trainer stz_trainer;
/* opts: the compressor options the pairs are generated with (eb, eb_mode,
 * predictor, multipliers...); its model field is ignored. */
stz_status stz_trainer_create(stz_context* ctx, const stz_opts* opts, const stz_train_opts* topts,
                              stz_trainer** out);
/* Adds the pairs of one field (device memory, x fastest). */
stz_status stz_trainer_add_field_dev(stz_trainer* t, const void* field_dev, stz_dtype dtype, size_t nx, size_t ny,
                                     size_t nz);
/* Trains both levels and returns the int8 model (free with stz_model_free). */
stz_status stz_trainer_fit(stz_trainer* t, stz_model** out);
stz_status stz_trainer_stats(const stz_trainer* t, stz_train_stats* st);
void stz_trainer_free(stz_trainer* t);

/* One forward + backward pass of the training kernels over n samples, for
 * gradient checks: params (1864 floats: W1[32][16], b1[32], W2[32][32],
 * b2[32], W3[8][32], b3[8]) as the master weights, x n x 16 features in eb
 * (rounded to BF16 as stored), t n x 8 targets in eb; s_in, s_t the scales,
 * qat 0/1 with activation scales sa[2]. Writes the mean loss (normalised
 * units) and the 1864 gradients. */
/* The exported int8 network on n rows of int8 inputs (16 per row, the last
 * two zero), host buffers: out (n x 8 int32) receives the output
 * accumulators of the 7 blocks (and a zero). tensor_cores = 1 runs the
 * tcgen05 kind::i8 kernel, 0 the dp4a form of the level kernels. */
stz_status stz_debug_learned_infer(stz_context* ctx, const int8_t* xq, size_t n, const void* model_record,
                                   int tensor_cores, int32_t* out);

stz_status stz_debug_mlp_grad(stz_context* ctx, const float* params, const float* x, const float* t, size_t n,
                              double s_in, double s_t, double huber_delta, int qat, const double sa[2], float* grad,
                              double* loss);

/* ---- reference function boundary (device pointers) --------------------- *
 * The reference's own stage functions, one for one, for callers that drive
 * the stages themselves. Block = sub_index - 1 (0..6); dims are the block's.  */

/* slice_full_data (FD5:107-122): 8 sub-blocks written back to back in subs. */
stz_status stz_split_dev(stz_context* ctx, stz_dtype dtype, const void* full, size_t nx, size_t ny, size_t nz,
                         void* subs);
/* merge_sub_blocks_to_full (FD5:68-90). */
stz_status stz_merge_dev(stz_context* ctx, stz_dtype dtype, const void* subs, size_t hx, size_t hy, size_t hz,
                         void* full);
/* preprocess_block_zslab (FD5:1161-1175): diff = sub - P(ref) on z in [z0,z1). */
stz_status stz_preprocess_block_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* sub,
                                    const void* ref, void* diff, int dx, int dy, int dz, int z0, int z1);
/* depreprocess_block_zslab (FD5:1177-1191): out = de + P(ref) on z in [z0,z1). */
stz_status stz_depreprocess_block_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* de,
                                      const void* ref, void* out, int dx, int dy, int dz, int z0, int z1);
/* depreprocess_block_zslab_to_full (FD5:1145-1159): scatter into the
 * (2dx,2dy,2dz) grid at the block's parity offsets. */
stz_status stz_depreprocess_block_to_full_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block,
                                              const void* de, const void* ref, void* full, int dx, int dy, int dz,
                                              int z0, int z1);
/* depreprocess_block with ROI bounds (FD5:978-999, 1193-1196): half-open
 * [start, end) per axis. */
stz_status stz_depreprocess_block_roi_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* de,
                                          const void* ref, void* out, int dx, int dy, int dz, int end_x, int end_y,
                                          int end_z, int start_x, int start_y, int start_z);
/* The staged predictor's stage functions of src/dependency.cpp on dense
 * sub-blocks of dx*dy*dz values: diff = sub - P (preprocess) or out = de + P
 * (depreprocess). Blocks 0, 1, 3 are preprocess_block / depreprocess_block
 * (dependency.cpp:333-431): refs[0] is the coarse sub-block 0, the other
 * entries are ignored. Blocks 2, 4, 5, 6 are preprocess_block_staged /
 * depreprocess_block_staged (dependency.cpp:294-331): refs[0..5] are ref_x,
 * ref_y, ref_z, ref_xy, ref_xz, ref_yz (the decoded sub-blocks 1, 2, 4, 3, 5,
 * 6); an entry the block does not read may be null (2: ref_x, ref_y; 4:
 * ref_x, ref_z; 5: ref_y, ref_z; 6: ref_xy, ref_xz, ref_yz). Asynchronous on
 * the context's stream, like the other calls of this group. */
stz_status stz_preprocess_block_staged_dev(stz_context* ctx, stz_dtype dtype, int block, const void* sub,
                                           const void* const refs[6], void* diff, size_t dx, size_t dy, size_t dz);
stz_status stz_depreprocess_block_staged_dev(stz_context* ctx, stz_dtype dtype, int block, const void* de,
                                             const void* const refs[6], void* out, size_t dx, size_t dy, size_t dz);
/* quantize_range_nodec (FD5:1204-1253): int32 codes, unpredictable values in
 * element order; *n_unpred receives their count. */
stz_status stz_quantize_dev(stz_context* ctx, stz_dtype dtype, const void* data, size_t n, double eb, int radius,
                            int32_t* q, void* unpred, size_t* n_unpred);
/* Recover (FD5:1531-1535 and the unpredictable fallback FD5:1556-1562). */
stz_status stz_dequantize_dev(stz_context* ctx, stz_dtype dtype, const int32_t* q, size_t n, double eb, int radius,
                              const void* unpred, void* out);

/* stz_quantize_noalloc_dev: the quantizer of stz_quantize_dev (same results,
 * bit for bit) for callers that cannot allocate device memory — code running
 * inside another framework's memory pool or arena, latency-critical loops that
 * must not hit the device-wide synchronization of cudaMalloc/cudaFree, hosts
 * that reserve all GPU memory up front. It needs no context: work runs on the
 * caller's CUDA stream (`stream` is a cudaStream_t; NULL = default stream) on
 * the current device, and its scratch is a fixed array inside the library
 * image (about 0.8 MB per GPU that loads the library, kept until the process
 * exits), so at most STZ_NOALLOC_MAX_VALUES values per call; larger n returns
 * STZ_ERR_RANGE. Every call looks up that array's device address in the
 * current context (cudaGetSymbolAddress, a host-side lookup). All calls share
 * the one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialized by the caller. The call copies the
 * unpredictable count back and waits for its stream to finish, so it must not
 * be called while its stream, or the legacy default stream, is being captured
 * into a CUDA graph. It returns that count in *n_unpred.
 * This entry point has no counterpart in the reference. */
#define STZ_NOALLOC_MAX_VALUES ((size_t)65536 * 1024)
stz_status stz_quantize_noalloc_dev(stz_dtype dtype, const void* data, size_t n, double eb, int radius, int32_t* q,
                                    void* unpred, size_t* n_unpred, void* stream);

/* ROI planner (FD5:1578-1839) for a query [a, b] on a field of dims
 * (nx,ny,nz), as a flat int64 record:
 *   query x.b x.e y.b y.e z.b z.e is_slice,
 *   n_high, then per high plan: block x.b x.e y.b y.e z.b z.e n_chunks chunks...,
 *   n_regions, then per region: x.b x.e y.b y.e z.b z.e is_slice,
 *   n_low, then per low plan: block x.b x.e y.b y.e z.b z.e n_chunks chunks...
 * Returns the number of values written in *n_out (STZ_ERR_RANGE if cap is too
 * small). */
stz_status stz_plan_box(size_t nx, size_t ny, size_t nz, int chunk_high, int chunk_low, const int64_t a[3],
                        const int64_t b[3], int64_t* out, size_t cap, size_t* n_out);

/* ---- request server ------------------------------------------------------------
 * Serves box, slice and progressive-resolution requests against streams kept
 * resident in HBM (tables, payload, decoded base). The reference answers one
 * query per process run (run_typed, FD5:2460-2660, and the no-marker ROI
 * baseline of src/stz-rd.cpp); this is the long-lived form of the same path.
 *
 * Continuous batching: a worker thread admits queued requests while their
 * outputs fit in the output arena (device memory reserved at create) and a
 * batch slot is free, plans them on the host, and runs each batch as one
 * replay of a captured CUDA graph per stream: one persistent chunk-decode
 * kernel over the union of the batch's marker chunks, one low-level kernel
 * over all mid-grid regions and one high-level kernel over all outputs.
 * Requests that arrive while a batch is on the GPU join the next batch.
 * Full-resolution and half-resolution requests (levels 0 and 1) run in a
 * separate lane on a low-priority CUDA stream, so boxes and slices do not
 * wait behind them. Results do not depend on the batch or lane a request
 * lands in. All functions are thread-safe. */
typedef struct stz_server stz_server;

typedef struct stz_server_opts {
    size_t arena_bytes; /* device memory for request outputs; 0 = 1 GiB */
    int max_batch;      /* requests per batch; 0 = 64 */
    int slots;          /* batches in flight (pinned + device batch buffers); 0 = 2 */
    int autotune;       /* 1 = time launch shapes on each added stream and keep the fastest */
    int threads;        /* host threads for zstd on stream upload; 0 = all cores */
    size_t fast_reserve; /* arena bytes level 0/1 outputs may not take (kept for boxes,
                            slices, coarse levels); (size_t)-1 = a quarter of the arena */
} stz_server_opts;

typedef enum stz_request_kind {
    STZ_REQ_BOX = 0,   /* lo/hi: inclusive (x, y, z) corners, as stz_decompress_box */
    STZ_REQ_LEVEL = 1  /* level: 0 = full resolution, l = every 2^l-th point, as stz_decompress_level */
} stz_request_kind;

typedef struct stz_request {
    int stream_id;
    int kind;
    int64_t lo[3], hi[3];
    int level;
} stz_request;

typedef struct stz_result {
    stz_status status;
    const void* out_dev; /* result on the server's device; valid until stz_server_release */
    size_t dims[3];      /* x, y, z extents */
    size_t bytes;
    double queue_ms;     /* submit -> launch of its batch */
    double latency_ms;   /* submit -> result complete on the device */
    uint64_t batch;      /* id of the batch that served it */
    int batch_size;      /* requests in that batch */
} stz_result;

typedef struct stz_server_stats {
    uint64_t submitted, completed, batches;
    int decode_grid, roi_block, roi_grid; /* launch shapes in use (autotuned or default) */
    size_t arena_bytes, arena_in_use;
} stz_server_stats;

/* One batch of the server's recent history (times in ms since the server was
 * created; device_ms = CUDA-event time from the batch record's copy to its
 * last kernel, -1 until known). */
typedef struct stz_batch_record {
    uint64_t batch;
    int n_requests;
    int lane;             /* 0 = fast (boxes, slices, levels >= 2), 1 = bulk (levels 1 and 0) */
    int slot;
    double t_start_ms;    /* worker took the batch */
    double t_planned_ms;  /* host planning and packing done */
    double t_launched_ms; /* all of the batch's GPU work enqueued */
    double t_done_ms;     /* the completion thread saw its end event */
    double device_ms;
} stz_batch_record;

void stz_server_default_opts(stz_server_opts* o);
stz_status stz_server_create(int device, const stz_server_opts* opts, stz_server** out);
/* Stops the worker after the batches in flight; pending requests fail with
 * STZ_ERR_ARG. */
void stz_server_destroy(stz_server* srv);
/* Parse a container stream, upload its tables and payload, decode its base
 * (levels up to quarter resolution) and capture its batch graphs. */
stz_status stz_server_add_stream(stz_server* srv, const void* data, size_t size, int* stream_id);
/* Queue a request; *ticket identifies it. A request whose output can never
 * fit in the arena returns STZ_ERR_NOMEM here. */
stz_status stz_server_submit(stz_server* srv, const stz_request* req, uint64_t* ticket);
/* Wait up to timeout_ms (< 0: forever) for a ticket; STZ_ERR_RANGE on
 * timeout. The result's own status is in res->status. */
stz_status stz_server_wait(stz_server* srv, uint64_t ticket, double timeout_ms, stz_result* res);
/* Copy a completed result to host memory (res.bytes bytes). */
stz_status stz_server_copy_out(stz_server* srv, uint64_t ticket, void* host);
/* Return a completed ticket's output memory to the arena. */
stz_status stz_server_release(stz_server* srv, uint64_t ticket);
stz_status stz_server_stats_get(stz_server* srv, stz_server_stats* st);
/* The most recent batches (up to 4096 are kept), oldest first: up to cap
 * records into out, the number written in *n. */
stz_status stz_server_batch_log(stz_server* srv, stz_batch_record* out, size_t cap, size_t* n);

/* ---- inspection (tests) --------------------------------------------------- */
/* Quant codes of one residual stream in chunk-major order (the entropy
 * coder's symbol order). level_from_coarse is 1..n_levels. */
stz_status stz_debug_stream_codes(stz_context* ctx, const stz_stream* s, int level_from_coarse, int block,
                                  uint16_t* codes, size_t cap, size_t* n_out);
/* The f32 quantizer table of the plain level encoders for (eb, radius), host
 * only: 64 entries of 4 floats {S_h, S_h+1, lo_h, hi_h} (see QuantTable in
 * the sources), the float 0.5 / eb and whether the table is used. It
 * restates quantize_range_nodec (FD5:1216-1229) for |d| < S_64. */
stz_status stz_debug_quant_table(double eb, int radius, float* entries, float* r2, int* on);
/* Canonical codebook the container format derives from a histogram of nbins
 * code counts (host only): n_used symbols and lengths in canonical order. The
 * reference's equivalent is SZ3-ncp HuffmanEncoder::preprocess_encode_fast
 * (call site FD5:1401-1402), whose format is not available. */
stz_status stz_debug_codebook(const uint32_t* hist, int nbins, uint16_t* sym, uint8_t* len, int* n_used);
/* Run-symbol slots (container version 3) of a stream with code histogram
 * hist (nbins = 2 * radius) and planes of `plane` codes: *run_n slots from
 * *run_base (0: no runs). Host only. */
stz_status stz_debug_run_slots(const uint32_t* hist, int nbins, int plane, uint32_t* run_base, uint32_t* run_n);

#ifdef __cplusplus
}
#endif
#endif /* STZ_B200_STZ_H */
