/*
 * CPU oracle for the STZ streaming compress/decompress path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm (FabioGrosso/SC25-STZ2, file
 * src/zero_all_line_dynamic_random_access_optfast3_optcr_lb_fastdec5.cpp,
 * cited below as FD5:<line>) plus a restatement of this project's own
 * container / canonical-Huffman format. Only tests/, the smoke check and the
 * benchmark's CPU-baseline leg may load it, and only as the checker. The
 * product library never links or calls it.
 *
 * Parity pin: the predictor, quantizer, recover, split/merge and planner
 * restatements are checked against the reference's own functions compiled
 * from its sources (oracle/_ref, see oracle/Makefile) and against the golden
 * vectors in tests/golden/. The Huffman/marker/base-codec byte formats of the
 * reference's SZ3-ncp dependency are not available, so the entropy-coded
 * container is this project's own format; for it the oracle is the second,
 * independent implementation that the GPU path must match byte for byte.
 */
#ifndef STZ_ORACLE_H
#define STZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pointwise FD5 "dynamic lines" predictor P_block(ref; x,y,z) on a coarse grid
 * of dims (dx,dy,dz) (FD5:690-748 with FD5:624-688, 163-203). block = sub_index-1. */
float stzo_predict_f32(int block, const float* ref, int x, int y, int z, int dx, int dy, int dz);
double stzo_predict_f64(int block, const double* ref, int x, int y, int z, int dx, int dy, int dz);

/* Plain tricubic-family predictor of src/float.cpp:84-273 / src/stz-rd.cpp. */
float stzo_predict_plain_f32(int block, const float* ref, int x, int y, int z, int dx, int dy, int dz);
double stzo_predict_plain_f64(int block, const double* ref, int x, int y, int z, int dx, int dy, int dz);

/* Linear quantizer of FD5:1204-1253 on n residuals; returns #unpredictable
 * (appended to unpred in element order), -1 if cap is exceeded. */
long long stzo_quantize_f32(const float* d, size_t n, double eb, int radius, int* q, float* unpred, size_t cap);
long long stzo_quantize_f64(const double* d, size_t n, double eb, int radius, int* q, double* unpred, size_t cap);

/* One refinement level (row-major codes per block, 7 blocks back to back).
 * fine has dims (2dx,2dy,2dz); coarse (dx,dy,dz) holds decoded values.
 * decoded (optional, dims of fine) receives the reconstructed fine grid. */
int stzo_level_encode_f32(const float* fine, const float* coarse, int dx, int dy, int dz, int predictor,
                          double eb, int radius, int* q, float* unpred, size_t cap, size_t* counts,
                          float* decoded);
int stzo_level_encode_f64(const double* fine, const double* coarse, int dx, int dy, int dz, int predictor,
                          double eb, int radius, int* q, double* unpred, size_t cap, size_t* counts,
                          double* decoded);
void stzo_level_decode_f32(const int* q, const float* unpred, const size_t* counts, const float* coarse,
                           int dx, int dy, int dz, int predictor, double eb, int radius, float* out);
void stzo_level_decode_f64(const int* q, const double* unpred, const size_t* counts, const double* coarse,
                           int dx, int dy, int dz, int predictor, double eb, int radius, double* out);

/* Learned correction of one level (this project's addition; the reference has
 * none). An int8 MLP 14 -> 32 -> 32 -> 7 on the 14-point stencil of a coarse
 * cell (the 8 cell corners, then (-1,0,0), (0,-1,0), (0,0,-1), (2,1,1),
 * (1,2,1), (1,1,2)); inputs are the stencil values minus the corner mean,
 * times rs = 1 / (eb * s_in), rounded to int8; hidden layers are ReLU with a
 * fixed-point requantization a = clamp((acc * m + 2^(sh-1)) >> sh, 0, 127);
 * output o is the correction (acc_o * (s_out * eb)) added to the base
 * prediction of block o. Only interior cells (1 <= x,y,z <= dim-3) use it.
 * The struct is also the byte layout stored in the container (2112 bytes,
 * little endian). */
typedef struct stzo_model {
    double s_in, s_out;
    int8_t w1[32][16]; /* inputs 14 and 15 are zero */
    int32_t b1[32], m1, sh1;
    int8_t w2[32][32];
    int32_t b2[32], m2, sh2;
    int8_t w3[8][32];  /* row 7 unused */
    int32_t b3[8];
} stzo_model;

/* Corrections of the 7 blocks at interior coarse point (x,y,z) of a decoded
 * coarse grid, for a level of eb `eb` (tests). */
void stzo_mlp_corr_f32(const stzo_model* m, const float* coarse, int x, int y, int z, int dx, int dy, int dz,
                       double eb, float corr[7]);
void stzo_mlp_corr_f64(const stzo_model* m, const double* coarse, int x, int y, int z, int dx, int dy, int dz,
                       double eb, double corr[7]);

/* Whole-field codec in this project's container format (byte-identical to the
 * GPU path's output). dtype 0 = f32, 1 = f64. */
typedef struct stzo_params {
    int dtype;
    int predictor;      /* 0 = dynamic lines (FD5), 1 = plain cubic (float.cpp) */
    int radius;         /* quantizer radius, <= 32768 */
    int chunk_high;     /* marker chunk edge, finest level (FD5 default 32) */
    int chunk_low;      /* marker chunk edge, second-finest level (FD5 default 16) */
    int zstd_level;     /* 0 = frames stored raw; FD5/SZ3 default 3 */
    double eb;          /* absolute eb handed to the level multipliers */
    double mult_base, mult_low, mult_high; /* FD5:2127-2129 defaults 0.7 / 2.7 / 8.2 */
    const stzo_model* model[2];   /* learned correction of levels K-1 and K (NULL = none) */
    uint32_t learned_flags[2];    /* blocks (bit b) of those levels that use it */
} stzo_params;

/* Returns stream size, or a negative error. *out is malloc'ed. */
long long stzo_compress(const void* field, int nx, int ny, int nz, const stzo_params* p, uint8_t** out);
/* Decompress at resolution level `level` (0 = full, 1 = half, ...). out must
 * hold the grid at that level; dims are returned through odims. */
int stzo_decompress(const uint8_t* stream, size_t size, int level, void* out, int odims[3]);
/* Inspect the container header: dtype, dims, n_levels. */
int stzo_stream_info(const uint8_t* stream, size_t size, int* dtype, int dims[3], int* n_levels);
/* Per-stream quant codes (chunk-major order) for tests. */
long long stzo_debug_stream_codes(const uint8_t* stream, size_t size, int level_from_coarse, int block,
                                  uint16_t* codes, size_t cap);
void stzo_free(void* p);

/* Hierarchy shape shared with the product: number of refinement levels and
 * the chunk edge of each level (1-based from the coarsest). */
int stzo_num_levels(int nx, int ny, int nz);
int stzo_level_chunk(int nx, int ny, int nz, int k, int chunk_high, int chunk_low);

/* Canonical Huffman codebook of this project's format for one histogram of
 * 2*radius bins. Writes n_used symbols/lengths in canonical order. */
int stzo_codebook(const uint32_t* hist, int nbins, uint16_t* sym, uint8_t* len);
/* Run-symbol slots of a stream with code histogram hist (nbins = 2 * radius)
 * and planes of `plane` codes: returns run_n (0: no runs), *run_base the first
 * slot (direct run lengths 2..D, then powers of two; see stz_oracle.c). */
int stzo_run_slots(const uint32_t* hist, int nbins, int plane, uint32_t* run_base);

/* ROI planner restatement (FD5:1578-1839) with the same flat record layout as
 * fd5ref_plan in oracle/ref_shim.cpp. */
long long stzo_plan(int nx, int ny, int nz, int chunk_high, int chunk_low, int ax, int ay, int az,
                    int bx, int by, int bz, long long* out, long long cap);

/* ROI box/slice decode from a container: inclusive box [a,b] per axis in
 * full-resolution coordinates, output row-major (z,y,x) over the box. */
int stzo_decompress_box(const uint8_t* stream, size_t size, const int lo[3], const int hi[3], void* out);

#ifdef __cplusplus
}
#endif
#endif
