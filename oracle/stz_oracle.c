/*
 * CPU oracle for the STZ streaming compress/decompress path — TEST
 * INFRASTRUCTURE ONLY (see stz_oracle.h for what may load it).
 *
 * Sections:
 *   1. FP environment and zstd prototypes.
 *   2. Typed predictor / quantizer / level code (stz_oracle_typed.h, x2).
 *   3. Hierarchy shape (levels, chunk edges).
 *   4. Canonical Huffman codebook of this project's container format.
 *   5. Container writer / reader (whole-field compress and decompress).
 *   6. ROI planner restatement (FD5:1578-1839) and box decode.
 */
#define _GNU_SOURCE
#include "stz_oracle.h"

#include <math.h>
#include <pmmintrin.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>

/* ---- 1. FP environment ------------------------------------------------- */
/* The reference main() runs with FTZ and DAZ on (FD5:3046-3047). */
static void ftz_on(void)
{
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
}

/* libzstd 1.5.5 ships here as a runtime library only; these are its public
 * prototypes (zstd.h). */
size_t ZSTD_compress(void* dst, size_t dstCapacity, const void* src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
size_t ZSTD_compressBound(size_t srcSize);
unsigned ZSTD_isError(size_t code);

/* ---- 2. typed code ------------------------------------------------------ */
/* Learned correction: stencil of a coarse cell (x, y, z offsets) and the
 * hidden layers' fixed-point requantization (stz_oracle.h, stzo_model). */
static const int kStencil[14][3] = {{0, 0, 0},  {1, 0, 0},  {0, 1, 0},  {1, 1, 0}, {0, 0, 1},
                                    {1, 0, 1},  {0, 1, 1},  {1, 1, 1},  {-1, 0, 0}, {0, -1, 0},
                                    {0, 0, -1}, {2, 1, 1},  {1, 2, 1},  {1, 1, 2}};

static int requant(int32_t acc, int32_t m, int32_t sh)
{
    const int64_t p = ((int64_t)acc * m + ((int64_t)1 << (sh - 1))) >> sh;
    return p < 0 ? 0 : p > 127 ? 127 : (int)p;
}

#define T float
#define SUF f32
#include "stz_oracle_typed.h"
#undef T
#undef SUF
#define T double
#define SUF f64
#include "stz_oracle_typed.h"
#undef T
#undef SUF

float stzo_predict_f32(int block, const float* ref, int x, int y, int z, int dx, int dy, int dz)
{
    ftz_on();
    return t_predict_f32(block, ref, x, y, z, dx, dy, dz);
}
double stzo_predict_f64(int block, const double* ref, int x, int y, int z, int dx, int dy, int dz)
{
    ftz_on();
    return t_predict_f64(block, ref, x, y, z, dx, dy, dz);
}
float stzo_predict_plain_f32(int block, const float* ref, int x, int y, int z, int dx, int dy, int dz)
{
    ftz_on();
    return t_predict_plain_f32(block, ref, x, y, z, dx, dy, dz);
}
double stzo_predict_plain_f64(int block, const double* ref, int x, int y, int z, int dx, int dy, int dz)
{
    ftz_on();
    return t_predict_plain_f64(block, ref, x, y, z, dx, dy, dz);
}

/* ---- 3. hierarchy shape -------------------------------------------------- */
/* Refinement levels: halve while every dim is even and the halved minimum is
 * at least 4; at least the reference's two residual levels (low, high). */
int stzo_num_levels(int nx, int ny, int nz)
{
    int k = 0;
    while (nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0) {
        int m = nx < ny ? nx : ny;
        m = m < nz ? m : nz;
        if (m / 2 < 4) break;
        nx /= 2, ny /= 2, nz /= 2, ++k;
    }
    return k < 2 ? 2 : k;
}

/* Chunk edge of level k (1 = coarsest refinement, K = finest): the marker
 * chunk sizes of FD5 (high/low, FD5:33-35) on the two finest levels, below
 * them the largest power of two <= 16 dividing all block dims. */
int stzo_level_chunk(int nx, int ny, int nz, int k, int chunk_high, int chunk_low)
{
    const int K = stzo_num_levels(nx, ny, nz);
    if (k == K) return chunk_high;
    if (k == K - 1) return chunk_low;
    const int sh = K - k + 1;
    const int dx = nx >> sh, dy = ny >> sh, dz = nz >> sh;
    int c = 16;
    while (c > 1 && (dx % c || dy % c || dz % c)) c >>= 1;
    return c;
}

/* ---- 4. canonical Huffman codebook -------------------------------------- */
#define STZO_LMAX 24

typedef struct {
    uint64_t w;
    uint32_t sym;
} wsym;

static int cmp_wsym(const void* a, const void* b)
{
    const wsym* x = (const wsym*)a;
    const wsym* y = (const wsym*)b;
    if (x->w != y->w) return x->w < y->w ? -1 : 1;
    return x->sym < y->sym ? -1 : (x->sym > y->sym);
}

typedef struct {
    uint8_t len;
    uint16_t sym;
} lsym;

static int cmp_lsym(const void* a, const void* b)
{
    const lsym* x = (const lsym*)a;
    const lsym* y = (const lsym*)b;
    if (x->len != y->len) return x->len < y->len ? -1 : 1;
    return x->sym < y->sym ? -1 : (x->sym > y->sym);
}

/* Minimum-redundancy code lengths of weights sorted ascending, computed in
 * place (Moffat & Katajainen, "In-place calculation of minimum-redundancy
 * codes", WADS 1995): pass 1 builds parent links left to right, pass 2 turns
 * them into internal-node depths, pass 3 hands out leaf depths. */
static void mk_lengths(uint64_t* a, int n)
{
    if (n == 1) {
        a[0] = 0;
        return;
    }
    int root = 0, leaf = 2;
    a[0] += a[1];
    for (int next = 1; next < n - 1; ++next) {
        if (leaf >= n || a[root] < a[leaf]) {
            a[next] = a[root];
            a[root++] = (uint64_t)next;
        } else {
            a[next] = a[leaf++];
        }
        if (leaf >= n || (root < next && a[root] < a[leaf])) {
            a[next] += a[root];
            a[root++] = (uint64_t)next;
        } else {
            a[next] += a[leaf++];
        }
    }
    a[n - 2] = 0;
    for (int next = n - 3; next >= 0; --next) a[next] = a[a[next]] + 1;
    int avail = 1, used = 0, depth = 0;
    root = n - 2;
    int next = n - 1;
    while (avail > 0) {
        while (root >= 0 && a[root] == (uint64_t)depth) {
            ++used;
            --root;
        }
        while (avail > used) {
            a[next--] = (uint64_t)depth;
            --avail;
        }
        avail = 2 * used;
        ++depth;
        used = 0;
    }
}

/* Codebook rule of the container: symbols with a nonzero count, sorted by
 * (count, symbol); minimum-redundancy lengths; lengths capped at 24 by
 * lengthening, least frequent first, the first code shorter than the cap until
 * the Kraft sum fits; canonical order (length, symbol). A single used symbol
 * gets length 0 (no payload bits). Returns n_used. */
int stzo_codebook(const uint32_t* hist, int nbins, uint16_t* sym, uint8_t* len)
{
    int n = 0;
    for (int s = 0; s < nbins; ++s) n += hist[s] != 0;
    if (n == 0) return 0;
    wsym* ws = (wsym*)malloc(sizeof(wsym) * (size_t)n);
    uint64_t* a = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int k = 0;
    for (int s = 0; s < nbins; ++s)
        if (hist[s]) {
            ws[k].w = hist[s];
            ws[k].sym = (uint32_t)s;
            ++k;
        }
    qsort(ws, (size_t)n, sizeof(wsym), cmp_wsym);
    for (int i = 0; i < n; ++i) a[i] = ws[i].w;
    mk_lengths(a, n);
    if (n > 1) {
        uint64_t kraft = 0;
        for (int i = 0; i < n; ++i) {
            if (a[i] > STZO_LMAX) a[i] = STZO_LMAX;
            kraft += (uint64_t)1 << (STZO_LMAX - a[i]);
        }
        const uint64_t cap = (uint64_t)1 << STZO_LMAX;
        while (kraft > cap) {
            int i = 0;
            while (a[i] >= STZO_LMAX) ++i;
            kraft -= (uint64_t)1 << (STZO_LMAX - a[i] - 1);
            a[i] += 1;
        }
    }
    lsym* ls = (lsym*)malloc(sizeof(lsym) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        ls[i].len = (uint8_t)a[i];
        ls[i].sym = (uint16_t)ws[i].sym;
    }
    qsort(ls, (size_t)n, sizeof(lsym), cmp_lsym);
    for (int i = 0; i < n; ++i) {
        sym[i] = ls[i].sym;
        len[i] = ls[i].len;
    }
    free(ls);
    free(a);
    free(ws);
    return n;
}

/* Canonical codes in canonical order: first code 0, then
 * code <- (code + 1) << (len_i - len_{i-1}). */
static void canonical_codes(const uint8_t* len, int n, uint32_t* code)
{
    uint32_t c = 0;
    for (int i = 0; i < n; ++i) {
        if (i > 0) c = (c + 1) << (len[i] - len[i - 1]);
        code[i] = c;
    }
}

/* ---- 5. container ------------------------------------------------------ */
typedef struct {
    uint8_t* p;
    size_t n, cap;
} buf_t;

static void bput(buf_t* b, const void* src, size_t n)
{
    if (b->n + n > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + n) c *= 2;
        b->p = (uint8_t*)realloc(b->p, c);
        b->cap = c;
    }
    if (n) memcpy(b->p + b->n, src, n);
    b->n += n;
}
static void bu8(buf_t* b, uint8_t v) { bput(b, &v, 1); }
static void bu16(buf_t* b, uint16_t v) { bput(b, &v, 2); }
static void bu32(buf_t* b, uint32_t v) { bput(b, &v, 4); }
static void bi32(buf_t* b, int32_t v) { bput(b, &v, 4); }
static void bu64(buf_t* b, uint64_t v) { bput(b, &v, 8); }
static void bf64(buf_t* b, double v) { bput(b, &v, 8); }

typedef struct {
    const uint8_t* p;
    size_t n, pos;
    int err;
} rd_t;

static void rget(rd_t* r, void* dst, size_t n)
{
    if (r->err || r->pos + n > r->n) {
        r->err = 1;
        memset(dst, 0, n);
        return;
    }
    memcpy(dst, r->p + r->pos, n);
    r->pos += n;
}
static uint32_t ru32(rd_t* r) { uint32_t v; rget(r, &v, 4); return v; }
static int32_t ri32(rd_t* r) { int32_t v; rget(r, &v, 4); return v; }
static uint64_t ru64(rd_t* r) { uint64_t v; rget(r, &v, 8); return v; }
static double rf64(rd_t* r) { double v; rget(r, &v, 8); return v; }

static const char kMagic[8] = {'S', 'T', 'Z', 'B', '2', '0', '0', 0};

/* One zstd frame of the container: compressed when that is smaller, else the
 * raw bytes (a stored size equal to the raw size means raw). A payload frame
 * longer than ZSTD_PROBE bytes is tried only when zstd shrinks its first
 * ZSTD_PROBE bytes (this container's own rule; Huffman payload is rarely
 * compressible). */
#define ZSTD_PROBE 4096
static void put_frame(buf_t* data, const uint8_t* raw, size_t n, int level, int payload, uint64_t* stored)
{
    int try_zstd = level > 0 && n > 0;
    if (try_zstd && payload && n > ZSTD_PROBE) {
        const size_t pcap = ZSTD_compressBound(ZSTD_PROBE);
        uint8_t* tmp = (uint8_t*)malloc(pcap);
        const size_t c = ZSTD_compress(tmp, pcap, raw, ZSTD_PROBE, level);
        try_zstd = !ZSTD_isError(c) && c < ZSTD_PROBE;
        free(tmp);
    }
    if (try_zstd) {
        const size_t cap = ZSTD_compressBound(n);
        uint8_t* tmp = (uint8_t*)malloc(cap);
        const size_t c = ZSTD_compress(tmp, cap, raw, n, level);
        if (!ZSTD_isError(c) && c < n) {
            bput(data, tmp, c);
            *stored = c;
            free(tmp);
            return;
        }
        free(tmp);
    }
    bput(data, raw, n);
    *stored = n;
}

/* Encoded form of one residual stream (block b of one level). */
typedef struct {
    buf_t hdr;       /* raw stream header */
    uint32_t* words; /* payload */
    uint64_t nwords;
    uint64_t* chunk_off; /* n_chunks + 1 word offsets */
    int n_chunks, layers, chunks_per_layer;
} enc_stream;

/* Run symbols of a stream (this container's own rule, version 3): a maximal
 * run of the centre code (= radius) inside a plane is coded with run
 * symbols placed in consecutive code values the stream does not use,
 * [run_base, run_base + run_n):
 *   J  = min(14, floor(log2 plane)), D = min(32, 2^J), LD = log2 D;
 *   slots 0 .. D-2      : runs of exactly 2 .. D centre codes;
 *   slots D-1 .. run_n-1: runs of 2^k centre codes, k = LD+1 .. J;
 *   run_n = D - 1 + (J - LD). The window is the highest free one in
 *   [1, 2 * radius); none (or J = 0): run_n = 0, no runs. */
static int run_geometry(int plane, int* D, int* LD)
{
    int J = 0;
    while (J < 14 && ((size_t)2 << J) <= (size_t)plane) ++J;
    *LD = J < 5 ? J : 5;
    *D = 1 << *LD;
    return J;
}

int stzo_run_slots(const uint32_t* hist, int nbins, int plane, uint32_t* run_base)
{
    int D, LD;
    const int J = run_geometry(plane, &D, &LD);
    *run_base = 0;
    if (J == 0) return 0;
    const int S = D - 1 + (J - LD);
    for (int u0 = nbins - S; u0 >= 1; --u0) {
        int free_ = 1;
        for (int j = 0; j < S && free_; ++j) free_ = hist[u0 + j] == 0;
        if (free_) {
            *run_base = (uint32_t)u0;
            return S;
        }
    }
    return 0;
}

/* The symbols of one plane with runs. A run of r centre codes: while
 * r > D, the largest 2^k <= r (k <= J) when k > LD, else D; then a direct
 * symbol for 2 <= r <= D, or the centre code itself for r = 1. Returns the
 * symbol count; out needs plane entries. */
static size_t plane_symbols(const uint16_t* s, size_t plane, int radius, uint32_t run_base, int run_n, uint16_t* out)
{
    int D = 0, LD = 0;
    const int J = run_geometry((int)plane, &D, &LD);
    size_t m = 0, r = 0;
    for (size_t j = 0; j <= plane; ++j) {
        if (j < plane && run_n && s[j] == radius) {
            ++r;
            continue;
        }
        while (r > (size_t)D) {
            int k = 0;
            while (k < J && ((size_t)2 << k) <= r) ++k; /* k = min(floor(log2 r), J) */
            if (k > LD) {
                out[m++] = (uint16_t)(run_base + (uint32_t)(D - 1 + (k - LD - 1)));
                r -= (size_t)1 << k;
            } else {
                out[m++] = (uint16_t)(run_base + (uint32_t)(D - 2));
                r -= (size_t)D;
            }
        }
        if (r >= 2) out[m++] = (uint16_t)(run_base + (uint32_t)(r - 2));
        else if (r == 1) out[m++] = (uint16_t)radius;
        r = 0;
        if (j < plane) out[m++] = s[j];
    }
    return m;
}

/* Length of run symbol slot i (0 <= i < run_n) for planes of `plane` codes. */
static size_t run_length(uint32_t i, int plane)
{
    int D, LD;
    run_geometry(plane, &D, &LD);
    return i < (uint32_t)(D - 1) ? (size_t)i + 2 : (size_t)1 << (i - (uint32_t)(D - 1) + (uint32_t)LD + 1);
}

/* Entropy-code one stream given chunk-major codes and chunk-major unpred
 * values (elem = sizeof(T)). */
static void encode_stream(const uint16_t* codes, size_t n, int dx, int dy, int dz, int C, int radius,
                          const void* unpred, uint64_t nunpred, const uint32_t* unpred_count, size_t elem,
                          enc_stream* es)
{
    const int nbins = 2 * radius;
    const int ncx = dx / C, ncy = dy / C, ncz = dz / C;
    const int nch = ncx * ncy * ncz;
    const size_t cvol = (size_t)C * C * C, plane = (size_t)C * C;
    uint32_t* hist = (uint32_t*)calloc((size_t)nbins, 4);
    for (size_t i = 0; i < n; ++i) hist[codes[i]]++;
    uint32_t run_base = 0;
    int run_n = stzo_run_slots(hist, nbins, (int)plane, &run_base);
    /* runs only where they shorten the Huffman payload (else the decoder
     * keeps its plain path): compare sum(count * length) of both codebooks */
    uint64_t bits_plain = 0;
    if (run_n) {
        uint16_t* ps = (uint16_t*)malloc(2 * (size_t)nbins);
        uint8_t* pl = (uint8_t*)malloc((size_t)nbins);
        const int pn = stzo_codebook(hist, nbins, ps, pl);
        for (int i = 0; i < pn; ++i) bits_plain += (uint64_t)hist[ps[i]] * pl[i];
        free(ps);
        free(pl);
    }
    /* the symbol stream: runs inside every plane */
    uint16_t* syms = (uint16_t*)malloc(2 * (n ? n : 1));
    size_t* pstart = (size_t*)malloc(sizeof(size_t) * ((size_t)nch * C + 1));
    size_t m = 0;
    for (int c = 0; c < nch; ++c)
        for (int lz = 0; lz < C; ++lz) {
            pstart[(size_t)c * C + lz] = m;
            m += plane_symbols(codes + (size_t)c * cvol + (size_t)lz * plane, plane, radius, run_base, run_n, syms + m);
        }
    pstart[(size_t)nch * C] = m;
    uint32_t* rhist = (uint32_t*)calloc((size_t)nbins, 4);
    for (size_t i = 0; i < m; ++i) rhist[syms[i]]++;
    uint16_t* sym = (uint16_t*)malloc(2 * (size_t)nbins);
    uint8_t* len = (uint8_t*)malloc((size_t)nbins);
    int nu = stzo_codebook(rhist, nbins, sym, len);
    if (run_n) {
        uint64_t bits_runs = 0;
        for (int i = 0; i < nu; ++i) bits_runs += (uint64_t)rhist[sym[i]] * len[i];
        if (bits_runs >= bits_plain) { /* plain coding: symbols = codes */
            run_n = 0;
            run_base = 0;
            m = 0;
            for (int c = 0; c < nch; ++c)
                for (int lz = 0; lz < C; ++lz) {
                    pstart[(size_t)c * C + lz] = m;
                    m += plane_symbols(codes + (size_t)c * cvol + (size_t)lz * plane, plane, radius, 0, 0, syms + m);
                }
            pstart[(size_t)nch * C] = m;
            nu = stzo_codebook(hist, nbins, sym, len);
        }
    }
    free(rhist);
    uint32_t* code = (uint32_t*)malloc(4 * (size_t)(nu ? nu : 1));
    canonical_codes(len, nu, code);
    uint32_t* ctab = (uint32_t*)calloc((size_t)nbins, 4);
    uint8_t* ltab = (uint8_t*)calloc((size_t)nbins, 1);
    for (int i = 0; i < nu; ++i) {
        ctab[sym[i]] = code[i];
        ltab[sym[i]] = len[i];
    }
    uint32_t* sub_off = (uint32_t*)malloc(4 * (size_t)nch * C);
    uint64_t* choff = (uint64_t*)malloc(8 * ((size_t)nch + 1));
    choff[0] = 0;
    for (int c = 0; c < nch; ++c) {
        uint64_t bits = 0;
        for (int lz = 0; lz < C; ++lz) {
            const size_t p = (size_t)c * C + lz;
            sub_off[p] = (uint32_t)bits;
            for (size_t i = pstart[p]; i < pstart[p + 1]; ++i) bits += ltab[syms[i]];
        }
        choff[c + 1] = choff[c] + (bits + 31) / 32;
    }
    const uint64_t nw = choff[nch];
    uint32_t* w = (uint32_t*)calloc(nw ? nw : 1, 4);
    for (int c = 0; c < nch; ++c) {
        uint64_t bit = 0;
        uint32_t* cw = w + choff[c];
        for (size_t i = pstart[(size_t)c * C]; i < pstart[(size_t)(c + 1) * C]; ++i) {
            const int l = ltab[syms[i]];
            const uint32_t cd = ctab[syms[i]];
            for (int t = l - 1; t >= 0; --t) {
                if ((cd >> t) & 1u) cw[bit >> 5] |= 1u << (31 - (bit & 31));
                ++bit;
            }
        }
    }
    free(pstart);
    free(syms);
    /* raw stream header */
    memset(&es->hdr, 0, sizeof(es->hdr));
    bu32(&es->hdr, (uint32_t)nu);
    for (int i = 0; i < nu; ++i) bu16(&es->hdr, sym[i]);
    for (int i = 0; i < nu; ++i) bu8(&es->hdr, len[i]);
    bu32(&es->hdr, run_base);
    bu32(&es->hdr, (uint32_t)run_n);
    bu64(&es->hdr, nunpred);
    bput(&es->hdr, unpred, (size_t)nunpred * elem);
    for (int c = 0; c < nch; ++c) bu32(&es->hdr, unpred_count[c]);
    for (int c = 0; c <= nch; ++c) bu64(&es->hdr, choff[c]);
    /* plane table (version 4): per chunk the bit counts of its first C - 1
     * planes (the first starts at bit 0), 2 bytes each when all fit, else 4 */
    {
        uint32_t mx = 0;
        for (int c = 0; c < nch; ++c)
            for (int lz = 1; lz < C; ++lz) {
                const uint32_t d = sub_off[(size_t)c * C + lz] - sub_off[(size_t)c * C + lz - 1];
                if (d > mx) mx = d;
            }
        const int width = mx < 65536 ? 2 : 4;
        bu8(&es->hdr, (uint8_t)width);
        for (int c = 0; c < nch; ++c)
            for (int lz = 1; lz < C; ++lz) {
                const uint32_t d = sub_off[(size_t)c * C + lz] - sub_off[(size_t)c * C + lz - 1];
                if (width == 2) bu16(&es->hdr, (uint16_t)d);
                else bu32(&es->hdr, d);
            }
    }
    es->words = w;
    es->nwords = nw;
    es->chunk_off = choff;
    es->n_chunks = nch;
    es->layers = ncz;
    es->chunks_per_layer = ncx * ncy;
    free(sub_off);
    free(ltab);
    free(ctab);
    free(code);
    free(len);
    free(sym);
    free(hist);
}

/* Reorder one block's row-major codes (and its row-major unpred list) into
 * chunk-major symbol order: chunks row-major over (cz,cy,cx), each chunk
 * row-major over (lz,ly,lx). */
static void to_chunk_major(const int* q, const uint8_t* unpred_rm, uint64_t nunpred, size_t elem, int dx, int dy,
                           int dz, int C, uint16_t* codes, uint8_t* unpred_cm, uint32_t* unpred_count)
{
    const size_t n = (size_t)dx * dy * dz;
    /* rank of each row-major unpredictable position */
    uint64_t* rank = (uint64_t*)malloc(8 * (n ? n : 1));
    uint64_t r = 0;
    for (size_t i = 0; i < n; ++i) rank[i] = q[i] == 0 ? r++ : 0;
    (void)nunpred;
    const int ncx = dx / C, ncy = dy / C, ncz = dz / C;
    size_t o = 0;
    uint64_t u = 0;
    for (int cz = 0; cz < ncz; ++cz)
        for (int cy = 0; cy < ncy; ++cy)
            for (int cx = 0; cx < ncx; ++cx) {
                const int c = (cz * ncy + cy) * ncx + cx;
                uint32_t cnt = 0;
                for (int lz = 0; lz < C; ++lz)
                    for (int ly = 0; ly < C; ++ly)
                        for (int lx = 0; lx < C; ++lx) {
                            const size_t i = ((size_t)(cz * C + lz) * dy + (size_t)(cy * C + ly)) * dx + (size_t)(cx * C + lx);
                            codes[o++] = (uint16_t)q[i];
                            if (q[i] == 0) {
                                memcpy(unpred_cm + u * elem, unpred_rm + rank[i] * elem, elem);
                                ++u;
                                ++cnt;
                            }
                        }
                unpred_count[c] = cnt;
            }
    free(rank);
}

typedef struct {
    int dtype, predictor, nx, ny, nz, K, radius, chunk_high, chunk_low, zstd_level;
    double eb, mb, ml, mh;
    int c0[3];
    size_t elem;
} hdr_t;

static double level_eb(const hdr_t* h, int k)
{
    if (k == h->K) return h->mh * h->eb;
    if (k == h->K - 1) return h->ml * h->eb;
    return h->mb * h->eb;
}

static void level_dims(const hdr_t* h, int k, int d[3])
{
    const int sh = h->K - k + 1;
    d[0] = h->nx >> sh, d[1] = h->ny >> sh, d[2] = h->nz >> sh;
}

long long stzo_compress(const void* field, int nx, int ny, int nz, const stzo_params* p, uint8_t** out)
{
    ftz_on();
    *out = NULL;
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 4 || ny % 4 || nz % 4) return -2;
    if (p->chunk_high <= 0 || p->chunk_low <= 0) return -2;
    if ((nx / 2) % p->chunk_high || (ny / 2) % p->chunk_high || (nz / 2) % p->chunk_high) return -2;
    if ((nx / 4) % p->chunk_low || (ny / 4) % p->chunk_low || (nz / 4) % p->chunk_low) return -2;
    if (p->radius < 1 || p->radius > 32768 || !(p->eb > 0)) return -3;
    hdr_t h;
    h.dtype = p->dtype, h.predictor = p->predictor, h.nx = nx, h.ny = ny, h.nz = nz;
    h.K = stzo_num_levels(nx, ny, nz);
    h.radius = p->radius, h.chunk_high = p->chunk_high, h.chunk_low = p->chunk_low, h.zstd_level = p->zstd_level;
    h.eb = p->eb, h.mb = p->mult_base, h.ml = p->mult_low, h.mh = p->mult_high;
    h.elem = p->dtype == 1 ? 8 : 4;
    h.c0[0] = nx >> h.K, h.c0[1] = ny >> h.K, h.c0[2] = nz >> h.K;

    /* learned correction of levels K-1 and K: container version 2 */
    const stzo_model* lm[64] = {0};
    uint32_t lf[64] = {0};
    const int version = 4; /* per-level learned fields, run symbols, plane bit counts */
    for (int i = 0; i < 2; ++i) {
        const int k = h.K - 1 + i;
        if (k >= 1 && p->model[i] && (p->learned_flags[i] & 0x7fu)) {
            lm[k] = p->model[i];
            lf[k] = p->learned_flags[i] & 0x7fu;
        }
    }
    buf_t dir = {0}, data = {0};
    bput(&dir, kMagic, 8);
    bu32(&dir, (uint32_t)version);
    bu32(&dir, (uint32_t)h.dtype);
    bu32(&dir, (uint32_t)h.predictor);
    bu32(&dir, (uint32_t)nx);
    bu32(&dir, (uint32_t)ny);
    bu32(&dir, (uint32_t)nz);
    bu32(&dir, (uint32_t)h.K);
    bu32(&dir, (uint32_t)h.radius);
    bu32(&dir, (uint32_t)h.chunk_high);
    bu32(&dir, (uint32_t)h.chunk_low);
    bi32(&dir, h.zstd_level);
    bf64(&dir, h.eb);
    bf64(&dir, h.mb);
    bf64(&dir, h.ml);
    bf64(&dir, h.mh);
    bu32(&dir, (uint32_t)h.c0[0]);
    bu32(&dir, (uint32_t)h.c0[1]);
    bu32(&dir, (uint32_t)h.c0[2]);

    const size_t ncoarse = (size_t)h.c0[0] * h.c0[1] * h.c0[2];
    void* G = malloc(ncoarse * h.elem);
    if (h.dtype == 1) subsample_f64((const double*)field, nx, ny, nz, 1 << h.K, (double*)G);
    else subsample_f32((const float*)field, nx, ny, nz, 1 << h.K, (float*)G);
    bput(&dir, G, ncoarse * h.elem);

    for (int k = 1; k <= h.K; ++k) {
        int d[3];
        level_dims(&h, k, d);
        const int C = stzo_level_chunk(nx, ny, nz, k, h.chunk_high, h.chunk_low);
        const double ebk = level_eb(&h, k);
        const size_t n = (size_t)d[0] * d[1] * d[2];
        const int s = 1 << (h.K - k);
        void* fine = malloc(8 * n * h.elem);
        if (h.dtype == 1) subsample_f64((const double*)field, nx, ny, nz, s, (double*)fine);
        else subsample_f32((const float*)field, nx, ny, nz, s, (float*)fine);
        int* q = (int*)malloc(sizeof(int) * 7 * n);
        void* unpred = malloc(7 * n * h.elem);
        size_t counts[7];
        void* Gn = k < h.K ? malloc(8 * n * h.elem) : NULL;
        int rc;
        if (h.dtype == 1)
            rc = t_level_encode_f64((const double*)fine, (const double*)G, d[0], d[1], d[2], h.predictor, ebk,
                                    h.radius, q, (double*)unpred, 7 * n, counts, (double*)Gn, lm[k], lf[k]);
        else
            rc = t_level_encode_f32((const float*)fine, (const float*)G, d[0], d[1], d[2], h.predictor, ebk,
                                    h.radius, q, (float*)unpred, 7 * n, counts, (float*)Gn, lm[k], lf[k]);
        (void)rc;
        bu32(&dir, (uint32_t)d[0]);
        bu32(&dir, (uint32_t)d[1]);
        bu32(&dir, (uint32_t)d[2]);
        bu32(&dir, (uint32_t)C);
        bf64(&dir, ebk);
        bu32(&dir, lf[k]);
        if (lf[k]) bput(&dir, lm[k], sizeof(stzo_model));
        uint16_t* codes = (uint16_t*)malloc(2 * n);
        uint8_t* ucm = (uint8_t*)malloc(n * h.elem + 1);
        const int nch = (d[0] / C) * (d[1] / C) * (d[2] / C);
        uint32_t* ucount = (uint32_t*)malloc(4 * (size_t)nch);
        size_t uoff = 0;
        for (int b = 0; b < 7; ++b) {
            to_chunk_major(q + (size_t)b * n, (const uint8_t*)unpred + uoff * h.elem, counts[b], h.elem, d[0], d[1],
                           d[2], C, codes, ucm, ucount);
            enc_stream es;
            encode_stream(codes, n, d[0], d[1], d[2], C, h.radius, ucm, counts[b], ucount, h.elem, &es);
            uoff += counts[b];
            uint64_t hs;
            put_frame(&data, es.hdr.p, es.hdr.n, h.zstd_level, 0, &hs);
            bu32(&dir, (uint32_t)es.layers);
            bu64(&dir, hs);
            bu64(&dir, es.hdr.n);
            uint64_t* ls = (uint64_t*)malloc(8 * (size_t)es.layers);
            uint64_t* lr = (uint64_t*)malloc(8 * (size_t)es.layers);
            for (int L = 0; L < es.layers; ++L) {
                const uint64_t w0 = es.chunk_off[(size_t)L * es.chunks_per_layer];
                const uint64_t w1 = es.chunk_off[(size_t)(L + 1) * es.chunks_per_layer];
                lr[L] = 4 * (w1 - w0);
                put_frame(&data, (const uint8_t*)(es.words + w0), (size_t)lr[L], h.zstd_level, 1, &ls[L]);
            }
            for (int L = 0; L < es.layers; ++L) bu64(&dir, ls[L]);
            for (int L = 0; L < es.layers; ++L) bu64(&dir, lr[L]);
            free(ls);
            free(lr);
            free(es.hdr.p);
            free(es.words);
            free(es.chunk_off);
        }
        free(ucount);
        free(ucm);
        free(codes);
        free(unpred);
        free(q);
        free(fine);
        free(G);
        G = Gn;
    }
    free(G);
    bput(&dir, data.p, data.n);
    free(data.p);
    *out = dir.p;
    return (long long)dir.n;
}

/* Parsed directory entry of one stream. */
typedef struct {
    int layers;
    uint64_t hdr_stored, hdr_raw;
    uint64_t* ls;
    uint64_t* lr;
    size_t data_off; /* offset of the header frame in the stream bytes */
} sdir_t;

typedef struct {
    hdr_t h;
    const uint8_t* coarsest;
    int d[64][3];
    int C[64];
    double ebk[64];
    int version;             /* 1: plain, 2: learned fields, 3: learned fields and run symbols */
    uint32_t lflags[64];     /* learned-correction blocks of the level (version >= 2) */
    stzo_model lmodel[64];   /* its model when lflags != 0 */
    sdir_t s[64][7];
} parsed_t;

static void free_parsed(parsed_t* ps)
{
    for (int k = 1; k <= ps->h.K && k < 64; ++k)
        for (int b = 0; b < 7; ++b) {
            free(ps->s[k][b].ls);
            free(ps->s[k][b].lr);
        }
}

static int parse(const uint8_t* st, size_t size, parsed_t* ps)
{
    memset(ps, 0, sizeof(*ps));
    rd_t r = {st, size, 0, 0};
    char mg[8];
    rget(&r, mg, 8);
    if (r.err || memcmp(mg, kMagic, 8) != 0) return -10;
    const uint32_t version = ru32(&r);
    if (version < 1 || version > 4) return -11;
    ps->version = (int)version;
    hdr_t* h = &ps->h;
    h->dtype = (int)ru32(&r);
    h->predictor = (int)ru32(&r);
    h->nx = (int)ru32(&r), h->ny = (int)ru32(&r), h->nz = (int)ru32(&r);
    h->K = (int)ru32(&r);
    h->radius = (int)ru32(&r);
    h->chunk_high = (int)ru32(&r), h->chunk_low = (int)ru32(&r);
    h->zstd_level = ri32(&r);
    h->eb = rf64(&r), h->mb = rf64(&r), h->ml = rf64(&r), h->mh = rf64(&r);
    h->c0[0] = (int)ru32(&r), h->c0[1] = (int)ru32(&r), h->c0[2] = (int)ru32(&r);
    if (r.err || h->K < 1 || h->K >= 64 || (h->dtype != 0 && h->dtype != 1)) return -12;
    if (h->predictor < 0 || h->predictor > 3) return -12; /* dynamic, cubic, staged, truncated */
    h->elem = h->dtype == 1 ? 8 : 4;
    ps->coarsest = st + r.pos;
    r.pos += (size_t)h->c0[0] * h->c0[1] * h->c0[2] * h->elem;
    for (int k = 1; k <= h->K; ++k) {
        ps->d[k][0] = (int)ru32(&r), ps->d[k][1] = (int)ru32(&r), ps->d[k][2] = (int)ru32(&r);
        ps->C[k] = (int)ru32(&r);
        ps->ebk[k] = rf64(&r);
        if (version >= 2) {
            ps->lflags[k] = ru32(&r);
            if (ps->lflags[k] > 0x7f) return -16;
            if (ps->lflags[k]) rget(&r, &ps->lmodel[k], sizeof(stzo_model));
        }
        for (int b = 0; b < 7; ++b) {
            sdir_t* s = &ps->s[k][b];
            s->layers = (int)ru32(&r);
            s->hdr_stored = ru64(&r);
            s->hdr_raw = ru64(&r);
            if (r.err || s->layers < 0 || s->layers > (1 << 20)) return -13;
            s->ls = (uint64_t*)malloc(8 * (size_t)(s->layers + 1));
            s->lr = (uint64_t*)malloc(8 * (size_t)(s->layers + 1));
            for (int L = 0; L < s->layers; ++L) s->ls[L] = ru64(&r);
            for (int L = 0; L < s->layers; ++L) s->lr[L] = ru64(&r);
        }
    }
    if (r.err) return -14;
    size_t off = r.pos;
    for (int k = 1; k <= h->K; ++k)
        for (int b = 0; b < 7; ++b) {
            sdir_t* s = &ps->s[k][b];
            s->data_off = off;
            off += s->hdr_stored;
            for (int L = 0; L < s->layers; ++L) off += s->ls[L];
        }
    if (off > size) return -15;
    return 0;
}

static int get_frame(const uint8_t* src, uint64_t stored, uint64_t raw, uint8_t* dst)
{
    if (stored == raw) {
        if (raw) memcpy(dst, src, (size_t)raw);
        return 0;
    }
    const size_t r = ZSTD_decompress(dst, (size_t)raw, src, (size_t)stored);
    return (ZSTD_isError(r) || r != raw) ? -20 : 0;
}

/* Decode one stream into chunk-major codes and chunk-major unpred values. */
static int decode_stream(const uint8_t* st, const parsed_t* ps, int k, int b, uint16_t* codes, uint8_t* unpred,
                         uint64_t* nunpred_out)
{
    const hdr_t* h = &ps->h;
    const sdir_t* s = &ps->s[k][b];
    const int dx = ps->d[k][0], dy = ps->d[k][1], dz = ps->d[k][2], C = ps->C[k];
    const int nch = (dx / C) * (dy / C) * (dz / C);
    const size_t cvol = (size_t)C * C * C, plane = (size_t)C * C;
    uint8_t* hraw = (uint8_t*)malloc((size_t)s->hdr_raw + 1);
    const uint8_t* src = st + s->data_off;
    if (get_frame(src, s->hdr_stored, s->hdr_raw, hraw)) {
        free(hraw);
        return -21;
    }
    src += s->hdr_stored;
    uint64_t total = 0;
    for (int L = 0; L < s->layers; ++L) total += s->lr[L];
    uint8_t* praw = (uint8_t*)malloc((size_t)total + 4);
    uint64_t po = 0;
    for (int L = 0; L < s->layers; ++L) {
        if (get_frame(src, s->ls[L], s->lr[L], praw + po)) {
            free(hraw);
            free(praw);
            return -22;
        }
        src += s->ls[L];
        po += s->lr[L];
    }
    const uint32_t* words = (const uint32_t*)praw;
    int rc_hdr_bad = 0;
    rd_t r = {hraw, (size_t)s->hdr_raw, 0, 0};
    const int nu = (int)ru32(&r);
    uint16_t* sym = (uint16_t*)malloc(2 * (size_t)(nu + 1));
    uint8_t* len = (uint8_t*)malloc((size_t)nu + 1);
    rget(&r, sym, 2 * (size_t)nu);
    rget(&r, len, (size_t)nu);
    uint32_t run_base = 0, run_n = 0;
    if (ps->version >= 3) {
        run_base = ru32(&r);
        run_n = ru32(&r);
        int D_, LD_;
        const int J_ = run_geometry((int)plane, &D_, &LD_);
        if (run_n && (J_ == 0 || run_n != (uint32_t)(D_ - 1 + (J_ - LD_)) || run_base < 1 ||
                      run_base + run_n > (uint32_t)(2 * h->radius)))
            rc_hdr_bad = 1;
    }
    const uint64_t nunp = ru64(&r);
    rget(&r, unpred, (size_t)nunp * h->elem);
    *nunpred_out = nunp;
    r.pos += 4 * (size_t)nch; /* unpred counts: implied by the code order */
    uint64_t* choff = (uint64_t*)malloc(8 * ((size_t)nch + 1));
    for (int c = 0; c <= nch; ++c) choff[c] = ru64(&r);
    uint32_t* sub = (uint32_t*)malloc(4 * (size_t)nch * C);
    if (ps->version >= 4) {
        uint8_t width = 0;
        rget(&r, &width, 1);
        if (width != 2 && width != 4) rc_hdr_bad = 1;
        for (int c = 0; c < nch; ++c) {
            uint64_t acc = 0;
            sub[(size_t)c * C] = 0;
            for (int lz = 1; lz < C; ++lz) {
                uint32_t d = 0;
                if (width == 2) {
                    uint16_t d16 = 0;
                    rget(&r, &d16, 2);
                    d = d16;
                } else {
                    d = ru32(&r);
                }
                acc += d;
                if (acc > 0xffffffffull) rc_hdr_bad = 1;
                sub[(size_t)c * C + lz] = (uint32_t)acc;
            }
        }
    } else {
        for (size_t i = 0; i < (size_t)nch * C; ++i) sub[i] = ru32(&r);
    }
    int rc = (r.err || rc_hdr_bad) ? -23 : 0;
    /* canonical decode tables: count / first code / first index per length */
    uint32_t* code = (uint32_t*)malloc(4 * (size_t)(nu + 1));
    canonical_codes(len, nu, code);
    int cnt[STZO_LMAX + 2] = {0}, first_idx[STZO_LMAX + 2] = {0};
    uint32_t first_code[STZO_LMAX + 2] = {0};
    for (int i = nu - 1; i >= 0; --i) {
        cnt[len[i]]++;
        first_idx[len[i]] = i;
        first_code[len[i]] = code[i];
    }
    for (int c = 0; c < nch && !rc; ++c)
        for (int lz = 0; lz < C && !rc; ++lz) {
            uint64_t bit = 32 * choff[c] + sub[(size_t)c * C + lz];
            uint16_t* out = codes + (size_t)c * cvol + (size_t)lz * plane;
            for (size_t j = 0; j < plane;) {
                uint32_t sy = 0;
                if (nu == 1) {
                    sy = sym[0];
                } else {
                    uint32_t v = 0;
                    int l = 0, found = 0;
                    while (l < STZO_LMAX) {
                        v = (v << 1) | ((words[bit >> 5] >> (31 - (bit & 31))) & 1u);
                        ++bit;
                        ++l;
                        if (cnt[l] && v >= first_code[l] && v - first_code[l] < (uint32_t)cnt[l]) {
                            sy = sym[first_idx[l] + (int)(v - first_code[l])];
                            found = 1;
                            break;
                        }
                    }
                    if (!found) {
                        rc = -24;
                        break;
                    }
                }
                if (run_n && sy - run_base < run_n) { /* a run of centre codes */
                    size_t rl = run_length(sy - run_base, (int)plane);
                    if (rl > plane - j) {
                        rc = -25;
                        break;
                    }
                    for (; rl; --rl) out[j++] = (uint16_t)h->radius;
                } else {
                    out[j++] = (uint16_t)sy;
                }
            }
        }
    free(code);
    free(sub);
    free(choff);
    free(len);
    free(sym);
    free(praw);
    free(hraw);
    return rc;
}

/* Decode one level into dense dq values (7 blocks, row-major each) and
 * reconstruct the fine grid. */
static int decode_level(const uint8_t* st, const parsed_t* ps, int k, const void* G, void* Gn)
{
    const hdr_t* h = &ps->h;
    const int dx = ps->d[k][0], dy = ps->d[k][1], dz = ps->d[k][2], C = ps->C[k];
    const size_t n = (size_t)dx * dy * dz, cvol = (size_t)C * C * C;
    const int ncx = dx / C, ncy = dy / C;
    uint16_t* codes = (uint16_t*)malloc(2 * n);
    uint8_t* unpred = (uint8_t*)malloc(n * h->elem + 8);
    int* q = (int*)malloc(sizeof(int) * 7 * n);
    uint8_t* urm = (uint8_t*)malloc(7 * n * h->elem + 8);
    size_t uo = 0;
    int rc = 0;
    for (int b = 0; b < 7 && !rc; ++b) {
        uint64_t nunp = 0;
        rc = decode_stream(st, ps, k, b, codes, unpred, &nunp);
        if (rc) break;
        /* chunk-major -> row-major codes; unpred values to row-major order */
        uint64_t* at = (uint64_t*)malloc(8 * (n ? n : 1));
        uint64_t u = 0;
        for (size_t ci = 0; ci < n; ++ci) {
            const size_t c = ci / cvol, w = ci % cvol;
            const int cx = (int)(c % (size_t)ncx), cy = (int)((c / (size_t)ncx) % (size_t)ncy),
                      cz = (int)(c / ((size_t)ncx * ncy));
            const int lx = (int)(w % (size_t)C), ly = (int)((w / (size_t)C) % (size_t)C), lz = (int)(w / ((size_t)C * C));
            const size_t i = ((size_t)(cz * C + lz) * dy + (size_t)(cy * C + ly)) * dx + (size_t)(cx * C + lx);
            q[(size_t)b * n + i] = codes[ci];
            at[i] = codes[ci] == 0 ? u++ : 0;
        }
        if (u != nunp) rc = -25;
        for (size_t i = 0; i < n && !rc; ++i)
            if (q[(size_t)b * n + i] == 0) memcpy(urm + uo++ * h->elem, unpred + at[i] * h->elem, h->elem);
        free(at);
    }
    if (!rc) {
        size_t counts[7] = {0};
        const stzo_model* M = ps->lflags[k] ? &ps->lmodel[k] : NULL;
        if (h->dtype == 1)
            t_level_decode_f64(q, (const double*)urm, counts, (const double*)G, dx, dy, dz, h->predictor,
                               ps->ebk[k], h->radius, (double*)Gn, M, ps->lflags[k]);
        else
            t_level_decode_f32(q, (const float*)urm, counts, (const float*)G, dx, dy, dz, h->predictor,
                               ps->ebk[k], h->radius, (float*)Gn, M, ps->lflags[k]);
    }
    free(urm);
    free(q);
    free(unpred);
    free(codes);
    return rc;
}

int stzo_stream_info(const uint8_t* stream, size_t size, int* dtype, int dims[3], int* n_levels)
{
    parsed_t* ps = (parsed_t*)malloc(sizeof(parsed_t));
    int rc = parse(stream, size, ps);
    if (!rc) {
        *dtype = ps->h.dtype;
        dims[0] = ps->h.nx, dims[1] = ps->h.ny, dims[2] = ps->h.nz;
        *n_levels = ps->h.K;
    }
    free_parsed(ps);
    free(ps);
    return rc;
}

int stzo_decompress(const uint8_t* stream, size_t size, int level, void* out, int odims[3])
{
    ftz_on();
    parsed_t* ps = (parsed_t*)malloc(sizeof(parsed_t));
    int rc = parse(stream, size, ps);
    if (rc) {
        free_parsed(ps);
        free(ps);
        return rc;
    }
    const hdr_t* h = &ps->h;
    if (level < 0 || level > h->K) {
        free_parsed(ps);
        free(ps);
        return -30;
    }
    const int last = h->K - level;
    size_t ng = (size_t)h->c0[0] * h->c0[1] * h->c0[2];
    void* G = malloc(ng * h->elem);
    memcpy(G, ps->coarsest, ng * h->elem);
    int gd[3] = {h->c0[0], h->c0[1], h->c0[2]};
    for (int k = 1; k <= last && !rc; ++k) {
        const size_t n = (size_t)ps->d[k][0] * ps->d[k][1] * ps->d[k][2];
        void* Gn = malloc(8 * n * h->elem);
        rc = decode_level(stream, ps, k, G, Gn);
        free(G);
        G = Gn;
        gd[0] = 2 * ps->d[k][0], gd[1] = 2 * ps->d[k][1], gd[2] = 2 * ps->d[k][2];
        ng = 8 * n;
    }
    if (!rc) {
        memcpy(out, G, ng * h->elem);
        if (odims) odims[0] = gd[0], odims[1] = gd[1], odims[2] = gd[2];
    }
    free(G);
    free_parsed(ps);
    free(ps);
    return rc;
}

long long stzo_debug_stream_codes(const uint8_t* stream, size_t size, int k, int block, uint16_t* codes, size_t cap)
{
    parsed_t* ps = (parsed_t*)malloc(sizeof(parsed_t));
    long long rc = parse(stream, size, ps);
    if (!rc && (k < 1 || k > ps->h.K || block < 0 || block > 6)) rc = -31;
    if (!rc) {
        const size_t n = (size_t)ps->d[k][0] * ps->d[k][1] * ps->d[k][2];
        if (n > cap) rc = -32;
        else {
            uint8_t* u = (uint8_t*)malloc(n * ps->h.elem + 8);
            uint64_t nu = 0;
            rc = decode_stream(stream, ps, k, block, codes, u, &nu);
            free(u);
            if (!rc) rc = (long long)n;
        }
    }
    free_parsed(ps);
    free(ps);
    return rc;
}

void stzo_free(void* p) { free(p); }

/* ---- 6. ROI planner (FD5:1578-1839) and box decode ---------------------- */
typedef struct {
    int b, e;
} axr;

static axr normalize_axis(int a, int b, int dim, int* is_slice)
{
    axr r;
    if (a == b) {
        *is_slice = 1;
        int v = a < dim - 1 ? a : dim - 1;
        v = v > 0 ? v : 0;
        r.b = r.e = v;
        return r;
    }
    int lo = a < b ? a : b;
    lo = lo > 0 ? lo : 0;
    int hi = a > b ? a : b;
    hi = hi < dim - 1 ? hi : dim - 1;
    if (hi < lo) hi = lo;
    r.b = lo, r.e = hi;
    return r;
}

static axr range_for_parity(axr full, int parity)
{
    int first = full.b;
    if ((first & 1) != parity) ++first;
    axr r = {1, 0};
    if (first > full.e) return r;
    int last = full.e;
    if ((last & 1) != parity) --last;
    r.b = first / 2, r.e = last / 2;
    return r;
}

static int chunks_for_box(int bx, int by, int bz, int C, axr x, axr y, axr z, long long* out)
{
    if (x.b > x.e || y.b > y.e || z.b > z.e) return 0;
    const int ncx = bx / C, ncy = by / C, ncz = bz / C;
    const int cx0 = x.b / C > 0 ? x.b / C : 0, cy0 = y.b / C > 0 ? y.b / C : 0, cz0 = z.b / C > 0 ? z.b / C : 0;
    const int cx1 = x.e / C < ncx - 1 ? x.e / C : ncx - 1;
    const int cy1 = y.e / C < ncy - 1 ? y.e / C : ncy - 1;
    const int cz1 = z.e / C < ncz - 1 ? z.e / C : ncz - 1;
    int n = 0;
    for (int cz = cz0; cz <= cz1; ++cz)
        for (int cy = cy0; cy <= cy1; ++cy)
            for (int cx = cx0; cx <= cx1; ++cx) out[n++] = ((long long)cz * ncy + cy) * ncx + cx;
    return n;
}

static axr ref_range_for_used_axis(axr t, int dim)
{
    if (t.b > t.e) return t;
    int lo = t.b, hi = t.e;
    const int ib = t.b > 1 ? t.b : 1;
    const int ie = t.e < dim - 3 ? t.e : dim - 3;
    if (ib <= ie) {
        lo = lo < ib - 1 ? lo : ib - 1;
        hi = hi > ie + 2 ? hi : ie + 2;
    }
    const int nb = t.b > 0 ? t.b : 0;
    const int ne = t.e < dim - 2 ? t.e : dim - 2;
    if (nb <= ne) hi = hi > ne + 1 ? hi : ne + 1;
    axr r;
    r.b = lo > 0 ? lo : 0;
    r.e = hi < dim - 1 ? hi : dim - 1;
    return r;
}

static void merge_axis(axr* dst, axr src)
{
    if (src.b > src.e) return;
    if (dst->b > dst->e) {
        *dst = src;
        return;
    }
    dst->b = dst->b < src.b ? dst->b : src.b;
    dst->e = dst->e > src.e ? dst->e : src.e;
}

typedef struct {
    long long* p;
    long long n, cap;
    int err;
} lv_t;

static void lpush(lv_t* v, long long x)
{
    if (v->n >= v->cap) {
        v->err = 1;
        return;
    }
    v->p[v->n++] = x;
}

static int cmp_ll(const void* a, const void* b)
{
    const long long x = *(const long long*)a, y = *(const long long*)b;
    return x < y ? -1 : (x > y);
}

long long stzo_plan(int nx, int ny, int nz, int chunk_high, int chunk_low, int ax, int ay, int az, int bx, int by,
                    int bz, long long* out, long long cap)
{
    lv_t v = {out, 0, cap, 0};
    const int dx = nx / 2, dy = ny / 2, dz = nz / 2;
    const int lx = nx / 4, ly = ny / 4, lz = nz / 4;
    int is_slice = 0;
    axr q[3];
    q[0] = normalize_axis(ax, bx, nx, &is_slice);
    q[1] = normalize_axis(ay, by, ny, &is_slice);
    q[2] = normalize_axis(az, bz, nz, &is_slice);
    for (int a = 0; a < 3; ++a) {
        lpush(&v, q[a].b);
        lpush(&v, q[a].e);
    }
    lpush(&v, is_slice);
    /* high plans (build_residual_plan, FD5:1689-1711) */
    axr hp[7][3];
    int hblock[7], nh = 0;
    long long* tmp = (long long*)malloc(sizeof(long long) * 1024 * 1024);
    const long long nh_pos = v.n;
    lpush(&v, 0);
    for (int b = 0; b < 7; ++b) {
        const int s = b + 1;
        axr r[3] = {range_for_parity(q[0], s & 1), range_for_parity(q[1], (s >> 1) & 1),
                    range_for_parity(q[2], (s >> 2) & 1)};
        if (r[0].b > r[0].e || r[1].b > r[1].e || r[2].b > r[2].e) continue;
        const int nc = chunks_for_box(dx, dy, dz, chunk_high, r[0], r[1], r[2], tmp);
        lpush(&v, b);
        for (int a = 0; a < 3; ++a) {
            lpush(&v, r[a].b);
            lpush(&v, r[a].e);
        }
        lpush(&v, nc);
        for (int i = 0; i < nc; ++i) lpush(&v, tmp[i]);
        hblock[nh] = b;
        memcpy(hp[nh], r, sizeof(r));
        ++nh;
    }
    if (!v.err) out[nh_pos] = nh;
    /* high reference regions (FD5:1751-1770) + the query's sub-block-0 region (FD5:1772-1782) */
    axr reg[8][3];
    int nreg = 0;
    for (int i = 0; i < nh; ++i) {
        const int s = hblock[i] + 1;
        reg[nreg][0] = (s & 1) ? ref_range_for_used_axis(hp[i][0], dx) : hp[i][0];
        reg[nreg][1] = (s & 2) ? ref_range_for_used_axis(hp[i][1], dy) : hp[i][1];
        reg[nreg][2] = (s & 4) ? ref_range_for_used_axis(hp[i][2], dz) : hp[i][2];
        ++nreg;
    }
    axr s0[3] = {range_for_parity(q[0], 0), range_for_parity(q[1], 0), range_for_parity(q[2], 0)};
    if (s0[0].b <= s0[0].e && s0[1].b <= s0[1].e && s0[2].b <= s0[2].e) {
        memcpy(reg[nreg], s0, sizeof(s0));
        ++nreg;
    }
    lpush(&v, nreg);
    for (int i = 0; i < nreg; ++i) {
        for (int a = 0; a < 3; ++a) {
            lpush(&v, reg[i][a].b);
            lpush(&v, reg[i][a].e);
        }
        lpush(&v, (reg[i][0].b == reg[i][0].e) || (reg[i][1].b == reg[i][1].e) || (reg[i][2].b == reg[i][2].e));
    }
    /* low plan (build_low_residual_plan, FD5:1784-1830): union of chunk sets
     * (sorted, unique) and the bounding ranges per block */
    const long long nl_pos = v.n;
    lpush(&v, 0);
    int nl = 0;
    long long* cs = (long long*)malloc(sizeof(long long) * 1024 * 1024);
    for (int b = 0; b < 7; ++b) {
        axr acc[3] = {{1, 0}, {1, 0}, {1, 0}};
        long long ncs = 0;
        for (int i = 0; i < nreg; ++i) {
            if (reg[i][0].b > reg[i][0].e || reg[i][1].b > reg[i][1].e || reg[i][2].b > reg[i][2].e) continue;
            const int s = b + 1;
            axr r[3] = {range_for_parity(reg[i][0], s & 1), range_for_parity(reg[i][1], (s >> 1) & 1),
                        range_for_parity(reg[i][2], (s >> 2) & 1)};
            if (r[0].b > r[0].e || r[1].b > r[1].e || r[2].b > r[2].e) continue;
            ncs += chunks_for_box(lx, ly, lz, chunk_low, r[0], r[1], r[2], cs + ncs);
            for (int a = 0; a < 3; ++a) merge_axis(&acc[a], r[a]);
        }
        if (ncs == 0) continue;
        qsort(cs, (size_t)ncs, sizeof(long long), cmp_ll);
        long long u = 0;
        for (long long i = 0; i < ncs; ++i)
            if (i == 0 || cs[i] != cs[i - 1]) cs[u++] = cs[i];
        lpush(&v, b);
        for (int a = 0; a < 3; ++a) {
            lpush(&v, acc[a].b);
            lpush(&v, acc[a].e);
        }
        lpush(&v, u);
        for (long long i = 0; i < u; ++i) lpush(&v, cs[i]);
        ++nl;
    }
    if (!v.err) out[nl_pos] = nl;
    free(cs);
    free(tmp);
    return v.err ? -1 : v.n;
}

/* The reference validates every ROI answer against the full decode at the
 * same coordinates (FD5:2625-2640); the oracle's box answer is exactly that:
 * the full decode cropped to the normalized box. */
int stzo_decompress_box(const uint8_t* stream, size_t size, const int lo[3], const int hi[3], void* out)
{
    int dtype, dims[3], K;
    int rc = stzo_stream_info(stream, size, &dtype, dims, &K);
    if (rc) return rc;
    const size_t elem = dtype == 1 ? 8 : 4;
    int is_slice = 0;
    axr q[3];
    for (int a = 0; a < 3; ++a) q[a] = normalize_axis(lo[a], hi[a], dims[a], &is_slice);
    void* full = malloc((size_t)dims[0] * dims[1] * dims[2] * elem);
    rc = stzo_decompress(stream, size, 0, full, NULL);
    if (!rc) {
        size_t o = 0;
        for (int z = q[2].b; z <= q[2].e; ++z)
            for (int y = q[1].b; y <= q[1].e; ++y)
                for (int x = q[0].b; x <= q[0].e; ++x, ++o)
                    memcpy((uint8_t*)out + o * elem,
                           (const uint8_t*)full + (((size_t)z * dims[1] + y) * dims[0] + x) * elem, elem);
    }
    free(full);
    return rc;
}

/* exported typed wrappers */
long long stzo_quantize_f32(const float* d, size_t n, double eb, int radius, int* q, float* unpred, size_t cap)
{
    return t_quantize_f32(d, n, eb, radius, q, unpred, cap);
}
long long stzo_quantize_f64(const double* d, size_t n, double eb, int radius, int* q, double* unpred, size_t cap)
{
    return t_quantize_f64(d, n, eb, radius, q, unpred, cap);
}
int stzo_level_encode_f32(const float* fine, const float* coarse, int dx, int dy, int dz, int predictor, double eb,
                          int radius, int* q, float* unpred, size_t cap, size_t* counts, float* decoded)
{
    return t_level_encode_f32(fine, coarse, dx, dy, dz, predictor, eb, radius, q, unpred, cap, counts, decoded,
                              NULL, 0);
}
int stzo_level_encode_f64(const double* fine, const double* coarse, int dx, int dy, int dz, int predictor, double eb,
                          int radius, int* q, double* unpred, size_t cap, size_t* counts, double* decoded)
{
    return t_level_encode_f64(fine, coarse, dx, dy, dz, predictor, eb, radius, q, unpred, cap, counts, decoded,
                              NULL, 0);
}
void stzo_level_decode_f32(const int* q, const float* unpred, const size_t* counts, const float* coarse, int dx, int dy,
                           int dz, int predictor, double eb, int radius, float* out)
{
    t_level_decode_f32(q, unpred, counts, coarse, dx, dy, dz, predictor, eb, radius, out, NULL, 0);
}
void stzo_level_decode_f64(const int* q, const double* unpred, const size_t* counts, const double* coarse, int dx,
                           int dy, int dz, int predictor, double eb, int radius, double* out)
{
    t_level_decode_f64(q, unpred, counts, coarse, dx, dy, dz, predictor, eb, radius, out, NULL, 0);
}
void stzo_mlp_corr_f32(const stzo_model* m, const float* coarse, int x, int y, int z, int dx, int dy, int dz,
                       double eb, float corr[7])
{
    ftz_on();
    (void)dz;
    mlp_corr_f32(m, coarse, x, y, z, dx, dy, (float)(1.0 / (eb * m->s_in)), (float)(m->s_out * eb), corr);
}
void stzo_mlp_corr_f64(const stzo_model* m, const double* coarse, int x, int y, int z, int dx, int dy, int dz,
                       double eb, double corr[7])
{
    ftz_on();
    (void)dz;
    mlp_corr_f64(m, coarse, x, y, z, dx, dy, 1.0 / (eb * m->s_in), m->s_out * eb, corr);
}
