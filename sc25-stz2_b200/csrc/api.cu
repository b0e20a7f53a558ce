// C ABI and pipeline orchestration of the STZ B200 library.
//
// Compress (stz_compress_dev):
//   1. value range on the GPU when the bound is relative (computeRange,
//      FD5:92-104);
//   2. coarsest grid = field sampled every 2^K points (stored raw);
//   3. one fused level-encode launch per level, coarse to fine (levels.cu);
//   4. histogram windows to the host, canonical codebooks on the host pool;
//   5. entropy coding on the GPU: code tables, plane bit counts, offsets scan
//      (marker tables), encode, unpredictable-value gather, payload pack;
//   6. per-layer zstd frames on the host pool and the container.
// Decompress: zstd frames on the host pool into one pinned staging buffer, one
// host->device copy, one decode launch for every chunk of every stream, then
// one fused level-decode launch per level into the output (or an intermediate
// grid). Box/slice queries decode only the planner's chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "host.h"
#include "huffman.h"
#include "levels.h"
#include "roi.h"
#include "runtime.h"
#include "stz/stz.h"
#include "stz_internal.h"

namespace {
thread_local std::string g_err;
}  // namespace

namespace stz {

void set_last_error(const std::string& msg) { g_err = msg; }

QuantParams make_quant_params(double eb, int radius)
{
    QuantParams q;
    q.eb = eb;
    q.recip = 1.0 / eb;
    q.radius = radius;
    // largest float / double t with t <= eb and t * recip < 1 in double
    float f = (float)eb;
    while (f > 0.f && ((double)f > eb || (double)f * q.recip >= 1.0)) f = std::nextafter(f, 0.f);
    double d = eb;
    while (d > 0.0 && d * q.recip >= 1.0) d = std::nextafter(d, 0.0);
    q.tlo32 = f > 0.f ? f : 0.f;
    q.tlo64 = d > 0.0 ? d : 0.0;
    return q;
}

namespace {
// Host mirrors of the device's f32 quantizer operations.
float ftz32(float x) { return std::fabs(x) < FLT_MIN ? std::copysign(0.0f, x) : x; }
float next_up(float x) { return std::nextafter(x, INFINITY); }
float next_down(float x) { return std::nextafter(x, 0.0f); }
// The least float a >= 0 with pred(a), pred monotone (false then true),
// searched from guess g; +inf when none below FLT_MAX.
template <class P>
float least_true(float g, P pred)
{
    if (!(g >= 0.0f) || !std::isfinite(g)) g = 0.0f;
    int steps = 0;
    if (pred(g)) {
        while (g > 0.0f && pred(next_down(g)) && ++steps < 256) g = next_down(g);
        if (steps < 256) return g;
    } else {
        while (g < FLT_MAX && !pred(g) && ++steps < 256) g = next_up(g);
        if (steps < 256) return pred(g) ? g : INFINITY;
    }
    // far from the guess: bisection over the positive float bit patterns
    uint32_t lo = 0, hi = 0x7f7fffffu;  // pred(hi) assumed; answer in [lo, hi]
    auto f = [](uint32_t u) {
        float x;
        std::memcpy(&x, &u, 4);
        return x;
    };
    if (!pred(f(hi))) return INFINITY;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (pred(f(mid))) hi = mid;
        else lo = mid + 1;
    }
    return f(lo);
}
}  // namespace

QuantTable make_quant_table(const QuantParams& qp)
{
    QuantTable t{};
    const double eb = qp.eb, recip = qp.recip;
    const int H = std::min(kQuantTableH, qp.radius - 2);  // every entry in range (ad < 2 radius - 1)
    for (int h = 0; h < kQuantTableH; ++h) t.e[h] = make_float4(INFINITY, INFINITY, INFINITY, -INFINITY);
    t.r2 = (float)(0.5 / eb);
    t.on = 0;
    if (!(eb >= 1e-30) || !(eb <= 1e30) || !std::isfinite(recip) || H < 1) return t;
    // S_h for h = 0..H: least |d| with trunc(fl64(|d| * recip)) >= 2h - 1
    std::vector<float> S(H + 1);
    S[0] = 0.0f;
    for (int h = 1; h <= H; ++h) {
        const double m = 2.0 * h - 1.0;
        S[h] = least_true((float)(m * eb), [&](float a) { return (double)a * recip >= m; });
    }
    for (int h = 0; h < H; ++h) {
        if (!std::isfinite(S[h + 1])) break;
        float lo, hi;
        const float top = next_down(S[h + 1]);  // the interval's last float
        if (h == 0) {
            // half 0: the decompressed value is +-0, the check is |d| <= eb
            lo = 0.0f;
            const float hmax = least_true((float)eb, [&](float a) { return (double)a > eb; });
            hi = std::min(top, next_down(hmax));
        } else {
            const float mag = ftz32((float)((double)(2 * h) * eb));
            // |fl32(mag - a)| <= eb, fl32 flushed as the device's sub.rn.ftz
            const float a1 = least_true(std::max(0.0f, (float)(mag - eb)),
                                        [&](float a) { return (double)ftz32(mag - a) <= eb; });
            const float a2n = least_true((float)(mag + eb), [&](float a) { return (double)ftz32(mag - a) < -eb; });
            lo = std::max(S[h], a1);
            hi = std::min(top, next_down(a2n));
        }
        if (lo > hi) lo = INFINITY, hi = -INFINITY;  // nothing in the interval passes
        t.e[h] = make_float4(S[h], S[h + 1], lo, hi);
    }
    t.on = 1;
    return t;
}

Geometry make_geometry(int nx, int ny, int nz, int chunk_high, int chunk_low, int radius)
{
    Geometry g;
    g.nx = nx, g.ny = ny, g.nz = nz;
    g.radius = radius, g.chunk_high = chunk_high, g.chunk_low = chunk_low;
    g.K = num_levels(nx, ny, nz);
    g.c0[0] = nx >> g.K, g.c0[1] = ny >> g.K, g.c0[2] = nz >> g.K;
    g.lv.resize(g.K + 1);
    g.n_fine_max = (size_t)g.c0[0] * g.c0[1] * g.c0[2];
    for (int k = 1; k <= g.K; ++k) {
        LevelGeom& L = g.lv[k];
        const int sh = g.K - k + 1;
        L.dx = nx >> sh, L.dy = ny >> sh, L.dz = nz >> sh;
        L.C = level_chunk(nx, ny, nz, g.K, k, chunk_high, chunk_low);
        L.ncx = L.dx / L.C, L.ncy = L.dy / L.C, L.ncz = L.dz / L.C;
        L.n = (size_t)L.dx * L.dy * L.dz;
        if (k < g.K) g.n_fine_max = std::max(g.n_fine_max, 8 * L.n);
        for (int b = 0; b < 7; ++b) {
            StreamDesc s{};
            s.code_off = g.total_codes;
            g.total_codes += L.n;
            s.chunk_base = g.total_chunk_slots;
            g.total_chunk_slots += (uint64_t)L.nchunks() + 1;
            s.sub_base = g.total_sub;
            g.total_sub += (uint64_t)L.nchunks() * L.C;
            s.word_base = g.total_words;
            s.word_cap = (L.n * kMaxCodeLen + 31) / 32 + L.nchunks() + 4;
            g.total_words += s.word_cap;
            s.C = L.C;
            s.ncx = L.ncx, s.ncy = L.ncy, s.ncz = L.ncz;
            s.nchunks = L.nchunks();
            s.radius = radius;
            g.sd.push_back(s);
        }
    }
    return g;
}

void add_work(std::vector<CtaWork>& work, std::vector<uint32_t>& ids, uint32_t stream, const uint32_t* chunks,
              size_t n, int C)
{
    const size_t G = std::max(1, kCoderThreads / C);
    for (size_t i = 0; i < n; i += G) {
        const uint32_t cnt = (uint32_t)std::min(G, n - i);
        work.push_back({stream, (uint32_t)ids.size(), cnt, 0});
        ids.insert(ids.end(), chunks + i, chunks + i + cnt);
    }
}

void add_all_chunks(std::vector<CtaWork>& work, std::vector<uint32_t>& ids, uint32_t stream, uint32_t nchunks, int C)
{
    std::vector<uint32_t> all(nchunks);
    for (uint32_t i = 0; i < nchunks; ++i) all[i] = i;
    add_work(work, ids, stream, all.data(), all.size(), C);
}

int pool_threads(int requested)
{
    if (requested > 0) return requested;
    if (const char* e = std::getenv("STZ_POOL_THREADS"))
        if (std::atoi(e) > 0) return std::min(std::atoi(e), 64);
    const unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h ? h : 1u, 64u));
}

namespace {
constexpr size_t kXferChunk = 16ull << 20;

bool host_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer: pageable
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy of n bytes on the pool, in pieces of at least 1 MiB
void pool_copy(ThreadPool& pool, void* dst, const void* src, size_t n)
{
    const size_t parts = std::max<size_t>(1, std::min<size_t>((size_t)pool.size(), n >> 20));
    const size_t per = (n + parts - 1) / parts;
    pool.parallel_for(parts, [&](size_t i) {
        const size_t a = i * per, b = std::min(n, a + per);
        if (a < b) std::memcpy((uint8_t*)dst + a, (const uint8_t*)src + a, b - a);
    });
}

struct XferEvents {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~XferEvents()
    {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
};

// On an early return (a failed CUDA call mid-loop), waits for the copies
// already queued on the stream, so the next host-buffer call never refills a
// staging chunk that a DMA still reads or writes. The wait's own status is
// ignored: the caller already reports the first error.
struct DrainOnExit {
    cudaStream_t st;
    bool done = false;
    ~DrainOnExit()
    {
        if (!done) cudaStreamSynchronize(st);
    }
};
}  // namespace

stz_status copy_to_host(stz_context* ctx, void* dst, const void* src_dev, size_t n)
{
    cudaStream_t st = ctx->st;
    if (n <= kXferChunk || host_pinned(dst)) {
        STZ_CUDA(cudaMemcpyAsync(dst, src_dev, n, cudaMemcpyDeviceToHost, st));
        STZ_CUDA(cudaStreamSynchronize(st));
        return STZ_OK;
    }
    XferEvents ev;
    DrainOnExit drain{st};
    for (int b = 0; b < 2; ++b) {
        STZ_CUDA(ctx->h_xfer[b].ensure(kXferChunk));
        STZ_CUDA(cudaEventCreateWithFlags(&ev.e[b], cudaEventDisableTiming));
    }
    const size_t nch = (n + kXferChunk - 1) / kXferChunk;
    auto issue = [&](size_t i) -> cudaError_t {
        const size_t a = i * kXferChunk, len = std::min(kXferChunk, n - a);
        cudaError_t e = cudaMemcpyAsync(ctx->h_xfer[i & 1].p, (const uint8_t*)src_dev + a, len, cudaMemcpyDeviceToHost, st);
        return e == cudaSuccess ? cudaEventRecord(ev.e[i & 1], st) : e;
    };
    STZ_CUDA(issue(0));
    for (size_t i = 0; i < nch; ++i) {
        if (i + 1 < nch) STZ_CUDA(issue(i + 1));  // into the other chunk, free since chunk i - 1 was copied out
        STZ_CUDA(cudaEventSynchronize(ev.e[i & 1]));
        const size_t a = i * kXferChunk;
        pool_copy(*ctx->pool, (uint8_t*)dst + a, ctx->h_xfer[i & 1].p, std::min(kXferChunk, n - a));
    }
    drain.done = true;  // every DMA was waited for above
    return STZ_OK;
}

stz_status copy_from_host(stz_context* ctx, void* dst_dev, const void* src, size_t n)
{
    cudaStream_t st = ctx->st;
    if (n <= kXferChunk || host_pinned(src)) {
        STZ_CUDA(cudaMemcpyAsync(dst_dev, src, n, cudaMemcpyHostToDevice, st));
        STZ_CUDA(cudaStreamSynchronize(st));
        return STZ_OK;
    }
    XferEvents ev;
    DrainOnExit drain{st};
    for (int b = 0; b < 2; ++b) {
        STZ_CUDA(ctx->h_xfer[b].ensure(kXferChunk));
        STZ_CUDA(cudaEventCreateWithFlags(&ev.e[b], cudaEventDisableTiming));
    }
    const size_t nch = (n + kXferChunk - 1) / kXferChunk;
    for (size_t i = 0; i < nch; ++i) {
        if (i >= 2) STZ_CUDA(cudaEventSynchronize(ev.e[i & 1]));  // chunk i - 2's DMA has left this buffer
        const size_t a = i * kXferChunk, len = std::min(kXferChunk, n - a);
        pool_copy(*ctx->pool, ctx->h_xfer[i & 1].p, (const uint8_t*)src + a, len);
        STZ_CUDA(cudaMemcpyAsync((uint8_t*)dst_dev + a, ctx->h_xfer[i & 1].p, len, cudaMemcpyHostToDevice, st));
        STZ_CUDA(cudaEventRecord(ev.e[i & 1], st));
    }
    STZ_CUDA(cudaStreamSynchronize(st));  // the staging chunks are reused by the next call
    drain.done = true;
    return STZ_OK;
}

stz_status check_opts(const stz_opts* o)
{
    if (!o) STZ_FAIL(STZ_ERR_ARG, "opts is null");
    if (!(o->eb > 0) || !std::isfinite(o->eb)) STZ_FAIL(STZ_ERR_ARG, "eb must be a positive finite number");
    if (o->eb_mode != STZ_EB_ABS && o->eb_mode != STZ_EB_REL) STZ_FAIL(STZ_ERR_ARG, "bad eb_mode");
    if (o->bound_mode != STZ_BOUND_POINTWISE && o->bound_mode != STZ_BOUND_REFERENCE)
        STZ_FAIL(STZ_ERR_ARG, "bad bound_mode");
    if (!(o->mult_base > 0) || !(o->mult_low > 0) || !(o->mult_high > 0)) STZ_FAIL(STZ_ERR_ARG, "multipliers must be > 0");
    if (o->radius < 1 || o->radius > 32768) STZ_FAIL(STZ_ERR_ARG, "radius must be in [1, 32768]");
    if (o->zstd_level < 0 || o->zstd_level > 22) STZ_FAIL(STZ_ERR_ARG, "zstd_level must be in [0, 22]");
    if (o->predictor != STZ_PRED_DYNAMIC && o->predictor != STZ_PRED_CUBIC && o->predictor != STZ_PRED_STAGED &&
        o->predictor != STZ_PRED_TRUNCATED)
        STZ_FAIL(STZ_ERR_ARG, "bad predictor");
    if (o->predictor >= STZ_PRED_STAGED && o->model)
        STZ_FAIL(STZ_ERR_ARG, "the staged and truncated predictors take no learned correction");
    if (o->learned_flags < -1 || (o->learned_flags >= 0 && (o->learned_flags & ~0x7f7f)))
        STZ_FAIL(STZ_ERR_ARG, "learned_flags must be -1 or a mask of bits 0-6 and 8-14");
    return STZ_OK;
}

// Estimated coded bits of a sampled code histogram (kEvalBins bins, the last
// one for far and unpredictable codes): ideal code lengths, plus the stored
// value for every entry of the last bin.
double sample_bits(const uint32_t* h, size_t elem)
{
    double n = 0, bits = 0;
    for (int i = 0; i < kEvalBins; ++i) n += h[i];
    if (n == 0) return 0;
    for (int i = 0; i < kEvalBins; ++i)
        if (h[i]) bits += h[i] * std::log2(n / h[i]);
    return bits + (double)h[kEvalBins - 1] * 8.0 * (double)elem;
}

// Blocks of level k where the learned correction pays, from the sampled
// histograms of both predictions: a block is flagged when its estimate
// drops below 0.995 of the base one, and the level only when the saving
// (scaled from the 1/8 sample) exceeds the model record it costs.
uint32_t choose_learned_flags(const uint32_t* hist, size_t elem)
{
    uint32_t flags = 0;
    double saved = 0;
    for (int b = 0; b < 7; ++b) {
        const double b0 = sample_bits(hist + (size_t)b * kEvalBins, elem);
        const double b1 = sample_bits(hist + (size_t)(7 + b) * kEvalBins, elem);
        if (b1 < 0.995 * b0) {
            flags |= 1u << b;
            saved += b0 - b1;
        }
    }
    return 8.0 * saved > 8.0 * (double)(sizeof(LearnedModel) + 4) ? flags : 0u;
}

// ---- error bounds ----------------------------------------------------------------
template <typename T>
stz_status level_error_bounds(stz_context* ctx, const T* field, size_t N, const stz_opts& o, int K, double& eb,
                              std::vector<double>& ebk)
{
    cudaStream_t st = ctx->st;
    // value range as computeRange (FD5:92-104)
    STZ_CUDA(ctx->minmax.ensure(16));
    STZ_CUDA(ctx->h_small.ensure(64));
    {
        KScope ks(ctx, "k_minmax");
        launch_minmax<T>(field, N, ctx->minmax.as<double>(), st);
    }
    STZ_CUDA(cudaMemcpyAsync(ctx->h_small.p, ctx->minmax.p, 16, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaStreamSynchronize(st));
    const unsigned long long* mk = ctx->h_small.as<unsigned long long>();
    const double lo = minmax_key_to_double(mk[0]), hi = minmax_key_to_double(mk[1]);
    double E = o.eb;
    if (o.eb_mode == STZ_EB_REL) {
        E = o.eb * (hi - lo);
        if (!(E > 0) || !std::isfinite(E)) E = o.eb;  // constant (or non-finite) field: bound taken as absolute
    }
    // The quantizer bounds each residual by eb, but the reconstruction
    // dq + P is rounded once more in T, so the reference overshoots its bound
    // by up to ~1.5 ulp of the largest magnitude. The pointwise mode leaves
    // 4 ulp of slack so that max|x - x'| <= E holds when checked in FP64.
    eb = E;
    if (o.bound_mode == STZ_BOUND_POINTWISE) {
        const double ulp = sizeof(T) == 4 ? 1.1920928955078125e-07 : 2.220446049250313e-16;
        const double slack = 4.0 * std::max(std::fabs(lo), std::fabs(hi)) * ulp;
        const double Eb = (std::isfinite(slack) && E > 2.0 * slack) ? E - slack : 0.5 * E;
        eb = Eb / std::max({o.mult_base, o.mult_low, o.mult_high});
    }
    ebk.assign(K + 1, 0.0);
    for (int k = 1; k <= K; ++k) ebk[k] = (k == K ? o.mult_high : k == K - 1 ? o.mult_low : o.mult_base) * eb;
    return STZ_OK;
}
template stz_status level_error_bounds<float>(stz_context*, const float*, size_t, const stz_opts&, int, double&,
                                              std::vector<double>&);
template stz_status level_error_bounds<double>(stz_context*, const double*, size_t, const stz_opts&, int, double&,
                                               std::vector<double>&);

// ---- compress ----------------------------------------------------------------
template <typename T>
stz_status compress_impl(stz_context* ctx, const T* field, int nx, int ny, int nz, const stz_opts& o,
                         stz_stream** out)
{
    Lap lap("compress");
    cudaStream_t st = ctx->st;
    const Geometry g = make_geometry(nx, ny, nz, o.chunk_high, o.chunk_low, o.radius);
    const int K = g.K, R2 = 2 * o.radius;
    const int nstreams = 7 * K;
    const size_t N = (size_t)nx * ny * nz;
    const size_t elem = sizeof(T);
    double eb = 0;
    std::vector<double> ebk;

    // buffers, cleared ahead of the value range
    STZ_CUDA(ctx->grid[0].ensure(g.n_fine_max * elem));
    STZ_CUDA(ctx->grid[1].ensure(g.n_fine_max * elem));
    // the staged predictor's finest level keeps its decoded values too (its
    // later stages predict from them): the grid level K would write, at
    // full size
    const bool staged = o.predictor == STZ_PRED_STAGED;
    if (staged) STZ_CUDA(ctx->grid[K & 1].ensure(std::max(g.n_fine_max, N) * elem));
    STZ_CUDA(ctx->codes.ensure(g.total_codes * 2));
    STZ_CUDA(ctx->unpred_dense.ensure(g.total_codes * elem));
    STZ_CUDA(ctx->unpred_cnt.ensure(g.total_chunk_slots * 4));
    STZ_CUDA(ctx->hist.ensure((size_t)nstreams * R2 * 4));
    STZ_CUDA(ctx->hist_out.ensure((size_t)nstreams * 4));
    STZ_CUDA(cudaMemsetAsync(ctx->hist.p, 0, (size_t)nstreams * R2 * 4, st));
    STZ_CUDA(cudaMemsetAsync(ctx->hist_out.p, 0, (size_t)nstreams * 4, st));
    STZ_CUDA(cudaMemsetAsync(ctx->unpred_cnt.p, 0, g.total_chunk_slots * 4, st));
    STZ_TRY(level_error_bounds<T>(ctx, field, N, o, K, eb, ebk));
    lap.mark("value range");

    // coarsest grid
    const size_t n0 = (size_t)g.c0[0] * g.c0[1] * g.c0[2];
    int cur = 0;
    {
        KScope ks(ctx, "k_subsample");
        launch_subsample<T>(field, nx, ny, nz, 1 << K, ctx->grid[cur].as<T>(), st);
    }
    // to pinned memory, so the host goes on enqueueing (read after the levels)
    STZ_CUDA(ctx->h_small.ensure(64 + n0 * elem));
    STZ_CUDA(cudaMemcpyAsync(ctx->h_small.as<uint8_t>() + 64, ctx->grid[cur].p, n0 * elem, cudaMemcpyDeviceToHost, st));

    // learned models of levels K-1 (record 0) and K (record 1) on the device
    const stz_model* M = o.model;
    std::vector<uint32_t> lflags(K + 1, 0);
    if (M && M->mask) {
        STZ_CUDA(ctx->models.ensure(2 * sizeof(LearnedModel)));
        STZ_CUDA(cudaMemcpyAsync(ctx->models.p, M->lv, 2 * sizeof(LearnedModel), cudaMemcpyHostToDevice, st));
        STZ_CUDA(ctx->eval.ensure(2 * 7 * kEvalBins * 4));
    }
    auto level_model = [&](int k) -> int {  // record index of level k, -1 if none
        const int i = k - (K - 1);
        return (M && i >= 0 && i < 2 && (M->mask >> i & 1u)) ? i : -1;
    };

    // levels, coarse to fine
    for (int k = 1; k <= K; ++k) {
        const StreamDesc& s0 = g.sd[(size_t)(k - 1) * 7];
        LevelEncodeArgs<T> a;
        a.field = field;
        a.fsx = (size_t)nx;
        a.fsy = (size_t)nx * ny;
        a.stride = 1 << (K - k);
        a.coarse = ctx->grid[cur].as<T>();
        a.geo = g.lv[k];
        a.predictor = o.predictor;
        a.codes = ctx->codes.as<uint16_t>() + s0.code_off;
        a.unpred_dense = ctx->unpred_dense.as<T>() + s0.code_off;
        a.unpred_cnt = ctx->unpred_cnt.as<uint32_t>() + s0.chunk_base;
        a.hist_full = ctx->hist.as<uint32_t>() + (size_t)(k - 1) * 7 * R2;
        a.hist_outside = ctx->hist_out.as<uint32_t>() + (size_t)(k - 1) * 7;
        a.decoded = k < K || staged ? ctx->grid[1 - cur].as<T>() : nullptr;
        a.qp = make_quant_params(ebk[k], o.radius);
        a.learned.tensor_cores = learned_tensor_cores();
        if (const int mi = level_model(k); mi >= 0) {
            const LearnedModel& lm = M->lv[mi];
            a.learned.model = ctx->models.as<LearnedModel>() + mi;
            a.learned.rs = (T)(1.0 / (ebk[k] * lm.s_in));
            a.learned.so = (T)(lm.s_out * ebk[k]);
            if (o.learned_flags >= 0) {
                lflags[k] = (uint32_t)(o.learned_flags >> (mi == 0 ? 0 : 8)) & 0x7fu;
            } else {
                a.learned.flags = 0x7f;
                STZ_CUDA(cudaMemsetAsync(ctx->eval.p, 0, 2 * 7 * kEvalBins * 4, st));
                {
                    KScope ks(ctx, "k_learned_eval");
                    launch_learned_eval<T>(a, ctx->eval.as<uint32_t>(), st);
                }
                STZ_CUDA(ctx->h_hist.ensure(2 * 7 * kEvalBins * 4));
                STZ_CUDA(cudaMemcpyAsync(ctx->h_hist.p, ctx->eval.p, 2 * 7 * kEvalBins * 4, cudaMemcpyDeviceToHost,
                                         st));
                STZ_CUDA(cudaStreamSynchronize(st));
                lflags[k] = choose_learned_flags(ctx->h_hist.as<uint32_t>(), elem);
            }
            a.learned.flags = lflags[k];
            if (!lflags[k]) a.learned.model = nullptr, a.learned.flags = 0;
        }
        {
            KScope ks(ctx, k == K ? "k_level_encode[finest]" : "k_level_encode[coarser]");
            a.side = ctx->side();
            launch_level_encode<T>(a, st);
        }
        cur = 1 - cur;
    }
    STZ_CUDA(cudaGetLastError());

    std::vector<StreamDesc> sd = g.sd;
    // work list over every chunk of every stream
    std::vector<CtaWork> work;
    std::vector<uint32_t> ids;
    for (int s = 0; s < nstreams; ++s) add_all_chunks(work, ids, (uint32_t)s, sd[s].nchunks, (int)sd[s].C);
    // Run statistics of every stream whose planes can take run symbols: one
    // pass over the codes right after the level encodes, while the histograms
    // go to the host. The counts per run class depend only on the plane size
    // and the codes, not on which free code values the stream's run symbols
    // later take; here they are numbered from R2, above every code, so no
    // literal is taken for one. Work list and counters go up on the copy
    // stream while the device runs the levels.
    std::vector<unsigned long long> rstats((size_t)nstreams * kRunStats, 0);
    bool rs_any = false;
    size_t r_sd = 0, r_work = 0, r_ids = 0;
    cudaEvent_t ev_up = ctx->event();
    {
        std::vector<StreamDesc> rsd = sd;
        for (auto& d : rsd) {
            d.run_n = run_slot_count(d.C * d.C);
            d.run_base = (uint32_t)R2;
            rs_any = rs_any || d.run_n;
        }
        if (rs_any) {
            r_work = align256(rsd.size() * sizeof(StreamDesc));
            r_ids = align256(r_work + work.size() * sizeof(CtaWork));
            const size_t r_bytes = align256(r_ids + ids.size() * 4);
            STZ_CUDA(ctx->h_stage.ensure(r_bytes));
            uint8_t* hr = ctx->h_stage.as<uint8_t>();
            std::memcpy(hr + r_sd, rsd.data(), rsd.size() * sizeof(StreamDesc));
            std::memcpy(hr + r_work, work.data(), work.size() * sizeof(CtaWork));
            std::memcpy(hr + r_ids, ids.data(), ids.size() * 4);
            STZ_CUDA(ctx->work.ensure(r_bytes));
            STZ_CUDA(cudaMemcpyAsync(ctx->work.p, hr, r_bytes, cudaMemcpyHostToDevice, ctx->st_copy));
            STZ_CUDA(ctx->rstats.ensure(rstats.size() * 8));
            STZ_CUDA(cudaMemsetAsync(ctx->rstats.p, 0, rstats.size() * 8, ctx->st_copy));
            STZ_CUDA(ctx->h_rstats.ensure(rstats.size() * 8));
            STZ_CUDA(cudaEventRecord(ev_up, ctx->st_copy));
        }
    }

    // histogram windows + outside counts + unpred counts to the host, on the
    // copy stream, while ctx->st counts the run symbols
    const int wlo = std::max(0, o.radius - kHistWindow / 2);
    const int wn = std::min(kHistWindow, R2 - wlo);
    STZ_CUDA(ctx->h_hist.ensure((size_t)nstreams * wn * 4));
    const size_t meta_bytes = (size_t)nstreams * 4 + g.total_chunk_slots * 4;
    STZ_CUDA(ctx->h_meta.ensure(meta_bytes));
    cudaStream_t sc = ctx->st_copy;
    cudaEvent_t ev_lv = ctx->event(), ev_hist = ctx->event();
    STZ_CUDA(cudaEventRecord(ev_lv, st));
    STZ_CUDA(cudaStreamWaitEvent(sc, ev_lv, 0));
    STZ_CUDA(cudaMemcpy2DAsync(ctx->h_hist.p, (size_t)wn * 4, ctx->hist.as<uint32_t>() + wlo, (size_t)R2 * 4,
                               (size_t)wn * 4, (size_t)nstreams, cudaMemcpyDeviceToHost, sc));
    uint32_t* h_out = ctx->h_meta.as<uint32_t>();
    uint32_t* h_ucnt = h_out + nstreams;
    STZ_CUDA(cudaMemcpyAsync(h_out, ctx->hist_out.p, (size_t)nstreams * 4, cudaMemcpyDeviceToHost, sc));
    STZ_CUDA(cudaMemcpyAsync(h_ucnt, ctx->unpred_cnt.p, g.total_chunk_slots * 4, cudaMemcpyDeviceToHost, sc));
    STZ_CUDA(cudaEventRecord(ev_hist, sc));
    if (rs_any) {
        STZ_CUDA(cudaStreamWaitEvent(st, ev_up, 0));
        const uint8_t* dw = ctx->work.as<uint8_t>();
        {
            KScope ks(ctx, "k_run_stats");
            launch_run_stats((const CtaWork*)(dw + r_work), (const uint32_t*)(dw + r_ids), (int)work.size(),
                             (const StreamDesc*)(dw + r_sd), ctx->codes.as<uint16_t>(),
                             ctx->rstats.as<unsigned long long>(), st);
        }
        STZ_CUDA(cudaGetLastError());
        STZ_CUDA(cudaMemcpyAsync(ctx->h_rstats.p, ctx->rstats.p, rstats.size() * 8, cudaMemcpyDeviceToHost, st));
    }
    {
        const cudaError_t e = cudaEventSynchronize(ev_hist);
        ctx->ev_pool.push_back(ev_lv);
        ctx->ev_pool.push_back(ev_hist);
        ctx->ev_pool.push_back(ev_up);
        STZ_CUDA(e);
    }
    std::vector<T> coarsest(n0);
    std::memcpy(coarsest.data(), ctx->h_small.as<uint8_t>() + 64, n0 * elem);
    if (level_error_take()) STZ_FAIL(STZ_ERR_CUDA, "level kernel: a TMA tile load did not complete in time");
    if (M && M->mask && learned_tc_error_take(st))
        STZ_FAIL(STZ_ERR_CUDA, "learned correction: a tensor-core MMA did not complete in time");
    lap.mark("levels + histograms");

    // codebooks
    std::vector<std::vector<uint16_t>> syms(nstreams);
    std::vector<std::vector<uint8_t>> lens(nstreams);
    // full histograms of the streams with codes outside the window: one
    // pinned buffer, asynchronous copies, one wait
    std::vector<const uint32_t*> fullh(nstreams, nullptr);
    {
        size_t nfull = 0;
        for (int s = 0; s < nstreams; ++s) nfull += h_out[s] ? 1 : 0;
        if (nfull) {
            STZ_CUDA(ctx->h_fullh.ensure(nfull * (size_t)R2 * 4));
            size_t k = 0;
            for (int s = 0; s < nstreams; ++s)
                if (h_out[s]) {
                    uint32_t* dst = ctx->h_fullh.as<uint32_t>() + k++ * (size_t)R2;
                    STZ_CUDA(cudaMemcpyAsync(dst, ctx->hist.as<uint32_t>() + (size_t)s * R2, (size_t)R2 * 4,
                                             cudaMemcpyDeviceToHost, ctx->st_copy));
                    fullh[s] = dst;
                }
            // on the copy stream: ctx->st is counting run symbols (the level
            // encodes, all these copies need, are complete)
            STZ_CUDA(cudaStreamSynchronize(ctx->st_copy));
        }
    }
    lap.mark("full histograms");
    // run symbols: J slots in unused code values, else none
    for (int s = 0; s < nstreams; ++s) {
        const uint32_t* hw = ctx->h_hist.as<uint32_t>() + s * (size_t)wn;
        auto count = [&](uint32_t c) -> uint64_t {
            if (h_out[s]) return (uint64_t)fullh[s][c];
            return (c >= (uint32_t)wlo && c < (uint32_t)(wlo + wn)) ? hw[c - wlo] : 0;
        };
        sd[s].run_n = (uint32_t)run_slots(count, R2, (int)(sd[s].C * sd[s].C), sd[s].run_base);
    }
    lap.mark("run slots");
    // the plain codebooks while the device counts the run symbols
    ctx->pool->parallel_for((size_t)nstreams, [&](size_t s) {
        const uint32_t* hw = h_out[s] ? fullh[s] : ctx->h_hist.as<uint32_t>() + s * (size_t)wn;
        const int hn = h_out[s] ? R2 : wn, hb = h_out[s] ? 0 : wlo;
        build_codebook(hw, hn, hb, syms[s], lens[s]);
    });
    lap.mark("plain codebooks");
    if (rs_any) {
        STZ_CUDA(cudaStreamSynchronize(st));
        std::memcpy(rstats.data(), ctx->h_rstats.p, rstats.size() * 8);
    }
    lap.mark("run stats wait");
    ctx->pool->parallel_for((size_t)nstreams, [&](size_t s) {
        if (!sd[s].run_n) return;
        const uint32_t* hw = h_out[s] ? fullh[s] : ctx->h_hist.as<uint32_t>() + s * (size_t)wn;
        const int hn = h_out[s] ? R2 : wn, hb = h_out[s] ? 0 : wlo;
        auto code_count = [&](uint32_t c) -> uint64_t {
            return c >= (uint32_t)hb && c < (uint32_t)(hb + hn) ? hw[c - hb] : 0;
        };
        // runs only where they shorten the Huffman payload (else the decoder
        // keeps its plain path): sum(count * length) of both codebooks
        uint64_t bits_plain = 0;
        for (size_t i = 0; i < syms[s].size(); ++i) bits_plain += code_count(syms[s][i]) * lens[s][i];
        std::vector<std::pair<uint32_t, uint64_t>> set;
        set.push_back({(uint32_t)o.radius, rstats[s * kRunStats]});
        for (uint32_t i = 0; i < sd[s].run_n; ++i) set.push_back({sd[s].run_base + i, rstats[s * kRunStats + 1 + i]});
        std::vector<uint16_t> rs;
        std::vector<uint8_t> rl;
        build_codebook_adjusted(hw, hn, hb, set, rs, rl);
        uint64_t bits_runs = 0;
        for (size_t i = 0; i < rs.size(); ++i) {
            uint64_t c = code_count(rs[i]);
            for (const auto& e : set)
                if (e.first == rs[i]) c = e.second;
            bits_runs += c * rl[i];
        }
        if (bits_runs < bits_plain) {
            syms[s].swap(rs);
            lens[s].swap(rl);
        } else {
            sd[s].run_n = 0;
            sd[s].run_base = 0;
        }
    });
    lap.mark("run codebooks");
    uint32_t cb_total = 0;
    for (int s = 0; s < nstreams; ++s) {
        sd[s].cb_off = cb_total;
        sd[s].n_used = (uint32_t)syms[s].size();
        cb_total += sd[s].n_used;
    }
    // unpredictable values: per chunk list offsets
    std::vector<UnpredWork> uwork;
    std::vector<uint64_t> unpred_off(nstreams + 1, 0);
    for (int s = 0; s < nstreams; ++s) {
        uint64_t acc = unpred_off[s];
        const uint32_t* cnt = h_ucnt + sd[s].chunk_base;
        for (uint32_t c = 0; c < sd[s].nchunks; ++c) {
            if (cnt[c]) uwork.push_back({(uint32_t)s, c, acc, cnt[c]});
            acc += cnt[c];
        }
        unpred_off[s + 1] = acc;
    }
    const uint64_t total_unpred = unpred_off[nstreams];

    // upload: sd | cb_sym | cb_len | work | ids | uwork
    const size_t o_sd = 0, o_sym = align256(o_sd + sd.size() * sizeof(StreamDesc));
    const size_t o_len = align256(o_sym + (size_t)cb_total * 2), o_work = align256(o_len + cb_total);
    const size_t o_ids = align256(o_work + work.size() * sizeof(CtaWork));
    const size_t o_uw = align256(o_ids + ids.size() * 4), up_bytes = align256(o_uw + uwork.size() * sizeof(UnpredWork));
    STZ_CUDA(ctx->h_stage.ensure(up_bytes));
    uint8_t* hs = ctx->h_stage.as<uint8_t>();
    std::memcpy(hs + o_sd, sd.data(), sd.size() * sizeof(StreamDesc));
    for (int s = 0; s < nstreams; ++s) {
        std::memcpy(hs + o_sym + 2 * (size_t)sd[s].cb_off, syms[s].data(), 2 * syms[s].size());
        std::memcpy(hs + o_len + sd[s].cb_off, lens[s].data(), lens[s].size());
    }
    std::memcpy(hs + o_work, work.data(), work.size() * sizeof(CtaWork));
    std::memcpy(hs + o_ids, ids.data(), ids.size() * 4);
    if (!uwork.empty()) std::memcpy(hs + o_uw, uwork.data(), uwork.size() * sizeof(UnpredWork));
    STZ_CUDA(ctx->sd.ensure(up_bytes));
    STZ_CUDA(cudaMemcpyAsync(ctx->sd.p, hs, up_bytes, cudaMemcpyHostToDevice, st));
    uint8_t* dstage = ctx->sd.as<uint8_t>();
    const StreamDesc* d_sd = (const StreamDesc*)(dstage + o_sd);
    const uint16_t* d_sym = (const uint16_t*)(dstage + o_sym);
    const uint8_t* d_len = (const uint8_t*)(dstage + o_len);
    const CtaWork* d_work = (const CtaWork*)(dstage + o_work);
    const uint32_t* d_ids = (const uint32_t*)(dstage + o_ids);
    const UnpredWork* d_uw = (const UnpredWork*)(dstage + o_uw);

    lap.mark("codebooks + upload");
    // entropy coding
    STZ_CUDA(ctx->ctab.ensure((size_t)nstreams * R2 * 4));
    STZ_CUDA(ctx->sub_bits.ensure(g.total_sub * 4));
    STZ_CUDA(ctx->sub_off.ensure(g.total_sub * 4));
    STZ_CUDA(ctx->chunk_off.ensure(g.total_chunk_slots * 8));
    STZ_CUDA(ctx->stream_words.ensure((size_t)nstreams * 8 * 3));
    STZ_CUDA(ctx->payload.ensure(g.total_words * 4));
    STZ_CUDA(ctx->ulist.ensure(std::max<uint64_t>(total_unpred, 1) * elem));
    {
        KScope ks(ctx, "k_expand_codebook");
        launch_expand_codebook(d_sd, nstreams, d_sym, d_len, ctx->ctab.as<uint32_t>(), st);
    }
    STZ_CUDA(ctx->rbits.ensure((size_t)nstreams * kRunBitsStride));
    {
        KScope ks(ctx, "k_run_bits");
        launch_run_bits(d_sd, nstreams, ctx->ctab.as<uint32_t>(), ctx->rbits.as<uint8_t>(), st);
    }
    {
        KScope ks(ctx, "k_sub_bits");
        launch_sub_bits(d_work, d_ids, (int)work.size(), d_sd, ctx->codes.as<uint16_t>(), ctx->ctab.as<uint32_t>(),
                        ctx->rbits.as<uint8_t>(), ctx->sub_bits.as<uint32_t>(), st);
    }
    {
        KScope ks(ctx, "k_scan_stream");
        uint32_t max_chunks = 0;
        for (int s = 0; s < nstreams; ++s) max_chunks = std::max(max_chunks, sd[s].nchunks);
        launch_scan_streams(d_sd, nstreams, max_chunks, ctx->sub_bits.as<uint32_t>(), ctx->sub_off.as<uint32_t>(),
                            ctx->chunk_off.as<uint64_t>(), ctx->stream_words.as<uint64_t>(),
                            ctx->payload.as<uint32_t>(), st);
    }
    if (!uwork.empty()) {
        KScope ks(ctx, "k_unpred_move");
        launch_unpred_move<T>(true, d_uw, (int)uwork.size(), d_sd, ctx->codes.as<uint16_t>(),
                              ctx->unpred_dense.as<T>(), ctx->ulist.as<T>(), st);
    }
    STZ_CUDA(cudaGetLastError());

    // stream sizes and tables to the host (the payload is encoded next)
    const size_t t_words = 0, t_choff = align256(t_words + (size_t)nstreams * 8);
    const size_t t_sub = align256(t_choff + g.total_chunk_slots * 8);
    const size_t t_ul = align256(t_sub + g.total_sub * 4), t_bytes = align256(t_ul + total_unpred * elem);
    STZ_CUDA(ctx->h_io.ensure(t_bytes));
    uint8_t* ht = ctx->h_io.as<uint8_t>();
    // on the copy stream, so the encode launches below do not wait for them
    {
        cudaEvent_t ev_scan = ctx->event();
        STZ_CUDA(cudaEventRecord(ev_scan, st));
        STZ_CUDA(cudaStreamWaitEvent(sc, ev_scan, 0));
        ctx->ev_pool.push_back(ev_scan);  // the wait is enqueued: the event may be recorded again
    }
    STZ_CUDA(cudaMemcpyAsync(ht + t_words, ctx->stream_words.p, (size_t)nstreams * 8, cudaMemcpyDeviceToHost, sc));
    STZ_CUDA(cudaMemcpyAsync(ht + t_choff, ctx->chunk_off.p, g.total_chunk_slots * 8, cudaMemcpyDeviceToHost, sc));
    STZ_CUDA(cudaMemcpyAsync(ht + t_sub, ctx->sub_off.p, g.total_sub * 4, cudaMemcpyDeviceToHost, sc));
    if (total_unpred)
        STZ_CUDA(cudaMemcpyAsync(ht + t_ul, ctx->ulist.p, total_unpred * elem, cudaMemcpyDeviceToHost, sc));
    struct Events {
        std::vector<cudaEvent_t> e;
        ~Events()
        {
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } ev;
    // Encode, pack and copy back in groups: every stream of the coarser
    // levels, then the finest level's streams in two halves of their chunk
    // z-layers (all 7 streams per group, so every launch still fills the
    // device); the host zstd-compresses a group's frames while the device
    // encodes the next (one, two, four or eight finest groups measured within
    // noise of each other once payload frames skip zstd; two is the fewest
    // launches that still overlap the copy back). The encodes are enqueued
    // before the host waits for the tables; the copies once it has them.
    const int fin0 = std::max(0, nstreams - 7);
    const int fin_layers = (int)sd[nstreams - 1].ncz;
    const int lpg = std::max(1, (fin_layers + 1) / 2);  // layers per group: two finest groups
    const size_t ngroups = 1 + (size_t)((fin_layers + lpg - 1) / lpg);
    // ev.e[gi]: group gi's words are on the host; ev.e[ngroups + gi]: its
    // encode is done; ev.e[2 * ngroups]: the tables are on the host. The
    // copies run on the context's copy stream, so group gi's copy overlaps
    // group gi + 1's encode.
    ev.e.assign(2 * ngroups + 1, nullptr);
    // the pool's threads wait on the copy events ev.e[0, ngroups) while others
    // compress frames: those waits block instead of spinning on a core
    for (size_t i = 0; i < ev.e.size(); ++i)
        STZ_CUDA(cudaEventCreateWithFlags(&ev.e[i], cudaEventDisableTiming | (i < ngroups ? cudaEventBlockingSync : 0)));
    STZ_CUDA(cudaEventRecord(ev.e[2 * ngroups], sc));
    std::vector<CtaWork> gwork;
    std::vector<uint32_t> gids;
    std::vector<size_t> gw(ngroups + 1, 0);
    for (int s = 0; s < fin0; ++s) add_all_chunks(gwork, gids, (uint32_t)s, sd[s].nchunks, (int)sd[s].C);
    for (size_t gi = 1; gi < ngroups; ++gi) {
        gw[gi] = gwork.size();
        const int L0 = (int)(gi - 1) * lpg, L1 = std::min(fin_layers, L0 + lpg);
        for (int s = fin0; s < nstreams; ++s) {
            const uint32_t cpl = sd[s].ncx * sd[s].ncy;
            std::vector<uint32_t> cs;
            for (uint32_t c = (uint32_t)L0 * cpl; c < (uint32_t)L1 * cpl; ++c) cs.push_back(c);
            add_work(gwork, gids, (uint32_t)s, cs.data(), cs.size(), (int)sd[s].C);
        }
    }
    gw[0] = 0;
    gw[ngroups] = gwork.size();
    const size_t g_work = 0, g_ids = align256(gwork.size() * sizeof(CtaWork)), g_bytes = align256(g_ids + gids.size() * 4);
    STZ_CUDA(ctx->h_meta2.ensure(g_bytes));
    std::memcpy(ctx->h_meta2.as<uint8_t>() + g_work, gwork.data(), gwork.size() * sizeof(CtaWork));
    std::memcpy(ctx->h_meta2.as<uint8_t>() + g_ids, gids.data(), gids.size() * 4);
    STZ_CUDA(ctx->gwork.ensure(g_bytes));
    STZ_CUDA(cudaMemcpyAsync(ctx->gwork.p, ctx->h_meta2.p, g_bytes, cudaMemcpyHostToDevice, st));
    const CtaWork* d_gwork = (const CtaWork*)(ctx->gwork.as<uint8_t>() + g_work);
    const uint32_t* d_gids = (const uint32_t*)(ctx->gwork.as<uint8_t>() + g_ids);
    // the coarser levels' streams (group 0) are many small ones: packed back
    // to back on the device, they go to the host in one transfer
    if (fin0 > 0) STZ_CUDA(ctx->packed.ensure(sd[fin0].word_base * 4));
    for (size_t gi = 0; gi < ngroups; ++gi) {
        {
            KScope ks(ctx, "k_encode");
            launch_encode(d_gwork + gw[gi], d_gids, (int)(gw[gi + 1] - gw[gi]), d_sd, ctx->codes.as<uint16_t>(),
                          ctx->ctab.as<uint32_t>(), ctx->rbits.as<uint8_t>(), ctx->sub_bits.as<uint32_t>(),
                          ctx->sub_off.as<uint32_t>(), ctx->chunk_off.as<uint64_t>(), ctx->payload.as<uint32_t>(), st);
        }
        if (gi == 0 && fin0 > 0) {
            KScope ks(ctx, "k_pack_streams");
            launch_pack_streams(d_sd, ctx->stream_words.as<uint64_t>(), 0, fin0, ctx->payload.as<uint32_t>(),
                                ctx->packed.as<uint32_t>(), st);
        }
        STZ_CUDA(cudaEventRecord(ev.e[ngroups + gi], st));
    }
    STZ_CUDA(cudaGetLastError());
    STZ_CUDA(cudaEventSynchronize(ev.e[2 * ngroups]));
    lap.mark("code lengths + tables");
    const uint64_t* words = (const uint64_t*)(ht + t_words);

    // packed payload layout
    std::vector<uint64_t> meta(3 * (size_t)nstreams);
    uint64_t packed_total = 0;
    for (int s = 0; s < nstreams; ++s) {
        meta[s] = sd[s].word_base;
        meta[nstreams + s] = packed_total;
        meta[2 * (size_t)nstreams + s] = words[s];
        packed_total += words[s];
    }
    STZ_CUDA(ctx->h_payload.ensure(std::max<uint64_t>(packed_total, 1) * 4));
    struct Piece {  // a word range of one stream's payload
        int s;
        uint64_t w0, w1;  // words from the stream's start
    };
    std::vector<std::vector<Piece>> pieces(ngroups);
    const uint64_t* choff_h = (const uint64_t*)(ht + t_choff);
    for (int s = 0; s < fin0; ++s) pieces[0].push_back({s, 0, words[s]});
    for (size_t gi = 1; gi < ngroups; ++gi) {
        const int L0 = (int)(gi - 1) * lpg, L1 = std::min(fin_layers, L0 + lpg);
        for (int s = fin0; s < nstreams; ++s) {
            const uint32_t cpl = sd[s].ncx * sd[s].ncy;
            const uint64_t* co = choff_h + sd[s].chunk_base;
            pieces[gi].push_back({s, co[(size_t)L0 * cpl], co[(size_t)L1 * cpl]});
        }
    }
    for (size_t gi = 0; gi < ngroups; ++gi) {
        STZ_CUDA(cudaStreamWaitEvent(ctx->st_copy, ev.e[ngroups + gi], 0));
        if (gi == 0 && fin0 > 0) {  // packed on the device, at the start of the host payload
            const uint64_t n0 = meta[nstreams + fin0];
            if (n0)
                STZ_CUDA(cudaMemcpyAsync(ctx->h_payload.as<uint32_t>(), ctx->packed.p, n0 * 4, cudaMemcpyDeviceToHost,
                                         ctx->st_copy));
            STZ_CUDA(cudaEventRecord(ev.e[gi], ctx->st_copy));
            continue;
        }
        // the group's words straight from the stream buffers to their place in
        // the packed host payload (one copy per piece)
        for (const Piece& pc : pieces[gi])
            if (pc.w1 > pc.w0)
                STZ_CUDA(cudaMemcpyAsync(ctx->h_payload.as<uint32_t>() + meta[nstreams + pc.s] + pc.w0,
                                         ctx->payload.as<uint32_t>() + sd[pc.s].word_base + pc.w0,
                                         (pc.w1 - pc.w0) * 4, cudaMemcpyDeviceToHost, ctx->st_copy));
        STZ_CUDA(cudaEventRecord(ev.e[gi], ctx->st_copy));
    }
    STZ_CUDA(cudaGetLastError());

    // container: stream headers from the tables while the device encodes
    FileHeader h;
    h.dtype = sizeof(T) == 8 ? 1 : 0;
    h.predictor = o.predictor;
    h.nx = nx, h.ny = ny, h.nz = nz, h.K = K, h.radius = o.radius;
    h.chunk_high = o.chunk_high, h.chunk_low = o.chunk_low, h.zstd_level = o.zstd_level;
    h.eb = eb, h.mult_base = o.mult_base, h.mult_low = o.mult_low, h.mult_high = o.mult_high;
    h.c0[0] = g.c0[0], h.c0[1] = g.c0[1], h.c0[2] = g.c0[2];
    std::vector<LevelDir> levels(K + 1);
    for (int k = 1; k <= K; ++k) {
        levels[k].dx = g.lv[k].dx, levels[k].dy = g.lv[k].dy, levels[k].dz = g.lv[k].dz;
        levels[k].C = g.lv[k].C;
        levels[k].eb = ebk[k];
        levels[k].lflags = lflags[k];
        if (lflags[k]) levels[k].model = M->lv[level_model(k)];
    }
    std::vector<StreamParts> parts(nstreams);
    const uint64_t* choff = (const uint64_t*)(ht + t_choff);
    const uint32_t* subo = (const uint32_t*)(ht + t_sub);
    const uint8_t* ul = ht + t_ul;
    for (int s = 0; s < nstreams; ++s) {
        const StreamDesc& d = sd[s];
        StreamParts& p = parts[s];
        p.words = ctx->h_payload.as<uint32_t>() + meta[nstreams + s];
        p.chunk_word_off = choff + d.chunk_base;
        p.layers = (int)d.ncz;
        p.chunks_per_layer = (int)(d.ncx * d.ncy);
    }
    // each stream header is built by the pool job that compresses it (the
    // finest streams', the largest, first)
    auto build_header = [&](size_t s) {
        const StreamDesc& d = sd[s];
        append_stream_header(parts[s].hdr, syms[s].data(), lens[s].data(), d.n_used, d.run_base, d.run_n,
                             unpred_off[s + 1] - unpred_off[s], ul + unpred_off[s] * elem, elem,
                             h_ucnt + d.chunk_base, choff + d.chunk_base, subo + d.sub_base, (int)d.nchunks,
                             (int)d.C);
    };
    ContainerWriter cw(h, parts, *ctx->pool);
    std::atomic<int> ev_err{0};
    // a group's copy seen complete once: later frames of the group make no
    // CUDA call (concurrent calls from the pool's threads serialize in the
    // driver, and frames queued behind a finished copy waited on each other)
    std::unique_ptr<std::atomic<int>[]> copied(new std::atomic<int>[ngroups]);
    for (size_t i = 0; i < ngroups; ++i) copied[i].store(0);
    // zstd groups: every stream header first (nothing to wait for), then
    // the payload of encode group g after its copy (event g)
    cw.compress_groups(
        ngroups + 1,
        [&](size_t st_, int layer) -> size_t {
            if (layer < 0) return 0;
            if ((int)st_ < fin0) return 1;  // coarser levels: encode group 0
            return 2 + (size_t)(layer / lpg);
        },
        [&](size_t g) {
            if (g == 0 || copied[g - 1].load(std::memory_order_acquire)) return;
            if (cudaEventSynchronize(ev.e[g - 1]) != cudaSuccess) ev_err = 1;
            copied[g - 1].store(1, std::memory_order_release);
        },
        build_header);
    if (ev_err) {  // reports the device error
        STZ_CUDA(cudaStreamSynchronize(ctx->st_copy));
        STZ_CUDA(cudaStreamSynchronize(st));
    }
    STZ_CUDA(cudaStreamSynchronize(ctx->st_copy));  // every group's copy (the payload buffer is reused next call)
    lap.mark("encode + copy + zstd");
    auto* so = new (std::nothrow) stz_stream();
    if (!so) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    so->bytes = cw.finish(coarsest.data(), levels);
    lap.mark("container");
    so->raw_payload_bytes = packed_total * 4;
    const std::string pe = parse_stream(so->bytes.data(), so->bytes.size(), so->dir);
    if (!pe.empty()) {
        delete so;
        STZ_FAIL(STZ_ERR_FORMAT, "internal: written stream does not parse: " + pe);
    }
    lap.mark("parse check");
    *out = so;
    return STZ_OK;
}

// ---- decode preparation -------------------------------------------------------
namespace {
// Checks one parsed stream header against its directory entry; nullptr when
// it is consistent. Fills the stream's per-chunk unpredictable-value prefix.
const char* check_stream(const FileHeader& h, const LevelDir& L, const StreamDir& sdir, const StreamHeader& H,
                         std::vector<uint64_t>& pre)
{
    const uint32_t C = (uint32_t)L.C;
    const uint32_t nchunks = (uint32_t)((L.dx / L.C) * (L.dy / L.C) * (L.dz / L.C));
    const uint32_t n_used = (uint32_t)H.sym.size();
    if (H.run_n && (uint64_t)H.run_base + H.run_n > 2 * (uint64_t)h.radius) return "run symbols outside the code range";
    uint64_t raw = 0;
    for (uint64_t v : sdir.lr) raw += v;
    if (H.chunk_word_off.back() * 4 != raw) return "marker table does not match payload size";
    if (n_used == 0 || (n_used == 1 && raw != 0)) return "bad codebook";
    // codebook: symbols in range, sorted canonically, Kraft sum <= 1
    uint64_t kraft = 0;
    for (uint32_t j = 0; j < n_used; ++j) {
        if (H.sym[j] >= 2 * h.radius) return "codebook symbol out of range";
        if (j && (H.len[j] < H.len[j - 1] || (H.len[j] == H.len[j - 1] && H.sym[j] <= H.sym[j - 1])))
            return "codebook not in canonical order";
        if (n_used > 1) {
            if (H.len[j] == 0) return "zero-length code";
            kraft += 1ull << (kMaxCodeLen - H.len[j]);
        }
        if (H.sym[j] == 0 && H.n_unpred == 0) return "code 0 without unpredictable values";
    }
    if (kraft > (1ull << kMaxCodeLen)) return "codebook violates the Kraft inequality";
    for (uint32_t c = 0; c < nchunks; ++c) {
        if (H.chunk_word_off[c] > H.chunk_word_off[c + 1]) return "bad marker table";
        const uint64_t cbits = 32 * (H.chunk_word_off[c + 1] - H.chunk_word_off[c]);
        const uint32_t* so = H.sub_off.data() + (size_t)c * C;
        for (uint32_t lz = 0; lz < C; ++lz)
            if (so[lz] > cbits || (lz && so[lz] < so[lz - 1])) return "bad plane offsets";
    }
    pre.resize(nchunks + 1);
    uint64_t acc = 0;
    for (uint32_t c = 0; c < nchunks; ++c) {
        pre[c] = acc;
        acc += H.unpred_count[c];
    }
    pre[nchunks] = acc;
    if (acc != H.n_unpred) return "unpredictable counts do not match";
    return nullptr;
}
}  // namespace

std::vector<DecodeBatch> decode_batches(const ParsedStream& ps, int kmax)
{
    std::vector<DecodeBatch> v;
    if (kmax < 1) return v;
    const int f0 = 7 * (kmax - 1);
    if (kmax > 1) v.push_back({0, f0, 0, -1});
    const int L = (int)ps.lv[kmax].s[0].layers;
    if (L >= 2) {
        v.push_back({f0, f0 + 7, 0, L / 2});
        v.push_back({f0, f0 + 7, L / 2, L});
    } else {
        v.push_back({f0, f0 + 7, 0, -1});
    }
    return v;
}

stz_status prepare(stz_context* ctx, const stz_stream* s, int kmax, Prepared& p, const BatchFn* on_batch)
{
    Lap lap("prepare");
    const ParsedStream& ps = s->dir;
    const FileHeader& h = ps.h;
    const size_t elem = h.elem();
    const int nstreams = 7 * kmax;
    p.kmax = kmax;
    p.sd.assign(nstreams, StreamDesc{});
    p.hdr.assign(nstreams, StreamHeader{});
    p.unpred_prefix.assign(nstreams, {});
    std::atomic<int> bad{0};
    std::vector<const char*> why(nstreams, nullptr);
    const uint8_t* bytes = s->bytes.data();
    ctx->pool->parallel_for((size_t)nstreams, [&](size_t r) {
        const size_t i = (size_t)nstreams - 1 - r;  // finest streams (largest headers) first
        const int k = (int)i / 7 + 1, b = (int)i % 7;
        const LevelDir& L = ps.lv[k];
        const StreamDir& d = L.s[b];
        std::vector<uint8_t> raw(d.hdr_raw);
        const int nch = (L.dx / L.C) * (L.dy / L.C) * (L.dz / L.C);
        if (!decode_frame(bytes + d.data_off, d.hdr_stored, d.hdr_raw, raw.data())) bad = 1;
        else if (!parse_stream_header(raw.data(), raw.size(), nch, L.C, elem, ps.version, p.hdr[i])) bad = 2;
        else why[i] = check_stream(h, L, d, p.hdr[i], p.unpred_prefix[i]);
    });
    if (bad) STZ_FAIL(STZ_ERR_FORMAT, bad == 1 ? "stream header frame does not decode" : "bad stream header");
    for (const char* w : why)
        if (w) STZ_FAIL(STZ_ERR_FORMAT, w);
    lap.mark("header frames");
    // layout
    uint64_t codes = 0, chunks = 0, subs = 0, words = 0, syms = 0, unp = 0;
    p.ulist_off.assign(nstreams + 1, 0);
    for (int i = 0; i < nstreams; ++i) {
        const int k = i / 7 + 1;
        const LevelDir& L = ps.lv[k];
        const StreamHeader& H = p.hdr[i];
        StreamDesc& d = p.sd[i];
        d.C = L.C;
        d.ncx = L.dx / L.C, d.ncy = L.dy / L.C, d.ncz = L.dz / L.C;
        d.nchunks = d.ncx * d.ncy * d.ncz;
        d.radius = h.radius;
        d.code_off = codes;
        codes += (uint64_t)L.dx * L.dy * L.dz;
        d.chunk_base = chunks;
        chunks += d.nchunks + 1;
        d.sub_base = subs;
        subs += (uint64_t)d.nchunks * d.C;
        d.cb_off = (uint32_t)syms;
        d.n_used = (uint32_t)H.sym.size();
        syms += d.n_used;
        d.run_base = H.run_base;
        d.run_n = H.run_n;
        d.word_base = words;
        d.word_cap = H.chunk_word_off.back() + 4;
        words += d.word_cap;
        p.ulist_off[i] = unp;
        unp += H.n_unpred;
    }
    p.ulist_off[nstreams] = unp;
    p.total_codes = codes;
    p.total_unpred = unp;
    const size_t o_sd = 0, o_sym = align256(nstreams * sizeof(StreamDesc)), o_len = align256(o_sym + syms * 2);
    const size_t o_sub = align256(o_len + syms), o_ch = align256(o_sub + subs * 4), o_ul = align256(o_ch + chunks * 8);
    // learned models of levels 0..kmax (index k), with the tables
    const bool learned = stream_learned(ps);
    const size_t o_md = align256(o_ul + unp * elem);
    const size_t o_pl = align256(o_md + (learned ? (size_t)(kmax + 1) * sizeof(LearnedModel) : 0));
    const size_t total = align256(o_pl + words * 4);
    STZ_CUDA(ctx->h_stage.ensure(total));
    uint8_t* hs = ctx->h_stage.as<uint8_t>();
    if (learned)
        for (int k = 0; k <= kmax; ++k)
            std::memcpy(hs + o_md + k * sizeof(LearnedModel), &ps.lv[k].model, sizeof(LearnedModel));
    std::memcpy(hs + o_sd, p.sd.data(), nstreams * sizeof(StreamDesc));
    ctx->pool->parallel_for((size_t)nstreams, [&](size_t i) {
        const StreamHeader& H = p.hdr[i];
        const StreamDesc& d = p.sd[i];
        std::memcpy(hs + o_sym + 2 * (size_t)d.cb_off, H.sym.data(), 2 * H.sym.size());
        std::memcpy(hs + o_len + d.cb_off, H.len.data(), H.len.size());
        std::memcpy(hs + o_sub + 4 * d.sub_base, H.sub_off.data(), 4 * H.sub_off.size());
        std::memcpy(hs + o_ch + 8 * d.chunk_base, H.chunk_word_off.data(), 8 * H.chunk_word_off.size());
        if (H.n_unpred) std::memcpy(hs + o_ul + p.ulist_off[i] * elem, H.unpred.data(), H.unpred.size());
    });
    lap.mark("layout + tables");
    // payload frames straight into the staging buffer
    struct Job {
        const uint8_t* src;
        uint64_t stored, raw;
        uint8_t* dst;
    };
    std::vector<Job> jobs;
    std::vector<size_t> stream_first_job(nstreams + 1);
    for (int i = 0; i < nstreams; ++i) {
        stream_first_job[i] = jobs.size();
        const StreamDir& d = ps.lv[i / 7 + 1].s[i % 7];
        const uint8_t* src = bytes + d.data_off + d.hdr_stored;
        uint8_t* dst = hs + o_pl + 4 * p.sd[i].word_base;
        for (uint32_t L = 0; L < d.layers; ++L) {
            jobs.push_back({src, d.ls[L], d.lr[L], dst});
            src += d.ls[L];
            dst += d.lr[L];
        }
        std::memset(dst, 0, 16);  // read-ahead padding of the decoder
    }
    stream_first_job[nstreams] = jobs.size();
    // Tables and the coarsest grid first, then the payload in batches of
    // whole streams: each batch's host->device copy (and, with on_batch, its
    // decoding) runs while the next batch is being zstd-decoded.
    const size_t o_tab = align256(total), dev_total = o_tab + (size_t)nstreams * decode_tables_bytes();
    STZ_CUDA(p.stage->ensure(dev_total));
    STZ_CUDA(cudaMemcpyAsync(p.stage->p, hs, o_pl, cudaMemcpyHostToDevice, ctx->st));
    uint8_t* ds = p.stage->as<uint8_t>();
    p.d_sd = (StreamDesc*)(ds + o_sd);
    p.d_sym = (uint16_t*)(ds + o_sym);
    p.d_len = ds + o_len;
    p.d_sub = (uint32_t*)(ds + o_sub);
    p.d_choff = (uint64_t*)(ds + o_ch);
    p.d_ulist = ds + o_ul;
    p.d_models = learned ? (LearnedModel*)(ds + o_md) : nullptr;
    p.d_payload = (uint32_t*)(ds + o_pl);
    p.d_tables = ds + o_tab;
    launch_build_tables(p.d_sd, nstreams, p.d_sym, p.d_len, p.d_tables, ctx->st);
    STZ_CUDA(cudaGetLastError());
    const size_t n0 = (size_t)h.c0[0] * h.c0[1] * h.c0[2];
    STZ_CUDA(p.coarsest->ensure(n0 * elem));
    STZ_CUDA(cudaMemcpyAsync(p.coarsest->p, bytes + ps.coarsest_off, n0 * elem, cudaMemcpyHostToDevice, ctx->st));
    // batches: with on_batch, decode_batches; else whole streams, at least
    // two frames per pool thread
    std::vector<DecodeBatch> batches;
    if (on_batch) {
        batches = decode_batches(ps, kmax);
    } else {
        const size_t min_batch = 2 * (size_t)ctx->pool->size();
        for (int s0 = 0; s0 < nstreams;) {
            int s1 = s0 + 1;
            while (s1 < nstreams && stream_first_job[s1] - stream_first_job[s0] < min_batch) ++s1;
            batches.push_back({s0, s1, 0, -1});
            s0 = s1;
        }
    }
    // bytes of each stream's payload before chunk layer l
    auto layer_bytes = [&](int si, int l) -> size_t {
        const StreamDir& d = ps.lv[si / 7 + 1].s[si % 7];
        size_t b = 0;
        for (int i = 0; i < l; ++i) b += d.lr[i];
        return b;
    };
    auto stream_end = [&](int si) -> size_t { return si + 1 < nstreams ? o_pl + 4 * p.sd[si + 1].word_base : total; };
    // Payload copies go on the context's copy stream, so a batch's copy
    // overlaps the decoding of the batch before it; ctx->st waits on each
    // batch's event before decoding it (or, without on_batch, on the last).
    struct Events {
        std::vector<cudaEvent_t> e;
        ~Events()
        {
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } ev;
    auto sync_both = [&]() {
        cudaStreamSynchronize(ctx->st_copy);
        cudaStreamSynchronize(ctx->st_dec);
        cudaStreamSynchronize(ctx->st);
    };
    std::vector<size_t> bjobs;
    for (const DecodeBatch& B : batches) {
        // the batch's frames: whole streams, or layers [l0, l1) of each
        bjobs.clear();
        for (int si = B.s0; si < B.s1; ++si) {
            const size_t a = stream_first_job[si] + (B.l1 < 0 ? 0 : (size_t)B.l0);
            const size_t b = B.l1 < 0 ? stream_first_job[si + 1] : stream_first_job[si] + (size_t)B.l1;
            for (size_t j = a; j < b; ++j) bjobs.push_back(j);
        }
        ctx->pool->parallel_for(bjobs.size(), [&](size_t i) {
            const Job& J = jobs[bjobs[i]];
            if (!decode_frame(J.src, J.stored, J.raw, J.dst)) bad = 3;
        });
        if (bad) {
            sync_both();
            STZ_FAIL(STZ_ERR_ZSTD, "payload frame does not decode");
        }
        cudaEvent_t e = nullptr;
        cudaError_t ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (ce == cudaSuccess) ev.e.push_back(e);
        auto copy = [&](size_t b0, size_t b1) {
            if (ce == cudaSuccess && b1 > b0)
                ce = cudaMemcpyAsync(ds + b0, hs + b0, b1 - b0, cudaMemcpyHostToDevice, ctx->st_copy);
        };
        if (B.l1 < 0) {
            copy(o_pl + 4 * p.sd[B.s0].word_base, stream_end(B.s1 - 1));
        } else {
            const int L = (int)ps.lv[B.s0 / 7 + 1].s[B.s0 % 7].layers;
            for (int si = B.s0; si < B.s1; ++si) {
                const size_t base = o_pl + 4 * p.sd[si].word_base;
                copy(base + layer_bytes(si, B.l0), B.l1 >= L ? stream_end(si) : base + layer_bytes(si, B.l1));
            }
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(e, ctx->st_copy);
        if (ce == cudaSuccess && !on_batch && B.s1 == nstreams) ce = cudaStreamWaitEvent(ctx->st, e, 0);
        if (ce != cudaSuccess) {
            sync_both();
            STZ_CUDA(ce);
        }
        if (on_batch) {
            const stz_status st = (*on_batch)(B, e);
            if (st != STZ_OK) {
                sync_both();
                return st;
            }
        }
    }
    lap.mark("payload frames + h2d");
    STZ_CUDA(cudaStreamSynchronize(ctx->st_copy));  // the pinned staging buffer is reused by the next call
    STZ_CUDA(cudaStreamSynchronize(ctx->st_dec));
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    lap.mark("host->device");
    return STZ_OK;
}

// Entropy-decode the listed chunks (and scatter their unpredictable values).
template <typename T>
stz_status decode_chunks(stz_context* ctx, const Prepared& p, const std::vector<CtaWork>& work,
                         const std::vector<uint32_t>& ids, const std::vector<UnpredWork>& uwork)
{
    const size_t o_w = 0, o_i = align256(work.size() * sizeof(CtaWork));
    const size_t o_u = align256(o_i + ids.size() * 4), total = align256(o_u + uwork.size() * sizeof(UnpredWork));
    STZ_CUDA(ctx->h_meta.ensure(total));
    uint8_t* hm = ctx->h_meta.as<uint8_t>();
    std::memcpy(hm + o_w, work.data(), work.size() * sizeof(CtaWork));
    std::memcpy(hm + o_i, ids.data(), ids.size() * 4);
    if (!uwork.empty()) std::memcpy(hm + o_u, uwork.data(), uwork.size() * sizeof(UnpredWork));
    STZ_CUDA(ctx->work.ensure(total));
    STZ_CUDA(cudaMemcpyAsync(ctx->work.p, hm, total, cudaMemcpyHostToDevice, ctx->st));
    const uint8_t* dw = ctx->work.as<uint8_t>();
    STZ_CUDA(ctx->codes.ensure(p.total_codes * 2));
    if (p.total_unpred) STZ_CUDA(ctx->unpred_dense.ensure(p.total_codes * sizeof(T)));
    if (!work.empty()) {
        KScope ks(ctx, "k_decode");
        launch_decode((const CtaWork*)(dw + o_w), (const uint32_t*)(dw + o_i), (int)work.size(), p.d_sd, p.d_sym,
                      p.d_tables, p.d_sub, p.d_choff, p.d_payload, ctx->codes.as<uint16_t>(), ctx->st);
    }
    if (!uwork.empty()) {
        KScope ks(ctx, "k_unpred_move");
        launch_unpred_move<T>(false, (const UnpredWork*)(dw + o_u), (int)uwork.size(), p.d_sd,
                              ctx->codes.as<uint16_t>(), ctx->unpred_dense.as<T>(), (T*)p.d_ulist, ctx->st);
    }
    STZ_CUDA(cudaGetLastError());
    // the pinned work buffer is reused by the next call
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    return STZ_OK;
}

void add_unpred_work(const Prepared& p, uint32_t s, const uint32_t* chunks, size_t n, std::vector<UnpredWork>& uw)
{
    const StreamHeader& H = p.hdr[s];
    if (!H.n_unpred) return;
    for (size_t i = 0; i < n; ++i) {
        const uint32_t c = chunks[i];
        if (H.unpred_count[c]) uw.push_back({s, c, p.ulist_off[s] + p.unpred_prefix[s][c], H.unpred_count[c]});
    }
}

QuantParams qparams(const ParsedStream& ps, int k)
{
    QuantParams q;
    q.eb = ps.lv[k].eb;
    q.recip = 1.0 / q.eb;
    q.radius = ps.h.radius;
    return q;
}

LevelGeom level_geom(const ParsedStream& ps, int k)
{
    LevelGeom g;
    const LevelDir& L = ps.lv[k];
    g.dx = L.dx, g.dy = L.dy, g.dz = L.dz, g.C = L.C;
    g.ncx = L.dx / L.C, g.ncy = L.dy / L.C, g.ncz = L.dz / L.C;
    g.n = (size_t)L.dx * L.dy * L.dz;
    return g;
}

// Launches of a decode of levels 1..kdec in batches of streams (in level
// order): the chunks of a batch are entropy-decoded, then every level whose
// seven streams are all decoded is reconstructed; the last one lands in out.
template <typename T>
struct DecodePipe {
    stz_context* ctx;
    const stz_stream* s;
    const Prepared& p;
    int kdec;
    T* out;
    std::vector<DecodeBatch> batches;
    bool planned = false;
    size_t next_batch = 0;
    std::vector<size_t> wfirst, ufirst;  // per batch: first work / unpredictable item (+ end)
    size_t o_w = 0, o_i = 0, o_u = 0;
    int next_level = 1, cur = 0;
    int fin_bricks = 0, fin_done = 0;  // the finest level's z-bricks, and those launched
    const T* coarse = nullptr;
    std::vector<cudaEvent_t> events;  // ordering between ctx->st and ctx->st_dec

    DecodePipe(stz_context* c, const stz_stream* st, const Prepared& pp, int k, T* o, std::vector<DecodeBatch> b)
        : ctx(c), s(st), p(pp), kdec(k), out(o), batches(std::move(b))
    {
    }
    ~DecodePipe()
    {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
    }
    cudaError_t record(cudaStream_t on, cudaStream_t waiter)
    {
        cudaEvent_t e = nullptr;
        cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (r != cudaSuccess) return r;
        events.push_back(e);
        r = cudaEventRecord(e, on);
        return r == cudaSuccess ? cudaStreamWaitEvent(waiter, e, 0) : r;
    }

    // Work lists of every batch, uploaded once; buffers sized.
    stz_status plan()
    {
        const ParsedStream& ps = s->dir;
        std::vector<CtaWork> work;
        std::vector<uint32_t> ids;
        std::vector<UnpredWork> uw;
        wfirst.assign(batches.size() + 1, 0);
        ufirst.assign(batches.size() + 1, 0);
        std::vector<uint32_t> cs;
        for (size_t bi = 0; bi < batches.size(); ++bi) {
            const DecodeBatch& B = batches[bi];
            wfirst[bi] = work.size();
            ufirst[bi] = uw.size();
            for (int i = B.s0; i < B.s1; ++i) {
                const StreamDesc& d = p.sd[i];
                const uint32_t per_layer = d.ncx * d.ncy;
                const uint32_t c0 = B.l1 < 0 ? 0 : (uint32_t)B.l0 * per_layer;
                const uint32_t c1 = B.l1 < 0 ? d.nchunks : std::min(d.nchunks, (uint32_t)B.l1 * per_layer);
                cs.resize(c1 > c0 ? c1 - c0 : 0);
                for (uint32_t c = c0; c < c1; ++c) cs[c - c0] = c;
                add_work(work, ids, (uint32_t)i, cs.data(), cs.size(), (int)d.C);
                add_unpred_work(p, (uint32_t)i, cs.data(), cs.size(), uw);
            }
        }
        wfirst[batches.size()] = work.size();
        ufirst[batches.size()] = uw.size();
        o_w = 0, o_i = align256(work.size() * sizeof(CtaWork));
        o_u = align256(o_i + ids.size() * 4);
        const size_t total = align256(o_u + uw.size() * sizeof(UnpredWork));
        STZ_CUDA(ctx->h_meta.ensure(total));
        uint8_t* hm = ctx->h_meta.as<uint8_t>();
        std::memcpy(hm + o_w, work.data(), work.size() * sizeof(CtaWork));
        std::memcpy(hm + o_i, ids.data(), ids.size() * 4);
        if (!uw.empty()) std::memcpy(hm + o_u, uw.data(), uw.size() * sizeof(UnpredWork));
        STZ_CUDA(ctx->work.ensure(total));
        STZ_CUDA(cudaMemcpyAsync(ctx->work.p, hm, total, cudaMemcpyHostToDevice, ctx->st));
        STZ_CUDA(ctx->codes.ensure(p.total_codes * 2));
        if (p.total_unpred) STZ_CUDA(ctx->unpred_dense.ensure(p.total_codes * sizeof(T)));
        const FileHeader& h = ps.h;
        size_t gmax = (size_t)h.c0[0] * h.c0[1] * h.c0[2];
        for (int k = 1; k < kdec; ++k) gmax = std::max(gmax, 8 * (size_t)ps.lv[k].dx * ps.lv[k].dy * ps.lv[k].dz);
        STZ_CUDA(ctx->grid[0].ensure(gmax * sizeof(T)));
        STZ_CUDA(ctx->grid[1].ensure(gmax * sizeof(T)));
        coarse = p.coarsest->as<T>();
        // the finest level decodes by z-bricks as its chunk layers arrive
        // (plain kernels only; else the whole level after the last batch;
        // the staged and truncated predictors' kernels take whole levels)
        fin_bricks = level_decode_bricks(level_geom(ps, kdec),
                                         (learned_args<T>(ps, kdec, p.d_models).model != nullptr &&
                                          learned_args<T>(ps, kdec, p.d_models).flags) ||
                                             ps.h.predictor >= STZ_PRED_STAGED,
                                         0, nullptr);
        // the entropy decodes (ctx->st_dec) follow everything enqueued on
        // ctx->st so far: tables, coarsest grid, work lists, earlier calls
        STZ_CUDA(record(ctx->st, ctx->st_dec));
        planned = true;
        return STZ_OK;
    }

    LevelDecodeArgs<T> level_args(int k)
    {
        const ParsedStream& ps = s->dir;
        LevelDecodeArgs<T> a;
        a.coarse = coarse;
        a.geo = level_geom(ps, k);
        a.predictor = ps.h.predictor;
        a.qp = qparams(ps, k);
        a.codes = ctx->codes.as<uint16_t>() + p.sd[(size_t)(k - 1) * 7].code_off;
        a.unpred_dense = p.total_unpred ? ctx->unpred_dense.as<T>() + p.sd[(size_t)(k - 1) * 7].code_off : nullptr;
        a.out = k == kdec ? out : ctx->grid[cur].as<T>();
        a.learned = learned_args<T>(ps, k, p.d_models);
        a.side = ctx->side();
        return a;
    }

    // The next batch's entropy decode on ctx->st_dec (after `copied`, null:
    // already on the device), then on ctx->st every level it completes, and
    // for a layer batch of the finest level the z-bricks its layers cover.
    stz_status batch(const DecodeBatch& B, cudaEvent_t copied)
    {
        if (!planned) STZ_TRY(plan());
        const size_t bi = next_batch++;
        cudaStream_t sd = ctx->st_dec;
        if (copied) STZ_CUDA(cudaStreamWaitEvent(sd, copied, 0));
        const uint8_t* dw = ctx->work.as<uint8_t>();
        const size_t w0 = wfirst[bi], w1 = wfirst[bi + 1], u0 = ufirst[bi], u1 = ufirst[bi + 1];
        if (w1 > w0) {
            KScope ks(ctx, "k_decode", 1, sd);
            launch_decode((const CtaWork*)(dw + o_w) + w0, (const uint32_t*)(dw + o_i), (int)(w1 - w0), p.d_sd,
                          p.d_sym, p.d_tables, p.d_sub, p.d_choff, p.d_payload, ctx->codes.as<uint16_t>(), sd);
        }
        if (u1 > u0) {
            KScope ks(ctx, "k_unpred_move", 1, sd);
            launch_unpred_move<T>(false, (const UnpredWork*)(dw + o_u) + u0, (int)(u1 - u0), p.d_sd,
                                  ctx->codes.as<uint16_t>(), ctx->unpred_dense.as<T>(), (T*)p.d_ulist, sd);
        }
        const ParsedStream& ps = s->dir;
        const bool last = bi + 1 == batches.size();
        const bool whole = B.l1 < 0 || B.l1 >= (int)ps.lv[kdec].s[0].layers;
        // streams complete after this batch. The coarser levels of the first
        // batch start after the second batch's entropy decode instead of
        // beside it: its CTAs delayed theirs 3-4x, and the finest level's
        // first bricks wait for both anyway (STZ_DECODE_DEFER=0: beside it)
        static const bool defer = [] {
            const char* e = std::getenv("STZ_DECODE_DEFER");
            return !e || std::atoi(e) != 0;
        }();
        const int s1 = defer && bi == 0 && batches.size() > 1 ? 0 : whole ? B.s1 : B.s0;
        bool waited = false;  // ctx->st waits for this batch's entropy decode
        auto wait_decode = [&]() -> cudaError_t {
            if (waited) return cudaSuccess;
            waited = true;
            return record(sd, ctx->st);
        };
        if (next_level < kdec && 7 * next_level <= s1) STZ_CUDA(wait_decode());
        for (; next_level < kdec && 7 * next_level <= s1; ++next_level) {
            const LevelDecodeArgs<T> a = level_args(next_level);
            {
                KScope ks(ctx, next_level == ps.h.K ? "k_level_decode[finest]" : "k_level_decode[coarser]");
                launch_level_decode<T>(a, ctx->st);
            }
            coarse = a.out;
            cur = 1 - cur;
        }
        int bricks_to = fin_done;
        if (next_level == kdec && B.s0 == 7 * (kdec - 1) && fin_bricks && !last) {
            const LevelGeom g = level_geom(ps, kdec);
            level_decode_bricks(g, false, B.l1 * g.C, &bricks_to);
        }
        const bool finest_part = bricks_to > fin_done;
        if ((next_level == kdec && 7 * kdec <= s1) || finest_part) STZ_CUDA(wait_decode());
        if (next_level == kdec) {
            LevelDecodeArgs<T> a = level_args(kdec);
            const char* nm = kdec == ps.h.K ? "k_level_decode[finest]" : "k_level_decode[coarser]";
            if (finest_part) {  // the bricks of the layers on the device so far
                a.zb_lo = fin_done, a.zb_hi = bricks_to;
                KScope ks(ctx, nm);
                launch_level_decode<T>(a, ctx->st);
                fin_done = bricks_to;
            }
            if (7 * kdec <= s1) {  // every layer decoded: the rest of the level
                if (fin_bricks) a.zb_lo = fin_done, a.zb_hi = fin_bricks;
                {
                    KScope ks(ctx, nm);
                    launch_level_decode<T>(a, ctx->st);
                }
                fin_done = fin_bricks;
                ++next_level;
            }
        }
        STZ_CUDA(cudaGetLastError());
        return STZ_OK;
    }
};

// Reconstruct levels 1..kdec; the last one lands in out_dev.
template <typename T>
stz_status decode_levels(stz_context* ctx, const stz_stream* s, const Prepared& p, int kdec, T* out_dev)
{
    const ParsedStream& ps = s->dir;
    const FileHeader& h = ps.h;
    const size_t n0 = (size_t)h.c0[0] * h.c0[1] * h.c0[2];
    if (kdec == 0) {
        STZ_CUDA(cudaMemcpyAsync(out_dev, p.coarsest->p, n0 * sizeof(T), cudaMemcpyDeviceToDevice, ctx->st));
        return STZ_OK;
    }
    DecodePipe<T> pipe(ctx, s, p, kdec, out_dev, {DecodeBatch{0, 7 * kdec, 0, -1}});
    STZ_TRY(pipe.plan());
    STZ_CUDA(cudaStreamSynchronize(ctx->st));  // the pinned work-list buffer is free for the caller
    return pipe.batch(pipe.batches[0], nullptr);
}

template <typename T>
stz_status decompress_level_dev(stz_context* ctx, const stz_stream* s, int level, T* out_dev)
{
    const int K = s->dir.h.K;
    const int kdec = K - level;
    if (s->resident && s->resident->kmax >= kdec) {
        STZ_TRY(decode_levels<T>(ctx, s, *s->resident, kdec, out_dev));
        STZ_CUDA(cudaStreamSynchronize(ctx->st));  // the output is complete on return
        if (level_error_take()) STZ_FAIL(STZ_ERR_CUDA, "level kernel: a TMA tile load did not complete in time");
        if (stream_learned(s->dir) && learned_tc_error_take(ctx->st))
            STZ_FAIL(STZ_ERR_CUDA, "learned correction: a tensor-core MMA did not complete in time");
        return STZ_OK;
    }
    Prepared p;
    ctx->borrow(p);
    if (kdec == 0) {
        STZ_TRY(prepare(ctx, s, 0, p));
        STZ_TRY(decode_levels<T>(ctx, s, p, 0, out_dev));
    } else {
        // each batch of streams is decoded while the host zstd-decodes the next
        Trace t("decompress: prepare + decode");
        DecodePipe<T> pipe(ctx, s, p, kdec, out_dev, decode_batches(s->dir, kdec));
        const BatchFn fn = [&](const DecodeBatch& B, cudaEvent_t copied) { return pipe.batch(B, copied); };
        STZ_TRY(prepare(ctx, s, kdec, p, &fn));
    }
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    if (level_error_take()) STZ_FAIL(STZ_ERR_CUDA, "level kernel: a TMA tile load did not complete in time");
    if (stream_learned(s->dir) && learned_tc_error_take(ctx->st))
        STZ_FAIL(STZ_ERR_CUDA, "learned correction: a tensor-core MMA did not complete in time");
    return STZ_OK;
}

// Box / slice: base levels in full, low and high levels only on the
// planner's chunks.
template <typename T>
stz_status decompress_box_dev(stz_context* ctx, stz_stream* s, const int64_t lo[3], const int64_t hi[3], T* out_dev,
                              size_t odims[3])
{
    Lap lap("box");
    const ParsedStream& ps = s->dir;
    const FileHeader& h = ps.h;
    const int K = h.K;
    const QueryPlan plan = plan_query(h.nx, h.ny, h.nz, h.chunk_high, h.chunk_low, lo, hi);
    lap.mark("plan");
    if (odims) {
        odims[0] = (size_t)(plan.q[0].e - plan.q[0].b + 1);
        odims[1] = (size_t)(plan.q[1].e - plan.q[1].b + 1);
        odims[2] = (size_t)(plan.q[2].e - plan.q[2].b + 1);
    }
    if (h.predictor >= STZ_PRED_STAGED) {
        // The ROI cell kernels carry the one-pass predictors only, and a
        // staged block also needs its siblings' decoded values up to two
        // coarse points outside the box, whose codes can lie in chunks the
        // planner does not pick: decode the field, then copy the box out (as
        // a decoder without chunk markers does, src/stz-rd.cpp:591-596).
        STZ_CUDA(ctx->staged_full.ensure((size_t)h.nx * h.ny * h.nz * sizeof(T)));
        STZ_TRY(decompress_level_dev<T>(ctx, s, 0, ctx->staged_full.as<T>()));
        const size_t ox = (size_t)(plan.q[0].e - plan.q[0].b + 1), oy = (size_t)(plan.q[1].e - plan.q[1].b + 1),
                     oz = (size_t)(plan.q[2].e - plan.q[2].b + 1);
        cudaMemcpy3DParms cp{};
        cp.srcPtr = make_cudaPitchedPtr(ctx->staged_full.p, (size_t)h.nx * sizeof(T), (size_t)h.nx, (size_t)h.ny);
        cp.srcPos = make_cudaPos((size_t)plan.q[0].b * sizeof(T), (size_t)plan.q[1].b, (size_t)plan.q[2].b);
        cp.dstPtr = make_cudaPitchedPtr(out_dev, ox * sizeof(T), ox, oy);
        cp.extent = make_cudaExtent(ox * sizeof(T), oy, oz);
        cp.kind = cudaMemcpyDeviceToDevice;
        STZ_CUDA(cudaMemcpy3DAsync(&cp, ctx->st));
        STZ_CUDA(cudaStreamSynchronize(ctx->st));
        return STZ_OK;
    }
    Prepared local;
    Prepared* p = s->resident.get();
    if (!p || p->kmax < K) {
        ctx->borrow(local);
        STZ_TRY(prepare(ctx, s, K, local));
        p = &local;
    }
    const size_t elem = sizeof(T);
    // decoded base (the reference decodes the whole base per query, FD5:2645-2648)
    const LevelGeom low = level_geom(ps, K - 1), high = level_geom(ps, K);
    const size_t nbase = low.n;
    if (!p->base_valid) {
        STZ_CUDA(p->base->ensure(nbase * elem));
        STZ_TRY(decode_levels<T>(ctx, s, *p, K - 2, p->base->as<T>()));
        p->base_valid = true;
    }
    // Mid-grid window: the planner's reference regions; with a learned
    // correction on the finest level, also the full -1..+2 stencil of every
    // query cell, and then the low chunks of the whole window in all blocks.
    const bool learned_high = ps.lv[K].lflags != 0;
    int m0[3], m1[3];
    const bool have_mid = mid_window(plan, low.dx * 2, low.dy * 2, low.dz * 2, learned_high, m0, m1);
    // entropy-decode the planned chunks of the low and high levels
    std::vector<CtaWork> work;
    std::vector<uint32_t> ids;
    std::vector<UnpredWork> uw;
    if (learned_high) {
        std::vector<int64_t> wc;
        if (have_mid) {
            const int nc[3] = {low.ncx, low.ncy, low.ncz};
            window_chunks(m0, m1, low.C, nc, wc);
        }
        std::vector<uint32_t> cs(wc.begin(), wc.end());
        for (int b = 0; b < 7 && !cs.empty(); ++b) {
            const uint32_t si = (uint32_t)((K - 2) * 7 + b);
            add_work(work, ids, si, cs.data(), cs.size(), low.C);
            add_unpred_work(*p, si, cs.data(), cs.size(), uw);
        }
    } else {
        for (const BlockPlan& bp : plan.low) {
            const uint32_t si = (uint32_t)((K - 2) * 7 + bp.block);
            std::vector<uint32_t> cs(bp.chunks.begin(), bp.chunks.end());
            add_work(work, ids, si, cs.data(), cs.size(), low.C);
            add_unpred_work(*p, si, cs.data(), cs.size(), uw);
        }
    }
    for (const BlockPlan& bp : plan.high) {
        const uint32_t si = (uint32_t)((K - 1) * 7 + bp.block);
        std::vector<uint32_t> cs(bp.chunks.begin(), bp.chunks.end());
        add_work(work, ids, si, cs.data(), cs.size(), high.C);
        add_unpred_work(*p, si, cs.data(), cs.size(), uw);
    }
    lap.mark("work lists");
    // ROI jobs: the mid grid on the bounding box of the reference regions,
    // then the query box
    STZ_CUDA(ctx->mid.ensure(8 * nbase * elem));
    std::vector<RoiJob> mj, rj;
    if (have_mid) {
        const int o0[3] = {0, 0, 0};
        mj.push_back(cells_job(m0, m1, ctx->mid.p, o0, 2 * (uint64_t)low.dx, 4 * (uint64_t)low.dx * low.dy, 0));
    }
    const int w0[3] = {plan.q[0].b, plan.q[1].b, plan.q[2].b}, w1[3] = {plan.q[0].e, plan.q[1].e, plan.q[2].e};
    const uint64_t ex = (uint64_t)(w1[0] - w0[0] + 1), ey = (uint64_t)(w1[1] - w0[1] + 1);
    rj.push_back(cells_job(w0, w1, out_dev, w0, ex, ex * ey, 0));
    // one record (work lists + job lists), one copy, one synchronization
    BatchHdr hd{};
    hd.n_work = (uint32_t)work.size(), hd.n_uwork = (uint32_t)uw.size();
    hd.n_mid = (uint32_t)mj.size(), hd.n_req = (uint32_t)rj.size();
    hd.mid_total = mj.empty() ? 0 : job_units(mj[0]);
    hd.req_total = job_units(rj[0]);
    size_t off = align256(sizeof(BatchHdr));
    hd.o_work = (uint32_t)off;
    off = align256(off + work.size() * sizeof(CtaWork));
    hd.o_ids = (uint32_t)off;
    off = align256(off + ids.size() * 4);
    hd.o_uwork = (uint32_t)off;
    off = align256(off + uw.size() * sizeof(UnpredWork));
    hd.o_mid = (uint32_t)off;
    off = align256(off + mj.size() * sizeof(RoiJob));
    hd.o_req = (uint32_t)off;
    off = align256(off + rj.size() * sizeof(RoiJob));
    STZ_CUDA(ctx->h_meta.ensure(off));
    uint8_t* hm = ctx->h_meta.as<uint8_t>();
    std::memcpy(hm, &hd, sizeof hd);
    if (!work.empty()) std::memcpy(hm + hd.o_work, work.data(), work.size() * sizeof(CtaWork));
    if (!ids.empty()) std::memcpy(hm + hd.o_ids, ids.data(), ids.size() * 4);
    if (!uw.empty()) std::memcpy(hm + hd.o_uwork, uw.data(), uw.size() * sizeof(UnpredWork));
    if (!mj.empty()) std::memcpy(hm + hd.o_mid, mj.data(), mj.size() * sizeof(RoiJob));
    std::memcpy(hm + hd.o_req, rj.data(), rj.size() * sizeof(RoiJob));
    STZ_CUDA(ctx->work.ensure(off));
    STZ_CUDA(cudaMemcpyAsync(ctx->work.p, hm, off, cudaMemcpyHostToDevice, ctx->st));
    lap.mark("record + copy");
    const uint8_t* dm = ctx->work.as<uint8_t>();
    STZ_CUDA(ctx->codes.ensure(p->total_codes * 2));
    if (p->total_unpred) STZ_CUDA(ctx->unpred_dense.ensure(p->total_codes * sizeof(T)));
    if (!work.empty()) {
        KScope ks(ctx, "k_decode");
        launch_decode((const CtaWork*)(dm + hd.o_work), (const uint32_t*)(dm + hd.o_ids), (int)work.size(), p->d_sd,
                      p->d_sym, p->d_tables, p->d_sub, p->d_choff, p->d_payload, ctx->codes.as<uint16_t>(), ctx->st);
    }
    if (!uw.empty()) {
        KScope ks(ctx, "k_unpred_move");
        launch_unpred_move<T>(false, (const UnpredWork*)(dm + hd.o_uwork), (int)uw.size(), p->d_sd,
                              ctx->codes.as<uint16_t>(), ctx->unpred_dense.as<T>(), (T*)p->d_ulist, ctx->st);
    }
    const T* ud = p->total_unpred ? ctx->unpred_dense.as<T>() : nullptr;
    const uint64_t lo_off = p->sd[(size_t)(K - 2) * 7].code_off, hi_off = p->sd[(size_t)(K - 1) * 7].code_off;
    auto blocks = [](uint64_t n) { return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 16)); };
    if (hd.mid_total) {
        KScope ks(ctx, "k_roi_cells[low]");
        launch_roi_cells<T>(blocks(hd.mid_total), 256, dm, 0, p->base->as<T>(), low, p->base->as<T>(), low,
                            qparams(ps, K - 1), h.predictor, ctx->codes.as<uint16_t>() + lo_off,
                            ud ? ud + lo_off : nullptr, ctx->st, learned_args<T>(ps, K - 1, p->d_models));
    }
    {
        KScope ks(ctx, "k_roi_cells[high]");
        launch_roi_cells<T>(blocks(hd.req_total), 256, dm, 1, ctx->mid.as<T>(), high, p->base->as<T>(), low,
                            qparams(ps, K), h.predictor, ctx->codes.as<uint16_t>() + hi_off,
                            ud ? ud + hi_off : nullptr, ctx->st, learned_args<T>(ps, K, p->d_models));
    }
    STZ_CUDA(cudaGetLastError());
    lap.mark("launches");
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    lap.mark("device");
    return STZ_OK;
}

size_t dtype_size(int dtype) { return dtype == STZ_F64 ? 8 : 4; }

stz_status enter(stz_context* ctx)
{
    if (!ctx) STZ_FAIL(STZ_ERR_ARG, "context is null");
    g_err.clear();
    STZ_CUDA(cudaSetDevice(ctx->device));
    return STZ_OK;
}

template stz_status decode_chunks<float>(stz_context*, const Prepared&, const std::vector<CtaWork>&,
                                         const std::vector<uint32_t>&, const std::vector<UnpredWork>&);
template stz_status decode_chunks<double>(stz_context*, const Prepared&, const std::vector<CtaWork>&,
                                          const std::vector<uint32_t>&, const std::vector<UnpredWork>&);
template stz_status decode_levels<float>(stz_context*, const stz_stream*, const Prepared&, int, float*);
template stz_status decode_levels<double>(stz_context*, const stz_stream*, const Prepared&, int, double*);

}  // namespace stz

using namespace stz;

extern "C" {

void stz_default_opts(stz_opts* o)
{
    if (!o) return;
    o->eb = 1e-3;
    o->eb_mode = STZ_EB_REL;
    o->bound_mode = STZ_BOUND_POINTWISE;
    o->mult_base = 0.7;
    o->mult_low = 2.7;
    o->mult_high = 8.2;
    o->radius = 32768;
    o->chunk_high = 32;
    o->chunk_low = 16;
    o->zstd_level = 3;
    o->predictor = STZ_PRED_DYNAMIC;
    o->threads = 0;
    o->model = nullptr;
    o->learned_flags = -1;
}

const char* stz_status_string(stz_status s)
{
    switch (s) {
    case STZ_OK: return "ok";
    case STZ_ERR_ARG: return "invalid argument";
    case STZ_ERR_DIMS: return "unsupported dimensions";
    case STZ_ERR_CUDA: return "CUDA error";
    case STZ_ERR_NOMEM: return "out of memory";
    case STZ_ERR_FORMAT: return "invalid stream";
    case STZ_ERR_ZSTD: return "zstd error";
    case STZ_ERR_RANGE: return "out of range";
    case STZ_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

const char* stz_last_error(void) { return g_err.c_str(); }

stz_status stz_context_create(int device, stz_context** out)
{
    g_err.clear();
    if (!out) STZ_FAIL(STZ_ERR_ARG, "out is null");
    int n = 0;
    STZ_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) STZ_FAIL(STZ_ERR_ARG, "no such CUDA device");
    STZ_CUDA(cudaSetDevice(device));
    auto* c = new (std::nothrow) stz_context();
    if (!c) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st_side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st_dec, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (c->st) cudaStreamDestroy(c->st);
        if (c->st_copy) cudaStreamDestroy(c->st_copy);
        if (c->st_side) cudaStreamDestroy(c->st_side);
        if (c->st_dec) cudaStreamDestroy(c->st_dec);
        if (c->ev_fork) cudaEventDestroy(c->ev_fork);
        delete c;
        STZ_FAIL(STZ_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    c->pool.reset(new ThreadPool(pool_threads(0)));
    e = level_error_init();
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->st);
        cudaStreamDestroy(c->st_copy);
        cudaStreamDestroy(c->st_side);
        cudaStreamDestroy(c->st_dec);
        cudaEventDestroy(c->ev_fork);
        cudaEventDestroy(c->ev_join);
        delete c;
        STZ_FAIL(STZ_ERR_CUDA, std::string("level error word: ") + cudaGetErrorString(e));
    }
    *out = c;
    return STZ_OK;
}

void stz_context_destroy(stz_context* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->st);
    cudaStreamSynchronize(ctx->st_copy);
    cudaStreamSynchronize(ctx->st_side);
    cudaStreamSynchronize(ctx->st_dec);
    cudaStreamDestroy(ctx->st_dec);
    cudaStreamDestroy(ctx->st);
    cudaStreamDestroy(ctx->st_copy);
    cudaStreamDestroy(ctx->st_side);
    cudaEventDestroy(ctx->ev_fork);
    cudaEventDestroy(ctx->ev_join);
    delete ctx;
}

stz_status stz_context_sync(stz_context* ctx)
{
    STZ_TRY(enter(ctx));
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    return STZ_OK;
}

stz_status stz_context_stream(stz_context* ctx, void** stream)
{
    if (!ctx || !stream) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *stream = (void*)ctx->st;
    return STZ_OK;
}

stz_status stz_profile_enable(stz_context* ctx, int on)
{
    STZ_TRY(enter(ctx));
    ctx->flush_prof();
    ctx->prof_on = on != 0;
    return STZ_OK;
}

stz_status stz_profile_reset(stz_context* ctx)
{
    STZ_TRY(enter(ctx));
    ctx->flush_prof();
    std::fill(ctx->prof_ms.begin(), ctx->prof_ms.end(), 0.0);
    std::fill(ctx->prof_launches.begin(), ctx->prof_launches.end(), 0);
    return STZ_OK;
}

stz_status stz_profile_count(stz_context* ctx, int* n)
{
    STZ_TRY(enter(ctx));
    if (!n) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    ctx->flush_prof();
    *n = (int)ctx->prof_names.size();
    return STZ_OK;
}

stz_status stz_profile_entry(stz_context* ctx, int i, const char** name, double* total_ms, uint64_t* launches)
{
    STZ_TRY(enter(ctx));
    ctx->flush_prof();
    if (i < 0 || i >= (int)ctx->prof_names.size()) STZ_FAIL(STZ_ERR_RANGE, "no such profile entry");
    if (name) *name = ctx->prof_names[i].c_str();
    if (total_ms) *total_ms = ctx->prof_ms[i];
    if (launches) *launches = ctx->prof_launches[i];
    return STZ_OK;
}

stz_status stz_compress_dev(stz_context* ctx, const void* field, stz_dtype dtype, size_t nx, size_t ny, size_t nz,
                            const stz_opts* opts, stz_stream** out)
{
    STZ_TRY(enter(ctx));
    if (!field || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (dtype != STZ_F32 && dtype != STZ_F64) STZ_FAIL(STZ_ERR_ARG, "bad dtype");
    STZ_TRY(check_opts(opts));
    const std::string dm = validate_dims((long long)nx, (long long)ny, (long long)nz, opts->chunk_high, opts->chunk_low);
    if (!dm.empty()) STZ_FAIL(STZ_ERR_DIMS, dm);
    if ((uintptr_t)field % 16) STZ_FAIL(STZ_ERR_ARG, "device field must be 16-byte aligned");
    if (dtype == STZ_F32)
        return compress_impl<float>(ctx, (const float*)field, (int)nx, (int)ny, (int)nz, *opts, out);
    return compress_impl<double>(ctx, (const double*)field, (int)nx, (int)ny, (int)nz, *opts, out);
}

stz_status stz_compress(stz_context* ctx, const void* field, stz_dtype dtype, size_t nx, size_t ny, size_t nz,
                        const stz_opts* opts, stz_stream** out)
{
    STZ_TRY(enter(ctx));
    if (!field || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (dtype != STZ_F32 && dtype != STZ_F64) STZ_FAIL(STZ_ERR_ARG, "bad dtype");
    STZ_TRY(check_opts(opts));
    const std::string dm = validate_dims((long long)nx, (long long)ny, (long long)nz, opts->chunk_high, opts->chunk_low);
    if (!dm.empty()) STZ_FAIL(STZ_ERR_DIMS, dm);
    const size_t bytes = nx * ny * nz * dtype_size(dtype);
    STZ_CUDA(ctx->field.ensure(bytes));
    STZ_TRY(copy_from_host(ctx, ctx->field.p, field, bytes));
    return stz_compress_dev(ctx, ctx->field.p, dtype, nx, ny, nz, opts, out);
}

stz_status stz_decompress_level_dev(stz_context* ctx, const stz_stream* s, int level, void* out, size_t od[3])
{
    STZ_TRY(enter(ctx));
    if (!s || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const FileHeader& h = s->dir.h;
    if (level < 0 || level > h.K) STZ_FAIL(STZ_ERR_RANGE, "level out of range");
    if ((uintptr_t)out % 16) STZ_FAIL(STZ_ERR_ARG, "device output must be 16-byte aligned");
    if (od) od[0] = (size_t)(h.nx >> level), od[1] = (size_t)(h.ny >> level), od[2] = (size_t)(h.nz >> level);
    if (h.dtype == 1) return decompress_level_dev<double>(ctx, s, level, (double*)out);
    return decompress_level_dev<float>(ctx, s, level, (float*)out);
}

stz_status stz_decompress_level(stz_context* ctx, const stz_stream* s, int level, void* out, size_t od[3])
{
    STZ_TRY(enter(ctx));
    if (!s || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const FileHeader& h = s->dir.h;
    if (level < 0 || level > h.K) STZ_FAIL(STZ_ERR_RANGE, "level out of range");
    const size_t n = (size_t)(h.nx >> level) * (h.ny >> level) * (h.nz >> level) * h.elem();
    STZ_CUDA(ctx->out.ensure(n));
    STZ_TRY(stz_decompress_level_dev(ctx, s, level, ctx->out.p, od));
    return copy_to_host(ctx, out, ctx->out.p, n);
}

stz_status stz_decompress_full_dev(stz_context* ctx, const stz_stream* s, void* out)
{
    return stz_decompress_level_dev(ctx, s, 0, out, nullptr);
}

stz_status stz_decompress_full(stz_context* ctx, const stz_stream* s, void* out)
{
    return stz_decompress_level(ctx, s, 0, out, nullptr);
}

stz_status stz_decompress_box_dev(stz_context* ctx, const stz_stream* s, const int64_t lo[3], const int64_t hi[3],
                                  void* out, size_t od[3])
{
    STZ_TRY(enter(ctx));
    if (!s || !lo || !hi || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    stz_stream* ms = const_cast<stz_stream*>(s);  // only the cached decoded base changes
    if (s->dir.h.dtype == 1) return decompress_box_dev<double>(ctx, ms, lo, hi, (double*)out, od);
    return decompress_box_dev<float>(ctx, ms, lo, hi, (float*)out, od);
}

stz_status stz_decompress_box(stz_context* ctx, const stz_stream* s, const int64_t lo[3], const int64_t hi[3],
                              void* out, size_t od[3])
{
    STZ_TRY(enter(ctx));
    if (!s || !lo || !hi || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const FileHeader& h = s->dir.h;
    const QueryPlan plan = plan_query(h.nx, h.ny, h.nz, h.chunk_high, h.chunk_low, lo, hi);
    const size_t n = (size_t)(plan.q[0].e - plan.q[0].b + 1) * (plan.q[1].e - plan.q[1].b + 1) *
                     (plan.q[2].e - plan.q[2].b + 1) * h.elem();
    STZ_CUDA(ctx->out.ensure(n));
    STZ_TRY(stz_decompress_box_dev(ctx, s, lo, hi, ctx->out.p, od));
    return copy_to_host(ctx, out, ctx->out.p, n);
}

stz_status stz_stream_bytes(const stz_stream* s, const void** data, size_t* size)
{
    if (!s || !data || !size) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *data = s->bytes.data();
    *size = s->bytes.size();
    return STZ_OK;
}

stz_status stz_stream_parse(stz_context* ctx, const void* data, size_t size, stz_stream** out)
{
    (void)ctx;
    g_err.clear();
    if (!data || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    auto* s = new (std::nothrow) stz_stream();
    if (!s) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    s->bytes.assign((const uint8_t*)data, (const uint8_t*)data + size);
    const std::string e = parse_stream(s->bytes.data(), s->bytes.size(), s->dir);
    if (!e.empty()) {
        delete s;
        STZ_FAIL(STZ_ERR_FORMAT, e);
    }
    for (int k = 1; k <= s->dir.h.K; ++k)
        for (int b = 0; b < 7; ++b)
            for (uint64_t v : s->dir.lv[k].s[b].lr) s->raw_payload_bytes += v;
    *out = s;
    return STZ_OK;
}

stz_status stz_stream_info(const stz_stream* s, stz_info* info)
{
    if (!s || !info) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const FileHeader& h = s->dir.h;
    info->dtype = h.dtype;
    info->predictor = h.predictor;
    info->nx = (size_t)h.nx, info->ny = (size_t)h.ny, info->nz = (size_t)h.nz;
    info->n_levels = h.K;
    info->radius = h.radius;
    info->chunk_high = h.chunk_high, info->chunk_low = h.chunk_low;
    info->eb = h.eb;
    info->mult_base = h.mult_base, info->mult_low = h.mult_low, info->mult_high = h.mult_high;
    info->max_error = h.eb * std::max({h.mult_base, h.mult_low, h.mult_high});
    info->stream_bytes = s->bytes.size();
    info->raw_payload_bytes = s->raw_payload_bytes;
    info->learned_flags = 0;
    if (h.K >= 2) info->learned_flags |= (int)s->dir.lv[h.K - 1].lflags;
    if (h.K >= 1) info->learned_flags |= (int)s->dir.lv[h.K].lflags << 8;
    return STZ_OK;
}

stz_status stz_stream_upload(stz_context* ctx, stz_stream* s)
{
    STZ_TRY(enter(ctx));
    if (!s) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    std::unique_ptr<Prepared> p(new Prepared());
    STZ_TRY(prepare(ctx, s, s->dir.h.K, *p));
    s->resident = std::move(p);
    return STZ_OK;
}

void stz_stream_free(stz_stream* s) { delete s; }

// ---- learned correction models ------------------------------------------------
stz_status stz_model_parse(const void* data, size_t size, stz_model** out)
{
    if (!data || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *out = nullptr;
    const uint8_t* b = (const uint8_t*)data;
    if (size < 12 || std::memcmp(b, "STZLMDL1", 8) != 0) STZ_FAIL(STZ_ERR_FORMAT, "not an STZ model file");
    uint32_t mask;
    std::memcpy(&mask, b + 8, 4);
    if (mask == 0 || mask > 3) STZ_FAIL(STZ_ERR_FORMAT, "model mask must be 1, 2 or 3");
    const size_t nrec = (size_t)(mask & 1u) + (mask >> 1 & 1u);
    if (size != 12 + nrec * sizeof(LearnedModel)) STZ_FAIL(STZ_ERR_FORMAT, "model file size does not match its mask");
    auto* m = new (std::nothrow) stz_model();
    if (!m) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    m->mask = mask;
    size_t off = 12;
    for (int i = 0; i < 2; ++i)
        if (mask >> i & 1u) {
            std::memcpy(&m->lv[i], b + off, sizeof(LearnedModel));
            off += sizeof(LearnedModel);
            if (!learned_model_valid(m->lv[i])) {
                delete m;
                STZ_FAIL(STZ_ERR_FORMAT, "bad learned model record");
            }
        }
    m->serialize();
    *out = m;
    return STZ_OK;
}

stz_status stz_model_bytes(const stz_model* m, const void** data, size_t* size)
{
    if (!m || !data || !size) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *data = m->bytes.data();
    *size = m->bytes.size();
    return STZ_OK;
}

void stz_model_free(stz_model* m) { delete m; }

// ---- reference function boundary ------------------------------------------------
stz_status stz_split_dev(stz_context* ctx, stz_dtype dtype, const void* full, size_t nx, size_t ny, size_t nz,
                         void* subs)
{
    STZ_TRY(enter(ctx));
    if (!full || !subs) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (nx % 2 || ny % 2 || nz % 2 || !nx || !ny || !nz) STZ_FAIL(STZ_ERR_DIMS, "dims must be even and positive");
    if ((uintptr_t)full % 16) STZ_FAIL(STZ_ERR_ARG, "full must be 16-byte aligned");
    KScope ks(ctx, "k_split");
    if (dtype == STZ_F64) launch_split<double>((const double*)full, (int)nx, (int)ny, (int)nz, (double*)subs, ctx->st);
    else launch_split<float>((const float*)full, (int)nx, (int)ny, (int)nz, (float*)subs, ctx->st);
    STZ_CUDA(cudaGetLastError());
    return STZ_OK;
}

stz_status stz_merge_dev(stz_context* ctx, stz_dtype dtype, const void* subs, size_t hx, size_t hy, size_t hz,
                         void* full)
{
    STZ_TRY(enter(ctx));
    if (!full || !subs) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (!hx || !hy || !hz) STZ_FAIL(STZ_ERR_DIMS, "dims must be positive");
    if ((uintptr_t)full % 16) STZ_FAIL(STZ_ERR_ARG, "full must be 16-byte aligned");
    KScope ks(ctx, "k_merge");
    if (dtype == STZ_F64) launch_merge<double>((const double*)subs, (int)hx, (int)hy, (int)hz, (double*)full, ctx->st);
    else launch_merge<float>((const float*)subs, (int)hx, (int)hy, (int)hz, (float*)full, ctx->st);
    STZ_CUDA(cudaGetLastError());
    return STZ_OK;
}

static stz_status block_op(stz_context* ctx, int mode, stz_dtype dtype, int predictor, int block, const void* src,
                           const void* ref, void* dst, int dx, int dy, int dz, int x0, int x1, int y0, int y1, int z0,
                           int z1)
{
    STZ_TRY(enter(ctx));
    if (!src || !ref || !dst) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (block < 0 || block > 6) STZ_FAIL(STZ_ERR_RANGE, "block must be in [0, 6]");
    if (predictor != 0 && predictor != 1) STZ_FAIL(STZ_ERR_ARG, "bad predictor");
    if (dx <= 0 || dy <= 0 || dz <= 0) STZ_FAIL(STZ_ERR_DIMS, "dims must be positive");
    x0 = std::max(0, x0), y0 = std::max(0, y0), z0 = std::max(0, z0);
    x1 = std::min(dx, x1), y1 = std::min(dy, y1), z1 = std::min(dz, z1);
    if (x0 >= x1 || y0 >= y1 || z0 >= z1) return STZ_OK;
    KScope ks(ctx, "k_block_op");
    if (dtype == STZ_F64)
        launch_block_op<double>(mode, predictor, block, (const double*)src, (const double*)ref, (double*)dst, dx, dy, dz,
                                x0, x1, y0, y1, z0, z1, ctx->st);
    else
        launch_block_op<float>(mode, predictor, block, (const float*)src, (const float*)ref, (float*)dst, dx, dy, dz, x0,
                               x1, y0, y1, z0, z1, ctx->st);
    STZ_CUDA(cudaGetLastError());
    return STZ_OK;
}

static stz_status block_staged(stz_context* ctx, int mode, stz_dtype dtype, int block, const void* src,
                               const void* const refs[6], void* dst, size_t dx, size_t dy, size_t dz)
{
    STZ_TRY(enter(ctx));
    if (!src || !refs || !dst) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (dtype != STZ_F32 && dtype != STZ_F64) STZ_FAIL(STZ_ERR_ARG, "bad dtype");
    if (block < 0 || block > 6) STZ_FAIL(STZ_ERR_RANGE, "block must be in [0, 6]");
    if (!dx || !dy || !dz) STZ_FAIL(STZ_ERR_DIMS, "dims must be positive");
    if (dx > INT32_MAX || dy > INT32_MAX || dz > INT32_MAX || dx * dy > (size_t(1) << 40) / dz)
        STZ_FAIL(STZ_ERR_DIMS, "dims too large");
    // the refs each block's lines read (ref_x, ref_y, ref_z, ref_xy, ref_xz,
    // ref_yz; blocks 0, 1, 3: the coarse sub-block 0 in refs[0])
    static const unsigned kNeeds[7] = {0x01, 0x01, 0x03, 0x01, 0x05, 0x06, 0x38};
    for (int k = 0; k < 6; ++k)
        if ((kNeeds[block] >> k & 1u) && !refs[k]) STZ_FAIL(STZ_ERR_ARG, "a reference sub-block this block reads is null");
    KScope ks(ctx, "k_block_staged");
    if (dtype == STZ_F64)
        launch_block_staged<double>(mode, block, (const double*)src, refs, (double*)dst, (int)dx, (int)dy, (int)dz,
                                    ctx->st);
    else
        launch_block_staged<float>(mode, block, (const float*)src, refs, (float*)dst, (int)dx, (int)dy, (int)dz,
                                   ctx->st);
    STZ_CUDA(cudaGetLastError());
    return STZ_OK;
}

stz_status stz_preprocess_block_staged_dev(stz_context* ctx, stz_dtype dtype, int block, const void* sub,
                                           const void* const refs[6], void* diff, size_t dx, size_t dy, size_t dz)
{
    return block_staged(ctx, 0, dtype, block, sub, refs, diff, dx, dy, dz);
}

stz_status stz_depreprocess_block_staged_dev(stz_context* ctx, stz_dtype dtype, int block, const void* de,
                                             const void* const refs[6], void* out, size_t dx, size_t dy, size_t dz)
{
    return block_staged(ctx, 1, dtype, block, de, refs, out, dx, dy, dz);
}

stz_status stz_preprocess_block_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* sub,
                                    const void* ref, void* diff, int dx, int dy, int dz, int z0, int z1)
{
    return block_op(ctx, 0, dtype, predictor, block, sub, ref, diff, dx, dy, dz, 0, dx, 0, dy, z0, z1);
}

stz_status stz_depreprocess_block_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* de,
                                      const void* ref, void* out, int dx, int dy, int dz, int z0, int z1)
{
    return block_op(ctx, 1, dtype, predictor, block, de, ref, out, dx, dy, dz, 0, dx, 0, dy, z0, z1);
}

stz_status stz_depreprocess_block_to_full_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block,
                                              const void* de, const void* ref, void* full, int dx, int dy, int dz,
                                              int z0, int z1)
{
    return block_op(ctx, 2, dtype, predictor, block, de, ref, full, dx, dy, dz, 0, dx, 0, dy, z0, z1);
}

stz_status stz_depreprocess_block_roi_dev(stz_context* ctx, stz_dtype dtype, int predictor, int block, const void* de,
                                          const void* ref, void* out, int dx, int dy, int dz, int end_x, int end_y,
                                          int end_z, int start_x, int start_y, int start_z)
{
    // roi end < 0 means "to the end of the axis" (FD5:984-986)
    if (end_x < 0) end_x = dx;
    if (end_y < 0) end_y = dy;
    if (end_z < 0) end_z = dz;
    return block_op(ctx, 1, dtype, predictor, block, de, ref, out, dx, dy, dz, start_x, end_x, start_y, end_y, start_z,
                    end_z);
}

stz_status stz_quantize_dev(stz_context* ctx, stz_dtype dtype, const void* data, size_t n, double eb, int radius,
                            int32_t* q, void* unpred, size_t* n_unpred)
{
    STZ_TRY(enter(ctx));
    if ((!data || !q || !unpred || !n_unpred) && n) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (!(eb > 0) || radius < 1 || radius > (1 << 30)) STZ_FAIL(STZ_ERR_ARG, "bad eb or radius");
    if (n_unpred) *n_unpred = 0;
    if (!n) return STZ_OK;
    const size_t tiles = (n + 1023) / 1024;
    STZ_CUDA(ctx->tiles.ensure(align256(tiles * 4) + (tiles + 1) * 8));
    uint32_t* cnt = ctx->tiles.as<uint32_t>();
    uint64_t* off = (uint64_t*)(ctx->tiles.as<uint8_t>() + align256(tiles * 4));
    const QuantParams qp = make_quant_params(eb, radius);
    {
        KScope ks(ctx, "k_quantize", 3);
        if (dtype == STZ_F64) launch_quantize<double>((const double*)data, n, qp, q, (double*)unpred, cnt, off, ctx->st);
        else launch_quantize<float>((const float*)data, n, qp, q, (float*)unpred, cnt, off, ctx->st);
    }
    STZ_CUDA(cudaGetLastError());
    uint64_t total = 0;
    STZ_CUDA(cudaMemcpyAsync(&total, off + tiles, 8, cudaMemcpyDeviceToHost, ctx->st));
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    *n_unpred = (size_t)total;
    return STZ_OK;
}

stz_status stz_dequantize_dev(stz_context* ctx, stz_dtype dtype, const int32_t* q, size_t n, double eb, int radius,
                              const void* unpred, void* out)
{
    STZ_TRY(enter(ctx));
    if ((!q || !out) && n) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (!(eb > 0) || radius < 1 || radius > (1 << 30)) STZ_FAIL(STZ_ERR_ARG, "bad eb or radius");
    if (!n) return STZ_OK;
    const size_t tiles = (n + 1023) / 1024;
    STZ_CUDA(ctx->tiles.ensure(align256(tiles * 4) + (tiles + 1) * 8));
    uint32_t* cnt = ctx->tiles.as<uint32_t>();
    uint64_t* off = (uint64_t*)(ctx->tiles.as<uint8_t>() + align256(tiles * 4));
    const QuantParams qp = make_quant_params(eb, radius);
    KScope ks(ctx, "k_dequantize", 3);
    if (dtype == STZ_F64) launch_dequantize<double>(q, n, qp, (const double*)unpred, (double*)out, cnt, off, ctx->st);
    else launch_dequantize<float>(q, n, qp, (const float*)unpred, (float*)out, cnt, off, ctx->st);
    STZ_CUDA(cudaGetLastError());
    return STZ_OK;
}

stz_status stz_plan_box(size_t nx, size_t ny, size_t nz, int chunk_high, int chunk_low, const int64_t a[3],
                        const int64_t b[3], int64_t* out, size_t cap, size_t* n_out)
{
    g_err.clear();
    if (!a || !b || !n_out || (!out && cap)) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const std::string dm = validate_dims((long long)nx, (long long)ny, (long long)nz, chunk_high, chunk_low);
    if (!dm.empty()) STZ_FAIL(STZ_ERR_DIMS, dm);
    const QueryPlan p = plan_query((int)nx, (int)ny, (int)nz, chunk_high, chunk_low, a, b);
    std::vector<int64_t> flat;
    flatten_plan(p, flat);
    *n_out = flat.size();
    if (flat.size() > cap) STZ_FAIL(STZ_ERR_RANGE, "output capacity too small");
    std::memcpy(out, flat.data(), flat.size() * 8);
    return STZ_OK;
}

stz_status stz_debug_quant_table(double eb, int radius, float* entries, float* r2, int* on)
{
    g_err.clear();
    if (!entries || !r2 || !on) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (!(eb > 0) || radius < 1) STZ_FAIL(STZ_ERR_ARG, "bad eb or radius");
    const QuantTable t = make_quant_table(make_quant_params(eb, radius));
    for (int h = 0; h < kQuantTableH; ++h) {
        entries[4 * h] = t.e[h].x, entries[4 * h + 1] = t.e[h].y;
        entries[4 * h + 2] = t.e[h].z, entries[4 * h + 3] = t.e[h].w;
    }
    *r2 = t.r2;
    *on = t.on;
    return STZ_OK;
}

stz_status stz_debug_codebook(const uint32_t* hist, int nbins, uint16_t* sym, uint8_t* len, int* n_used)
{
    g_err.clear();
    if (!hist || !sym || !len || !n_used || nbins <= 0 || nbins > 65536) STZ_FAIL(STZ_ERR_ARG, "bad arguments");
    std::vector<uint16_t> s;
    std::vector<uint8_t> l;
    const int n = build_codebook(hist, nbins, 0, s, l);
    std::memcpy(sym, s.data(), 2 * (size_t)n);
    std::memcpy(len, l.data(), (size_t)n);
    *n_used = n;
    return STZ_OK;
}

stz_status stz_debug_run_slots(const uint32_t* hist, int nbins, int plane, uint32_t* run_base, uint32_t* run_n)
{
    g_err.clear();
    if (!hist || !run_base || !run_n || nbins <= 0 || nbins > 65536 || plane < 1) STZ_FAIL(STZ_ERR_ARG, "bad arguments");
    *run_n = (uint32_t)run_slots([&](uint32_t c) -> uint64_t { return hist[c]; }, nbins, plane, *run_base);
    return STZ_OK;
}

stz_status stz_debug_stream_codes(stz_context* ctx, const stz_stream* s, int k, int block, uint16_t* codes, size_t cap,
                                  size_t* n_out)
{
    STZ_TRY(enter(ctx));
    if (!s || !codes || !n_out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const int K = s->dir.h.K;
    if (k < 1 || k > K || block < 0 || block > 6) STZ_FAIL(STZ_ERR_RANGE, "level or block out of range");
    const LevelDir& L = s->dir.lv[k];
    const size_t n = (size_t)L.dx * L.dy * L.dz;
    *n_out = n;
    if (n > cap) STZ_FAIL(STZ_ERR_RANGE, "output capacity too small");
    Prepared p;
    ctx->borrow(p);
    STZ_TRY(prepare(ctx, s, k, p));
    const uint32_t si = (uint32_t)((k - 1) * 7 + block);
    std::vector<CtaWork> work;
    std::vector<uint32_t> ids;
    std::vector<uint32_t> all(p.sd[si].nchunks);
    for (uint32_t c = 0; c < all.size(); ++c) all[c] = c;
    add_work(work, ids, si, all.data(), all.size(), (int)p.sd[si].C);
    std::vector<UnpredWork> none;
    STZ_TRY(decode_chunks<float>(ctx, p, work, ids, none));
    STZ_CUDA(cudaMemcpy(codes, ctx->codes.as<uint16_t>() + p.sd[si].code_off, n * 2, cudaMemcpyDeviceToHost));
    return STZ_OK;
}

}  // extern "C"
