// Host runtime shared by the C ABI (api.cu) and the request server
// (server.cu): device/pinned buffers, the context, the parsed stream object,
// kernel accounting, and the decode pipeline stages.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "host.h"
#include "huffman.h"
#include "trace.h"
#include "stz/stz.h"
#include "stz_internal.h"

#define STZ_FAIL(code, msg)            \
    do {                               \
        ::stz::set_last_error((msg));  \
        return (code);                 \
    } while (0)

#define STZ_CUDA(x)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) {                                                            \
            ::stz::set_last_error(std::string(#x) + ": " + cudaGetErrorString(e_));        \
            return e_ == cudaErrorMemoryAllocation ? STZ_ERR_NOMEM : STZ_ERR_CUDA;          \
        }                                                                                   \
    } while (0)

#define STZ_TRY(x)                   \
    do {                             \
        stz_status s_ = (x);         \
        if (s_ != STZ_OK) return s_; \
    } while (0)

namespace stz {

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t b = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) cap = b;
        else p = nullptr;
        return e;
    }
    template <class T>
    T* as() const
    {
        return (T*)p;
    }
};

// Grow-only pinned host buffer.
struct PinBuf {
    void* p = nullptr;
    size_t cap = 0;
    PinBuf() = default;
    PinBuf(const PinBuf&) = delete;
    PinBuf& operator=(const PinBuf&) = delete;
    ~PinBuf()
    {
        if (p) cudaFreeHost(p);
    }
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t b = std::max<size_t>(bytes, 4096);
        cudaError_t e = cudaHostAlloc(&p, b, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = b;
        else p = nullptr;
        return e;
    }
    template <class T>
    T* as() const
    {
        return (T*)p;
    }
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device-resident decode inputs of levels 1..kmax of one stream object.
struct Prepared {
    int kmax = 0;
    std::vector<StreamDesc> sd;
    std::vector<StreamHeader> hdr;
    std::vector<std::vector<uint64_t>> unpred_prefix;  // per stream, per chunk: list offset
    std::vector<uint64_t> ulist_off;                   // per stream: element offset in the unpred list
    uint64_t total_codes = 0, total_unpred = 0;
    // device buffers: owned by a resident stream, borrowed from the context
    // for one-off decodes (no allocation per call)
    DevBuf own_stage, own_coarsest, own_base;
    DevBuf* stage = &own_stage;
    DevBuf* coarsest = &own_coarsest;
    DevBuf* base = &own_base;
    StreamDesc* d_sd = nullptr;
    uint16_t* d_sym = nullptr;
    uint8_t* d_len = nullptr;
    uint32_t* d_sub = nullptr;
    uint64_t* d_choff = nullptr;
    uint8_t* d_ulist = nullptr;
    uint32_t* d_payload = nullptr;
    LearnedModel* d_models = nullptr;  // per level k (index k), when the stream has learned corrections
    void* d_tables = nullptr;          // decode tables per stream (launch_build_tables)
    bool base_valid = false;  // *base holds the decoded base grid (level K-2 output) for box queries
};

// Where the level kernels evaluate the learned network: block-wide on the
// tensor cores (default) or per thread with dp4a (STZ_LEARNED_PATH=dp4a);
// both give the same integers.
inline bool learned_tensor_cores()
{
    const char* e = std::getenv("STZ_LEARNED_PATH");
    return !(e && std::string(e) == "dp4a");
}

// Learned-correction arguments of level k (none when the level has no flags).
template <typename T>
LearnedArgs<T> learned_args(const ParsedStream& ps, int k, const LearnedModel* d_models)
{
    LearnedArgs<T> a;
    a.tensor_cores = learned_tensor_cores();
    const LevelDir& L = ps.lv[k];
    if (!L.lflags || !d_models) return a;
    a.model = d_models + k;
    a.flags = L.lflags;
    a.rs = (T)(1.0 / (L.eb * L.model.s_in));
    a.so = (T)(L.model.s_out * L.eb);
    return a;
}

// Any level of the stream carries a learned correction.
inline bool stream_learned(const ParsedStream& ps)
{
    for (size_t k = 1; k < ps.lv.size(); ++k)
        if (ps.lv[k].lflags) return true;
    return false;
}

// Shape of the hierarchy for given dims and options.
struct Geometry {
    int nx = 0, ny = 0, nz = 0, K = 0, radius = 0, chunk_high = 0, chunk_low = 0;
    int c0[3] = {0, 0, 0};
    std::vector<LevelGeom> lv;  // 1..K
    std::vector<StreamDesc> sd; // stream (k-1)*7+b
    uint64_t total_codes = 0, total_chunk_slots = 0, total_sub = 0, total_words = 0;
    size_t n_fine_max = 0;      // largest intermediate decoded grid (elements)
};
Geometry make_geometry(int nx, int ny, int nz, int chunk_high, int chunk_low, int radius);

// Absolute eb the level multipliers apply to (value range on the GPU for a
// relative bound, pointwise slack) and the per-level bounds ebk[1..K].
template <typename T>
stz_status level_error_bounds(stz_context* ctx, const T* field, size_t N, const stz_opts& o, int K, double& eb,
                              std::vector<double>& ebk);

// CTA work items for chunk lists: groups of up to kCoderThreads / C chunks.
void add_work(std::vector<CtaWork>& work, std::vector<uint32_t>& ids, uint32_t stream, const uint32_t* chunks,
              size_t n, int C);
void add_all_chunks(std::vector<CtaWork>& work, std::vector<uint32_t>& ids, uint32_t stream, uint32_t nchunks, int C);

}  // namespace stz

struct stz_context {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaStream_t st_copy = nullptr;  // payload host->device copies of decode preparation
    cudaStream_t st_side = nullptr;  // boundary-shell kernels of level launches (SideStream)
    cudaStream_t st_dec = nullptr;   // entropy decoding of full decodes, beside the level decodes
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    stz::SideStream side() const { return stz::SideStream{st_side, ev_fork, ev_join}; }
    std::unique_ptr<stz::ThreadPool> pool;
    // kernel profiling (stz_profile_*)
    struct ProfRec {
        const char* name;
        cudaEvent_t a, b;
    };
    bool prof_on = false;
    std::vector<ProfRec> pending;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::string> prof_names;
    std::vector<double> prof_ms;
    std::vector<uint64_t> prof_launches;
    size_t prof_slot(const char* name)
    {
        for (size_t i = 0; i < prof_names.size(); ++i)
            if (prof_names[i] == name) return i;
        prof_names.emplace_back(name);
        prof_ms.push_back(0.0);
        prof_launches.push_back(0);
        return prof_names.size() - 1;
    }
    cudaEvent_t event()
    {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void flush_prof()
    {
        // STZ_TIMELINE: every bracketed launch of this flush with its start and
        // end relative to the first one's start (events of all the context's
        // streams share the device clock).
        static const bool timeline = std::getenv("STZ_TIMELINE") != nullptr;
        if (timeline && !pending.empty() && cudaEventSynchronize(pending.back().b) == cudaSuccess)
            for (auto& r : pending) {
                float t0 = 0.f, t1 = 0.f;
                if (cudaEventSynchronize(r.b) == cudaSuccess &&
                    cudaEventElapsedTime(&t0, pending[0].a, r.a) == cudaSuccess &&
                    cudaEventElapsedTime(&t1, pending[0].a, r.b) == cudaSuccess)
                    std::fprintf(stderr, "[stz] timeline %-28s %9.4f %9.4f %8.4f\n", r.name, t0, t1, t1 - t0);
            }
        for (auto& r : pending) {
            float ms = 0.f;
            if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess)
                prof_ms[prof_slot(r.name)] += ms;
            ev_pool.push_back(r.a);
            ev_pool.push_back(r.b);
        }
        pending.clear();
    }
    ~stz_context()
    {
        flush_prof();
        for (auto e : ev_pool) cudaEventDestroy(e);
    }
    stz::DevBuf field, grid[2], codes, unpred_dense, unpred_cnt, hist, hist_out, ctab, sub_bits, sub_off, chunk_off,
        stream_words, payload, sd, work, ids, uwork, ulist, cb_sym, cb_len, minmax, packed, rbits, out, mid, boxes,
        tiles, models, eval, rstats, gwork, staged_full;
    stz::PinBuf h_hist, h_meta, h_meta2, h_payload, h_stage, h_io, h_small, h_rstats, h_fullh;
    stz::PinBuf h_xfer[2];  // staging chunks of host <-> device copies of pageable caller buffers
    // device buffers lent to one-off decodes
    stz::DevBuf p_stage, p_coarsest, p_base;
    void borrow(stz::Prepared& p)
    {
        p.stage = &p_stage;
        p.coarsest = &p_coarsest;
        p.base = &p_base;
    }
};

struct stz_stream {
    stz::Bytes bytes;
    stz::ParsedStream dir;
    size_t raw_payload_bytes = 0;
    std::unique_ptr<stz::Prepared> resident;
};

// Learned models of the second-finest (lv[0]) and finest (lv[1]) levels.
struct stz_model {
    uint32_t mask = 0;  // bit i: lv[i] present
    stz::LearnedModel lv[2]{};
    std::vector<uint8_t> bytes;  // serialized form, kept for stz_model_bytes
    void serialize()
    {
        bytes.assign({'S', 'T', 'Z', 'L', 'M', 'D', 'L', '1'});
        const uint8_t* m = (const uint8_t*)&mask;
        bytes.insert(bytes.end(), m, m + 4);
        for (int i = 0; i < 2; ++i)
            if (mask >> i & 1u) {
                const uint8_t* r = (const uint8_t*)&lv[i];
                bytes.insert(bytes.end(), r, r + sizeof(stz::LearnedModel));
            }
    }
};

namespace stz {

// Counts the launches of one kernel and, when profiling is on, brackets them
// with events on the context's stream.
struct KScope {
    stz_context* c;
    cudaEvent_t b = nullptr;
    cudaStream_t s;
    KScope(stz_context* ctx, const char* name, int launches = 1, cudaStream_t on = nullptr)
        : c(ctx), s(on ? on : ctx->st)
    {
        c->prof_launches[c->prof_slot(name)] += (uint64_t)launches;
        if (c->prof_on) {
            if (c->pending.size() > 4096) c->flush_prof();
            cudaEvent_t a = c->event();
            b = c->event();
            cudaEventRecord(a, s);
            c->pending.push_back({name, a, b});
        }
    }
    ~KScope()
    {
        if (b) cudaEventRecord(b, s);
    }
};

int pool_threads(int requested);
// Host <-> device copies of a caller's host buffer on ctx->st, complete on
// return. A page-locked buffer takes one DMA; a pageable one goes through
// two pinned chunks, the DMA of one chunk overlapping the host pool's copy
// of the other (the driver's own staging of pageable memory is serial).
stz_status copy_to_host(stz_context* ctx, void* dst, const void* src_dev, size_t n);
stz_status copy_from_host(stz_context* ctx, void* dst_dev, const void* src, size_t n);
// Validates compressor options (STZ_ERR_ARG with a message).
stz_status check_opts(const stz_opts* o);
size_t dtype_size(int dtype);
// Make ctx current on this thread and clear the thread's last error.
stz_status enter(stz_context* ctx);
// A batch of the pipelined decode: streams [s0, s1), their chunk z-layers
// [l0, l1) (l1 < 0: every layer).
struct DecodeBatch {
    int s0, s1, l0, l1;
};
// The batches of a decode of levels 1..kmax: every stream of the levels
// below kmax, then the finest level's 7 streams in two halves of their chunk
// z-layers (one batch when they have a single layer).
std::vector<DecodeBatch> decode_batches(const ParsedStream& ps, int kmax);
// Parse stream headers, lay out and upload the tables and payload of levels
// 1..kmax (zstd frames decoded on the host pool) and the coarsest grid.
// on_batch(b, copied), when given, runs for each batch of
// decode_batches(kmax) in order, after the copy of its payload is enqueued;
// `copied` is the event after that copy, and the callback orders its own
// work after it. Without on_batch, ctx->st waits for every copy. prepare
// returns once the context's streams are idle.
using BatchFn = std::function<stz_status(const DecodeBatch&, cudaEvent_t)>;
stz_status prepare(stz_context* ctx, const stz_stream* s, int kmax, Prepared& p, const BatchFn* on_batch = nullptr);
// Entropy-decode the listed chunks into ctx->codes (and scatter their
// unpredictable values into ctx->unpred_dense).
template <typename T>
stz_status decode_chunks(stz_context* ctx, const Prepared& p, const std::vector<CtaWork>& work,
                         const std::vector<uint32_t>& ids, const std::vector<UnpredWork>& uwork);
void add_unpred_work(const Prepared& p, uint32_t s, const uint32_t* chunks, size_t n, std::vector<UnpredWork>& uw);
QuantParams qparams(const ParsedStream& ps, int k);
LevelGeom level_geom(const ParsedStream& ps, int k);
// Reconstruct levels 1..kdec; the last one lands in out_dev.
template <typename T>
stz_status decode_levels(stz_context* ctx, const stz_stream* s, const Prepared& p, int kdec, T* out_dev);

}  // namespace stz
