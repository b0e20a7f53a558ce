// Request server (stz_server_* in stz/stz.h): streams resident in HBM,
// continuous batching of box / slice / progressive-level requests, and a
// batched decode replayed from captured CUDA graphs.
//
// The reference answers one query per process: it plans the query
// (FD5:1578-1839), entropy-decodes the planned marker chunks
// (SZ_decompress_nopred_marked_chunks, FD5:1841-1911), rebuilds the
// half-resolution reference regions from the decoded base (FD5:2507-2538) and
// then the box (FD5:2573-2605). Here the same steps run for a whole batch of
// requests at once:
//   host   : plan every request, take the union of their marker chunks
//            (each chunk decoded once per batch), pack one batch record;
//   device : one H2D copy of the record, then one graph replay per stream:
//            k_decode_dyn (all chunks) -> k_unpred_scatter_dyn ->
//            k_roi_cells (the mid-grid windows) -> k_roi_cells (all outputs).
// Progressive levels >= 2 are strided samples of the resident decoded base
// (the decoded grid of level l+1 is the even-parity sub-grid of level l) and
// ride in the same graph.
//
// Two lanes, each with its own CUDA stream, batch slots and completion
// thread: the fast lane (boxes, slices, levels >= 2) on a high-priority
// stream, and the bulk lane (full decodes of levels 1 and 0, whole-grid
// outputs) on a low-priority stream, so small requests never queue behind a
// full-resolution decode. Both lanes write the stream's shared decode
// buffers (codes, mid grid) only with the values a full decode gives, so
// their overlap cannot change a result.
//
// Admission: a request is taken from the queue when its output fits in the
// output arena and a slot of its lane is free; requests that arrive while
// batches run join the next batch of their lane.
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "levels.h"
#include "roi.h"
#include "runtime.h"

namespace stz {
namespace {

using Clock = std::chrono::steady_clock;
constexpr int kMaxSlots = 8;
constexpr size_t kLogSize = 4096;
constexpr int kLaneFast = 0, kLaneBulk = 1, kLanes = 2;
constexpr int kBulkSlots = 1, kBulkBatch = 8;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// First-fit allocator over [0, cap) in 256-byte units.
class Arena {
public:
    void reset(size_t cap)
    {
        free_.clear();
        cap_ = cap & ~(size_t)255;
        used_ = 0;
        if (cap_) free_[0] = cap_;
    }
    bool alloc(size_t bytes, size_t& off)
    {
        bytes = align256(std::max<size_t>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            off = it->first;
            const size_t rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = align256(std::max<size_t>(bytes, 1));
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t capacity() const { return cap_; }
    size_t used() const { return used_; }
    // An allocation of `bytes` that leaves at least `reserve` bytes unused
    // could be made some day / now.
    bool fits_ever(size_t bytes, size_t reserve = 0) const
    {
        return reserve <= cap_ && align256(std::max<size_t>(bytes, 1)) <= cap_ - reserve;
    }
    bool alloc_leaving(size_t bytes, size_t reserve, size_t& off)
    {
        if (!fits_ever(bytes, reserve) || used_ + align256(std::max<size_t>(bytes, 1)) > cap_ - reserve) return false;
        return alloc(bytes, off);
    }

private:
    std::map<size_t, size_t> free_;
    size_t cap_ = 0, used_ = 0;
};

struct LaunchShape {
    int decode_grid = 148 * 4;
    int unpred_grid = 148 * 2;
    int roi_block = 256;
    int roi_grid = 148 * 8;
};

struct SrvStream {
    int id = 0;
    std::unique_ptr<stz_stream> s;
    Prepared* p = nullptr;
    int K = 0, dtype = 0, predictor = 0;
    size_t elem = 4;
    LevelGeom low, high;
    QuantParams qlow, qhigh;
    uint32_t low_s0 = 0, high_s0 = 0;  // index of block 0 of the low / high level among the streams
    DevBuf codes, unpred, mid;
    std::vector<uint32_t> stamp;  // per chunk of the 14 low/high streams: last batch that listed it
    uint64_t stamp_off[15] = {};
    uint32_t epoch = 0;
    size_t meta_cap = 0;
    DevBuf meta[kLanes][kMaxSlots];          // batch records on the device, per lane and slot
    cudaGraphExec_t graph[kMaxSlots] = {};  // fast-lane batch kernels, per slot
    LaunchShape shape;
    ~SrvStream()
    {
        for (auto g : graph)
            if (g) cudaGraphExecDestroy(g);
    }
    const StreamDesc& sd(uint32_t i) const { return p->sd[i]; }
    const uint16_t* low_codes() const { return codes.as<uint16_t>() + sd(low_s0).code_off; }
    const uint16_t* high_codes() const { return codes.as<uint16_t>() + sd(high_s0).code_off; }
    template <typename T>
    const T* low_unpred() const
    {
        return p->total_unpred ? unpred.as<T>() + sd(low_s0).code_off : nullptr;
    }
    template <typename T>
    const T* high_unpred() const
    {
        return p->total_unpred ? unpred.as<T>() + sd(high_s0).code_off : nullptr;
    }
};

struct Ticket {
    stz_request req{};
    SrvStream* ss = nullptr;
    int lane = kLaneFast;
    int state = 0;  // 0 queued, 1 in a batch, 2 done
    stz_status status = STZ_OK;
    std::string error;
    size_t off = 0, bytes = 0;
    size_t dims[3] = {0, 0, 0};
    Clock::time_point t_submit, t_launch, t_done;
    uint64_t batch = 0;
    int batch_size = 0;
};

// A level request's full decodes (bulk lane).
struct LevelJob {
    SrvStream* ss;
    int level;  // 0 or 1
    void* out;
};

// Host-side record of one batch for one stream.
struct Build {
    std::vector<uint32_t> lists[14];
    std::vector<CtaWork> work;
    std::vector<uint32_t> ids;
    std::vector<UnpredWork> uw;
    std::vector<RoiJob> mid;  // low-level cells: mid-grid windows
    std::vector<RoiJob> req;  // high-level cells of boxes, base samples of coarse levels
    uint64_t mid_total = 0, req_total = 0;
    std::vector<LevelJob> jobs;
};

// A launched batch waiting for its end event.
struct InFlight {
    int slot;
    uint64_t batch;
    std::vector<uint64_t> ids;
};

// One lane: a CUDA stream, its batch slots (pinned record buffers, events
// bracketing each batch's GPU work) and the batches in flight on it.
struct Lane {
    cudaStream_t st = nullptr;
    int slots = 0;
    bool busy[kMaxSlots] = {};
    PinBuf hmeta[kMaxSlots];
    cudaEvent_t ev_a[kMaxSlots] = {}, ev_b[kMaxSlots] = {};
    std::deque<InFlight> inflight;
    std::condition_variable cv;
    std::thread completer;
    int free_slot() const
    {
        for (int k = 0; k < slots; ++k)
            if (!busy[k]) return k;
        return -1;
    }
};

}  // namespace
}  // namespace stz

using namespace stz;

struct stz_server {
    stz_context* ctx = nullptr;
    stz_server_opts opts{};
    DevBuf arena_buf;
    Arena arena;
    std::mutex mu;  // queue, tickets, lane slots and in-flight lists, arena, stats
    std::condition_variable cv_work, cv_done;
    std::list<uint64_t> queue;
    std::unordered_map<uint64_t, Ticket> tickets;
    uint64_t next_ticket = 1;
    std::vector<std::unique_ptr<SrvStream>> streams;
    Lane lanes[kLanes];
    std::mutex exec_mu;  // GPU submission (worker batches vs stream upload / capture)
    std::thread worker;  // admits, plans and launches batches
    bool stop = false, stop_completers = false;
    uint64_t submitted = 0, completed = 0, batches = 0;
    LaunchShape last_shape;
    // batch history (ring)
    Clock::time_point t0 = Clock::now();
    std::vector<stz_batch_record> log = std::vector<stz_batch_record>(kLogSize);
    double ms_now() const { return ms_between(t0, Clock::now()); }
    stz_batch_record& rec(uint64_t batch) { return log[batch % kLogSize]; }
};

namespace stz {
namespace {

// Completion thread of one lane: its batches finish in launch order (one
// CUDA stream), so it waits on the oldest batch's end event, then publishes
// its results and frees its slot. (A host-function callback in the stream
// would hold back the next batch's kernels until the driver ran it.)
void completer_main(stz_server* S, int lane)
{
    cudaSetDevice(S->ctx->device);
    Lane& L = S->lanes[lane];
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        L.cv.wait(lk, [&]() { return S->stop_completers || !L.inflight.empty(); });
        if (L.inflight.empty()) break;  // stopping, nothing left in flight
        const int slot = L.inflight.front().slot;
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(L.ev_b[slot]);
        float ms = -1.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, L.ev_a[slot], L.ev_b[slot]);
        // a bulk-lane level decode whose TMA tile load gave up (the word is
        // process-wide; the batch that sees it fails)
        const bool tile_err = e == cudaSuccess && lane == kLaneBulk && level_error_take();
        lk.lock();
        InFlight f = std::move(L.inflight.front());
        L.inflight.pop_front();
        const auto now = Clock::now();
        stz_batch_record& r = S->rec(f.batch);
        r.t_done_ms = ms_between(S->t0, now);
        r.device_ms = ms;
        for (uint64_t id : f.ids) {
            auto it = S->tickets.find(id);
            if (it == S->tickets.end()) continue;
            Ticket& t = it->second;
            if (e != cudaSuccess || tile_err) {
                S->arena.release(t.off, t.bytes);
                t.status = STZ_ERR_CUDA;
                t.error = tile_err ? std::string("batch failed on the device: a TMA tile load did not complete in time")
                                   : std::string("batch failed on the device: ") + cudaGetErrorString(e);
            }
            t.state = 2;
            t.t_done = now;
        }
        L.busy[f.slot] = false;
        S->completed += f.ids.size();
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

uint32_t chunk_count(const SrvStream& ss, int j) { return ss.sd(j < 7 ? ss.low_s0 + j : ss.high_s0 + j - 7).nchunks; }

void list_chunk(SrvStream& ss, Build& b, int j, uint32_t c)
{
    uint32_t& st = ss.stamp[ss.stamp_off[j] + c];
    if (st == ss.epoch) return;
    st = ss.epoch;
    b.lists[j].push_back(c);
}

void list_all(SrvStream& ss, Build& b, int j0, int j1)
{
    for (int j = j0; j < j1; ++j) {
        const uint32_t n = chunk_count(ss, j);
        for (uint32_t c = 0; c < n; ++c) list_chunk(ss, b, j, c);
    }
}

// Plan one request into the batch record.
void plan_request(SrvStream& ss, Build& b, const Ticket& t, void* out)
{
    const FileHeader& h = ss.s->dir.h;
    const stz_request& r = t.req;
    if (r.kind == STZ_REQ_BOX) {
        const QueryPlan plan = plan_query(h.nx, h.ny, h.nz, h.chunk_high, h.chunk_low, r.lo, r.hi);
        for (const BlockPlan& bp : plan.high)
            for (int64_t c : bp.chunks) list_chunk(ss, b, 7 + bp.block, (uint32_t)c);
        int m0[3], m1[3];
        const bool learned_high = ss.s->dir.lv[ss.K].lflags != 0;
        if (mid_window(plan, 2 * ss.low.dx, 2 * ss.low.dy, 2 * ss.low.dz, learned_high, m0, m1)) {
            // The mid grid is rebuilt on the regions' bounding box (grown to
            // the learned stencil of every query cell when the finest level
            // has a learned correction): decode the low chunks of every cell
            // of that box (a superset of the planner's low chunks,
            // FD5:1784-1830), so every mid value written is the full decode's
            // value.
            const int C = ss.low.C;
            const int c0[3] = {(m0[0] >> 1) / C, (m0[1] >> 1) / C, (m0[2] >> 1) / C};
            const int c1[3] = {(m1[0] >> 1) / C, (m1[1] >> 1) / C, (m1[2] >> 1) / C};
            for (int blk = 0; blk < 7; ++blk)
                for (int cz = c0[2]; cz <= c1[2]; ++cz)
                    for (int cy = c0[1]; cy <= c1[1]; ++cy)
                        for (int cx = c0[0]; cx <= c1[0]; ++cx)
                            list_chunk(ss, b, blk, (uint32_t)((cz * ss.low.ncy + cy) * ss.low.ncx + cx));
            const int o0[3] = {0, 0, 0};
            b.mid.push_back(cells_job(m0, m1, ss.mid.p, o0, 2 * (uint64_t)ss.low.dx,
                                      4 * (uint64_t)ss.low.dx * ss.low.dy, b.mid_total));
            b.mid_total += job_units(b.mid.back());
        }
        const int w0[3] = {plan.q[0].b, plan.q[1].b, plan.q[2].b}, w1[3] = {plan.q[0].e, plan.q[1].e, plan.q[2].e};
        b.req.push_back(cells_job(w0, w1, out, w0, t.dims[0], (uint64_t)t.dims[0] * t.dims[1], b.req_total));
        b.req_total += job_units(b.req.back());
        return;
    }
    if (r.level >= 2) {
        RoiJob j{};
        j.ncx = (int)t.dims[0], j.ncy = (int)t.dims[1], j.ncz = (int)t.dims[2];
        j.kind = kJobSample;
        j.shift = r.level - 2;
        j.osx = t.dims[0], j.osy = (uint64_t)t.dims[0] * t.dims[1];
        j.start = b.req_total;
        j.out = (uint64_t)(uintptr_t)out;
        b.req.push_back(j);
        b.req_total += job_units(j);
        return;
    }
    list_all(ss, b, 0, 7);
    if (r.level == 0) list_all(ss, b, 7, 14);
    b.jobs.push_back({&ss, r.level, out});
}

// Work lists and the packed record (header + arrays) in host memory.
size_t pack(SrvStream& ss, Build& b, uint8_t* dst)
{
    for (int j = 0; j < 14; ++j) {
        if (b.lists[j].empty()) continue;
        const uint32_t si = j < 7 ? ss.low_s0 + j : ss.high_s0 + j - 7;
        std::sort(b.lists[j].begin(), b.lists[j].end());
        add_work(b.work, b.ids, si, b.lists[j].data(), b.lists[j].size(), (int)ss.sd(si).C);
        add_unpred_work(*ss.p, si, b.lists[j].data(), b.lists[j].size(), b.uw);
    }
    BatchHdr h{};
    h.n_work = (uint32_t)b.work.size();
    h.n_uwork = (uint32_t)b.uw.size();
    h.n_mid = (uint32_t)b.mid.size();
    h.n_req = (uint32_t)b.req.size();
    h.mid_total = b.mid_total;
    h.req_total = b.req_total;
    size_t off = align16(sizeof(BatchHdr));
    h.o_work = (uint32_t)off;
    off = align16(off + b.work.size() * sizeof(CtaWork));
    h.o_ids = (uint32_t)off;
    off = align16(off + b.ids.size() * 4);
    h.o_uwork = (uint32_t)off;
    off = align16(off + b.uw.size() * sizeof(UnpredWork));
    h.o_mid = (uint32_t)off;
    off = align16(off + b.mid.size() * sizeof(RoiJob));
    h.o_req = (uint32_t)off;
    off = align16(off + b.req.size() * sizeof(RoiJob));
    if (off > ss.meta_cap) return 0;
    std::memcpy(dst, &h, sizeof h);
    if (!b.work.empty()) std::memcpy(dst + h.o_work, b.work.data(), b.work.size() * sizeof(CtaWork));
    if (!b.ids.empty()) std::memcpy(dst + h.o_ids, b.ids.data(), b.ids.size() * 4);
    if (!b.uw.empty()) std::memcpy(dst + h.o_uwork, b.uw.data(), b.uw.size() * sizeof(UnpredWork));
    if (!b.mid.empty()) std::memcpy(dst + h.o_mid, b.mid.data(), b.mid.size() * sizeof(RoiJob));
    if (!b.req.empty()) std::memcpy(dst + h.o_req, b.req.data(), b.req.size() * sizeof(RoiJob));
    return off;
}

// The batch kernels of one stream on the context's stream (captured into the
// slot graphs, and run directly by the autotuner).
template <typename T>
void enqueue_kernels(const SrvStream& ss, const LaunchShape& sh, const uint8_t* meta, cudaStream_t st)
{
    const Prepared& p = *ss.p;
    uint16_t* codes = ss.codes.as<uint16_t>();
    launch_decode_dyn(sh.decode_grid, meta, p.d_sd, p.d_sym, p.d_tables, p.d_sub, p.d_choff, p.d_payload, codes, st);
    if (p.total_unpred)
        launch_unpred_scatter_dyn<T>(sh.unpred_grid, meta, p.d_sd, codes, ss.unpred.as<T>(), (T*)p.d_ulist, st);
    const T* base = p.base->as<T>();
    const ParsedStream& ps = ss.s->dir;
    launch_roi_cells<T>(sh.roi_grid, sh.roi_block, meta, 0, base, ss.low, base, ss.low, ss.qlow, ss.predictor,
                        ss.low_codes(), ss.low_unpred<T>(), st, learned_args<T>(ps, ss.K - 1, p.d_models));
    launch_roi_cells<T>(sh.roi_grid, sh.roi_block, meta, 1, ss.mid.as<T>(), ss.high, base, ss.low, ss.qhigh,
                        ss.predictor, ss.high_codes(), ss.high_unpred<T>(), st, learned_args<T>(ps, ss.K, p.d_models));
}

template <typename T>
void enqueue_level_job(const SrvStream& ss, const LevelJob& j, cudaStream_t st)
{
    LevelDecodeArgs<T> a;
    a.coarse = ss.p->base->as<T>();
    a.geo = ss.low;
    a.predictor = ss.predictor;
    a.qp = ss.qlow;
    a.codes = ss.low_codes();
    a.unpred_dense = ss.low_unpred<T>();
    a.out = j.level == 1 ? (T*)j.out : ss.mid.as<T>();
    a.learned = learned_args<T>(ss.s->dir, ss.K - 1, ss.p->d_models);
    launch_level_decode<T>(a, st);
    if (j.level == 1) return;
    a.coarse = ss.mid.as<T>();
    a.geo = ss.high;
    a.qp = ss.qhigh;
    a.codes = ss.high_codes();
    a.unpred_dense = ss.high_unpred<T>();
    a.out = (T*)j.out;
    a.learned = learned_args<T>(ss.s->dir, ss.K, ss.p->d_models);
    launch_level_decode<T>(a, st);
}

stz_status capture_graphs(stz_server* S, SrvStream& ss)
{
    cudaStream_t st = S->ctx->st;
    for (int k = 0; k < S->opts.slots; ++k) {
        if (ss.graph[k]) {
            cudaGraphExecDestroy(ss.graph[k]);
            ss.graph[k] = nullptr;
        }
        const uint8_t* meta = ss.meta[kLaneFast][k].as<uint8_t>();
        STZ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        if (ss.dtype == 1) enqueue_kernels<double>(ss, ss.shape, meta, st);
        else enqueue_kernels<float>(ss, ss.shape, meta, st);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            STZ_FAIL(STZ_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        }
        const cudaError_t e2 = cudaGraphInstantiate(&ss.graph[k], g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) STZ_FAIL(STZ_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    }
    return STZ_OK;
}

// Time the batch kernels on a synthetic batch of 16 boxes (edge 64, clipped
// to the field) for each candidate shape and keep the fastest.
stz_status autotune(stz_server* S, SrvStream& ss)
{
    cudaStream_t st = S->ctx->st;
    const FileHeader& h = ss.s->dir.h;
    Build b;
    ++ss.epoch;
    std::vector<Ticket> tk(16);
    uint64_t seed = 0x9e3779b97f4a7c15ull;
    auto rnd = [&](int n) {
        seed = seed * 6364136223846793005ull + 1442695040888963407ull;
        return n > 0 ? (int)((seed >> 33) % (uint64_t)n) : 0;
    };
    size_t out_elems = 0;
    const int dims[3] = {h.nx, h.ny, h.nz};
    for (auto& t : tk) {
        t.req.kind = STZ_REQ_BOX;
        for (int a = 0; a < 3; ++a) {
            const int e = std::min(64, dims[a]);
            t.req.lo[a] = rnd(dims[a] - e + 1);
            t.req.hi[a] = t.req.lo[a] + e - 1;
            t.dims[a] = (size_t)e;
        }
        out_elems += t.dims[0] * t.dims[1] * t.dims[2];
    }
    DevBuf out;
    STZ_CUDA(out.ensure(out_elems * ss.elem));
    size_t o = 0;
    for (auto& t : tk) {
        plan_request(ss, b, t, out.as<uint8_t>() + o * ss.elem);
        o += t.dims[0] * t.dims[1] * t.dims[2];
    }
    PinBuf& hm = S->lanes[kLaneFast].hmeta[0];
    const uint8_t* meta = ss.meta[kLaneFast][0].as<uint8_t>();
    STZ_CUDA(hm.ensure(ss.meta_cap));
    const size_t bytes = pack(ss, b, hm.as<uint8_t>());
    if (!bytes) STZ_FAIL(STZ_ERR_RANGE, "tuning batch exceeds the batch record");
    STZ_CUDA(cudaMemcpyAsync(ss.meta[kLaneFast][0].p, hm.p, bytes, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    STZ_CUDA(cudaEventCreate(&e0));
    STZ_CUDA(cudaEventCreate(&e1));
    auto time_shape = [&](const LaunchShape& sh) -> float {
        float best = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(e0, st);
            if (ss.dtype == 1) enqueue_kernels<double>(ss, sh, meta, st);
            else enqueue_kernels<float>(ss, sh, meta, st);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep) best = std::min(best, ms);  // first run warms up
        }
        return best;
    };
    LaunchShape best = ss.shape;
    float tbest = time_shape(best);
    for (int dg : {148, 148 * 2, 148 * 4, 148 * 8}) {
        LaunchShape c = best;
        c.decode_grid = dg;
        const float t = time_shape(c);
        if (t < tbest) tbest = t, best = c;
    }
    for (int blk : {128, 256})  // k_roi_cells is built for at most 256 threads
        for (int per_sm : {2, 4, 8, 16}) {
            LaunchShape c = best;
            c.roi_block = blk;
            c.roi_grid = 148 * per_sm;
            const float t = time_shape(c);
            if (t < tbest) tbest = t, best = c;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    STZ_CUDA(cudaGetLastError());
    STZ_CUDA(cudaStreamSynchronize(st));
    ss.shape = best;
    return STZ_OK;
}

// Bulk lane: every chunk of the levels the batch's full decodes need, then
// the level decodes (hrec: host copy of the record at drec).
template <typename T>
cudaError_t enqueue_bulk(SrvStream& ss, const uint8_t* hrec, const uint8_t* drec, const std::vector<LevelJob>& jobs,
                         cudaStream_t st)
{
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(hrec);
    const Prepared& p = *ss.p;
    uint16_t* codes = ss.codes.as<uint16_t>();
    if (h->n_work)
        launch_decode(reinterpret_cast<const CtaWork*>(drec + h->o_work),
                      reinterpret_cast<const uint32_t*>(drec + h->o_ids), (int)h->n_work, p.d_sd, p.d_sym, p.d_tables,
                      p.d_sub, p.d_choff, p.d_payload, codes, st);
    if (h->n_uwork)
        launch_unpred_move<T>(false, reinterpret_cast<const UnpredWork*>(drec + h->o_uwork), (int)h->n_uwork, p.d_sd,
                              codes, ss.unpred.as<T>(), (T*)p.d_ulist, st);
    for (const LevelJob& j : jobs) enqueue_level_job<T>(ss, j, st);
    return cudaGetLastError();
}

// Plan, pack and enqueue one batch on a lane (worker thread, exec_mu held).
stz_status launch_batch(stz_server* S, int lane, int slot, uint64_t bid, const std::vector<uint64_t>& ids)
{
    Lane& L = S->lanes[lane];
    cudaStream_t st = L.st;
    // group by stream, keep arrival order inside a group
    std::vector<SrvStream*> order;
    std::unordered_map<SrvStream*, std::vector<Ticket*>> groups;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        const auto now = Clock::now();
        for (uint64_t id : ids) {
            Ticket& t = S->tickets[id];
            t.t_launch = now;
            t.batch = bid;
            t.batch_size = (int)ids.size();
            if (!groups.count(t.ss)) order.push_back(t.ss);
            groups[t.ss].push_back(&t);
        }
        stz_batch_record& r = S->rec(bid);
        r = stz_batch_record{};
        r.batch = bid;
        r.n_requests = (int)ids.size();
        r.slot = slot;
        r.lane = lane;
        r.t_start_ms = ms_between(S->t0, now);
        r.t_planned_ms = r.t_launched_ms = r.t_done_ms = r.device_ms = -1.0;
    }
    uint8_t* arena = S->arena_buf.as<uint8_t>();
    // plan and pack every group into its own region of the slot's pinned buffer
    size_t need = 0;
    for (SrvStream* ss : order) need += align256(ss->meta_cap);
    STZ_CUDA(L.hmeta[slot].ensure(need));
    uint8_t* hbase = L.hmeta[slot].as<uint8_t>();
    std::vector<Build> builds(order.size());
    std::vector<size_t> bytes(order.size()), hoff(order.size());
    size_t off = 0;
    for (size_t g = 0; g < order.size(); ++g) {
        SrvStream* ss = order[g];
        ++ss->epoch;
        if (ss->epoch == 0) {  // wrapped: clear the stamps
            std::fill(ss->stamp.begin(), ss->stamp.end(), 0u);
            ss->epoch = 1;
        }
        for (Ticket* t : groups[ss]) plan_request(*ss, builds[g], *t, arena + t->off);
        hoff[g] = off;
        bytes[g] = pack(*ss, builds[g], hbase + off);
        if (!bytes[g]) STZ_FAIL(STZ_ERR_RANGE, "batch record exceeds its buffer");
        off += align256(ss->meta_cap);
    }
    const double t_planned = S->ms_now();
    STZ_CUDA(cudaEventRecord(L.ev_a[slot], st));
    for (size_t g = 0; g < order.size(); ++g) {
        SrvStream* ss = order[g];
        DevBuf& drec = ss->meta[lane][slot];
        STZ_CUDA(cudaMemcpyAsync(drec.p, hbase + hoff[g], bytes[g], cudaMemcpyHostToDevice, st));
        if (lane == kLaneFast) STZ_CUDA(cudaGraphLaunch(ss->graph[slot], st));
        else if (ss->dtype == 1)
            STZ_CUDA((enqueue_bulk<double>(*ss, hbase + hoff[g], drec.as<uint8_t>(), builds[g].jobs, st)));
        else STZ_CUDA((enqueue_bulk<float>(*ss, hbase + hoff[g], drec.as<uint8_t>(), builds[g].jobs, st)));
    }
    STZ_CUDA(cudaEventRecord(L.ev_b[slot], st));
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->rec(bid).t_planned_ms = t_planned;
        S->rec(bid).t_launched_ms = S->ms_now();
        L.inflight.push_back(InFlight{slot, bid, ids});
    }
    L.cv.notify_one();
    return STZ_OK;
}

// Admit the next batch (mu held): for the first lane with a free slot and a
// queued request, take that lane's requests in arrival order while their
// outputs fit in the arena.
bool admit(stz_server* S, int& lane, int& slot, std::vector<uint64_t>& ids)
{
    for (int ln = 0; ln < kLanes; ++ln) {
        Lane& L = S->lanes[ln];
        const int k = L.free_slot();
        if (k < 0) continue;
        const int cap = ln == kLaneFast ? S->opts.max_batch : kBulkBatch;
        ids.clear();
        for (auto it = S->queue.begin(); it != S->queue.end() && (int)ids.size() < cap;) {
            Ticket& t = S->tickets[*it];
            if (t.lane != ln) {
                ++it;
                continue;
            }
            const size_t reserve = ln == kLaneBulk ? S->opts.fast_reserve : 0;
            if (!S->arena.alloc_leaving(t.bytes, reserve, t.off)) break;  // the lane keeps its arrival order
            t.state = 1;
            ids.push_back(*it);
            it = S->queue.erase(it);
        }
        if (!ids.empty()) {
            lane = ln;
            slot = k;
            return true;
        }
    }
    return false;
}

void worker_main(stz_server* S)
{
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        int lane = 0, slot = -1;
        std::vector<uint64_t> ids;
        S->cv_work.wait(lk, [&]() { return S->stop || admit(S, lane, slot, ids); });
        if (S->stop) break;
        Lane& L = S->lanes[lane];
        L.busy[slot] = true;
        const uint64_t bid = ++S->batches;
        lk.unlock();
        stz_status st;
        std::string err;
        {
            std::lock_guard<std::mutex> ex(S->exec_mu);
            st = launch_batch(S, lane, slot, bid, ids);
            if (st != STZ_OK) err = stz_last_error();
        }
        lk.lock();
        if (st != STZ_OK) {
            // a batch that failed to launch never reached the completion
            // thread: fail its requests and give back the slot (after the
            // lane's stream drains)
            lk.unlock();
            cudaStreamSynchronize(L.st);
            lk.lock();
            const auto now = Clock::now();
            for (uint64_t id : ids) {
                Ticket& t = S->tickets[id];
                S->arena.release(t.off, t.bytes);  // a failed ticket holds no output
                t.state = 2;
                t.status = st;
                t.error = err;
                t.t_done = now;
            }
            L.busy[slot] = false;
            S->completed += ids.size();
            S->cv_done.notify_all();
        }
    }
}

stz_status enter_server(stz_server* S)
{
    if (!S) STZ_FAIL(STZ_ERR_ARG, "server is null");
    STZ_TRY(enter(S->ctx));
    return STZ_OK;
}

template <typename T>
stz_status decode_base(stz_context* ctx, SrvStream& ss)
{
    Prepared& p = *ss.p;
    STZ_CUDA(p.base->ensure(ss.low.n * sizeof(T)));
    STZ_TRY(decode_levels<T>(ctx, ss.s.get(), p, ss.K - 2, p.base->as<T>()));
    STZ_CUDA(cudaStreamSynchronize(ctx->st));
    p.base_valid = true;
    return STZ_OK;
}

}  // namespace
}  // namespace stz

extern "C" {

void stz_server_default_opts(stz_server_opts* o)
{
    if (!o) return;
    o->arena_bytes = (size_t)1 << 30;
    o->max_batch = 64;
    o->slots = 2;
    o->autotune = 1;
    o->threads = 0;
    o->fast_reserve = (size_t)-1;
}

stz_status stz_server_create(int device, const stz_server_opts* opts, stz_server** out)
{
    if (!out) STZ_FAIL(STZ_ERR_ARG, "out is null");
    *out = nullptr;
    stz_server_opts o;
    stz_server_default_opts(&o);
    if (opts) {
        if (opts->arena_bytes) o.arena_bytes = opts->arena_bytes;
        if (opts->max_batch > 0) o.max_batch = opts->max_batch;
        if (opts->slots > 0) o.slots = std::min(opts->slots, kMaxSlots);
        o.autotune = opts->autotune;
        o.threads = opts->threads;
        o.fast_reserve = opts->fast_reserve;
    }
    if (o.fast_reserve == (size_t)-1) o.fast_reserve = o.arena_bytes / 4;
    o.fast_reserve = std::min(o.fast_reserve, o.arena_bytes);
    std::unique_ptr<stz_server> S(new (std::nothrow) stz_server());
    if (!S) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    S->opts = o;
    STZ_TRY(stz_context_create(device, &S->ctx));
    if (o.threads > 0) S->ctx->pool.reset(new ThreadPool(o.threads));
    const cudaError_t e = S->arena_buf.ensure(o.arena_bytes);
    if (e != cudaSuccess) {
        stz_context_destroy(S->ctx);
        STZ_FAIL(STZ_ERR_NOMEM, "output arena allocation failed");
    }
    S->arena.reset(o.arena_bytes);
    // fast lane on the highest stream priority, bulk lane on the lowest
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    bool ok = true;
    for (int ln = 0; ln < kLanes && ok; ++ln) {
        Lane& L = S->lanes[ln];
        L.slots = ln == kLaneFast ? o.slots : kBulkSlots;
        ok = cudaStreamCreateWithPriority(&L.st, cudaStreamNonBlocking, ln == kLaneFast ? greatest : least) ==
             cudaSuccess;
        for (int k = 0; k < L.slots && ok; ++k)
            ok = cudaEventCreate(&L.ev_a[k]) == cudaSuccess && cudaEventCreate(&L.ev_b[k]) == cudaSuccess;
    }
    if (!ok) {
        for (Lane& L : S->lanes) {
            for (int k = 0; k < kMaxSlots; ++k) {
                if (L.ev_a[k]) cudaEventDestroy(L.ev_a[k]);
                if (L.ev_b[k]) cudaEventDestroy(L.ev_b[k]);
            }
            if (L.st) cudaStreamDestroy(L.st);
        }
        stz_context_destroy(S->ctx);
        STZ_FAIL(STZ_ERR_CUDA, "stream or event creation failed");
    }
    stz_server* raw = S.release();
    for (int ln = 0; ln < kLanes; ++ln) raw->lanes[ln].completer = std::thread(completer_main, raw, ln);
    raw->worker = std::thread(worker_main, raw);
    *out = raw;
    return STZ_OK;
}

void stz_server_destroy(stz_server* S)
{
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop_completers = true;  // they still drain the batches in flight
    }
    for (Lane& L : S->lanes) {
        L.cv.notify_all();
        if (L.completer.joinable()) L.completer.join();
    }
    cudaSetDevice(S->ctx->device);
    for (Lane& L : S->lanes) cudaStreamSynchronize(L.st);
    cudaStreamSynchronize(S->ctx->st);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (uint64_t id : S->queue) {
            Ticket& t = S->tickets[id];
            t.state = 2;
            t.status = STZ_ERR_ARG;
            t.error = "server stopped";
        }
        S->queue.clear();
    }
    S->cv_done.notify_all();
    S->streams.clear();
    for (Lane& L : S->lanes) {
        for (int k = 0; k < kMaxSlots; ++k) {
            if (L.ev_a[k]) cudaEventDestroy(L.ev_a[k]);
            if (L.ev_b[k]) cudaEventDestroy(L.ev_b[k]);
        }
        if (L.st) cudaStreamDestroy(L.st);
    }
    stz_context* ctx = S->ctx;
    delete S;
    stz_context_destroy(ctx);
}

stz_status stz_server_add_stream(stz_server* S, const void* data, size_t size, int* stream_id)
{
    STZ_TRY(enter_server(S));
    if (!data || !stream_id) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    std::lock_guard<std::mutex> ex(S->exec_mu);
    STZ_CUDA(cudaStreamSynchronize(S->ctx->st));
    std::unique_ptr<SrvStream> ss(new SrvStream());
    stz_stream* parsed = nullptr;
    STZ_TRY(stz_stream_parse(S->ctx, data, size, &parsed));
    ss->s.reset(parsed);
    const ParsedStream& ps = ss->s->dir;
    const FileHeader& h = ps.h;
    if (h.K < 2) STZ_FAIL(STZ_ERR_DIMS, "stream has fewer than two levels");
    if (h.predictor >= STZ_PRED_STAGED)
        STZ_FAIL(STZ_ERR_UNSUPPORTED,
                 "the server's batched decodes take dynamic and cubic streams, not staged or truncated ones");
    ss->K = h.K;
    ss->dtype = h.dtype;
    ss->elem = h.elem();
    ss->predictor = h.predictor;
    ss->low = level_geom(ps, h.K - 1);
    ss->high = level_geom(ps, h.K);
    ss->qlow = qparams(ps, h.K - 1);
    ss->qhigh = qparams(ps, h.K);
    ss->low_s0 = (uint32_t)(h.K - 2) * 7;
    ss->high_s0 = (uint32_t)(h.K - 1) * 7;
    ss->s->resident.reset(new Prepared());
    ss->p = ss->s->resident.get();
    STZ_TRY(prepare(S->ctx, ss->s.get(), h.K, *ss->p));
    if (h.dtype == 1) STZ_TRY(decode_base<double>(S->ctx, *ss));
    else STZ_TRY(decode_base<float>(S->ctx, *ss));
    const Prepared& p = *ss->p;
    STZ_CUDA(ss->codes.ensure(p.total_codes * 2));
    if (p.total_unpred) STZ_CUDA(ss->unpred.ensure(p.total_codes * ss->elem));
    STZ_CUDA(ss->mid.ensure(8 * ss->low.n * ss->elem));
    // chunk stamps and the batch record capacity
    uint64_t nch = 0;
    for (int j = 0; j < 14; ++j) {
        ss->stamp_off[j] = nch;
        nch += chunk_count(*ss, j);
    }
    ss->stamp_off[14] = nch;
    ss->stamp.assign(nch, 0u);
    ss->meta_cap = align16(sizeof(BatchHdr)) + align16(nch * sizeof(CtaWork)) + align16(nch * 4) +
                   align16(nch * sizeof(UnpredWork)) + 2 * align16((size_t)S->opts.max_batch * sizeof(RoiJob)) +
                   256;
    for (int ln = 0; ln < kLanes; ++ln)
        for (int k = 0; k < S->lanes[ln].slots; ++k) STZ_CUDA(ss->meta[ln][k].ensure(ss->meta_cap));
    if (S->opts.autotune) STZ_TRY(autotune(S, *ss));
    STZ_TRY(capture_graphs(S, *ss));
    STZ_CUDA(cudaStreamSynchronize(S->ctx->st));
    std::lock_guard<std::mutex> lk(S->mu);
    ss->id = (int)S->streams.size();
    S->last_shape = ss->shape;
    *stream_id = ss->id;
    S->streams.push_back(std::move(ss));
    return STZ_OK;
}

stz_status stz_server_submit(stz_server* S, const stz_request* r, uint64_t* ticket)
{
    if (!S || !r || !ticket) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    Ticket t;
    t.req = *r;
    t.t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stop) STZ_FAIL(STZ_ERR_ARG, "server stopped");
        if (r->stream_id < 0 || r->stream_id >= (int)S->streams.size()) STZ_FAIL(STZ_ERR_ARG, "no such stream");
        t.ss = S->streams[r->stream_id].get();
    }
    const FileHeader& h = t.ss->s->dir.h;
    if (r->kind == STZ_REQ_BOX) {
        AxisRange q[3];
        query_box(h.nx, h.ny, h.nz, r->lo, r->hi, q);
        for (int a = 0; a < 3; ++a) t.dims[a] = (size_t)(q[a].e - q[a].b + 1);
    } else if (r->kind == STZ_REQ_LEVEL) {
        if (r->level < 0 || r->level > h.K) STZ_FAIL(STZ_ERR_RANGE, "level out of range");
        t.dims[0] = (size_t)h.nx >> r->level;
        t.dims[1] = (size_t)h.ny >> r->level;
        t.dims[2] = (size_t)h.nz >> r->level;
        if (r->level <= 1) t.lane = kLaneBulk;  // full level decodes
    } else {
        STZ_FAIL(STZ_ERR_ARG, "unknown request kind");
    }
    t.bytes = t.dims[0] * t.dims[1] * t.dims[2] * h.elem();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (!S->arena.fits_ever(t.bytes, t.lane == kLaneBulk ? S->opts.fast_reserve : 0))
            STZ_FAIL(STZ_ERR_NOMEM, "request output exceeds the output arena (less the fast-lane reserve)");
        const uint64_t id = S->next_ticket++;
        S->tickets.emplace(id, std::move(t));
        S->queue.push_back(id);
        ++S->submitted;
        *ticket = id;
    }
    S->cv_work.notify_one();
    return STZ_OK;
}

stz_status stz_server_wait(stz_server* S, uint64_t ticket, double timeout_ms, stz_result* res)
{
    if (!S || !res) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->tickets.find(ticket);
    if (it == S->tickets.end()) STZ_FAIL(STZ_ERR_ARG, "unknown ticket");
    Ticket& t = it->second;
    auto done = [&]() { return t.state == 2; };
    if (timeout_ms < 0) S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done))
        STZ_FAIL(STZ_ERR_RANGE, "timed out");
    res->status = t.status;
    res->out_dev = t.status == STZ_OK ? S->arena_buf.as<uint8_t>() + t.off : nullptr;
    for (int a = 0; a < 3; ++a) res->dims[a] = t.dims[a];
    res->bytes = t.bytes;
    res->queue_ms = ms_between(t.t_submit, t.t_launch);
    res->latency_ms = ms_between(t.t_submit, t.t_done);
    res->batch = t.batch;
    res->batch_size = t.batch_size;
    if (t.status != STZ_OK) set_last_error(t.error);
    return STZ_OK;
}

stz_status stz_server_copy_out(stz_server* S, uint64_t ticket, void* host)
{
    STZ_TRY(enter_server(S));
    if (!host) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    const void* src = nullptr;
    size_t bytes = 0;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->tickets.find(ticket);
        if (it == S->tickets.end()) STZ_FAIL(STZ_ERR_ARG, "unknown ticket");
        if (it->second.state != 2) STZ_FAIL(STZ_ERR_ARG, "request not complete");
        if (it->second.status != STZ_OK) STZ_FAIL(it->second.status, it->second.error);
        src = S->arena_buf.as<uint8_t>() + it->second.off;
        bytes = it->second.bytes;
    }
    STZ_CUDA(cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost));
    return STZ_OK;
}

stz_status stz_server_release(stz_server* S, uint64_t ticket)
{
    if (!S) STZ_FAIL(STZ_ERR_ARG, "server is null");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->tickets.find(ticket);
        if (it == S->tickets.end()) STZ_FAIL(STZ_ERR_ARG, "unknown ticket");
        if (it->second.state != 2) STZ_FAIL(STZ_ERR_ARG, "request not complete");
        if (it->second.status == STZ_OK) S->arena.release(it->second.off, it->second.bytes);
        S->tickets.erase(it);
    }
    S->cv_work.notify_one();
    return STZ_OK;
}

stz_status stz_server_stats_get(stz_server* S, stz_server_stats* st)
{
    if (!S || !st) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    std::lock_guard<std::mutex> lk(S->mu);
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->batches = S->batches;
    st->decode_grid = S->last_shape.decode_grid;
    st->roi_block = S->last_shape.roi_block;
    st->roi_grid = S->last_shape.roi_grid;
    st->arena_bytes = S->arena.capacity();
    st->arena_in_use = S->arena.used();
    return STZ_OK;
}

stz_status stz_server_batch_log(stz_server* S, stz_batch_record* out, size_t cap, size_t* n)
{
    if (!S || !n || (!out && cap)) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    std::lock_guard<std::mutex> lk(S->mu);
    const uint64_t last = S->batches;
    const uint64_t cnt = std::min<uint64_t>({last, (uint64_t)kLogSize, (uint64_t)cap});
    for (uint64_t i = 0; i < cnt; ++i) out[i] = S->rec(last - cnt + 1 + i);
    *n = (size_t)cnt;
    return STZ_OK;
}

}  // extern "C"
