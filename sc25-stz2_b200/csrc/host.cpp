// Host-side pieces of the STZ B200 library (see host.h).
#include "host.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <functional>
#include <memory>
#include <numeric>

#include "stz_internal.h"
#include "trace.h"

// libzstd 1.5.5 is present as a runtime library only; public prototypes (zstd.h).
extern "C" {
typedef struct ZSTD_CCtx_s ZSTD_CCtx;
typedef struct ZSTD_DCtx_s ZSTD_DCtx;
size_t ZSTD_compressBound(size_t srcSize);
unsigned ZSTD_isError(size_t code);
ZSTD_CCtx* ZSTD_createCCtx(void);
size_t ZSTD_freeCCtx(ZSTD_CCtx* cctx);
size_t ZSTD_compressCCtx(ZSTD_CCtx* cctx, void* dst, size_t dstCapacity, const void* src, size_t srcSize,
                         int compressionLevel);
ZSTD_DCtx* ZSTD_createDCtx(void);
size_t ZSTD_freeDCtx(ZSTD_DCtx* dctx);
size_t ZSTD_decompressDCtx(ZSTD_DCtx* dctx, void* dst, size_t dstCapacity, const void* src, size_t srcSize);
}

namespace stz {

namespace {
// One zstd context per host thread, reused across frames (ZSTD_compress /
// ZSTD_decompress build a fresh one per call; the bytes are the same).
struct ZstdContexts {
    ZSTD_CCtx* c = nullptr;
    ZSTD_DCtx* d = nullptr;
    ~ZstdContexts()
    {
        if (c) ZSTD_freeCCtx(c);
        if (d) ZSTD_freeDCtx(d);
    }
};
thread_local ZstdContexts tl_zstd;

size_t zstd_compress(void* dst, size_t cap, const void* src, size_t n, int level)
{
    if (!tl_zstd.c) tl_zstd.c = ZSTD_createCCtx();
    return ZSTD_compressCCtx(tl_zstd.c, dst, cap, src, n, level);
}

size_t zstd_decompress(void* dst, size_t cap, const void* src, size_t n)
{
    if (!tl_zstd.d) tl_zstd.d = ZSTD_createDCtx();
    return ZSTD_decompressDCtx(tl_zstd.d, dst, cap, src, n);
}
}  // namespace

// ---- thread pool ------------------------------------------------------------
ThreadPool::ThreadPool(int threads)
{
    for (int i = 1; i < threads; ++i) workers_.emplace_back([this] { run(); });
}

ThreadPool::~ThreadPool()
{
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
}

// Workers claim items one at a time under the lock and read the job pointer at
// claim time, so a worker can never run an item of a finished job.
void ThreadPool::run()
{
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        cv_.wait(lk, [&] { return stop_ || (job_ != nullptr && next_ < n_); });
        if (stop_) return;
        const std::function<void(size_t)>* job = job_;
        const size_t i = next_++;
        ++active_;
        lk.unlock();
        (*job)(i);
        lk.lock();
        --active_;
        if (next_ >= n_ && active_ == 0) done_cv_.notify_all();
    }
}

void ThreadPool::parallel_for(size_t n, const std::function<void(size_t)>& fn)
{
    if (n == 0) return;
    if (workers_.empty() || n == 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::unique_lock<std::mutex> lk(mu_);
    job_ = &fn;
    n_ = n;
    next_ = 0;
    cv_.notify_all();
    while (next_ < n_) {
        const size_t i = next_++;
        ++active_;
        lk.unlock();
        fn(i);
        lk.lock();
        --active_;
    }
    done_cv_.wait(lk, [&] { return active_ == 0; });
    job_ = nullptr;
}

// ---- codebook -----------------------------------------------------------------
namespace {

// In-place minimum-redundancy code lengths for weights sorted ascending
// (Moffat & Katajainen 1995): parent links left to right, internal depths
// right to left, then leaf depths handed out level by level.
void min_redundancy_lengths(std::vector<uint64_t>& a)
{
    const int n = (int)a.size();
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
    int avail = 1, used = 0, depth = 0, next = n - 1;
    root = n - 2;
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

}  // namespace

int build_codebook(const uint32_t* hist, int nbins, int base, std::vector<uint16_t>& sym, std::vector<uint8_t>& len)
{
    return build_codebook_adjusted(hist, nbins, base, {}, sym, len);
}

int build_codebook_adjusted(const uint32_t* hist, int nbins, int base,
                            const std::vector<std::pair<uint32_t, uint64_t>>& set, std::vector<uint16_t>& sym,
                            std::vector<uint8_t>& len)
{
    struct Item {
        uint64_t w;
        uint32_t s;
    };
    std::vector<Item> items;
    for (int i = 0; i < nbins; ++i)
        if (hist[i]) items.push_back({hist[i], (uint32_t)(i + base)});
    if (!set.empty()) {  // items are in symbol order: replace or append the set's counts
        for (const auto& o : set) {
            auto it = std::lower_bound(items.begin(), items.end(), o.first,
                                       [](const Item& x, uint32_t sym) { return x.s < sym; });
            if (it != items.end() && it->s == o.first) it->w = o.second;
            else items.insert(it, {o.second, o.first});
        }
        items.erase(std::remove_if(items.begin(), items.end(), [](const Item& x) { return x.w == 0; }), items.end());
    }
    const int n = (int)items.size();
    sym.clear();
    len.clear();
    if (n == 0) return 0;
    // (count, symbol) order as one 64-bit key per item (counts stay below
    // 2^48), then (length, symbol) as one 32-bit key: plain integer sorts
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) key[i] = items[i].w << 16 | items[i].s;
    std::sort(key.begin(), key.end());
    std::vector<uint64_t> a(n);
    for (int i = 0; i < n; ++i) a[i] = key[i] >> 16;
    min_redundancy_lengths(a);
    if (n > 1) {
        const uint64_t cap = 1ull << kMaxCodeLen;
        uint64_t kraft = 0;
        for (auto& l : a) {
            l = std::min<uint64_t>(l, kMaxCodeLen);
            kraft += 1ull << (kMaxCodeLen - l);
        }
        int first_short = 0;
        while (kraft > cap) {
            while (a[first_short] >= (uint64_t)kMaxCodeLen) ++first_short;
            kraft -= 1ull << (kMaxCodeLen - a[first_short] - 1);
            ++a[first_short];
        }
    }
    std::vector<uint32_t> ls(n);
    for (int i = 0; i < n; ++i) ls[i] = (uint32_t)a[i] << 16 | (uint32_t)(key[i] & 0xffffu);
    std::sort(ls.begin(), ls.end());
    sym.resize(n);
    len.resize(n);
    for (int i = 0; i < n; ++i) {
        len[i] = (uint8_t)(ls[i] >> 16);
        sym[i] = (uint16_t)(ls[i] & 0xffffu);
    }
    return n;
}

// ---- hierarchy shape -------------------------------------------------------------
int num_levels(int nx, int ny, int nz)
{
    int k = 0;
    while (nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && std::min({nx, ny, nz}) / 2 >= 4) {
        nx /= 2, ny /= 2, nz /= 2;
        ++k;
    }
    return std::max(k, 2);
}

int level_chunk(int nx, int ny, int nz, int K, int k, int chunk_high, int chunk_low)
{
    if (k == K) return chunk_high;
    if (k == K - 1) return chunk_low;
    const int sh = K - k + 1;
    const int dx = nx >> sh, dy = ny >> sh, dz = nz >> sh;
    int c = 16;
    while (c > 1 && (dx % c || dy % c || dz % c)) c >>= 1;
    return c;
}

std::string validate_dims(long long nx, long long ny, long long nz, int chunk_high, int chunk_low)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 4 || ny % 4 || nz % 4)
        return "dims must be positive and divisible by 4, got " + std::to_string(nx) + " x " + std::to_string(ny) +
               " x " + std::to_string(nz);
    if (nx > (1 << 20) || ny > (1 << 20) || nz > (1 << 20) || nx * ny * nz > (1ll << 36))
        return "dims too large";
    if (chunk_high <= 0 || chunk_low <= 0 || chunk_high > 128 || chunk_low > 128)
        return "chunk dims must be in [1, 128]";
    if ((nx / 2) % chunk_high || (ny / 2) % chunk_high || (nz / 2) % chunk_high || (nx / 4) % chunk_low ||
        (ny / 4) % chunk_low || (nz / 4) % chunk_low)
        return "dims " + std::to_string(nx) + " x " + std::to_string(ny) + " x " + std::to_string(nz) +
               " are incompatible with high " + std::to_string(chunk_high) + "^3 and low " +
               std::to_string(chunk_low) + "^3 marker chunks";
    return "";
}

namespace {
struct BlockPool {
    std::mutex mu;
    std::vector<std::pair<void*, size_t>> free_;  // (block, capacity)
    size_t bytes = 0;
};
BlockPool& block_pool()
{
    static BlockPool* p = new BlockPool();  // never destroyed: frees may come from static destructors
    return *p;
}
// blocks below this size use malloc directly
constexpr size_t kPoolMin = (size_t)1 << 20;
constexpr size_t kPoolMaxBlocks = 4;
constexpr size_t kPoolMaxBytes = (size_t)2 << 30;
// header before each pooled block: its capacity (16 bytes keeps alignment)
constexpr size_t kPoolHdr = 16;
}  // namespace

void* pooled_alloc(size_t bytes)
{
    if (bytes < kPoolMin) return std::malloc(bytes ? bytes : 1);
    BlockPool& bp = block_pool();
    {
        std::lock_guard<std::mutex> lk(bp.mu);
        size_t best = SIZE_MAX;
        for (size_t i = 0; i < bp.free_.size(); ++i) {
            const size_t cap = bp.free_[i].second;
            if (cap >= bytes && cap <= 2 * bytes + kPoolMin && (best == SIZE_MAX || cap < bp.free_[best].second)) best = i;
        }
        if (best != SIZE_MAX) {
            void* blk = bp.free_[best].first;
            bp.bytes -= bp.free_[best].second;
            bp.free_.erase(bp.free_.begin() + (long)best);
            return static_cast<uint8_t*>(blk) + kPoolHdr;
        }
    }
    void* blk = std::malloc(bytes + kPoolHdr);
    if (!blk) return nullptr;
    *static_cast<size_t*>(blk) = bytes;
    return static_cast<uint8_t*>(blk) + kPoolHdr;
}

void pooled_free(void* p, size_t bytes)
{
    if (!p) return;
    if (bytes < kPoolMin) {
        std::free(p);
        return;
    }
    void* blk = static_cast<uint8_t*>(p) - kPoolHdr;
    const size_t cap = *static_cast<size_t*>(blk);
    BlockPool& bp = block_pool();
    {
        std::lock_guard<std::mutex> lk(bp.mu);
        if (bp.free_.size() < kPoolMaxBlocks && bp.bytes + cap <= kPoolMaxBytes) {
            bp.free_.push_back({blk, cap});
            bp.bytes += cap;
            return;
        }
    }
    std::free(blk);
}

int run_slots(const std::function<uint64_t(uint32_t)>& count, int nbins, int plane, uint32_t& run_base)
{
    const int J = (int)run_slot_count((uint32_t)plane);
    run_base = 0;
    if (J == 0) return 0;
    for (int u0 = nbins - J; u0 >= 1; --u0) {
        bool free_ = true;
        for (int j = 0; j < J && free_; ++j) free_ = count((uint32_t)(u0 + j)) == 0;
        if (free_) {
            run_base = (uint32_t)u0;
            return J;
        }
    }
    return 0;
}

// ---- container ------------------------------------------------------------------
bool learned_model_valid(const LearnedModel& m)
{
    return std::isfinite(m.s_in) && m.s_in > 0 && std::isfinite(m.s_out) && m.s_out > 0 && m.sh1 >= 1 &&
           m.sh1 <= 62 && m.sh2 >= 1 && m.sh2 <= 62;
}

namespace {

const char kMagic[8] = {'S', 'T', 'Z', 'B', '2', '0', '0', 0};

struct Writer {
    std::vector<uint8_t>& b;
    void put(const void* p, size_t n)
    {
        const uint8_t* c = (const uint8_t*)p;
        b.insert(b.end(), c, c + n);
    }
    void u8(uint8_t v) { put(&v, 1); }
    void u32(uint32_t v) { put(&v, 4); }
    void i32(int32_t v) { put(&v, 4); }
    void u64(uint64_t v) { put(&v, 8); }
    void f64(double v) { put(&v, 8); }
};

struct Reader {
    const uint8_t* p;
    size_t n, pos = 0;
    bool err = false;
    void get(void* dst, size_t k)
    {
        if (err || pos + k > n || pos + k < pos) {
            err = true;
            std::memset(dst, 0, k);
            return;
        }
        std::memcpy(dst, p + pos, k);
        pos += k;
    }
    uint8_t u8() { uint8_t v; get(&v, 1); return v; }
    uint16_t u16() { uint16_t v; get(&v, 2); return v; }
    uint32_t u32() { uint32_t v; get(&v, 4); return v; }
    int32_t i32() { int32_t v; get(&v, 4); return v; }
    uint64_t u64() { uint64_t v; get(&v, 8); return v; }
    double f64() { double v; get(&v, 8); return v; }
};

}  // namespace

void append_stream_header(std::vector<uint8_t>& out, const uint16_t* sym, const uint8_t* len, uint32_t n_used,
                          uint32_t run_base, uint32_t run_n, uint64_t n_unpred, const void* unpred, size_t elem,
                          const uint32_t* unpred_count, const uint64_t* chunk_word_off, const uint32_t* sub_off,
                          int nchunks, int C)
{
    Writer w{out};
    w.u32(n_used);
    w.put(sym, 2 * (size_t)n_used);
    w.put(len, n_used);
    w.u32(run_base);
    w.u32(run_n);
    w.u64(n_unpred);
    w.put(unpred, n_unpred * elem);
    w.put(unpred_count, 4 * (size_t)nchunks);
    w.put(chunk_word_off, 8 * ((size_t)nchunks + 1));
    // plane table (version 4): per chunk the bit counts of its first C - 1
    // planes (the first plane starts at bit 0), 2 bytes each when all fit
    uint32_t mx = 0;
    for (int c = 0; c < nchunks; ++c)
        for (int lz = 1; lz < C; ++lz)
            mx = std::max(mx, sub_off[(size_t)c * C + lz] - sub_off[(size_t)c * C + lz - 1]);
    const uint8_t width = mx < 65536 ? 2 : 4;
    w.u8(width);
    const size_t at = out.size(), m = (size_t)nchunks * (C > 0 ? C - 1 : 0);
    out.resize(at + m * width);
    uint8_t* dst = out.data() + at;
    for (int c = 0; c < nchunks; ++c)
        for (int lz = 1; lz < C; ++lz) {
            const uint32_t d = sub_off[(size_t)c * C + lz] - sub_off[(size_t)c * C + lz - 1];
            if (width == 2) {
                const uint16_t v = (uint16_t)d;
                std::memcpy(dst, &v, 2);
            } else {
                std::memcpy(dst, &d, 4);
            }
            dst += width;
        }
}

bool parse_stream_header(const uint8_t* raw, size_t n, int nchunks, int C, size_t elem, int version,
                         StreamHeader& out)
{
    Reader r{raw, n};
    const uint32_t nu = r.u32();
    if (r.err || nu > 65536) return false;
    out.sym.resize(nu);
    out.len.resize(nu);
    r.get(out.sym.data(), 2 * (size_t)nu);
    r.get(out.len.data(), nu);
    out.run_base = out.run_n = 0;
    if (version >= 3) {
        out.run_base = r.u32();
        out.run_n = r.u32();
        if (out.run_n && (out.run_n != run_slot_count((uint32_t)C * C) || out.run_base < 1)) return false;
    }
    out.n_unpred = r.u64();
    if (r.err || out.n_unpred > n) return false;
    out.unpred.resize(out.n_unpred * elem);
    r.get(out.unpred.data(), out.unpred.size());
    out.unpred_count.resize(nchunks);
    r.get(out.unpred_count.data(), 4 * (size_t)nchunks);
    out.chunk_word_off.resize((size_t)nchunks + 1);
    r.get(out.chunk_word_off.data(), 8 * ((size_t)nchunks + 1));
    out.sub_off.resize((size_t)nchunks * C);
    if (version >= 4) {
        // plane bit counts (all planes of a chunk but its last) -> offsets
        const uint8_t width = r.u8();
        if (width != 2 && width != 4) return false;
        for (int c = 0; c < nchunks && !r.err; ++c) {
            uint64_t acc = 0;
            out.sub_off[(size_t)c * C] = 0;
            for (int lz = 1; lz < C; ++lz) {
                acc += width == 2 ? r.u16() : r.u32();
                if (acc > 0xffffffffull) return false;
                out.sub_off[(size_t)c * C + lz] = (uint32_t)acc;
            }
        }
    } else {
        r.get(out.sub_off.data(), 4 * (size_t)nchunks * C);
    }
    if (r.err || r.pos != n) return false;
    for (uint8_t l : out.len)
        if (l > kMaxCodeLen) return false;
    if (nu == 1 && out.len[0] != 0) return false;
    return true;
}

bool decode_frame(const uint8_t* src, uint64_t stored, uint64_t raw, uint8_t* dst)
{
    if (stored == raw) {
        if (raw) std::memcpy(dst, src, raw);
        return true;
    }
    const size_t r = zstd_decompress(dst, raw, src, stored);
    return !ZSTD_isError(r) && r == raw;
}

std::string parse_stream(const uint8_t* data, size_t size, ParsedStream& out)
{
    Reader r{data, size};
    char mg[8];
    r.get(mg, 8);
    if (r.err || std::memcmp(mg, kMagic, 8) != 0) return "not an STZ-B200 stream (bad magic)";
    const uint32_t version = r.u32();
    if (version < 1 || version > 4) return "unsupported stream version";
    out.version = (int)version;
    FileHeader& h = out.h;
    h.dtype = (int)r.u32();
    h.predictor = (int)r.u32();
    h.nx = (int)r.u32(), h.ny = (int)r.u32(), h.nz = (int)r.u32();
    h.K = (int)r.u32();
    h.radius = (int)r.u32();
    h.chunk_high = (int)r.u32(), h.chunk_low = (int)r.u32();
    h.zstd_level = r.i32();
    h.eb = r.f64(), h.mult_base = r.f64(), h.mult_low = r.f64(), h.mult_high = r.f64();
    h.c0[0] = (int)r.u32(), h.c0[1] = (int)r.u32(), h.c0[2] = (int)r.u32();
    if (r.err) return "truncated stream header";
    if (h.dtype != 0 && h.dtype != 1) return "bad dtype";
    if (h.predictor < 0 || h.predictor > 3) return "bad predictor";
    if (h.radius < 1 || h.radius > 32768) return "bad radius";
    const std::string dm = validate_dims(h.nx, h.ny, h.nz, h.chunk_high, h.chunk_low);
    if (!dm.empty()) return dm;
    if (h.K != num_levels(h.nx, h.ny, h.nz)) return "level count does not match dims";
    if (h.c0[0] != (h.nx >> h.K) || h.c0[1] != (h.ny >> h.K) || h.c0[2] != (h.nz >> h.K)) return "bad coarsest dims";
    out.coarsest_off = r.pos;
    r.pos += (size_t)h.c0[0] * h.c0[1] * h.c0[2] * h.elem();
    out.lv.assign(h.K + 1, LevelDir());
    for (int k = 1; k <= h.K; ++k) {
        LevelDir& L = out.lv[k];
        L.dx = (int)r.u32(), L.dy = (int)r.u32(), L.dz = (int)r.u32();
        L.C = (int)r.u32();
        L.eb = r.f64();
        const int sh = h.K - k + 1;
        if (r.err || L.dx != (h.nx >> sh) || L.dy != (h.ny >> sh) || L.dz != (h.nz >> sh) ||
            L.C != level_chunk(h.nx, h.ny, h.nz, h.K, k, h.chunk_high, h.chunk_low))
            return "bad level record";
        if (version >= 2) {
            L.lflags = r.u32();
            if (L.lflags > 0x7f) return "bad learned-correction flags";
            if (L.lflags) {
                r.get(&L.model, sizeof(LearnedModel));
                if (!r.err && !learned_model_valid(L.model)) return "bad learned model record";
            }
        }
        for (int b = 0; b < 7; ++b) {
            StreamDir& s = L.s[b];
            s.layers = r.u32();
            s.hdr_stored = r.u64();
            s.hdr_raw = r.u64();
            if (r.err || s.layers != (uint32_t)(L.dz / L.C)) return "bad stream record";
            s.ls.resize(s.layers);
            s.lr.resize(s.layers);
            for (auto& v : s.ls) v = r.u64();
            for (auto& v : s.lr) v = r.u64();
        }
    }
    if (r.err) return "truncated directory";
    size_t off = r.pos;
    for (int k = 1; k <= h.K; ++k)
        for (int b = 0; b < 7; ++b) {
            StreamDir& s = out.lv[k].s[b];
            s.data_off = off;
            off += s.hdr_stored;
            if (s.hdr_stored > s.hdr_raw) return "bad frame sizes";
            for (uint32_t L = 0; L < s.layers; ++L) {
                if (s.ls[L] > s.lr[L] || s.lr[L] % 4) return "bad frame sizes";
                off += s.ls[L];
            }
            if (off > size) return "truncated stream data";
        }
    return "";
}

ContainerWriter::ContainerWriter(const FileHeader& h, std::vector<StreamParts>& parts, ThreadPool& pool)
    : h_(h), parts_(parts), pool_(pool)
{
    // per stream its header, then one frame per chunk z-layer
    first_.resize(parts.size() + 1);
    for (size_t i = 0; i < parts.size(); ++i) {
        first_[i] = frames_.size();
        frames_.push_back({parts[i].hdr.data(), parts[i].hdr.size()});
        for (int L = 0; L < parts[i].layers; ++L) {
            const uint64_t w0 = parts[i].chunk_word_off[(size_t)L * parts[i].chunks_per_layer];
            const uint64_t w1 = parts[i].chunk_word_off[(size_t)(L + 1) * parts[i].chunks_per_layer];
            frames_.push_back({(const uint8_t*)(parts[i].words + w0), (size_t)(4 * (w1 - w0))});
            frames_.back().payload = true;
        }
    }
    first_[parts.size()] = frames_.size();
}

void ContainerWriter::compress_streams(size_t s0, size_t s1)
{
    compress_groups(1, [&](size_t s, int) -> size_t { return s >= s0 && s < s1 ? 0 : SIZE_MAX; }, [](size_t) {});
}

void ContainerWriter::compress_groups(size_t ngroups, const std::function<size_t(size_t, int)>& group_of_frame,
                                      const std::function<void(size_t)>& wait_group,
                                      const std::function<void(size_t)>& build_header)
{
    // group by group, largest frames first inside a group (headers not built
    // yet: later streams, the finer levels, first): the pool's threads move
    // on to the next group's frames as soon as its bytes are ready
    std::vector<std::vector<size_t>> by_group(ngroups);
    std::vector<size_t> stream_of(frames_.size(), SIZE_MAX);
    for (size_t st = 0; st + 1 < first_.size(); ++st)
        for (size_t i = first_[st]; i < first_[st + 1]; ++i) {
            stream_of[i] = st;
            const size_t gi = group_of_frame(st, (int)(i - first_[st]) - 1);
            if (gi < ngroups) by_group[gi].push_back(i);
        }
    std::vector<size_t> order, group_of;
    for (size_t gi = 0; gi < ngroups; ++gi) {
        auto& v = by_group[gi];
        std::sort(v.begin(), v.end(),
                  [&](size_t a, size_t c) { return frames_[a].n != frames_[c].n ? frames_[a].n > frames_[c].n : a > c; });
        order.insert(order.end(), v.begin(), v.end());
        group_of.resize(order.size(), gi);
    }
    const int level = h_.zstd_level;
    const bool trace = std::getenv("STZ_TRACE") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    // trace: per group, when its first frame got past the wait and when its
    // last frame was done (microseconds from the start)
    std::vector<std::atomic<int64_t>> g_first(ngroups), g_last(ngroups), g_max(ngroups), g_zn(ngroups);
    for (size_t i = 0; i < ngroups; ++i) g_first[i] = INT64_MAX, g_last[i] = 0, g_max[i] = 0, g_zn[i] = 0;
    auto since = [&](std::chrono::steady_clock::time_point t) {
        return (int64_t)std::chrono::duration_cast<std::chrono::microseconds>(t - t0).count();
    };
    std::vector<int64_t> j_take(trace ? order.size() : 0), j_go(j_take.size()), j_end(j_take.size());
    pool_.parallel_for(order.size(), [&](size_t k) {
        if (trace) j_take[k] = since(std::chrono::steady_clock::now());
        wait_group(group_of[k]);
        const auto f0 = std::chrono::steady_clock::now();
        if (trace) j_go[k] = since(f0);
        if (build_header && !frames_[order[k]].payload) {
            const size_t st = stream_of[order[k]];
            build_header(st);
            frames_[order[k]].src = parts_[st].hdr.data();
            frames_[order[k]].n = parts_[st].hdr.size();
        }
        if (trace) {
            int64_t v = since(f0), cur = g_first[group_of[k]].load();
            while (v < cur && !g_first[group_of[k]].compare_exchange_weak(cur, v)) {
            }
        }
        Frame& f = frames_[order[k]];
        f.raw = true;
        f.stored = f.n;
        bool try_zstd = level > 0 && f.n > 0;
        if (try_zstd && f.payload && f.n > kZstdProbeBytes) {
            // Huffman payload is rarely compressible: zstd the whole frame only
            // when it shrinks the frame's first kZstdProbeBytes
            uint8_t probe[kZstdProbeBytes + kZstdProbeBytes / 64 + 512];
            const size_t c = zstd_compress(probe, sizeof(probe), f.src, kZstdProbeBytes, level);
            try_zstd = !ZSTD_isError(c) && c < kZstdProbeBytes;
        }
        if (try_zstd) {
            const size_t cap = ZSTD_compressBound(f.n);
            f.out.reset(new uint8_t[cap]);
            const size_t c = zstd_compress(f.out.get(), cap, f.src, f.n, level);
            if (!ZSTD_isError(c) && c < f.n) {
                f.stored = c;
                f.raw = false;
            } else {
                f.out.reset();
            }
        }
        if (trace) {
            const auto f1 = std::chrono::steady_clock::now();
            busy_ns_ += std::chrono::duration_cast<std::chrono::nanoseconds>(f1 - f0).count();
            int64_t v = since(f1), cur = g_last[group_of[k]].load();
            while (v > cur && !g_last[group_of[k]].compare_exchange_weak(cur, v)) {
            }
            const int64_t d = (int64_t)std::chrono::duration_cast<std::chrono::microseconds>(f1 - f0).count();
            cur = g_max[group_of[k]].load();
            while (d > cur && !g_max[group_of[k]].compare_exchange_weak(cur, d)) {
            }
            if (!f.raw) ++g_zn[group_of[k]];
            j_end[k] = since(f1);
        }
    });
    if (trace) {
        wall_ns_ += std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
        for (size_t i = 0; i < ngroups; ++i)
            if (g_last[i].load())
                std::fprintf(stderr,
                             "[stz] zstd group %zu: first frame at %.3f ms, last done at %.3f ms, longest frame "
                             "%.3f ms, %lld of %zu frames compressed\n",
                             i, g_first[i].load() / 1e3, g_last[i].load() / 1e3, g_max[i].load() / 1e3,
                             (long long)g_zn[i].load(), by_group[i].size());
        if (std::getenv("STZ_TRACE_JOBS"))
            for (size_t k = 0; k < order.size(); ++k)
                std::fprintf(stderr, "[stz] job %zu group %zu bytes %zu taken %lld started %lld done %lld us\n", k,
                             group_of[k], frames_[order[k]].n, (long long)j_take[k], (long long)j_go[k],
                             (long long)j_end[k]);
    }
}

Bytes ContainerWriter::finish(const void* coarsest, const std::vector<LevelDir>& levels)
{
    const FileHeader& h = h_;
    if (std::getenv("STZ_TRACE")) {
        size_t raw = 0, mx = 0;
        for (const Frame& f : frames_) raw += f.n, mx = std::max(mx, f.n);
        std::fprintf(stderr, "[stz] container: %zu frames, %.2f MB raw, largest %.3f MB, zstd busy %.3f ms on %d "
                             "threads, %.3f ms in zstd calls\n",
                     frames_.size(), raw / 1e6, mx / 1e6, busy_ns_.load() / 1e6, pool_.size(), wall_ns_ / 1e6);
    }
    Lap lap("container");
    std::vector<uint8_t> dir;
    Writer w{dir};
    w.put(kMagic, 8);
    w.u32(4);  // per-level learned-correction fields, run symbols, plane bit counts
    w.u32((uint32_t)h.dtype);
    w.u32((uint32_t)h.predictor);
    w.u32((uint32_t)h.nx);
    w.u32((uint32_t)h.ny);
    w.u32((uint32_t)h.nz);
    w.u32((uint32_t)h.K);
    w.u32((uint32_t)h.radius);
    w.u32((uint32_t)h.chunk_high);
    w.u32((uint32_t)h.chunk_low);
    w.i32(h.zstd_level);
    w.f64(h.eb);
    w.f64(h.mult_base);
    w.f64(h.mult_low);
    w.f64(h.mult_high);
    w.u32((uint32_t)h.c0[0]);
    w.u32((uint32_t)h.c0[1]);
    w.u32((uint32_t)h.c0[2]);
    w.put(coarsest, (size_t)h.c0[0] * h.c0[1] * h.c0[2] * h.elem());
    size_t si = 0;
    for (int k = 1; k <= h.K; ++k) {
        const LevelDir& L = levels[k];
        w.u32((uint32_t)L.dx);
        w.u32((uint32_t)L.dy);
        w.u32((uint32_t)L.dz);
        w.u32((uint32_t)L.C);
        w.f64(L.eb);
        w.u32(L.lflags);
        if (L.lflags) w.put(&L.model, sizeof(LearnedModel));
        for (int b = 0; b < 7; ++b, ++si) {
            const StreamParts& p = parts_[si];
            w.u32((uint32_t)p.layers);
            const Frame& hf = frames_[first_[si]];
            w.u64(hf.stored);
            w.u64(hf.n);
            for (int L2 = 0; L2 < p.layers; ++L2) w.u64(frames_[first_[si] + 1 + L2].stored);
            for (int L2 = 0; L2 < p.layers; ++L2) w.u64(frames_[first_[si] + 1 + L2].n);
        }
    }
    // the directory, then the frames in order, copied in parallel
    std::vector<size_t> off(frames_.size() + 1);
    off[0] = dir.size();
    for (size_t i = 0; i < frames_.size(); ++i) off[i + 1] = off[i] + frames_[i].stored;
    Bytes out;
    out.resize(off.back());
    std::memcpy(out.data(), dir.data(), dir.size());
    lap.mark("directory");
    uint8_t* base = out.data();
    pool_.parallel_for(frames_.size(), [&](size_t i) {
        if (frames_[i].stored) std::memcpy(base + off[i], frames_[i].bytes(), frames_[i].stored);
    });
    lap.mark("frame copy");
    return out;
}

Bytes write_container(const FileHeader& h, const void* coarsest, const std::vector<LevelDir>& levels,
                      std::vector<StreamParts>& parts, ThreadPool& pool)
{
    ContainerWriter w(h, parts, pool);
    w.compress_streams(0, parts.size());
    return w.finish(coarsest, levels);
}

// ---- ROI planner ------------------------------------------------------------------
namespace {

// normalize_axis (FD5:1622-1635)
AxisRange normalize_axis(int64_t a, int64_t b, int dim, bool& is_slice)
{
    AxisRange r;
    if (a == b) {
        is_slice = true;
        const int64_t v = std::max<int64_t>(0, std::min<int64_t>(a, dim - 1));
        r.b = r.e = (int)v;
        return r;
    }
    const int64_t lo = std::max<int64_t>(0, std::min(a, b));
    int64_t hi = std::min<int64_t>(dim - 1, std::max(a, b));
    if (hi < lo) hi = lo;
    r.b = (int)lo, r.e = (int)hi;
    return r;
}

// range_for_parity (FD5:1646-1660)
AxisRange range_for_parity(AxisRange f, int parity)
{
    int first = f.b;
    if ((first & 1) != parity) ++first;
    AxisRange r;
    if (first > f.e) return r;
    int last = f.e;
    if ((last & 1) != parity) --last;
    r.b = first / 2, r.e = last / 2;
    return r;
}

// chunks_for_box (FD5:1662-1687), row-major chunk ids (chunk_index_3d FD5:1578-1582)
void chunks_for_box(int bx, int by, int bz, int C, const AxisRange r[3], std::vector<int64_t>& out)
{
    if (r[0].empty() || r[1].empty() || r[2].empty()) return;
    const int ncx = bx / C, ncy = by / C, ncz = bz / C;
    const int c0[3] = {std::max(0, r[0].b / C), std::max(0, r[1].b / C), std::max(0, r[2].b / C)};
    const int c1[3] = {std::min(ncx - 1, r[0].e / C), std::min(ncy - 1, r[1].e / C), std::min(ncz - 1, r[2].e / C)};
    for (int cz = c0[2]; cz <= c1[2]; ++cz)
        for (int cy = c0[1]; cy <= c1[1]; ++cy)
            for (int cx = c0[0]; cx <= c1[0]; ++cx) out.push_back(((int64_t)cz * ncy + cy) * ncx + cx);
}

// ref_range_for_used_axis (FD5:1726-1749): the cubic stencil's reach.
AxisRange ref_range(AxisRange t, int dim)
{
    if (t.empty()) return t;
    int lo = t.b, hi = t.e;
    const int ib = std::max(t.b, 1), ie = std::min(t.e, dim - 3);
    if (ib <= ie) {
        lo = std::min(lo, ib - 1);
        hi = std::max(hi, ie + 2);
    }
    const int nb = std::max(t.b, 0), ne = std::min(t.e, dim - 2);
    if (nb <= ne) hi = std::max(hi, ne + 1);
    AxisRange r;
    r.b = std::max(0, lo), r.e = std::min(dim - 1, hi);
    return r;
}

void merge_axis(AxisRange& d, AxisRange s)
{
    if (s.empty()) return;
    if (d.empty()) {
        d = s;
        return;
    }
    d.b = std::min(d.b, s.b);
    d.e = std::max(d.e, s.e);
}

}  // namespace

bool region_bbox(const QueryPlan& p, int lo[3], int hi[3])
{
    bool any = false;
    for (const auto& rg : p.regions) {
        if (rg[0].empty() || rg[1].empty() || rg[2].empty()) continue;
        for (int a = 0; a < 3; ++a) {
            lo[a] = any ? std::min(lo[a], rg[a].b) : rg[a].b;
            hi[a] = any ? std::max(hi[a], rg[a].e) : rg[a].e;
        }
        any = true;
    }
    return any;
}

bool mid_window(const QueryPlan& p, int hx, int hy, int hz, bool learned, int lo[3], int hi[3])
{
    bool any = region_bbox(p, lo, hi);
    if (!learned) return any;
    const int hd[3] = {hx, hy, hz};
    for (int a = 0; a < 3; ++a)
        if (p.q[a].empty()) return any;
    for (int a = 0; a < 3; ++a) {
        const int b = std::max(0, (p.q[a].b >> 1) - 1), e = std::min(hd[a] - 1, (p.q[a].e >> 1) + 2);
        lo[a] = any ? std::min(lo[a], b) : b;
        hi[a] = any ? std::max(hi[a], e) : e;
    }
    return true;
}

void window_chunks(const int lo[3], const int hi[3], int C, const int nc[3], std::vector<int64_t>& out)
{
    AxisRange r[3];
    for (int a = 0; a < 3; ++a) r[a] = AxisRange{lo[a] >> 1, hi[a] >> 1};
    chunks_for_box(nc[0] * C, nc[1] * C, nc[2] * C, C, r, out);
}

bool query_box(int nx, int ny, int nz, const int64_t a[3], const int64_t b[3], AxisRange q[3])
{
    const int dims[3] = {nx, ny, nz};
    bool is_slice = false;
    for (int ax = 0; ax < 3; ++ax) q[ax] = normalize_axis(a[ax], b[ax], dims[ax], is_slice);
    return is_slice;
}

QueryPlan plan_query(int nx, int ny, int nz, int chunk_high, int chunk_low, const int64_t a[3], const int64_t b[3])
{
    QueryPlan p;
    const int dims[3] = {nx, ny, nz};
    const int hd[3] = {nx / 2, ny / 2, nz / 2}, ld[3] = {nx / 4, ny / 4, nz / 4};
    for (int ax = 0; ax < 3; ++ax) p.q[ax] = normalize_axis(a[ax], b[ax], dims[ax], p.is_slice);
    // build_residual_plan (FD5:1689-1711)
    for (int blk = 0; blk < 7; ++blk) {
        const int s = blk + 1;
        BlockPlan bp;
        bp.block = blk;
        for (int ax = 0; ax < 3; ++ax) bp.r[ax] = range_for_parity(p.q[ax], (s >> ax) & 1);
        if (bp.r[0].empty() || bp.r[1].empty() || bp.r[2].empty()) continue;
        chunks_for_box(hd[0], hd[1], hd[2], chunk_high, bp.r, bp.chunks);
        p.high.push_back(std::move(bp));
    }
    // build_high_ref_regions (FD5:1751-1770) + build_query_sub0_region (FD5:1772-1782)
    for (const auto& bp : p.high) {
        const int s = bp.block + 1;
        std::array<AxisRange, 3> reg;
        for (int ax = 0; ax < 3; ++ax) reg[ax] = ((s >> ax) & 1) ? ref_range(bp.r[ax], hd[ax]) : bp.r[ax];
        p.regions.push_back(reg);
    }
    {
        std::array<AxisRange, 3> s0;
        for (int ax = 0; ax < 3; ++ax) s0[ax] = range_for_parity(p.q[ax], 0);
        if (!s0[0].empty() && !s0[1].empty() && !s0[2].empty()) p.regions.push_back(s0);
    }
    for (const auto& reg : p.regions)
        p.region_slice.push_back(reg[0].b == reg[0].e || reg[1].b == reg[1].e || reg[2].b == reg[2].e);
    // build_low_residual_plan (FD5:1784-1830)
    for (int blk = 0; blk < 7; ++blk) {
        const int s = blk + 1;
        BlockPlan acc;
        acc.block = blk;
        std::vector<int64_t> cs;
        for (const auto& reg : p.regions) {
            if (reg[0].empty() || reg[1].empty() || reg[2].empty()) continue;
            AxisRange r[3];
            for (int ax = 0; ax < 3; ++ax) r[ax] = range_for_parity(reg[ax], (s >> ax) & 1);
            if (r[0].empty() || r[1].empty() || r[2].empty()) continue;
            chunks_for_box(ld[0], ld[1], ld[2], chunk_low, r, cs);
            for (int ax = 0; ax < 3; ++ax) merge_axis(acc.r[ax], r[ax]);
        }
        if (cs.empty()) continue;
        std::sort(cs.begin(), cs.end());
        cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
        acc.chunks = std::move(cs);
        p.low.push_back(std::move(acc));
    }
    return p;
}

void flatten_plan(const QueryPlan& p, std::vector<int64_t>& o)
{
    o.clear();
    for (int ax = 0; ax < 3; ++ax) {
        o.push_back(p.q[ax].b);
        o.push_back(p.q[ax].e);
    }
    o.push_back(p.is_slice ? 1 : 0);
    auto plans = [&](const std::vector<BlockPlan>& v) {
        o.push_back((int64_t)v.size());
        for (const auto& bp : v) {
            o.push_back(bp.block);
            for (int ax = 0; ax < 3; ++ax) {
                o.push_back(bp.r[ax].b);
                o.push_back(bp.r[ax].e);
            }
            o.push_back((int64_t)bp.chunks.size());
            o.insert(o.end(), bp.chunks.begin(), bp.chunks.end());
        }
    };
    plans(p.high);
    o.push_back((int64_t)p.regions.size());
    for (size_t i = 0; i < p.regions.size(); ++i) {
        for (int ax = 0; ax < 3; ++ax) {
            o.push_back(p.regions[i][ax].b);
            o.push_back(p.regions[i][ax].e);
        }
        o.push_back(p.region_slice[i] ? 1 : 0);
    }
    plans(p.low);
}

}  // namespace stz
