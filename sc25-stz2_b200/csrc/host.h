// Host-side pieces of the STZ B200 library: canonical Huffman codebooks, the
// stream container, the ROI planner and a small thread pool for zstd.
#pragma once
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "stz_internal.h"

namespace stz {

// Byte buffer whose resize leaves new bytes uninitialized (the container is
// written in parallel right after; zero-filling first costs a single-threaded
// pass over fresh pages).
// Large byte blocks come from a small process-wide pool of recently freed
// blocks (their pages stay mapped, so writing a new container does not fault
// and zero fresh pages); the pool keeps at most 4 blocks and 2 GiB.
void* pooled_alloc(size_t bytes);
void pooled_free(void* p, size_t bytes);

template <class T>
struct DefaultInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInitAlloc<U>;
    };
    DefaultInitAlloc() = default;
    template <class U>
    DefaultInitAlloc(const DefaultInitAlloc<U>&) noexcept
    {
    }
    T* allocate(size_t n)
    {
        void* p = pooled_alloc(n * sizeof(T));
        if (!p) throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t n) noexcept { pooled_free(p, n * sizeof(T)); }
    template <class U>
    void construct(U* p) noexcept
    {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a)
    {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
using Bytes = std::vector<uint8_t, DefaultInitAlloc<uint8_t>>;

// ---- thread pool ----------------------------------------------------------
class ThreadPool {
public:
    explicit ThreadPool(int threads);
    ~ThreadPool();
    int size() const { return (int)workers_.size() + 1; }
    // Runs fn(i) for i in [0, n) on the pool and the calling thread.
    void parallel_for(size_t n, const std::function<void(size_t)>& fn);

private:
    void run();
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(size_t)>* job_ = nullptr;
    size_t n_ = 0, next_ = 0, active_ = 0;
    bool stop_ = false;
};

// ---- codebook -------------------------------------------------------------
// Codebook of the container format for one histogram: symbols with a nonzero
// count sorted by (count, symbol); minimum-redundancy lengths (in-place
// algorithm of Moffat & Katajainen); lengths capped at kMaxCodeLen by
// lengthening the least frequent code below the cap until the Kraft sum fits;
// output in canonical (length, symbol) order. A lone symbol gets length 0.
// `base` is added to every histogram index (windowed histograms).
int build_codebook(const uint32_t* hist, int nbins, int base, std::vector<uint16_t>& sym, std::vector<uint8_t>& len);
// The same with the counts of the listed symbols set (symbols outside the
// window [base, base + nbins) are added).
int build_codebook_adjusted(const uint32_t* hist, int nbins, int base,
                            const std::vector<std::pair<uint32_t, uint64_t>>& set, std::vector<uint16_t>& sym,
                            std::vector<uint8_t>& len);

// ---- run symbols (container version 3) ---------------------------------------
// Runs of the centre code (= radius) inside a plane are coded with run
// symbols (run_geometry) in run_n consecutive code values the stream does
// not use, [run_base, run_base + run_n): the highest free window in
// [1, nbins) (count(code) = the stream's code count). Returns run_n (0: no
// runs).
int run_slots(const std::function<uint64_t(uint32_t)>& count, int nbins, int plane, uint32_t& run_base);

// ---- container ------------------------------------------------------------
struct FileHeader {
    int dtype = 0, predictor = 0;
    int nx = 0, ny = 0, nz = 0;
    int K = 0, radius = 0, chunk_high = 0, chunk_low = 0, zstd_level = 0;
    double eb = 0, mult_base = 0, mult_low = 0, mult_high = 0;
    int c0[3] = {0, 0, 0};
    size_t elem() const { return dtype == 1 ? 8 : 4; }
};

struct StreamDir {
    uint32_t layers = 0;
    uint64_t hdr_stored = 0, hdr_raw = 0;
    std::vector<uint64_t> ls, lr;  // stored / raw bytes per chunk z-layer
    size_t data_off = 0;           // byte offset of the header frame
};

struct LevelDir {
    int dx = 0, dy = 0, dz = 0, C = 0;
    double eb = 0;
    uint32_t lflags = 0;     // blocks with the learned correction (container version 2)
    LearnedModel model{};    // its model when lflags != 0
    StreamDir s[7];
};

// A learned model record is usable: finite positive scales, shifts 1..62.
bool learned_model_valid(const LearnedModel& m);

struct ParsedStream {
    int version = 0;  // 1: plain, 2: learned fields, 3: + run symbols, 4: + plane bit counts (not offsets)
    FileHeader h;
    size_t coarsest_off = 0;
    std::vector<LevelDir> lv;  // index 1..K (0 unused)
};

// Decoded (post-zstd) stream header.
struct StreamHeader {
    std::vector<uint16_t> sym;
    std::vector<uint8_t> len;
    uint64_t n_unpred = 0;
    std::vector<uint8_t> unpred;  // n_unpred * elem bytes
    std::vector<uint32_t> unpred_count;
    std::vector<uint64_t> chunk_word_off;  // nchunks + 1
    std::vector<uint32_t> sub_off;         // nchunks * C
    uint32_t run_base = 0, run_n = 0;      // run symbols (version 3)
};

// Levels of the hierarchy and chunk edge per level (shared rule with the
// container reader).
int num_levels(int nx, int ny, int nz);
int level_chunk(int nx, int ny, int nz, int K, int k, int chunk_high, int chunk_low);

std::string validate_dims(long long nx, long long ny, long long nz, int chunk_high, int chunk_low);

// Parse the directory; returns "" on success, else an error message.
std::string parse_stream(const uint8_t* data, size_t size, ParsedStream& out);
bool decode_frame(const uint8_t* src, uint64_t stored, uint64_t raw, uint8_t* dst);
bool parse_stream_header(const uint8_t* raw, size_t n, int nchunks, int C, size_t elem, int version,
                         StreamHeader& out);

// Writer input for one residual stream.
struct StreamParts {
    std::vector<uint8_t> hdr;        // raw stream header bytes
    const uint32_t* words = nullptr; // payload
    const uint64_t* chunk_word_off = nullptr;
    int layers = 0, chunks_per_layer = 0;
};

void append_stream_header(std::vector<uint8_t>& out, const uint16_t* sym, const uint8_t* len, uint32_t n_used,
                          uint32_t run_base, uint32_t run_n, uint64_t n_unpred, const void* unpred, size_t elem,
                          const uint32_t* unpred_count, const uint64_t* chunk_word_off, const uint32_t* sub_off,
                          int nchunks, int C);

// A payload frame longer than this many bytes is zstd-compressed only when
// zstd shrinks its first kZstdProbeBytes (stream headers and shorter frames
// are always tried); a frame is stored compressed when that is smaller.
constexpr size_t kZstdProbeBytes = 4096;

// The container in stages: the frame list of every stream (its header, one
// frame per chunk z-layer of payload), zstd of the frames of a range of
// streams on the pool (as soon as their bytes are on the host), then the
// directory, the coarsest grid and every frame. `parts` stays alive and
// unchanged until finish.
class ContainerWriter {
public:
    ContainerWriter(const FileHeader& h, std::vector<StreamParts>& parts, ThreadPool& pool);
    void compress_streams(size_t s0, size_t s1);
    // The frames in group order on the pool: group_of_frame(stream, layer)
    // (layer -1: the stream's header frame) gives a frame's group in
    // [0, ngroups) (anything else: not compressed by this call); a thread
    // calls wait_group(g) before each frame of group g. build_header (may be
    // empty): the job of stream s's header frame first calls it to fill
    // parts[s].hdr, so each header is built and compressed by one job.
    void compress_groups(size_t ngroups, const std::function<size_t(size_t, int)>& group_of_frame,
                         const std::function<void(size_t)>& wait_group,
                         const std::function<void(size_t)>& build_header = nullptr);
    Bytes finish(const void* coarsest, const std::vector<LevelDir>& levels);

private:
    struct Frame {
        const uint8_t* src;
        size_t n;
        bool payload = false;  // a chunk z-layer of payload (else a stream header)
        std::unique_ptr<uint8_t[]> out;
        size_t stored = 0;
        bool raw = true;
        const uint8_t* bytes() const { return raw ? src : out.get(); }
    };
    FileHeader h_;
    std::vector<StreamParts>& parts_;
    ThreadPool& pool_;
    std::vector<Frame> frames_;
    std::vector<size_t> first_;  // first frame of each stream (+ end)
    std::atomic<int64_t> busy_ns_{0};
    int64_t wall_ns_ = 0;
};

// All stages at once.
Bytes write_container(const FileHeader& h, const void* coarsest, const std::vector<LevelDir>& levels,
                      std::vector<StreamParts>& parts, ThreadPool& pool);

// ---- ROI planner (FD5:1578-1839) -------------------------------------------
struct AxisRange {
    int b = 1, e = 0;  // inclusive; empty when b > e
    bool empty() const { return b > e; }
};
struct BlockPlan {
    int block = 0;
    AxisRange r[3];
    std::vector<int64_t> chunks;  // row-major chunk ids, ascending
};
struct QueryPlan {
    AxisRange q[3];
    bool is_slice = false;
    std::vector<BlockPlan> high;
    std::vector<std::array<AxisRange, 3>> regions;  // high reference regions + query sub-block-0 region
    std::vector<bool> region_slice;
    std::vector<BlockPlan> low;
};
QueryPlan plan_query(int nx, int ny, int nz, int chunk_high, int chunk_low, const int64_t a[3], const int64_t b[3]);
// The query box alone (make_query, FD5:1637-1644); returns is_slice.
bool query_box(int nx, int ny, int nz, const int64_t a[3], const int64_t b[3], AxisRange q[3]);
// Bounding box (x, y, z, inclusive) of a plan's non-empty reference regions
// on the half-resolution grid; false when there are none.
bool region_bbox(const QueryPlan& p, int lo[3], int hi[3]);
// Half-resolution window a query decodes: the region bbox, grown when the
// finest level carries a learned correction (its stencil reaches -1..+2
// around every coarse cell of the query on all three axes) to the cells
// (q.b>>1)-1 .. (q.e>>1)+2, clamped to the grid. false when empty.
bool mid_window(const QueryPlan& p, int hx, int hy, int hz, bool learned, int lo[3], int hi[3]);
// Row-major ids (ascending) of the chunks (edge C, nc per axis) holding the
// cells lo>>1 .. hi>>1 of a half-resolution window.
void window_chunks(const int lo[3], const int hi[3], int C, const int nc[3], std::vector<int64_t>& out);
void flatten_plan(const QueryPlan& p, std::vector<int64_t>& out);

}  // namespace stz
