// Test-infrastructure shim: compiles the reference STZ translation unit
// (src/zero_all_line_dynamic_random_access_optfast3_optcr_lb_fastdec5.cpp,
// "FD5") unmodified, from where it lies, and exports its SZ3-independent
// functions through a C ABI so the tests can use the reference itself as the
// checker. The source path is passed in by the recipe as STZ_FD5_SOURCE; the
// SZ3-ncp headers it includes resolve to oracle/stub_sz3 (declarations only).
//
// Output goes to oracle/_ref/ only. Nothing in the product links this file.
//
// FP environment: the reference main() enables FTZ/DAZ before any work
// (FD5:3046-3047); every entry point below does the same on the calling thread
// and on each OpenMP worker, so results are those of the reference binary.
#include <xmmintrin.h>
#include <pmmintrin.h>

#define main stz_fd5_reference_main_unused
#include STZ_FD5_SOURCE
#undef main

namespace {

void enable_ftz_daz_all_threads()
{
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
#pragma omp parallel
    {
        _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
        _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
    }
}

struct FtzGuard {
    FtzGuard() { enable_ftz_daz_all_threads(); }
};

// Low/high level slab size used by run_typed's task lists (FD5:2179, 2253).
constexpr int kZChunk = 16;

template <typename T>
void split8(T* base, size_t n, T* out[8])
{
    for (int i = 0; i < 8; ++i) out[i] = base + static_cast<size_t>(i) * n;
}

template <typename T>
void split7(T* base, size_t n, T* out[7])
{
    for (int i = 0; i < 7; ++i) out[i] = base + static_cast<size_t>(i) * n;
}

// One refinement level of the reference compressor, as run_typed sequences
// it: split the fine grid into 8 parity sub-blocks (slice_full_data,
// FD5:107-122), predict the 7 odd-parity blocks from the decoded coarse grid
// in 16-plane z-slabs (preprocess_block_zslab, FD5:1161-1175; task list
// FD5:2176-2197), quantize with quantize_range_nodec (FD5:1204-1253; the
// high-level slab loop FD5:2263-2296 keeps unpredictable values in row-major
// order). When `decoded` is requested, the low-level closed loop is followed:
// the in-place "writeDec" quantizer output (FD5:1345-1397) is emulated from the
// codes (+/-dlut[half], raw value when unpredictable), reconstructed with
// depreprocess_block_zslab (FD5:2207-2212) and merged with
// merge_sub_blocks_to_full (FD5:2218-2230).
template <typename T>
int level_encode(const T* fine, const T* coarse, int dx, int dy, int dz, double eb, int radius,
                 int* q_out, T* unpred_out, size_t unpred_cap, size_t* unpred_counts, T* decoded)
{
    FtzGuard g;
    const size_t n = static_cast<size_t>(dx) * dy * dz;
    std::vector<T> subs_store(8 * n);
    T* subs[8];
    split8(subs_store.data(), n, subs);
    slice_full_data(fine, subs, 2 * dx, 2 * dy, 2 * dz);

    std::vector<T> diff_store(7 * n);
    T* diff[7];
    split7(diff_store.data(), n, diff);
    std::vector<std::array<int, 3>> tasks;
    for (int block = 0; block < 7; ++block)
        for (int z0 = 0; z0 < dz; z0 += kZChunk)
            tasks.push_back({block, z0, std::min(z0 + kZChunk, dz)});
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
        const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
        preprocess_block_zslab(block, subs[block + 1], coarse, diff[block], dx, dy, dz, z0, z1);
    }

    std::vector<T> dlut(static_cast<size_t>(radius) + 1);
    for (size_t h = 0; h < dlut.size(); ++h) dlut[h] = static_cast<T>(2 * static_cast<int>(h) * eb);

    size_t total = 0;
    const size_t plane = static_cast<size_t>(dx) * dy;
    for (int block = 0; block < 7; ++block) {
        std::vector<T> unpred;
        for (int z0 = 0; z0 < dz; z0 += kZChunk) {
            const int z1 = std::min(z0 + kZChunk, dz);
            const size_t i0 = static_cast<size_t>(z0) * plane;
            const size_t m = static_cast<size_t>(z1 - z0) * plane;
            quantize_range_nodec(diff[block] + i0, m, eb, radius, dlut.data(), q_out + block * n + i0, unpred);
        }
        unpred_counts[block] = unpred.size();
        if (total + unpred.size() > unpred_cap) return -1;
        std::copy(unpred.begin(), unpred.end(), unpred_out + total);
        total += unpred.size();
    }

    if (decoded) {
        std::vector<T> de_store(7 * n);
        T* de_sub[7];
        split7(de_store.data(), n, de_sub);
        // writeDec emulation: the decompressed residual left in place by the
        // low-level SZ_compress call.
        for (int block = 0; block < 7; ++block) {
            const int* q = q_out + block * n;
            T* d = diff[block];
            for (size_t i = 0; i < n; ++i) {
                if (q[i] == 0) continue;  // unpredictable: raw value stays
                const int half = q[i] >= radius ? q[i] - radius : radius - q[i];
                d[i] = (d[i] < 0) ? -dlut[half] : dlut[half];
            }
        }
#pragma omp parallel for schedule(dynamic)
        for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
            const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
            depreprocess_block_zslab(block, diff[block], coarse, de_sub[block], dx, dy, dz, z0, z1);
        }
        T* all[8] = {const_cast<T*>(coarse), de_sub[0], de_sub[1], de_sub[2],
                     de_sub[3], de_sub[4], de_sub[5], de_sub[6]};
        merge_sub_blocks_to_full(all, decoded, dx, dy, dz);
    }
    return 0;
}

// The same level step scheduled as run_typed schedules it, for timing: the
// fine level's fused (block, 16-plane slab) task loop with a thread-local slab
// buffer, preprocess_block_zslab + quantize_range_nodec per task and per-slab
// unpredictable lists (FD5:2249-2296); when `decoded` is requested the
// coarser-level tail follows: per-block writeDec emulation in parallel
// (SZ_compress runs once per block in parallel, FD5:2199-2205), the parallel
// depreprocess task loop and merge_sub_blocks_to_full (FD5:2207-2230).
// Codes land in q (7 x n, row-major per block); unpredictable values are only
// counted.
template <typename T>
long long level_encode_timed(const T* fine, const T* coarse, int dx, int dy, int dz, double eb, int radius, int* q,
                             T* decoded)
{
    FtzGuard g;
    const size_t n = static_cast<size_t>(dx) * dy * dz;
    std::vector<T> subs_store(8 * n);
    T* subs[8];
    split8(subs_store.data(), n, subs);
    slice_full_data(fine, subs, 2 * dx, 2 * dy, 2 * dz);
    std::vector<T> dlut(static_cast<size_t>(radius) + 1);
    for (size_t h = 0; h < dlut.size(); ++h) dlut[h] = static_cast<T>(2 * static_cast<int>(h) * eb);
    const int nslab = (dz + kZChunk - 1) / kZChunk;
    std::vector<std::array<int, 3>> tasks;
    for (int block = 0; block < 7; ++block)
        for (int z0 = 0; z0 < dz; z0 += kZChunk) tasks.push_back({block, z0, std::min(z0 + kZChunk, dz)});
    const size_t plane = static_cast<size_t>(dx) * dy;
    std::vector<std::vector<T>> unpred(7 * nslab);
    std::vector<T> diff_store(decoded ? 7 * n : 0);
    std::vector<std::vector<T>> slab_buf(omp_get_max_threads());
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
        const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
        T* out;
        if (decoded) {
            out = diff_store.data() + block * n;
        } else {
            std::vector<T>& sb = slab_buf[omp_get_thread_num()];
            if (sb.size() < static_cast<size_t>(kZChunk) * plane) sb.resize(static_cast<size_t>(kZChunk) * plane);
            out = sb.data() - static_cast<size_t>(z0) * plane;
        }
        preprocess_block_zslab(block, subs[block + 1], coarse, out, dx, dy, dz, z0, z1);
        const size_t i0 = static_cast<size_t>(z0) * plane, m = static_cast<size_t>(z1 - z0) * plane;
        quantize_range_nodec(out + i0, m, eb, radius, dlut.data(), q + block * n + i0, unpred[block * nslab + z0 / kZChunk]);
    }
    long long nu = 0;
    for (auto& u : unpred) nu += static_cast<long long>(u.size());
    if (decoded) {
#pragma omp parallel for
        for (int block = 0; block < 7; ++block) {
            const int* qb = q + block * n;
            T* d = diff_store.data() + block * n;
            for (size_t i = 0; i < n; ++i) {
                if (qb[i] == 0) continue;
                const int half = qb[i] >= radius ? qb[i] - radius : radius - qb[i];
                d[i] = (d[i] < 0) ? -dlut[half] : dlut[half];
            }
        }
        std::vector<T> de_store(7 * n);
        T* de_sub[7];
        split7(de_store.data(), n, de_sub);
#pragma omp parallel for schedule(dynamic)
        for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
            const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
            depreprocess_block_zslab(block, diff_store.data() + block * n, coarse, de_sub[block], dx, dy, dz, z0, z1);
        }
        T* all[8] = {const_cast<T*>(coarse), de_sub[0], de_sub[1], de_sub[2],
                     de_sub[3], de_sub[4], de_sub[5], de_sub[6]};
        merge_sub_blocks_to_full(all, decoded, dx, dy, dz);
    }
    return nu;
}

// Dequantize one residual stream exactly as SZ_decompress_separated does
// (recover LUT FD5:1528-1535, unpredictable values consumed in row-major order
// through LinearQuantizer::recover, FD5:1556-1562).
template <typename T>
void dequantize(const int* q, size_t n, double eb, int radius, const T* unpred, T* out)
{
    std::vector<T> lut(static_cast<size_t>(2 * radius) + 1);
    for (size_t i = 0; i < lut.size(); ++i) lut[i] = static_cast<T>(2 * (static_cast<int>(i) - radius) * eb);
    size_t u = 0;
    for (size_t i = 0; i < n; ++i) out[i] = q[i] == 0 ? unpred[u++] : lut[q[i]];
}

// Reference decoder for one level. mode 0: low-level path
// (depreprocess_block_zslab + merge_sub_blocks_to_full, FD5:2369-2394);
// mode 1: high-level fused path (depreprocess_block_zslab_to_full plus the
// sub-block-0 scatter task, FD5:2413-2451).
template <typename T>
void level_decode(const T* dq7, const T* coarse, int dx, int dy, int dz, int mode, T* out)
{
    FtzGuard g;
    const size_t n = static_cast<size_t>(dx) * dy * dz;
    if (mode == 0) {
        std::vector<T> de_store(7 * n);
        T* de_sub[7];
        split7(de_store.data(), n, de_sub);
        std::vector<std::array<int, 3>> tasks;
        for (int block = 0; block < 7; ++block)
            for (int z0 = 0; z0 < dz; z0 += kZChunk)
                tasks.push_back({block, z0, std::min(z0 + kZChunk, dz)});
#pragma omp parallel for schedule(dynamic)
        for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
            const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
            depreprocess_block_zslab(block, dq7 + block * n, coarse, de_sub[block], dx, dy, dz, z0, z1);
        }
        T* all[8] = {const_cast<T*>(coarse), de_sub[0], de_sub[1], de_sub[2],
                     de_sub[3], de_sub[4], de_sub[5], de_sub[6]};
        merge_sub_blocks_to_full(all, out, dx, dy, dz);
        return;
    }
    std::vector<std::array<int, 3>> tasks;
    for (int block = -1; block < 7; ++block)
        for (int z0 = 0; z0 < dz; z0 += kZChunk)
            tasks.push_back({block, z0, std::min(z0 + kZChunk, dz)});
    const size_t fdx = 2 * static_cast<size_t>(dx);
    const size_t fdxy = fdx * 2 * static_cast<size_t>(dy);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < static_cast<int>(tasks.size()); ++t) {
        const int block = tasks[t][0], z0 = tasks[t][1], z1 = tasks[t][2];
        if (block < 0) {
            for (int z = z0; z < z1; ++z)
                for (int y = 0; y < dy; ++y) {
                    const T* src = coarse + (static_cast<size_t>(z) * dy + y) * dx;
                    T* frow = out + 2 * static_cast<size_t>(z) * fdxy + 2 * static_cast<size_t>(y) * fdx;
                    for (int x = 0; x < dx; ++x) frow[2 * static_cast<size_t>(x)] = src[x];
                }
        } else {
            depreprocess_block_zslab_to_full(block, dq7 + block * n, coarse, out, dx, dy, dz, z0, z1);
        }
    }
}

// Flattened planner output (see fd5ref_plan).
void push_range(std::vector<long long>& o, const AxisRange& r)
{
    o.push_back(r.begin);
    o.push_back(r.end);
}

}  // namespace

#define STZ_REF_TYPED(SUF, T)                                                                         \
    extern "C" void fd5ref_slice_full_data_parity_##SUF(const T* full, T* subs, int dx, int dy,       \
                                                         int dz, int parity)                          \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        T* s[8];                                                                                      \
        split8(subs, static_cast<size_t>(dx / 2) * (dy / 2) * (dz / 2), s);                           \
        slice_full_data_parity(full, s, dx, dy, dz, parity);                                         \
    }                                                                                                 \
    extern "C" void fd5ref_slice_full_data_##SUF(const T* full, T* subs, int dx, int dy, int dz)      \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        T* s[8];                                                                                      \
        split8(subs, static_cast<size_t>(dx / 2) * (dy / 2) * (dz / 2), s);                           \
        slice_full_data(full, s, dx, dy, dz);                                                        \
    }                                                                                                 \
    extern "C" void fd5ref_merge_sub_blocks_to_full_##SUF(T* subs, T* full, int sdx, int sdy, int sdz) \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        T* s[8];                                                                                      \
        split8(subs, static_cast<size_t>(sdx) * sdy * sdz, s);                                        \
        merge_sub_blocks_to_full(s, full, sdx, sdy, sdz);                                            \
    }                                                                                                 \
    extern "C" void fd5ref_preprocess_block_zslab_##SUF(int block, const T* sub, const T* ref, T* diff, \
                                                         int dx, int dy, int dz, int z0, int z1)      \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        preprocess_block_zslab(block, sub, ref, diff, dx, dy, dz, z0, z1);                            \
    }                                                                                                 \
    extern "C" void fd5ref_depreprocess_block_zslab_##SUF(int block, const T* de, const T* ref, T* out, \
                                                           int dx, int dy, int dz, int z0, int z1)    \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        depreprocess_block_zslab(block, de, ref, out, dx, dy, dz, z0, z1);                            \
    }                                                                                                 \
    extern "C" void fd5ref_depreprocess_block_zslab_to_full_##SUF(int block, const T* de, const T* ref, \
                                                                   T* full, int dx, int dy, int dz,   \
                                                                   int z0, int z1)                    \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        depreprocess_block_zslab_to_full(block, de, ref, full, dx, dy, dz, z0, z1);                   \
    }                                                                                                 \
    extern "C" void fd5ref_depreprocess_block_roi_##SUF(int block, const T* de, const T* ref, T* out,  \
                                                         int dx, int dy, int dz, int ex, int ey,      \
                                                         int ez, int sx, int sy, int sz)              \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        depreprocess_block(block, de, ref, out, dx, dy, dz, ex, ey, ez, sx, sy, sz);                  \
    }                                                                                                 \
    extern "C" long long fd5ref_quantize_range_nodec_##SUF(const T* data, size_t n, double eb,        \
                                                           int radius, int* q, T* unpred,             \
                                                           size_t cap)                                \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        std::vector<T> dlut(static_cast<size_t>(radius) + 1);                                         \
        for (size_t h = 0; h < dlut.size(); ++h)                                                      \
            dlut[h] = static_cast<T>(2 * static_cast<int>(h) * eb);                                   \
        std::vector<T> u;                                                                             \
        quantize_range_nodec(data, n, eb, radius, dlut.data(), q, u);                                 \
        if (u.size() > cap) return -1;                                                                \
        std::copy(u.begin(), u.end(), unpred);                                                        \
        return static_cast<long long>(u.size());                                                      \
    }                                                                                                 \
    extern "C" int fd5ref_level_encode_##SUF(const T* fine, const T* coarse, int dx, int dy, int dz,  \
                                              double eb, int radius, int* q, T* unpred, size_t cap,   \
                                              size_t* counts, T* decoded)                             \
    {                                                                                                 \
        return level_encode<T>(fine, coarse, dx, dy, dz, eb, radius, q, unpred, cap, counts, decoded); \
    }                                                                                                 \
    extern "C" void fd5ref_dequantize_##SUF(const int* q, size_t n, double eb, int radius,            \
                                             const T* unpred, T* out)                                 \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        dequantize<T>(q, n, eb, radius, unpred, out);                                                 \
    }                                                                                                 \
    extern "C" long long fd5ref_level_encode_timed_##SUF(const T* fine, const T* coarse, int dx,      \
                                                         int dy, int dz, double eb, int radius,       \
                                                         int* q, T* decoded)                          \
    {                                                                                                 \
        return level_encode_timed<T>(fine, coarse, dx, dy, dz, eb, radius, q, decoded);               \
    }                                                                                                 \
    /* recover with the LUT, chunk-parallel as the decoder's fused pass (FD5:1528-1544);             \
       only for streams without unpredictable values */                                              \
    extern "C" void fd5ref_recover_parallel_##SUF(const int* q, size_t n, double eb, int radius,      \
                                                   T* out)                                            \
    {                                                                                                 \
        FtzGuard g;                                                                                   \
        std::vector<T> lut(static_cast<size_t>(2 * radius) + 1);                                      \
        for (size_t i = 0; i < lut.size(); ++i)                                                       \
            lut[i] = static_cast<T>(2 * (static_cast<int>(i) - radius) * eb);                         \
        _Pragma("omp parallel for") for (long long i = 0; i < static_cast<long long>(n); ++i)         \
            out[i] = lut[q[i]];                                                                       \
    }                                                                                                 \
    extern "C" void fd5ref_level_decode_##SUF(const T* dq7, const T* coarse, int dx, int dy, int dz,  \
                                               int mode, T* out)                                      \
    {                                                                                                 \
        level_decode<T>(dq7, coarse, dx, dy, dz, mode, out);                                          \
    }

STZ_REF_TYPED(f32, float)
STZ_REF_TYPED(f64, double)

// Reference ROI planner (FD5:1578-1839), run for one query exactly as the
// auto-query section of run_typed sequences it (FD5:2460-2470). Output is a
// flat int64 record:
//   query: x.b x.e y.b y.e z.b z.e is_slice
//   n_high, then per high plan: block x.b x.e y.b y.e z.b z.e n_chunks chunks...
//   n_regions, then per region: x.b x.e y.b y.e z.b z.e is_slice
//   n_low, then per low plan: block x.b x.e y.b y.e z.b z.e n_chunks chunks...
// Returns the number of int64 written, or -1 if `cap` is too small.
extern "C" long long fd5ref_plan(int nx, int ny, int nz, int chunk_high, int chunk_low, int ax, int ay,
                                 int az, int bx, int by, int bz, long long* out, long long cap)
{
    set_full_dims(nx, ny, nz);
    roi_high_dim = chunk_high;
    roi_low_dim = chunk_low;
    const QueryBox query = make_query(ax, ay, az, bx, by, bz);
    const auto highPlans = build_residual_plan(query, dim_x, dim_y, dim_z, roi_high_dim);
    auto highRefRegions = build_high_ref_regions(highPlans);
    const QueryBox querySub0Region = build_query_sub0_region(query);
    if (querySub0Region.x.begin <= querySub0Region.x.end &&
        querySub0Region.y.begin <= querySub0Region.y.end &&
        querySub0Region.z.begin <= querySub0Region.z.end) {
        highRefRegions.push_back(querySub0Region);
    }
    const auto lowPlans = build_low_residual_plan(highRefRegions);

    std::vector<long long> o;
    push_range(o, query.x);
    push_range(o, query.y);
    push_range(o, query.z);
    o.push_back(query.is_slice ? 1 : 0);
    auto push_plans = [&](const std::vector<BlockAccessPlan>& plans) {
        o.push_back(static_cast<long long>(plans.size()));
        for (const auto& p : plans) {
            o.push_back(p.block);
            push_range(o, p.x);
            push_range(o, p.y);
            push_range(o, p.z);
            o.push_back(static_cast<long long>(p.chunks.size()));
            for (size_t c : p.chunks) o.push_back(static_cast<long long>(c));
        }
    };
    push_plans(highPlans);
    o.push_back(static_cast<long long>(highRefRegions.size()));
    for (const auto& r : highRefRegions) {
        push_range(o, r.x);
        push_range(o, r.y);
        push_range(o, r.z);
        o.push_back(r.is_slice ? 1 : 0);
    }
    push_plans(lowPlans);
    if (static_cast<long long>(o.size()) > cap) return -1;
    std::copy(o.begin(), o.end(), out);
    return static_cast<long long>(o.size());
}
