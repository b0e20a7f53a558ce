// Level kernels of the STZ hierarchy on B200.
//
// Encode (one launch per level): a CTA covers a 32 x 8 x 8 brick of coarse
// points of a level; each thread owns one (x, y) column of it and handles all
// 8 parity positions of the 2x2x2 cell above each coarse point. The brick's
// coarse-grid halo (x-1..x+2 on every axis, the reach of the cubic stencils)
// is staged once in shared memory, so every stencil tap is one shared load
// with a compile-time offset. Per point the kernel reads the original fine
// values straight from the input field (the hierarchical split, FD5:107-139,
// is never materialised: level k reads the field at stride 2^(K-k)), predicts
// the 7 odd-parity sub-blocks (FD5:1005-1047, 690-748), quantizes the
// residuals (FD5:1204-1253), writes the codes in chunk-major order for the
// entropy coder, builds the per-stream code histogram, and, on every level but
// the finest, writes the decoded fine grid the next level predicts from (the
// encoder's closed loop, FD5:2195-2230).
//
// Decode (one launch per level): the same traversal, x' = recover(q) + P
// (FD5:1049-1143), written straight into the merged fine grid (the fused
// depreprocess+merge of FD5:1096-1143, including the sub-block-0 scatter of
// FD5:2430-2440).
//
// Standalone kernels mirror the reference's per-function boundary (split,
// merge, zslab preprocess/depreprocess, ROI depreprocess, quantize,
// dequantize) for callers that drive the stages themselves.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

#include <cuda.h>
#include <cuda_runtime.h>

#include "learned_tc.cuh"
#include "levels.h"
#include "stz_device.cuh"

namespace stz {

// Set by a level kernel whose tensor-core network gave up waiting on an MMA.
__device__ uint32_t g_learned_tc_error;

// A pinned, mapped host word that a level kernel sets when a TMA tile load
// did not complete within its bounded wait (null until level_error_init). The
// host reads it after the synchronizations it makes anyway.
__device__ volatile uint32_t* g_tile_error;
namespace {
volatile uint32_t* g_tile_error_host = nullptr;
std::mutex g_tile_error_mu;
}  // namespace

cudaError_t level_error_init()
{
    std::lock_guard<std::mutex> lk(g_tile_error_mu);
    if (!g_tile_error_host) {
        void* p = nullptr;
        const cudaError_t e = cudaHostAlloc(&p, 64, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) return e;
        std::memset(p, 0, 64);
        g_tile_error_host = static_cast<volatile uint32_t*>(p);
    }
    void* d = nullptr;
    cudaError_t e = cudaHostGetDevicePointer(&d, (void*)g_tile_error_host, 0);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_tile_error, &d, sizeof(d));
    return e;
}

bool level_error_take()
{
    if (!g_tile_error_host || !*g_tile_error_host) return false;
    *g_tile_error_host = 0;
    return true;
}

uint32_t learned_tc_error_take(cudaStream_t st)
{
    uint32_t v = 0;
    const uint32_t zero = 0;
    if (cudaMemcpyFromSymbolAsync(&v, g_learned_tc_error, 4, 0, cudaMemcpyDeviceToHost, st) != cudaSuccess) return 1;
    if (v) cudaMemcpyToSymbolAsync(g_learned_tc_error, &zero, 4, 0, cudaMemcpyHostToDevice, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 1;
    return v;
}

namespace {

template <typename T>
struct V2;
template <>
struct V2<float> {
    using type = float2;
};
template <>
struct V2<double> {
    using type = double2;
};

// Brick of coarse points per CTA and its halo tile: BX x BY columns, ZB
// planes deep. Levels of at least 2^23 coarse points take kZBig planes (a
// tile loads ZB + 3 planes, so deeper bricks load fewer halo planes per
// point: finest 512^3 encode 0.55 -> 0.48 ms, decode 0.40 -> 0.34 ms);
// smaller levels keep kZSmall so they still spread over the SMs, and so do
// the learned-correction kernels.
constexpr int BX = 32, BY = 8;
constexpr int kZSmall = 8, kZBig = 16;
constexpr size_t kZBigPoints = size_t(1) << 23;
// Levels of at most 2^18 coarse points (64^3) take 2-plane bricks: four times
// the CTAs and a quarter of each thread's serial chain, for levels that are
// too small to fill the device with 8-plane bricks.
constexpr int kZTiny = 2;
constexpr size_t kZTinyPoints = size_t(1) << 18;
// Tile rows hold BX + 3 values, padded to BX + 4 so a row is a multiple of
// 16 bytes: the inner extent of the TMA box that stages the tile.
constexpr int TSX = BX + 4, TSY = BY + 3;
constexpr int TPLANE = TSX * TSY;
template <int ZB>
__host__ __device__ constexpr int tile_elems()
{
    return TPLANE * (ZB + 3);
}

template <typename T, int ZB = kZSmall>
constexpr size_t tile_bytes()
{
    return sizeof(T) * tile_elems<ZB>();
}
// Offset of the learned model behind the tile in dynamic shared memory.
template <typename T, int ZB = kZSmall>
constexpr size_t kTileBytesAligned = (sizeof(T) * tile_elems<ZB>() + 15) & ~(size_t)15;

// Stage the coarse grid on [x0-1, x0+BX+1] x [y0-1, y0+BY+1] x [z0-1, z0+ZB+1]
// (zero outside the grid; the predictors never read those positions).
template <typename T, int ZB>
__device__ __forceinline__ void load_tile(T* tile, const T* __restrict__ R, int dx, int dy, int dz, int x0, int y0,
                                          int z0)
{
    const int tid = threadIdx.y * BX + threadIdx.x;
    for (int i = tid; i < tile_elems<ZB>(); i += BX * BY) {
        const int tz = i / TPLANE, rem = i - tz * TPLANE;
        const int ty = rem / TSX, tx = rem - ty * TSX;
        const int gx = x0 - 1 + tx, gy = y0 - 1 + ty, gz = z0 - 1 + tz;
        T v = T(0);
        if (gx >= 0 && gx < dx && gy >= 0 && gy < dy && gz >= 0 && gz < dz)
            v = __ldg(R + ((size_t)gz * dy + gy) * dx + gx);
        tile[i] = v;
    }
}

// TMA staging of the halo tile (sm_100a): one thread issues a 3-D bulk tensor
// load of the box [x0-1, x0+BX+3) x [y0-1, y0+BY+2) x [z0-1, z0+ZB+2) of the
// coarse grid into the tile, the tensor map filling zeros outside the grid;
// the CTA waits on an mbarrier. The box's x origin x0 - 1 = BX * blockIdx.x
// is a multiple of 16 bytes for any element size, as the TMA requires. The
// wait is bounded: past kTileSpin tries the kernel flags the error (host word
// g_tile_error), waits once more within the same bound and goes on; the
// host then fails the call.
constexpr int kTileSpin = 1 << 22;

template <typename T, int ZB>
__device__ __forceinline__ void tma_load_tile(T* tile, const CUtensorMap* map, int x0, int y0, int z0,
                                              uint64_t* bar)
{
    const int tid = threadIdx.y * BX + threadIdx.x;
    const uint32_t b = tc::smem_addr(bar);
    if (tid == 0) {
        tc::mbar_init(b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        constexpr uint32_t bytes = (uint32_t)(sizeof(T) * tile_elems<ZB>());
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4}], [%5];" ::"r"(tc::smem_addr(tile)),
            "l"(reinterpret_cast<uint64_t>(map)), "r"(x0 - 1), "r"(y0 - 1), "r"(z0 - 1), "r"(b)
            : "memory");
    }
    bool done = false;
    for (int i = 0; i < kTileSpin && !done; ++i) done = tc::mbar_try(b, 0);
    if (!done) {
        if (tid == 0 && g_tile_error) *g_tile_error = 1u;
        for (int i = 0; i < kTileSpin && !done; ++i) done = tc::mbar_try(b, 0);
    }
}

// The halo tile through the TMA (tmap non-null, and the tile's shared-memory
// address 128-byte aligned as a bulk tensor destination wants) or by the
// CTA's threads.
template <typename T, int ZB>
__device__ __forceinline__ void stage_tile(T* tile, const T* __restrict__ R, const CUtensorMap* tmap, int dx, int dy,
                                           int dz, int x0, int y0, int z0, uint64_t* bar)
{
    if (tmap && (tc::smem_addr(tile) & 127u) == 0) tma_load_tile<T, ZB>(tile, tmap, x0, y0, z0, bar);
    else load_tile<T, ZB>(tile, R, dx, dy, dz, x0, y0, z0);
}

// Shared histogram bins around the centre code per stream (codes outside go
// to global atomics); 448 keeps five finest-encode CTAs within an SM's
// shared memory.
constexpr int kSmemBins = 448;

struct HistArgs {
    uint32_t* full;     // 7 x 2r bins
    uint32_t* outside;  // 7 counters: codes outside the host window
    int radius;
};

__device__ __forceinline__ void hist_add(uint32_t (*sh)[kSmemBins], int wlo, int wn, const HistArgs& h, int b, int key,
                                         uint32_t cnt)
{
    const int w = key - wlo;
    if (w >= 0 && w < wn) atomicAdd(&sh[b][w], cnt);
    else atomicAdd(&h.full[(size_t)b * 2 * h.radius + key], cnt);
    const int off = key - h.radius;
    if (off < -kHistWindow / 2 || off >= kHistWindow / 2) atomicAdd(&h.outside[b], cnt);
}

// Histogram of one stream: codes equal to the radius (the dominant bin of a
// well-predicted level) are counted in a register per thread; any other code
// is one atomic on the block's shared bins (such codes are few, so lanes
// rarely collide; a warp-aggregated form cost more in match/vote
// instructions than it saved). `key` < 0 marks a lane without a code.
__device__ __forceinline__ void hist_code(uint32_t (*sh)[kSmemBins], int wlo, int wn, const HistArgs& h, int b, int key,
                                          uint32_t& center)
{
    center += key == h.radius;
    if (key >= 0 && key != h.radius) hist_add(sh, wlo, wn, h, b, key, 1u);
}

// Flush the per-thread dominant-bin counters: warp sum, one atomic per warp.
__device__ __forceinline__ void hist_flush_center(uint32_t (*sh)[kSmemBins], int wlo, int wn, const HistArgs& h,
                                                  const uint32_t (&center)[7])
{
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        uint32_t c = center[b];
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) hist_add(sh, wlo, wn, h, b, h.radius, c);
    }
}

// Chunk-major position of coarse point (x, y, z): the x/y parts are fixed per
// thread, the z part changes per plane.
struct ChunkIndex {
    int C, lc, ncx, ncy;  // lc = log2(C) for power-of-two edges, else -1
    int cx, lx, cy, ly;
    __device__ __forceinline__ void init(const LevelGeom& g, int x, int y)
    {
        C = g.C, ncx = g.ncx, ncy = g.ncy;
        lc = (C & (C - 1)) == 0 ? __ffs(C) - 1 : -1;
        if (lc >= 0) {
            cx = x >> lc, lx = x & (C - 1);
            cy = y >> lc, ly = y & (C - 1);
        } else {
            cx = x / C, lx = x - cx * C;
            cy = y / C, ly = y - cy * C;
        }
    }
    __device__ __forceinline__ size_t at(int z, int& chunk) const
    {
        if (lc >= 0) {
            const int cz = z >> lc, lz = z & (C - 1);
            chunk = (cz * ncy + cy) * ncx + cx;
            return ((size_t)chunk << (3 * lc)) + (size_t)((((lz << lc) + ly) << lc) + lx);
        }
        const int cz = z / C, lz = z - cz * C;
        chunk = (cz * ncy + cy) * ncx + cx;
        return (size_t)chunk * C * C * C + (size_t)((lz * C + ly) * C + lx);
    }
};

// The same position, advanced along z by one thread's walk down its column:
// inside a chunk the next z is C*C codes further, at a chunk boundary the walk
// jumps to the chunk above (ncx*ncy chunks on).
struct ZWalk {
    size_t cm;   // chunk-major position of (x, y, z)
    int chunk;   // its chunk
    int lz, C;
    size_t plane, jump;
    int chunk_step;
    __device__ __forceinline__ void init(const LevelGeom& g, int x, int y, int z)
    {
        ChunkIndex ci;
        ci.init(g, x, y);
        cm = ci.at(z, chunk);
        C = g.C;
        lz = z % C;
        plane = (size_t)C * C;
        chunk_step = g.ncx * g.ncy;
        jump = (size_t)chunk_step * C * C * C - (size_t)(C - 1) * C * C;
    }
    __device__ __forceinline__ void next()
    {
        if (++lz == C) {
            lz = 0;
            chunk += chunk_step;
            cm += jump;
        } else {
            cm += plane;
        }
    }
};

// Recover table for the codes around the radius (the reference's recover LUT,
// FD5:1528-1535): one shared load instead of int->double->T conversions.
constexpr int kRecW = 256;
template <typename T>
__device__ __forceinline__ void build_recover_lut(T* lut, const QuantParams& qp, int tid, int nthreads)
{
    for (int i = tid; i < 2 * kRecW; i += nthreads) lut[i] = recover<T>(qp.radius - kRecW + i, qp);
}
template <typename T>
__device__ __forceinline__ T recover_lut(const T* lut, int q, const QuantParams& qp)
{
    const unsigned i = (unsigned)(q - qp.radius + kRecW);
    return i < 2u * kRecW ? lut[i] : recover<T>(q, qp);
}

#include "level_kernels.cuh"
#include "staged_kernels.cuh"
#include "trunc_kernels.cuh"

// Coarsest grid of the hierarchy: every 2^K-th point of the field.
template <typename T>
__global__ void k_subsample(const T* __restrict__ field, size_t fsx, size_t fsy, int s, int ox, int oy, int oz,
                            T* __restrict__ out)
{
    const size_t n = (size_t)ox * oy * oz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % ox), y = (int)((i / ox) % oy), z = (int)(i / ((size_t)ox * oy));
        out[i] = field[(size_t)s * z * fsy + (size_t)s * y * fsx + (size_t)s * x];
    }
}

// Value range of a field (max and min, as computeRange FD5:92-104, NaN
// ignored). Reduces in T (exact), then converts.
template <typename T>
__global__ void k_minmax(const T* __restrict__ p, size_t n, double* out)
{
    T lo = T(INFINITY), hi = T(-INFINITY);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    auto take = [&](T a) {
        lo = fmin(lo, a);
        hi = fmax(hi, a);
    };
    // elements before the first 16-byte boundary, then 16-byte vectors (four
    // in flight per thread), then the tail
    constexpr size_t V = 16 / sizeof(T);
    const size_t h = min(n, ((16 - ((uintptr_t)p & 15)) & 15) / sizeof(T));
    const size_t nv = (n - h) / V;
    const uint4* __restrict__ pv = reinterpret_cast<const uint4*>(p + h);
    auto take4 = [&](const uint4& q) {
        const T* e = reinterpret_cast<const T*>(&q);
#pragma unroll
        for (size_t k = 0; k < V; ++k) take(e[k]);
    };
    size_t i = tid;
    for (; i + 3 * stride < nv; i += 4 * stride) {
        const uint4 a = __ldg(pv + i), b = __ldg(pv + i + stride), c = __ldg(pv + i + 2 * stride),
                    d = __ldg(pv + i + 3 * stride);
        take4(a), take4(b), take4(c), take4(d);
    }
    for (; i < nv; i += stride) take4(__ldg(pv + i));
    for (size_t j = tid; j < h; j += stride) take(__ldg(p + j));
    for (size_t j = h + nv * V + tid; j < n; j += stride) take(__ldg(p + j));
    for (int o = 16; o; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ double slo[32], shi[32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) slo[w] = (double)lo, shi[w] = (double)hi;
    __syncthreads();
    if (threadIdx.x == 0) {
        double l = slo[0], h = shi[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) l = fmin(l, slo[k]), h = fmax(h, shi[k]);
        // doubles compare as unsigned integers after a sign-magnitude fix-up
        unsigned long long* u = reinterpret_cast<unsigned long long*>(out);
        auto key = [](double d) {
            long long b = __double_as_longlong(d);
            return (unsigned long long)(b < 0 ? ~b : (b | 0x8000000000000000ll));
        };
        atomicMin(&u[0], key(l));
        atomicMax(&u[1], key(h));
    }
}

// ---- reference-boundary kernels ------------------------------------------

// slice_full_data (FD5:107-122): sub[((z&1)<<2)|((y&1)<<1)|(x&1)][z/2,y/2,x/2].
template <typename T>
__global__ void k_split(const T* __restrict__ full, int nx, int ny, int nz, T* __restrict__ subs)
{
    using T2 = typename V2<T>::type;
    const int hx = nx / 2, hy = ny / 2, hz = nz / 2;
    const size_t hn = (size_t)hx * hy * hz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < hn; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % hx), y = (int)((i / hx) % hy), z = (int)(i / ((size_t)hx * hy));
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int pz = r >> 1, py = r & 1;
            const T2 t = *reinterpret_cast<const T2*>(full + ((size_t)(2 * z + pz) * ny + (2 * y + py)) * nx + 2 * (size_t)x);
            subs[(size_t)(pz * 4 + py * 2) * hn + i] = t.x;
            subs[(size_t)(pz * 4 + py * 2 + 1) * hn + i] = t.y;
        }
    }
}

// merge_sub_blocks_to_full (FD5:68-90).
template <typename T>
__global__ void k_merge(const T* __restrict__ subs, int hx, int hy, int hz, T* __restrict__ full)
{
    using T2 = typename V2<T>::type;
    const size_t hn = (size_t)hx * hy * hz;
    const size_t nx = 2 * (size_t)hx, ny = 2 * (size_t)hy;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < hn; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % hx), y = (int)((i / hx) % hy), z = (int)(i / ((size_t)hx * hy));
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int pz = r >> 1, py = r & 1;
            T2 t;
            t.x = subs[(size_t)(pz * 4 + py * 2) * hn + i];
            t.y = subs[(size_t)(pz * 4 + py * 2 + 1) * hn + i];
            *reinterpret_cast<T2*>(full + ((size_t)(2 * z + pz) * ny + (2 * y + py)) * nx + 2 * (size_t)x) = t;
        }
    }
}

// mode 0: preprocess_block_zslab (diff = sub - P, FD5:1161-1175)
// mode 1: depreprocess_block_zslab (out = de + P, FD5:1177-1191)
// mode 2: depreprocess_block_zslab_to_full (scatter into the full grid, FD5:1145-1159)
// Points outside [x0,x1) x [y0,y1) x [z0,z1) are left untouched; mode 1 with
// a sub-range is the ROI depreprocess_block (FD5:978-999).
template <typename T, int PRED>
__global__ void k_block_op(int mode, int block, const T* __restrict__ src, Grid<T> R, T* __restrict__ dst, int x0,
                           int x1, int y0, int y1, int z0, int z1)
{
    using A = Ar<T>;
    const int ex = x1 - x0, ey = y1 - y0;
    const size_t m = (size_t)ex * ey * (z1 - z0);
    const int si = block + 1;
    const int px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const int x = x0 + (int)(i % ex), y = y0 + (int)((i / ex) % ey), z = z0 + (int)(i / ((size_t)ex * ey));
        const size_t idx = (size_t)z * R.sy + (size_t)y * R.sx + x;
        const T p = predict<PRED>(block, R, x, y, z);
        if (mode == 0) dst[idx] = A::sub(src[idx], p);
        else if (mode == 1) dst[idx] = A::add(src[idx], p);
        else
            dst[(size_t)(2 * z + pz) * 4 * R.sy + (size_t)(2 * y + py) * 2 * R.sx + 2 * (size_t)x + px] = A::add(src[idx], p);
    }
}

// Per-tile quantize: codes, per-tile unpredictable counts (tile = blockDim.x).
template <typename T>
__global__ void k_quantize(const T* __restrict__ d, size_t n, QuantParams qp, int* __restrict__ q,
                           uint32_t* __restrict__ tile_cnt)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int code = 1;
    if (i < n) {
        code = quantize(d[i], qp);
        q[i] = code;
    }
    const int c = __syncthreads_count(code == 0);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = (uint32_t)c;
}

// Exclusive scan of tile counts by one CTA (counts are few: n / 1024).
__global__ void k_scan_tiles(const uint32_t* __restrict__ cnt, size_t ntiles, uint64_t* __restrict__ off)
{
    __shared__ uint64_t carry;
    __shared__ uint64_t warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (size_t base = 0; base < ntiles; base += blockDim.x) {
        const size_t i = base + threadIdx.x;
        uint64_t v = i < ntiles ? cnt[i] : 0;
        uint64_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if ((threadIdx.x & 31) >= o) incl += t;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint64_t w = threadIdx.x < (blockDim.x >> 5) ? warp_sums[threadIdx.x] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += t;
            }
            warp_sums[threadIdx.x] = w;
        }
        __syncthreads();
        const uint64_t wprefix = (threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5) - 1] : 0;
        if (i < ntiles) off[i] = carry + wprefix + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += wprefix + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[ntiles] = carry;
}

// Rank of element i among the tile's unpredictable elements.
__device__ __forceinline__ uint32_t tile_rank(bool flag, uint32_t* warp_cnt)
{
    const unsigned full = 0xffffffffu;
    const unsigned bal = __ballot_sync(full, flag);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_cnt[w] = __popc(bal);
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < w; ++k) before += warp_cnt[k];
    return before + __popc(bal & ((1u << lane) - 1u));
}

template <typename T>
__global__ void k_quantize_unpred(const T* __restrict__ d, size_t n, const int* __restrict__ q,
                                  const uint64_t* __restrict__ off, T* __restrict__ unpred)
{
    __shared__ uint32_t wc[32];
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const bool f = i < n && q[i] == 0;
    const uint32_t r = tile_rank(f, wc);
    if (f) unpred[off[blockIdx.x] + r] = d[i];
}

__global__ void k_dequant_count(const int* __restrict__ q, size_t n, uint32_t* __restrict__ tile_cnt)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const int c = __syncthreads_count(i < n && q[i] == 0);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = (uint32_t)c;
}

template <typename T>
__global__ void k_dequantize(const int* __restrict__ q, size_t n, QuantParams qp, const uint64_t* __restrict__ off,
                             const T* __restrict__ unpred, T* __restrict__ out)
{
    __shared__ uint32_t wc[32];
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const int code = i < n ? q[i] : 1;
    const uint32_t r = tile_rank(code == 0, wc);
    if (i < n) out[i] = code ? recover<T>(code, qp) : unpred[off[blockIdx.x] + r];
}

int grid_for(size_t n, int threads)
{
    size_t g = (n + threads - 1) / threads;
    if (g > 148 * 64) g = 148 * 64;
    return (int)(g ? g : 1);
}

template <typename T>
Grid<T> make_grid(const T* p, int dx, int dy, int dz)
{
    Grid<T> g;
    g.p = p;
    g.dx = dx, g.dy = dy, g.dz = dz;
    g.sx = (size_t)dx;
    g.sy = (size_t)dx * dy;
    return g;
}

// Code histograms of the sampled interior points without (hist[0]) and with
// (hist[1]) the learned correction; thread per sample point, the network per
// thread (dp4a) or block-wide on the tensor cores (LM).
template <typename T, int PRED, int LM>
__global__ void __launch_bounds__(256) k_learned_eval(const T* __restrict__ field, size_t fsx, size_t fsy, int s,
                                                      const T* __restrict__ R, LevelGeom geo, QuantParams qp,
                                                      LearnedArgs<T> la, int sx, int sy, int sz,
                                                      uint32_t* __restrict__ hist)
{
    __shared__ __align__(16) LearnedModel model;
    __shared__ uint32_t h[2][7][kEvalBins];
    const int tid = threadIdx.x;
    for (int i = tid; i < 2 * 7 * kEvalBins; i += blockDim.x) (&h[0][0][0])[i] = 0;
    learned_load(&model, la.model, tid, blockDim.x);
    __syncthreads();
    using A = Ar<T>;
    const uint64_t total = (uint64_t)sx * sy * sz;
    const long long gx = geo.dx, gy = (long long)geo.dx * geo.dy;
    const int lo = qp.radius - kEvalHalf;
    [[maybe_unused]] uint32_t phase = 0;
    [[maybe_unused]] bool tc_failed = false;
    if constexpr (LM == kLearnTc) tc::net_setup(*net_smem(), model, tid);
    // uniform trip count per block (the tensor-core network is block-wide)
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < total; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = base + tid;
        const bool valid = i < total;
        const uint64_t ii = valid ? i : 0;
        const int ix = (int)(ii % sx), iy = (int)((ii / sx) % sy), iz = (int)(ii / ((uint64_t)sx * sy));
        const int x = 1 + 2 * ix, y = 1 + 2 * iy, z = 1 + 2 * iz;
        const GlobalAt<T> r{R + (size_t)z * gy + (size_t)y * gx + x, gx, gy};
        int acc3[7];
        if constexpr (LM == kLearnTc) {
            const uint4 xin = valid ? learned_inputs<T>(r, la.rs) : make_uint4(0u, 0u, 0u, 0u);
            if (!tc::net_run(*net_smem(), model, xin, phase, tid, acc3)) {
                tc_failed = true;
                break;
            }
        } else {
            learned_mlp_int(model, learned_inputs<T>(r, la.rs), acc3);
        }
        if (!valid) continue;
        T p[7];
        predict7<PRED>(r, true, x, y, z, geo.dx, geo.dy, geo.dz, p);
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            const int si = b + 1, px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
            const T o = __ldg(field + (size_t)s * (2 * z + pz) * fsy + (size_t)s * (2 * y + py) * fsx +
                              (size_t)s * (2 * x + px));
            const int c0 = quantize(A::sub(o, p[b]), qp);
            const int c1 = quantize(A::sub(o, A::add(p[b], A::mul((T)acc3[b], la.so))), qp);
            const int k0 = c0 == 0 ? kEvalBins - 1 : min(max(c0 - lo, -1), kEvalBins - 1);
            const int k1 = c1 == 0 ? kEvalBins - 1 : min(max(c1 - lo, -1), kEvalBins - 1);
            atomicAdd(&h[0][b][k0 < 0 ? kEvalBins - 1 : k0], 1u);
            atomicAdd(&h[1][b][k1 < 0 ? kEvalBins - 1 : k1], 1u);
        }
    }
    if constexpr (LM == kLearnTc) {
        tc::net_teardown(*net_smem(), tid);
        if (tc_failed && tid == 0) atomicOr(&g_learned_tc_error, 1u);
    }
    __syncthreads();
    for (int i = tid; i < 2 * 7 * kEvalBins; i += blockDim.x) {
        const uint32_t c = (&h[0][0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

// The kernel's dynamic shared memory (its static arrays come on top; above 48
// KB in total the launch needs this opt-in).
template <class K>
void allow_smem(K kernel, size_t bytes)
{
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // the whole unified L1 / shared array as shared memory: five finest-encode
    // CTAs (45.6 KB each) fit only in the largest carveout
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled_fn()
{
    static const EncodeTiledFn f = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return f;
}

// The f32 quantizer table is the default; STZ_QUANT_TABLE=0 sends every
// non-centre residual through quantize_full (same codes), for comparisons.
bool quant_table_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("STZ_QUANT_TABLE");
        return !(e && std::strcmp(e, "0") == 0);
    }();
    return on;
}

// TMA staging is the default; STZ_TILE_LOAD=threads loads the tile with the
// CTA's threads (same tile, for comparisons).
bool tma_tiles_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("STZ_TILE_LOAD");
        return !(e && std::strcmp(e, "threads") == 0);
    }();
    return on;
}

// Tensor map of a coarse grid for the halo tile of zb-deep bricks; false when
// the TMA cannot serve it (grid or row not 16-byte aligned, no driver entry
// point), and the threads load the tile instead.
template <typename T>
bool make_tile_map(const T* R, int dx, int dy, int dz, int zb, CUtensorMap* m)
{
    if (!tma_tiles_enabled() || !R) return false;
    if ((uintptr_t)R % 16 || ((size_t)dx * sizeof(T)) % 16) return false;
    const EncodeTiledFn f = encode_tiled_fn();
    if (!f) return false;
    const cuuint64_t gdim[3] = {(cuuint64_t)dx, (cuuint64_t)dy, (cuuint64_t)dz};
    const cuuint64_t gstride[2] = {(cuuint64_t)dx * sizeof(T), (cuuint64_t)dx * dy * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)TSX, (cuuint32_t)TSY, (cuuint32_t)(zb + 3)};
    const cuuint32_t estride[3] = {1, 1, 1};
    return f(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)R, gdim,
             gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Staged predictor: three dependent launches per level (staged_kernels.cuh);
// a.decoded is the decoded fine grid, a scratch grid on the finest level.
template <typename T>
void launch_staged_encode(const LevelEncodeArgs<T>& a, cudaStream_t st)
{
    const HistArgs h{a.hist_full, a.hist_outside, a.qp.radius};
    const EncodeIO<T> io{a.field, a.fsx, a.fsy, a.stride, a.codes, a.unpred_dense, a.unpred_cnt, a.decoded};
    const dim3 grd = staged_grid(a.geo), blk(kStagedTX, kStagedTY);
    k_staged_encode<T, 1><<<grd, blk, 0, st>>>(io, a.decoded, a.coarse, a.geo, a.qp, h);
    k_staged_encode<T, 2><<<grd, blk, 0, st>>>(io, a.decoded, a.coarse, a.geo, a.qp, h);
    k_staged_encode<T, 3><<<grd, blk, 0, st>>>(io, a.decoded, a.coarse, a.geo, a.qp, h);
}

template <typename T>
void launch_staged_decode(const LevelDecodeArgs<T>& a, cudaStream_t st)
{
    const dim3 grd = staged_grid(a.geo), blk(kStagedTX, kStagedTY);
    k_staged_decode<T, 1><<<grd, blk, 0, st>>>(a.coarse, a.geo, a.qp, a.codes, a.unpred_dense, a.out);
    k_staged_decode<T, 2><<<grd, blk, 0, st>>>(a.coarse, a.geo, a.qp, a.codes, a.unpred_dense, a.out);
    k_staged_decode<T, 3><<<grd, blk, 0, st>>>(a.coarse, a.geo, a.qp, a.codes, a.unpred_dense, a.out);
}

template <typename T>
void launch_level_encode(const LevelEncodeArgs<T>& a, cudaStream_t st)
{
    if (a.predictor == 2) {
        launch_staged_encode(a, st);
        return;
    }
    if (a.predictor == 3) {  // one global-tap pass (trunc_kernels.cuh)
        const HistArgs h{a.hist_full, a.hist_outside, a.qp.radius};
        const EncodeIO<T> io{a.field, a.fsx, a.fsy, a.stride, a.codes, a.unpred_dense, a.unpred_cnt, a.decoded};
        k_trunc_encode<T><<<trunc_grid(a.geo), dim3(kTruncTX, kTruncTY), 0, st>>>(io, a.coarse, a.geo, a.qp, h);
        return;
    }
    const LevelGeom& g = a.geo;
    const Shell shell = Shell::make(g.dx, g.dy, g.dz);
    dim3 blk(BX, BY, 1);
    const bool learned = a.learned.model && a.learned.flags;
    const size_t npts = (size_t)g.dx * g.dy * g.dz;
    const bool big = !learned && npts >= kZBigPoints;
    const bool tiny = !learned && npts <= kZTinyPoints;
    const int zb = big ? kZBig : tiny ? kZTiny : kZSmall;
    dim3 grd((shell.nix + BX - 1) / BX, (shell.niy + BY - 1) / BY, (shell.niz + zb - 1) / zb);
    const bool interior = shell.nix > 0 && shell.niy > 0 && shell.niz > 0;
    HistArgs h{a.hist_full, a.hist_outside, a.qp.radius};
    const EncodeIO<T> io{a.field, a.fsx, a.fsy, a.stride, a.codes, a.unpred_dense, a.unpred_cnt, a.decoded};
    const size_t sm = learned ? kTileBytesAligned<T> + sizeof(LearnedModel)
                      : big   ? tile_bytes<T, kZBig>()
                      : tiny  ? tile_bytes<T, kZTiny>()
                              : tile_bytes<T>();
    // the boundary shell runs beside the interior on the side stream (folding
    // all of it into the interior CTAs, as the decoder does, left the finest
    // encode level and slowed the coarser ones, whose shells are a large share
    // and whose z-plane CTAs run last). The finest level's plain interior
    // kernel takes the x-boundary columns itself: their owners are spread over
    // the launch, and a column point per shell thread read the field and grid
    // uncoalesced (142 -> 15 MB of shell traffic at 512^3).
    Shell shell_k = shell;
    if (interior && !learned && a.stride == 1) shell_k.g3 = 0;
    const uint64_t ns = shell_k.total();
    const int gs = (int)std::min<uint64_t>((ns + 255) / 256, 148 * 16);
    const bool par = a.side.st && interior && ns;
    cudaStream_t ss = par ? a.side.st : st;
    if (par) {
        cudaEventRecord(a.side.fork, st);
        cudaStreamWaitEvent(ss, a.side.fork, 0);
    }
    alignas(64) CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    const int use_tma = interior && make_tile_map(a.coarse, g.dx, g.dy, g.dz, zb, &tmap) ? 1 : 0;
    QuantTable qt{};
    if (std::is_same<T, float>::value && interior && !learned && quant_table_enabled()) qt = make_quant_table(a.qp);
#define STZ_ENC(P, F)                                                                                              \
    do {                                                                                                           \
        if (ns && par) k_level_encode_shell<T, P, F><<<gs, 256, 0, ss>>>(io, a.coarse, g, a.qp, h, shell_k);       \
        if (interior) {                                                                                            \
            auto kern = big                          ? k_level_encode<T, P, F, kLearnNone, kZBig>                  \
                        : tiny                   ? k_level_encode<T, P, F, kLearnNone, kZTiny>                 \
                        : !learned               ? k_level_encode<T, P, F, kLearnNone>                         \
                        : a.learned.tensor_cores ? k_level_encode<T, P, F, kLearnTc>                           \
                                                 : k_level_encode<T, P, F, kLearnDp4a>;                        \
            allow_smem(kern, sm);                                                                                  \
            kern<<<grd, blk, sm, st>>>(io, a.coarse, g, a.qp, h, a.learned, tmap, use_tma, qt);                    \
        }                                                                                                          \
        if (ns && !par) k_level_encode_shell<T, P, F><<<gs, 256, 0, st>>>(io, a.coarse, g, a.qp, h, shell_k);      \
    } while (0)
    const bool finest = a.stride == 1;
    if (a.predictor == 1) {
        if (finest) STZ_ENC(1, true);
        else STZ_ENC(1, false);
    } else {
        if (finest) STZ_ENC(0, true);
        else STZ_ENC(0, false);
    }
#undef STZ_ENC
    if (par) {
        cudaEventRecord(a.side.join, ss);
        cudaStreamWaitEvent(st, a.side.join, 0);
    }
}

template <typename T>
void launch_level_decode(const LevelDecodeArgs<T>& a, cudaStream_t st)
{
    if (a.predictor == 2) {  // whole level (level_decode_bricks: none)
        launch_staged_decode(a, st);
        return;
    }
    if (a.predictor == 3) {  // whole level
        k_trunc_decode<T><<<trunc_grid(a.geo), dim3(kTruncTX, kTruncTY), 0, st>>>(a.coarse, a.geo, a.qp, a.codes,
                                                                                  a.unpred_dense, a.out);
        return;
    }
    const LevelGeom& g = a.geo;
    const Shell shell = Shell::make(g.dx, g.dy, g.dz);
    dim3 blk(BX, BY, 1);
    const bool learned = a.learned.model && a.learned.flags;
    const size_t npts = (size_t)g.dx * g.dy * g.dz;
    const bool big = !learned && npts >= kZBigPoints;
    const bool tiny = !learned && npts <= kZTinyPoints;
    const int zb = big ? kZBig : tiny ? kZTiny : kZSmall;
    dim3 grd((shell.nix + BX - 1) / BX, (shell.niy + BY - 1) / BY, (shell.niz + zb - 1) / zb);
    const bool interior = shell.nix > 0 && shell.niy > 0 && shell.niz > 0;
    const int nzb = (int)grd.z;
    int zoff = 0;
    if (!learned && interior && a.zb_hi >= 0) {  // a range of z-bricks
        zoff = std::min(std::max(a.zb_lo, 0), nzb);
        const int zhi = std::min(std::max(a.zb_hi, zoff), nzb);
        if (zhi == zoff) return;
        grd.z = (unsigned)(zhi - zoff);
    }
    const size_t sm = learned ? kTileBytesAligned<T> + sizeof(LearnedModel)
                      : big   ? tile_bytes<T, kZBig>()
                      : tiny  ? tile_bytes<T, kZTiny>()
                              : tile_bytes<T>();
    // plain decode kernels predict their owned boundary points themselves
    // from the halo tile; the shell kernel serves learned levels and levels
    // without an interior
    const uint64_t ns = (interior && !learned) ? 0 : shell.total();
    const int gs = (int)std::min<uint64_t>((ns + 255) / 256, 148 * 16);
    const bool par = a.side.st && interior && ns;
    cudaStream_t ss = par ? a.side.st : st;
    if (par) {
        cudaEventRecord(a.side.fork, st);
        cudaStreamWaitEvent(ss, a.side.fork, 0);
    }
    alignas(64) CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    const int use_tma = interior && make_tile_map(a.coarse, g.dx, g.dy, g.dz, zb, &tmap) ? 1 : 0;
#define STZ_DEC(P)                                                                                                 \
    do {                                                                                                           \
        if (ns && par)                                                                                             \
            k_level_decode_shell<T, P><<<gs, 256, 0, ss>>>(a.coarse, g, a.qp, a.codes, a.unpred_dense, a.out, shell); \
        if (interior) {                                                                                            \
            auto kern = big                          ? k_level_decode<T, P, kLearnNone, kZBig>                     \
                        : tiny                   ? k_level_decode<T, P, kLearnNone, kZTiny>                    \
                        : !learned               ? k_level_decode<T, P, kLearnNone>                            \
                        : a.learned.tensor_cores ? k_level_decode<T, P, kLearnTc>                              \
                                                 : k_level_decode<T, P, kLearnDp4a>;                           \
            allow_smem(kern, sm);                                                                                  \
            kern<<<grd, blk, sm, st>>>(a.coarse, g, a.qp, a.codes, a.unpred_dense, a.out, a.learned, tmap, use_tma,   \
                                       zoff, nzb);                                                                 \
        }                                                                                                          \
        if (ns && !par)                                                                                            \
            k_level_decode_shell<T, P><<<gs, 256, 0, st>>>(a.coarse, g, a.qp, a.codes, a.unpred_dense, a.out, shell); \
    } while (0)
    if (a.predictor == 1) STZ_DEC(1);
    else STZ_DEC(0);
#undef STZ_DEC
    if (par) {
        cudaEventRecord(a.side.join, ss);
        cudaStreamWaitEvent(st, a.side.join, 0);
    }
}

int level_decode_bricks(const LevelGeom& g, bool learned, int zlim, int* below)
{
    const Shell shell = Shell::make(g.dx, g.dy, g.dz);
    const bool interior = shell.nix > 0 && shell.niy > 0 && shell.niz > 0;
    if (learned || !interior) {
        if (below) *below = 0;
        return 0;
    }
    const size_t npts = (size_t)g.dx * g.dy * g.dz;
    const int zb = npts >= kZBigPoints ? kZBig : npts <= kZTinyPoints ? kZTiny : kZSmall;
    const int n = (shell.niz + zb - 1) / zb;
    if (below) *below = std::max(0, std::min(n - 1, (zlim - 1) / zb));
    return n;
}

template <typename T>
void launch_learned_eval(const LevelEncodeArgs<T>& a, uint32_t* hist, cudaStream_t st)
{
    const LevelGeom& g = a.geo;
    const int sx = g.dx > 2 ? (g.dx - 2) / 2 : 0, sy = g.dy > 2 ? (g.dy - 2) / 2 : 0,
              sz = g.dz > 2 ? (g.dz - 2) / 2 : 0;
    const uint64_t total = (uint64_t)sx * sy * sz;
    if (!total || !a.learned.model) return;
    const int gs = (int)std::min<uint64_t>((total + 255) / 256, 148 * 8);
    const bool tcm = a.learned.tensor_cores;
    auto kern = a.predictor == 1 ? (tcm ? k_learned_eval<T, 1, kLearnTc> : k_learned_eval<T, 1, kLearnDp4a>)
                                 : (tcm ? k_learned_eval<T, 0, kLearnTc> : k_learned_eval<T, 0, kLearnDp4a>);
    kern<<<gs, 256, 0, st>>>(a.field, a.fsx, a.fsy, a.stride, a.coarse, g, a.qp, a.learned, sx, sy, sz, hist);
}

template <typename T>
void launch_subsample(const T* field, int nx, int ny, int nz, int s, T* out, cudaStream_t st)
{
    const int ox = nx / s, oy = ny / s, oz = nz / s;
    const size_t n = (size_t)ox * oy * oz;
    k_subsample<T><<<grid_for(n, 256), 256, 0, st>>>(field, (size_t)nx, (size_t)nx * ny, s, ox, oy, oz, out);
}

template <typename T>
void launch_minmax(const T* p, size_t n, double* out2, cudaStream_t st)
{
    // out2 holds order-preserving keys; init to (max key, min key)
    const unsigned long long init[2] = {~0ull, 0ull};
    cudaMemcpyAsync(out2, init, sizeof(init), cudaMemcpyHostToDevice, st);
    k_minmax<T><<<148 * 8, 256, 0, st>>>(p, n, out2);
}

double minmax_key_to_double(unsigned long long k)
{
    long long b = (k & 0x8000000000000000ull) ? (long long)(k & 0x7fffffffffffffffull) : (long long)~k;
    double d;
    memcpy(&d, &b, sizeof(d));
    return d;
}

template <typename T>
void launch_split(const T* full, int nx, int ny, int nz, T* subs, cudaStream_t st)
{
    const size_t hn = (size_t)(nx / 2) * (ny / 2) * (nz / 2);
    k_split<T><<<grid_for(hn, 256), 256, 0, st>>>(full, nx, ny, nz, subs);
}

template <typename T>
void launch_merge(const T* subs, int hx, int hy, int hz, T* full, cudaStream_t st)
{
    const size_t hn = (size_t)hx * hy * hz;
    k_merge<T><<<grid_for(hn, 256), 256, 0, st>>>(subs, hx, hy, hz, full);
}

template <typename T>
void launch_block_op(int mode, int predictor, int block, const T* src, const T* ref, T* dst, int dx, int dy, int dz,
                     int x0, int x1, int y0, int y1, int z0, int z1, cudaStream_t st)
{
    const size_t m = (size_t)(x1 - x0) * (y1 - y0) * (z1 - z0);
    if (m == 0) return;
    const Grid<T> R = make_grid(ref, dx, dy, dz);
    if (predictor == 1)
        k_block_op<T, 1><<<grid_for(m, 256), 256, 0, st>>>(mode, block, src, R, dst, x0, x1, y0, y1, z0, z1);
    else
        k_block_op<T, 0><<<grid_for(m, 256), 256, 0, st>>>(mode, block, src, R, dst, x0, x1, y0, y1, z0, z1);
}

template <typename T>
void launch_block_staged(int mode, int block, const T* src, const void* const refs[6], T* dst, int dx, int dy, int dz,
                         cudaStream_t st)
{
    const size_t m = (size_t)dx * dy * dz;
    if (m == 0) return;
    StagedRefs r;
    for (int k = 0; k < 6; ++k) r.p[k] = refs[k];
    k_block_staged<T><<<grid_for(m, 256), 256, 0, st>>>(mode, block, src, r, dst, dx, dy, dz);
}

template <typename T>
void launch_quantize(const T* d, size_t n, QuantParams qp, int* q, T* unpred, uint32_t* tile_cnt, uint64_t* tile_off,
                     cudaStream_t st)
{
    const size_t tiles = (n + 1023) / 1024;
    if (!tiles) return;
    k_quantize<T><<<(unsigned)tiles, 1024, 0, st>>>(d, n, qp, q, tile_cnt);
    k_scan_tiles<<<1, 1024, 0, st>>>(tile_cnt, tiles, tile_off);
    k_quantize_unpred<T><<<(unsigned)tiles, 1024, 0, st>>>(d, n, q, tile_off, unpred);
}

template <typename T>
void launch_dequantize(const int* q, size_t n, QuantParams qp, const T* unpred, T* out, uint32_t* tile_cnt,
                       uint64_t* tile_off, cudaStream_t st)
{
    const size_t tiles = (n + 1023) / 1024;
    if (!tiles) return;
    k_dequant_count<<<(unsigned)tiles, 1024, 0, st>>>(q, n, tile_cnt);
    k_scan_tiles<<<1, 1024, 0, st>>>(tile_cnt, tiles, tile_off);
    k_dequantize<T><<<(unsigned)tiles, 1024, 0, st>>>(q, n, qp, tile_off, unpred, out);
}

#define STZ_INST(T)                                                                                                 \
    template void launch_level_encode<T>(const LevelEncodeArgs<T>&, cudaStream_t);                                  \
    template void launch_level_decode<T>(const LevelDecodeArgs<T>&, cudaStream_t);                                  \
    template void launch_learned_eval<T>(const LevelEncodeArgs<T>&, uint32_t*, cudaStream_t);                       \
    template void launch_subsample<T>(const T*, int, int, int, int, T*, cudaStream_t);                              \
    template void launch_minmax<T>(const T*, size_t, double*, cudaStream_t);                                        \
    template void launch_split<T>(const T*, int, int, int, T*, cudaStream_t);                                       \
    template void launch_merge<T>(const T*, int, int, int, T*, cudaStream_t);                                       \
    template void launch_block_op<T>(int, int, int, const T*, const T*, T*, int, int, int, int, int, int, int, int, \
                                     int, cudaStream_t);                                                            \
    template void launch_block_staged<T>(int, int, const T*, const void* const*, T*, int, int, int, cudaStream_t);  \
    template void launch_quantize<T>(const T*, size_t, QuantParams, int*, T*, uint32_t*, uint64_t*, cudaStream_t);  \
    template void launch_dequantize<T>(const int*, size_t, QuantParams, const T*, T*, uint32_t*, uint64_t*,         \
                                       cudaStream_t);
STZ_INST(float)
STZ_INST(double)

}  // namespace stz
