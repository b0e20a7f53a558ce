// Level kernels of the STZ hierarchy on B200.
//
// Encode (one launch per level): each thread owns one coarse point (x,y,z) of
// a level and handles all 8 parity positions of the 2x2x2 cell above it. It
// reads the original fine values straight from the input field (the
// hierarchical split, FD5:107-139, is never materialised: level k reads the
// field at stride 2^(K-k)), predicts the 7 odd-parity sub-blocks from the
// decoded coarse grid (FD5:1005-1047 / 690-748), quantizes the residuals
// (FD5:1204-1253), writes the codes in chunk-major order for the entropy
// coder, builds the per-stream code histogram, and, for every level but the
// finest, writes the decoded fine grid the next level predicts from (the
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
#include <cstring>

#include <cuda_runtime.h>

#include "levels.h"
#include "stz_device.cuh"

namespace stz {
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

__device__ __forceinline__ size_t chunk_major(const LevelGeom& g, int x, int y, int z, int& chunk)
{
    const int C = g.C;
    const int cx = x / C, cy = y / C, cz = z / C;
    chunk = (cz * g.ncy + cy) * g.ncx + cx;
    const int lx = x - cx * C, ly = y - cy * C, lz = z - cz * C;
    return (size_t)chunk * C * C * C + (size_t)(lz * C + ly) * C + lx;
}

constexpr int kSmemBins = 1024;

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

// Warp-aggregated histogram update: one atomic per distinct code in the warp.
__device__ __forceinline__ void hist_warp(uint32_t (*sh)[kSmemBins], int wlo, int wn, const HistArgs& h, int b, int key)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int k0 = __shfl_sync(full, key, 0);
    if (__all_sync(full, key == k0)) {
        if (lane == 0 && k0 >= 0) hist_add(sh, wlo, wn, h, b, k0, 32u);
        return;
    }
    const unsigned peers = __match_any_sync(full, key);
    if (key >= 0 && lane == __ffs(peers) - 1) hist_add(sh, wlo, wn, h, b, key, (uint32_t)__popc(peers));
}

template <typename T, int PRED, bool FINEST>
__global__ void __launch_bounds__(256) k_level_encode(const T* __restrict__ field, size_t fsx, size_t fsy, int s,
                                                      Grid<T> R, LevelGeom geo, QuantParams qp,
                                                      uint16_t* __restrict__ codes, T* __restrict__ unpred_dense,
                                                      uint32_t* __restrict__ unpred_cnt, HistArgs hist,
                                                      T* __restrict__ G, size_t gsx, size_t gsy, int zper)
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    __shared__ uint32_t sh[7][kSmemBins];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < 7 * kSmemBins; i += blockDim.x * blockDim.y) (&sh[0][0])[i] = 0;
    const int wlo = max(0, qp.radius - kSmemBins / 2);
    const int wn = min(kSmemBins, 2 * qp.radius - wlo);
    __syncthreads();

    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const bool valid = x < geo.dx && y < geo.dy;
    const int z0 = blockIdx.z * zper, z1 = min(z0 + zper, geo.dz);
    const size_t n = geo.n;
    const int nch1 = geo.nchunks() + 1;

    for (int z = z0; z < z1; ++z) {
        T o[8];
        T v[8];
        int q[7];
        if (valid) {
            if constexpr (FINEST) {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int pz = r >> 1, py = r & 1;
                    const T2 t = *reinterpret_cast<const T2*>(field + (size_t)(2 * z + pz) * fsy +
                                                              (size_t)(2 * y + py) * fsx + 2 * (size_t)x);
                    o[2 * r] = t.x;
                    o[2 * r + 1] = t.y;
                }
            } else {
#pragma unroll
                for (int si = 1; si < 8; ++si) {
                    const int px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
                    o[si] = __ldg(field + (size_t)(s * (2 * z + pz)) * fsy + (size_t)(s * (2 * y + py)) * fsx +
                                  (size_t)s * (2 * x + px));
                }
            }
            int chunk;
            const size_t cm = chunk_major(geo, x, y, z, chunk);
#pragma unroll
            for (int b = 0; b < 7; ++b) {
                const T p = predict<PRED>(b, R, x, y, z);
                const T d = A::sub(o[b + 1], p);
                T dec;
                const int code = quantize(d, qp, dec);
                q[b] = code;
                codes[(size_t)b * n + cm] = (uint16_t)code;
                if (code == 0) {
                    unpred_dense[(size_t)b * n + cm] = d;
                    atomicAdd(&unpred_cnt[(size_t)b * nch1 + chunk], 1u);
                }
                if (G) v[b + 1] = A::add(code ? recover<T>(code, qp) : d, p);
            }
            if (G) {
                v[0] = R.at((size_t)z * R.sy + (size_t)y * R.sx + x);
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int pz = r >> 1, py = r & 1;
                    T2 t;
                    t.x = v[2 * r];
                    t.y = v[2 * r + 1];
                    *reinterpret_cast<T2*>(G + (size_t)(2 * z + pz) * gsy + (size_t)(2 * y + py) * gsx + 2 * (size_t)x) = t;
                }
            }
        } else {
#pragma unroll
            for (int b = 0; b < 7; ++b) q[b] = -1;
        }
#pragma unroll
        for (int b = 0; b < 7; ++b) hist_warp(sh, wlo, wn, hist, b, q[b]);
    }
    __syncthreads();
    for (int i = tid; i < 7 * kSmemBins; i += blockDim.x * blockDim.y) {
        const int b = i / kSmemBins, w = i % kSmemBins;
        const uint32_t c = sh[b][w];
        if (c) atomicAdd(&hist.full[(size_t)b * 2 * hist.radius + wlo + w], c);
    }
}

template <typename T, int PRED>
__global__ void __launch_bounds__(256) k_level_decode(Grid<T> R, LevelGeom geo, QuantParams qp,
                                                      const uint16_t* __restrict__ codes,
                                                      const T* __restrict__ unpred_dense, T* __restrict__ G,
                                                      size_t gsx, size_t gsy, int zper)
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= geo.dx || y >= geo.dy) return;
    const int z0 = blockIdx.z * zper, z1 = min(z0 + zper, geo.dz);
    const size_t n = geo.n;
    for (int z = z0; z < z1; ++z) {
        int chunk;
        const size_t cm = chunk_major(geo, x, y, z, chunk);
        T v[8];
        v[0] = R.at((size_t)z * R.sy + (size_t)y * R.sx + x);
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            const int code = __ldg(codes + (size_t)b * n + cm);
            const T dq = code ? recover<T>(code, qp) : __ldg(unpred_dense + (size_t)b * n + cm);
            v[b + 1] = A::add(dq, predict<PRED>(b, R, x, y, z));
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int pz = r >> 1, py = r & 1;
            T2 t;
            t.x = v[2 * r];
            t.y = v[2 * r + 1];
            *reinterpret_cast<T2*>(G + (size_t)(2 * z + pz) * gsy + (size_t)(2 * y + py) * gsx + 2 * (size_t)x) = t;
        }
    }
}

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

// Value range (max - min in double) of a field, as computeRange (FD5:92-104).
template <typename T>
__global__ void k_minmax(const T* __restrict__ p, size_t n, double* out)
{
    double lo = __longlong_as_double(0x7fefffffffffffffll), hi = -lo;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = (double)p[i];
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    for (int o = 16; o; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ double slo[32], shi[32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) slo[w] = lo, shi[w] = hi;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) lo = fmin(lo, slo[i]), hi = fmax(hi, shi[i]);
        // doubles compare as signed integers after a sign-magnitude fix-up
        unsigned long long* u = reinterpret_cast<unsigned long long*>(out);
        auto key = [](double d) {
            long long b = __double_as_longlong(d);
            return (unsigned long long)(b < 0 ? ~b : (b | 0x8000000000000000ll));
        };
        atomicMin(&u[0], key(lo));
        atomicMax(&u[1], key(hi));
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
        T p;
        switch (block) {
        case 0: p = predict<PRED>(0, R, x, y, z); break;
        case 1: p = predict<PRED>(1, R, x, y, z); break;
        case 2: p = predict<PRED>(2, R, x, y, z); break;
        case 3: p = predict<PRED>(3, R, x, y, z); break;
        case 4: p = predict<PRED>(4, R, x, y, z); break;
        case 5: p = predict<PRED>(5, R, x, y, z); break;
        default: p = predict<PRED>(6, R, x, y, z); break;
        }
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
        T dec;
        code = quantize(d[i], qp, dec);
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

template <typename T>
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

}  // namespace

template <typename T>
void launch_level_encode(const LevelEncodeArgs<T>& a, cudaStream_t st)
{
    const LevelGeom& g = a.geo;
    const int zper = 8;
    dim3 blk(32, 8, 1);
    dim3 grd((g.dx + 31) / 32, (g.dy + 7) / 8, (g.dz + zper - 1) / zper);
    const Grid<T> R = make_grid(a.coarse, g.dx, g.dy, g.dz);
    HistArgs h{a.hist_full, a.hist_outside, a.qp.radius};
    const size_t gsx = 2 * (size_t)g.dx, gsy = 4 * (size_t)g.dx * g.dy;
#define STZ_ENC(P, F)                                                                                            \
    k_level_encode<T, P, F><<<grd, blk, 0, st>>>(a.field, a.fsx, a.fsy, a.stride, R, g, a.qp, a.codes,          \
                                                 a.unpred_dense, a.unpred_cnt, h, a.decoded, gsx, gsy, zper)
    const bool finest = a.stride == 1;
    if (a.predictor == 1) {
        if (finest) STZ_ENC(1, true);
        else STZ_ENC(1, false);
    } else {
        if (finest) STZ_ENC(0, true);
        else STZ_ENC(0, false);
    }
#undef STZ_ENC
}

template <typename T>
void launch_level_decode(const LevelDecodeArgs<T>& a, cudaStream_t st)
{
    const LevelGeom& g = a.geo;
    const int zper = 8;
    dim3 blk(32, 8, 1);
    dim3 grd((g.dx + 31) / 32, (g.dy + 7) / 8, (g.dz + zper - 1) / zper);
    const Grid<T> R = make_grid(a.coarse, g.dx, g.dy, g.dz);
    const size_t gsx = 2 * (size_t)g.dx, gsy = 4 * (size_t)g.dx * g.dy;
    if (a.predictor == 1)
        k_level_decode<T, 1><<<grd, blk, 0, st>>>(R, g, a.qp, a.codes, a.unpred_dense, a.out, gsx, gsy, zper);
    else
        k_level_decode<T, 0><<<grd, blk, 0, st>>>(R, g, a.qp, a.codes, a.unpred_dense, a.out, gsx, gsy, zper);
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
    k_minmax<T><<<grid_for(n, 256), 256, 0, st>>>(p, n, out2);
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
    k_dequant_count<T><<<(unsigned)tiles, 1024, 0, st>>>(q, n, tile_cnt);
    k_scan_tiles<<<1, 1024, 0, st>>>(tile_cnt, tiles, tile_off);
    k_dequantize<T><<<(unsigned)tiles, 1024, 0, st>>>(q, n, qp, tile_off, unpred, out);
}

#define STZ_INST(T)                                                                                                 \
    template void launch_level_encode<T>(const LevelEncodeArgs<T>&, cudaStream_t);                                  \
    template void launch_level_decode<T>(const LevelDecodeArgs<T>&, cudaStream_t);                                  \
    template void launch_subsample<T>(const T*, int, int, int, int, T*, cudaStream_t);                              \
    template void launch_minmax<T>(const T*, size_t, double*, cudaStream_t);                                        \
    template void launch_split<T>(const T*, int, int, int, T*, cudaStream_t);                                       \
    template void launch_merge<T>(const T*, int, int, int, T*, cudaStream_t);                                       \
    template void launch_block_op<T>(int, int, int, const T*, const T*, T*, int, int, int, int, int, int, int, int, \
                                     int, cudaStream_t);                                                            \
    template void launch_quantize<T>(const T*, size_t, QuantParams, int*, T*, uint32_t*, uint64_t*, cudaStream_t);  \
    template void launch_dequantize<T>(const int*, size_t, QuantParams, const T*, T*, uint32_t*, uint64_t*,         \
                                       cudaStream_t);
STZ_INST(float)
STZ_INST(double)

}  // namespace stz
