// Chunk-indexed canonical Huffman coding of the quant codes on B200.
//
// The reference entropy-codes each residual stream with SZ3-ncp's
// HuffmanEncoder<int> and a per-chunk "marker" table of bit offsets
// (encode_marked_fast / decode_marked_transform / decode_marked_chunks_fast,
// call sites FD5:1264-1306, 1401-1413, 1512-1562, 1870-1875). That library is
// not available, so the byte format here is this project's own; the roles are
// the same: a codebook per stream, codes grouped in C^3 marker chunks with a
// word offset per chunk (the marker table), so any chunk decodes on its own.
//
// Parallel decomposition: every z-plane of a chunk (C^2 symbols, a
// "sub-chunk") has its bit offset inside the chunk in the stream header, so
// all planes of all chunks of all streams encode and decode independently.
// Inside a plane, a group of lanes shares the work: the encode side splits
// the codes into lane segments (runs are the gaps between literal masks),
// the decoder splits the bits into lane slices and resynchronises them
// (a dense stream in a large launch is decoded one thread per plane
// instead). Bits are packed MSB-first into 32-bit words; a chunk starts on a
// word boundary.
//
// Runs: inside a plane, a maximal run of r centre codes (code == radius) is
// coded with run symbols (run_geometry): while r > D, 2^k (the largest power
// of two <= r, k <= J) when k > LD, else D codes; then one symbol for the
// remaining 2..D codes, or the centre code itself for one. The run symbols
// occupy run_n code values the stream does not use (StreamDesc::run_base),
// so they share the codebook, the tables and the 16-bit symbol width with
// the codes; a well-predicted stream (mostly centre codes) then costs well
// under one bit per code.
#include <cstdlib>

#include <cuda_runtime.h>

#include "huffman.h"

namespace stz {
namespace {

// Canonical codes from the (length, symbol)-sorted list: first code of each
// length by the usual recurrence, then rank within the length.
__global__ void k_expand_codebook(const StreamDesc* __restrict__ sd, const uint16_t* __restrict__ cb_sym,
                                  const uint8_t* __restrict__ cb_len, uint32_t* __restrict__ ctab)
{
    const StreamDesc s = sd[blockIdx.x];
    __shared__ uint32_t cnt[kMaxCodeLen + 1];
    __shared__ uint32_t first_code[kMaxCodeLen + 1];
    __shared__ uint32_t first_idx[kMaxCodeLen + 1];
    if (threadIdx.x <= kMaxCodeLen) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < s.n_used; i += blockDim.x) atomicAdd(&cnt[cb_len[s.cb_off + i]], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t code = 0, idx = cnt[0];
        first_code[0] = 0;
        first_idx[0] = 0;
        for (int l = 1; l <= kMaxCodeLen; ++l) {
            code = (code + (l > 1 ? cnt[l - 1] : 0)) << 1;
            first_code[l] = code;
            first_idx[l] = idx;
            idx += cnt[l];
        }
    }
    __syncthreads();
    uint32_t* tab = ctab + (size_t)blockIdx.x * 2 * s.radius;
    for (uint32_t i = threadIdx.x; i < s.n_used; i += blockDim.x) {
        const uint32_t l = cb_len[s.cb_off + i];
        const uint32_t code = l ? first_code[l] + (i - first_idx[l]) : 0;
        tab[cb_sym[s.cb_off + i]] = (code << 5) | l;
    }
}

// ---- encode side: a lane group per plane ----------------------------------------
// (Planes of up to 1024 codes take the literal lists below; this segment form
// serves larger planes.)
// Lane i of a group of W lanes (W = 32 for planes of 1024 codes and more,
// fewer for smaller planes, see lanes_per_plane) owns the codes [a_i, b_i) of
// the plane (W consecutive segments of S = ceil(plane / W) codes). A run of centre codes is coded by
// the lane holding the literal that follows it, or, for a run that reaches
// the plane's end, by the lane holding the plane's last code (`tail`): a
// warp max-scan of the lanes' last literal positions gives every lane the
// centre codes just before its segment (`lead`), which belong to the run
// leading into its first literal. The lanes' bit counts, an exclusive warp
// scan of them and the plane's bit offset place every lane's bits, so the
// bitstream is the one a sequential pass over the plane writes.
constexpr int kLaneThreads = 256;  // 8 warps per CTA, each one plane at a time
constexpr int kPlaneSlices = 4;    // CTAs per work item (gridDim.y)

// Symbols of a run of r centre codes (none for r = 0), in order: while
// r > D, 2^k (the largest power of two <= r, k <= J) when k > LD, else D
// codes; then the symbol of the remaining 2..D codes, or the centre code.
template <class F>
__device__ __forceinline__ void run_symbols(uint32_t r, uint32_t R, uint32_t base, uint32_t J, uint32_t D, uint32_t LD,
                                            F&& f)
{
    while (r > D) {
        const uint32_t k = min((uint32_t)(31 - __clz(r)), J);
        if (k > LD) {
            f(base + D - 1 + (k - LD - 1));
            r -= 1u << k;
        } else {
            f(base + D - 2);
            r -= D;
        }
    }
    if (r >= 2) f(base + r - 2);
    else if (r) f(R);
}

// Lanes per plane: the largest power of two <= plane / 32, at most 32, so a
// lane holds about 32 codes; a warp takes 32 / W planes at a time (small
// planes of the coarser levels would otherwise leave each lane a few codes
// and the per-plane lane scans would dominate).
__host__ __device__ inline uint32_t lanes_per_plane(uint32_t P)
{
    uint32_t w = 1;
    while (w < 32 && 2 * w <= P / 32) w *= 2;
    return w;
}

// A lane group's view of one plane (a group without a plane has an empty
// segment but still takes part in the group's shuffles).
struct LaneSeg {
    uint32_t P, a, b;  // plane size; this lane's codes [a, b)
    uint32_t W, lane;  // lanes of the group; this lane's index in it
    bool vec;          // segments are whole 16-byte groups of 8 codes
};

__device__ __forceinline__ LaneSeg lane_seg(uint32_t C, const uint16_t* src, uint32_t W, bool active)
{
    LaneSeg g;
    g.P = C * C;
    g.W = W;
    g.lane = threadIdx.x & (W - 1);
    const uint32_t S = (g.P + W - 1) / W;
    g.a = active ? min(g.lane * S, g.P) : 0;
    g.b = active ? min(g.a + S, g.P) : 0;
    g.vec = g.P % (8 * W) == 0 && ((uintptr_t)src & 15) == 0;
    return g;
}

// Sum over a lane group of width W (a power of two).
__device__ __forceinline__ uint32_t group_sum(uint32_t v, uint32_t W)
{
    for (uint32_t o = W >> 1; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Inclusive prefix sum over a lane group of width W.
__device__ __forceinline__ uint32_t group_scan(uint32_t v, uint32_t W, uint32_t lane)
{
    for (uint32_t o = 1; o < W; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, o, W);
        if (lane >= o) v += u;
    }
    return v;
}

// The lane's codes in order (streams without runs): f(q) for each.
template <class G>
__device__ __forceinline__ void lane_codes(const uint16_t* __restrict__ src, const LaneSeg& g, G&& f)
{
    if (g.vec) {
        const uint4* v = reinterpret_cast<const uint4*>(src + g.a);
        for (uint32_t j = 0; j < (g.b - g.a) / 8; ++j) {
            const uint4 q = __ldg(v + j);
            f(q.x & 0xffffu), f(q.x >> 16), f(q.y & 0xffffu), f(q.y >> 16);
            f(q.z & 0xffffu), f(q.z >> 16), f(q.w & 0xffffu), f(q.w >> 16);
        }
    } else {
        for (uint32_t j = g.a; j < g.b; ++j) f(__ldg(src + j));
    }
}

// Bits 0 and 1 set for the 16-bit halves of w equal to those of R2.
__device__ __forceinline__ uint32_t pair_mask(uint32_t w, uint32_t R2)
{
    const uint32_t e = __vcmpeq2(w, R2);  // 0xffff per equal half
    return (e & 1u) | ((e >> 15) & 2u);
}

// Literal mask of the n <= 32 codes at plane position p: bit i set when code
// p + i is not the centre code R (with g.vec, p and n are multiples of 8).
__device__ __forceinline__ uint32_t literal_mask(const uint16_t* __restrict__ src, const LaneSeg& g, uint32_t p,
                                                 uint32_t n, uint32_t R)
{
    uint32_t m = 0;  // centre codes
    if (g.vec) {
        const uint4* v = reinterpret_cast<const uint4*>(src + p);
        const uint32_t R2 = R | (R << 16);
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
            if (j < n / 8) {
                const uint4 q = __ldg(v + j);
                m |= (pair_mask(q.x, R2) | pair_mask(q.y, R2) << 2 | pair_mask(q.z, R2) << 4 |
                      pair_mask(q.w, R2) << 6)
                     << (8 * j);
            }
    } else {
        for (uint32_t i = 0; i < n; ++i) m |= (uint32_t)(__ldg(src + p + i) == R) << i;
    }
    return ~m & (n == 32 ? ~0u : (1u << n) - 1);
}

// A lane's plane segment with runs, as 32-code blocks: the literal mask of
// the first block is kept (most segments are one block), later ones are
// rebuilt on each pass.
struct RunLane {
    uint32_t lit0 = 0;  // literal mask of the block at a
    uint32_t lead = 0;  // centre codes between the last literal before a and a
    bool tail = false;  // the lane holds the plane's last code

    template <class F>
    __device__ __forceinline__ void blocks(const uint16_t* __restrict__ src, const LaneSeg& g, uint32_t R, F&& fn) const
    {
        for (uint32_t p = g.a; p < g.b; p += 32) {
            const uint32_t n = min(32u, g.b - p);
            fn(p, n, p == g.a ? lit0 : literal_mask(src, g, p, n, R));
        }
    }

    // Literal masks, then a group max-scan of the lanes' last literal
    // positions for lead.
    __device__ __forceinline__ void init(const uint16_t* __restrict__ src, const LaneSeg& g, uint32_t R)
    {
        uint32_t last = 0;  // last literal + 1 (0: none)
        for (uint32_t p = g.a; p < g.b; p += 32) {
            const uint32_t n = min(32u, g.b - p);
            const uint32_t lit = literal_mask(src, g, p, n, R);
            if (p == g.a) lit0 = lit;
            if (lit) last = p + 32 - __clz(lit);
        }
        for (uint32_t o = 1; o < g.W; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, last, o, g.W);
            if (g.lane >= o) last = max(last, v);
        }
        uint32_t excl = __shfl_up_sync(0xffffffffu, last, 1, g.W);
        if (g.lane == 0) excl = 0;
        lead = g.a - excl;
        tail = g.a < g.b && g.b == g.P;
    }

    // The lane's symbols in order: f(sym). Between consecutive literals of a
    // block every code is a centre code, so the runs are the gaps.
    template <class F>
    __device__ __forceinline__ void symbols(const uint16_t* __restrict__ src, const LaneSeg& g, const StreamDesc& s,
                                            F&& f) const
    {
        uint32_t D, LD;
        const uint32_t J = run_geometry(g.P, D, LD);
        uint32_t run = lead;
        blocks(src, g, s.radius, [&](uint32_t p, uint32_t n, uint32_t lit) {
            uint32_t i = 0;
            while (lit) {
                const uint32_t j = __ffs(lit) - 1;
                run += j - i;
                if (run) {
                    run_symbols(run, s.radius, s.run_base, J, D, LD, f);
                    run = 0;
                }
                f((uint32_t)__ldg(src + p + j));
                i = j + 1;
                lit &= lit - 1;
            }
            run += n - i;
        });
        if (tail && run) run_symbols(run, s.radius, s.run_base, J, D, LD, f);
    }
};

// Planes of a work item for this lane group: warp i of the grid's
// (blockDim.x / 32) * gridDim.y warps on an item takes its planes
// [i * G, i * G + G), then every (warps * G)-th group of G after that (G =
// 32 / W planes per warp); p is this group's plane, valid when active (else
// pe, a valid plane of the same warp, stands in for reads).
#define STZ_GROUP_PLANES(nplanes, W)                                                                      \
    for (uint32_t base_ = (blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 / (W));            \
         base_ < (nplanes); base_ += (blockDim.x >> 5) * gridDim.y * (32 / (W)))
#define STZ_GROUP_PLANE(nplanes, W)                                     \
    const uint32_t p = base_ + (threadIdx.x & 31) / (W);               \
    const bool active = p < (nplanes);                                 \
    const uint32_t pe = active ? p : base_

// ---- literal lists: the symbols of a run-coded plane in warp-wide rounds ----
// A lane's literals vary in number from lane to lane, so a walk over each
// lane's own literals leaves most of the warp idle. Instead the group first
// lists the plane's literal positions in plane order in shared memory (a
// group scan of the lanes' literal counts places each lane's), then visits
// them in rounds of W: literal k (lane k mod W) with the run of centre codes
// before it (the gap to literal k - 1), then the run after the last literal.
// That is the symbol order of a sequential pass over the plane. Used where a
// lane holds at most 32 codes (planes of up to 1024 codes).
constexpr uint32_t kListPerWarp = 1024;  // list entries per warp: 32 / W groups of at most 32 W codes
constexpr uint32_t kStagePerWarp = 832;  // staging words per warp: groups of at most (32 W * 24 + 63) / 32

__device__ __forceinline__ bool lits_ok(uint32_t P, uint32_t W) { return (P + W - 1) / W <= 32; }

// The group's literal positions into list[0, L) in plane order; returns L.
__device__ __forceinline__ uint32_t plane_literals(const uint16_t* __restrict__ src, const LaneSeg& g, uint32_t R,
                                                   uint16_t* list)
{
    const uint32_t n = g.b - g.a;
    const uint32_t m = n ? literal_mask(src, g, g.a, n, R) : 0u;
    const uint32_t c = __popc(m);
    const uint32_t incl = group_scan(c, g.W, g.lane);
    const uint32_t L = __shfl_sync(0xffffffffu, incl, g.W - 1, g.W);
    uint32_t j = incl - c;
    for (uint32_t mm = m; mm; mm &= mm - 1) list[j++] = (uint16_t)(g.a + (__ffs(mm) - 1));
    __syncwarp();
    return L;
}

// Rounds over the group's literals with a warp-uniform trip count (every lane
// takes part in the shuffles f may make): f(valid, pos, run).
template <class F>
__device__ __forceinline__ void literal_rounds(const uint16_t* list, uint32_t L, const LaneSeg& g, F&& f)
{
    const uint32_t rounds = __reduce_max_sync(0xffffffffu, (L + g.W - 1) / g.W);
    for (uint32_t t = 0; t < rounds; ++t) {
        const uint32_t k = t * g.W + g.lane;
        const bool valid = k < L;
        uint32_t pos = 0, run = 0;
        if (valid) {
            pos = list[k];
            run = pos - (k ? list[k - 1] + 1u : 0u);
        }
        f(valid, pos, run);
    }
}

// The same, two consecutive literals per lane per round (2 lane, 2 lane + 1
// of the round's 2W): two independent load chains per lane.
template <class F>
__device__ __forceinline__ void literal_rounds2(const uint16_t* list, uint32_t L, const LaneSeg& g, F&& f)
{
    const uint32_t rounds = __reduce_max_sync(0xffffffffu, (L + 2 * g.W - 1) / (2 * g.W));
    for (uint32_t t = 0; t < rounds; ++t) {
        const uint32_t k = t * 2 * g.W + 2 * g.lane;
        const bool v0 = k < L, v1 = k + 1 < L;
        uint32_t pos0 = 0, run0 = 0, pos1 = 0, run1 = 0;
        if (v0) {
            pos0 = list[k];
            run0 = pos0 - (k ? list[k - 1] + 1u : 0u);
        }
        if (v1) {
            pos1 = list[k + 1];
            run1 = pos1 - pos0 - 1u;
        }
        f(v0, pos0, run0, v1, pos1, run1);
    }
}

// Centre codes after the plane's last literal.
__device__ __forceinline__ uint32_t tail_run(const uint16_t* list, uint32_t L, uint32_t P)
{
    return P - (L ? list[L - 1] + 1u : 0u);
}

// Bits of the run symbols of a run of r centre codes (r <= P), per stream:
// rb[r], r = 0 .. kRunBitsStride - 1 (planes of up to 1024 codes).
__global__ void k_run_bits(const StreamDesc* __restrict__ sd, const uint32_t* __restrict__ ctab,
                           uint8_t* __restrict__ rbits)
{
    const StreamDesc s = sd[blockIdx.x];
    const uint32_t P = s.C * s.C;
    if (s.run_n == 0 || P >= kRunBitsStride) return;
    const uint32_t* tab = ctab + (size_t)blockIdx.x * 2 * s.radius;
    uint32_t D, LD;
    const uint32_t J = run_geometry(P, D, LD);
    for (uint32_t r = threadIdx.x; r <= P; r += blockDim.x) {
        uint32_t b = 0;
        run_symbols(r, s.radius, s.run_base, J, D, LD, [&](uint32_t sym) { b += __ldg(tab + sym) & 31u; });
        rbits[(size_t)blockIdx.x * kRunBitsStride + r] = (uint8_t)b;
    }
}

// Run-symbol counts of every listed plane (streams with runs).
__global__ void __launch_bounds__(kLaneThreads) k_run_stats(const CtaWork* __restrict__ work,
                                                            const uint32_t* __restrict__ chunk_ids,
                                                            const StreamDesc* __restrict__ sd,
                                                            const uint16_t* __restrict__ codes,
                                                            unsigned long long* __restrict__ stats)
{
    __shared__ uint32_t cnt[kRunStats];
    const CtaWork w = work[blockIdx.x];
    const StreamDesc s = sd[w.stream];
    if (s.run_n == 0) return;  // uniform per block
    if (threadIdx.x < kRunStats) cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t C = s.C, P = C * C, W = lanes_per_plane(P), np = w.count * C;
    uint32_t singles = 0;
    auto count = [&](uint32_t sym) {
        if (sym == s.radius) ++singles;
        else if (sym - s.run_base < s.run_n) atomicAdd(&cnt[sym - s.run_base + 1], 1u);
    };
    if (lits_ok(P, W)) {
        __shared__ uint16_t lists[kLaneThreads / 32][kListPerWarp];
        uint16_t* list = lists[threadIdx.x >> 5] + ((threadIdx.x & 31) / W) * 32 * W;
        uint32_t D, LD;
        const uint32_t J = run_geometry(P, D, LD);
        STZ_GROUP_PLANES(np, W)
        {
            STZ_GROUP_PLANE(np, W);
            const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
            const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
            const LaneSeg g = lane_seg(C, src, W, active);
            const uint32_t L = plane_literals(src, g, s.radius, list);
            literal_rounds2(list, L, g, [&](bool v0, uint32_t, uint32_t run0, bool v1, uint32_t, uint32_t run1) {
                if (v0 && run0) run_symbols(run0, s.radius, s.run_base, J, D, LD, count);
                if (v1 && run1) run_symbols(run1, s.radius, s.run_base, J, D, LD, count);
            });
            if (active && g.lane == 0) run_symbols(tail_run(list, L, P), s.radius, s.run_base, J, D, LD, count);
            __syncwarp();  // the list is rewritten for the next plane
        }
    } else {
        STZ_GROUP_PLANES(np, W)
        {
            STZ_GROUP_PLANE(np, W);
            const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
            const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
            const LaneSeg g = lane_seg(C, src, W, active);
            RunLane rl;
            rl.init(src, g, s.radius);
            rl.symbols(src, g, s, count);
        }
    }
    singles = group_sum(singles, 32);
    if ((threadIdx.x & 31) == 0 && singles) atomicAdd(&cnt[0], singles);
    __syncthreads();
    if (threadIdx.x < kRunStats && cnt[threadIdx.x])
        atomicAdd(&stats[(size_t)w.stream * kRunStats + threadIdx.x], cnt[threadIdx.x]);
}

// Bits of every plane.
__global__ void __launch_bounds__(kLaneThreads) k_sub_bits(const CtaWork* __restrict__ work,
                                                           const uint32_t* __restrict__ chunk_ids,
                                                           const StreamDesc* __restrict__ sd,
                                                           const uint16_t* __restrict__ codes,
                                                           const uint32_t* __restrict__ ctab,
                                                           const uint8_t* __restrict__ rbits,
                                                           uint32_t* __restrict__ sub_bits)
{
    const CtaWork w = work[blockIdx.x];
    const StreamDesc s = sd[w.stream];
    const uint32_t C = s.C, P = C * C, W = lanes_per_plane(P), np = w.count * C;
    const uint32_t* tab = ctab + (size_t)w.stream * 2 * s.radius;
    if (s.run_n && lits_ok(P, W)) {
        __shared__ uint16_t lists[kLaneThreads / 32][kListPerWarp];
        uint16_t* list = lists[threadIdx.x >> 5] + ((threadIdx.x & 31) / W) * 32 * W;
        const uint8_t* rb = rbits + (size_t)w.stream * kRunBitsStride;
        STZ_GROUP_PLANES(np, W)
        {
            STZ_GROUP_PLANE(np, W);
            const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
            const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
            const LaneSeg g = lane_seg(C, src, W, active);
            const uint32_t L = plane_literals(src, g, s.radius, list);
            uint32_t bits = 0;
            literal_rounds2(list, L, g, [&](bool v0, uint32_t pos0, uint32_t run0, bool v1, uint32_t pos1, uint32_t run1) {
                const uint32_t q0 = v0 ? __ldg(src + pos0) : 0u, q1 = v1 ? __ldg(src + pos1) : 0u;
                if (v0) bits += __ldg(rb + run0) + (__ldg(tab + q0) & 31u);
                if (v1) bits += __ldg(rb + run1) + (__ldg(tab + q1) & 31u);
            });
            if (active && g.lane == 0) bits += __ldg(rb + tail_run(list, L, P));
            bits = group_sum(bits, W);
            if (active && g.lane == 0) sub_bits[s.sub_base + (size_t)c * C + lz] = bits;
            __syncwarp();  // the list is rewritten for the next plane
        }
        return;
    }
    STZ_GROUP_PLANES(np, W)
    {
        STZ_GROUP_PLANE(np, W);
        const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
        const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
        const LaneSeg g = lane_seg(C, src, W, active);
        uint32_t bits = 0;
        auto add = [&](uint32_t sym) { bits += __ldg(tab + sym) & 31u; };
        if (s.run_n) {
            RunLane rl;
            rl.init(src, g, s.radius);
            rl.symbols(src, g, s, add);
        } else {
            lane_codes(src, g, add);
        }
        bits = group_sum(bits, W);
        if (active && g.lane == 0) sub_bits[s.sub_base + (size_t)c * C + lz] = bits;
    }
}

// Plane bit offsets inside each chunk (one warp per chunk: a scan of the
// planes' bit counts); the chunk's word count goes to chunk_word_off, which
// k_scan_stream then turns into offsets. Block (s, y) takes chunks 32y..32y+31
// of stream s.
__global__ void __launch_bounds__(1024) k_plane_offsets(const StreamDesc* __restrict__ sd,
                                                        const uint32_t* __restrict__ sub_bits,
                                                        uint32_t* __restrict__ sub_off,
                                                        uint64_t* __restrict__ chunk_word_off)
{
    const StreamDesc s = sd[blockIdx.x];
    const uint32_t c = blockIdx.y * 32 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (c >= s.nchunks) return;  // uniform per warp
    const size_t k0 = s.sub_base + (size_t)c * s.C;
    uint64_t carry = 0;
    for (uint32_t lz0 = 0; lz0 < s.C; lz0 += 32) {
        const uint32_t lz = lz0 + lane;
        const uint32_t bits = lz < s.C ? sub_bits[k0 + lz] : 0u;
        uint32_t incl = bits;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        if (lz < s.C) sub_off[k0 + lz] = (uint32_t)(carry + incl - bits);
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) chunk_word_off[s.chunk_base + c] = (carry + 31) / 32;
}

// Per stream: chunk word counts -> word offsets (the marker table) and the
// stream's word count; then the boundary words of every plane are cleared
// for the encoder's atomic ORs.
__global__ void __launch_bounds__(1024) k_scan_stream(const StreamDesc* __restrict__ sd,
                                                      const uint32_t* __restrict__ sub_bits,
                                                      const uint32_t* __restrict__ sub_off,
                                                      uint64_t* __restrict__ chunk_word_off,
                                                      uint64_t* __restrict__ stream_words,
                                                      uint32_t* __restrict__ payload)
{
    const StreamDesc s = sd[blockIdx.x];
    const uint32_t C = s.C;
    __shared__ uint64_t carry;
    __shared__ uint64_t wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < s.nchunks; base += blockDim.x) {
        const uint32_t c = base + threadIdx.x;
        const uint64_t words = c < s.nchunks ? chunk_word_off[s.chunk_base + c] : 0;
        uint64_t incl = words;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if ((threadIdx.x & 31) >= o) incl += v;
        }
        if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint64_t v = wsum[threadIdx.x];
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t u = __shfl_up_sync(0xffffffffu, v, o);
                if (threadIdx.x >= o) v += u;
            }
            wsum[threadIdx.x] = v;
        }
        __syncthreads();
        const uint64_t pre = carry + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0) + incl - words;
        if (c < s.nchunks) chunk_word_off[s.chunk_base + c] = pre;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        chunk_word_off[s.chunk_base + s.nchunks] = carry;
        stream_words[blockIdx.x] = carry;
    }
    __syncthreads();  // every chunk offset is written
    // four planes per thread in flight (one block per stream: the loop is
    // latency-bound)
    const uint64_t np = (uint64_t)s.nchunks * C;
    for (uint64_t p0 = threadIdx.x; p0 < np; p0 += 4 * (uint64_t)blockDim.x) {
        uint32_t b0[4], nb[4];
        uint64_t cw[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint64_t p = p0 + (uint64_t)j * blockDim.x;
            nb[j] = 0;
            if (p < np) {
                const size_t k = s.sub_base + p;
                b0[j] = sub_off[k];
                nb[j] = sub_bits[k];
                cw[j] = chunk_word_off[s.chunk_base + p / C];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (nb[j]) {
                uint32_t* w = payload + s.word_base + cw[j];
                w[b0[j] >> 5] = 0;
                w[(b0[j] + nb[j] - 1) >> 5] = 0;
            }
    }
}

// Encode: a warp packs one plane MSB-first, each lane its own bits from the
// plane's offset plus the bits of the lanes before it. The plane's first and
// last words (shared with its neighbours, cleared by k_scan_stream) and each
// lane's first and last words are merged with atomicOr; the warp clears the
// plane's inner words first, and words inside one lane's range are stored.
__global__ void __launch_bounds__(kLaneThreads) k_encode(const CtaWork* __restrict__ work,
                                                         const uint32_t* __restrict__ chunk_ids,
                                                         const StreamDesc* __restrict__ sd,
                                                         const uint16_t* __restrict__ codes,
                                                         const uint32_t* __restrict__ ctab,
                                                         const uint8_t* __restrict__ rbits,
                                                         const uint32_t* __restrict__ sub_bits,
                                                         const uint32_t* __restrict__ sub_off,
                                                         const uint64_t* __restrict__ chunk_word_off,
                                                         uint32_t* __restrict__ payload)
{
    const CtaWork w = work[blockIdx.x];
    const StreamDesc s = sd[w.stream];
    const uint32_t C = s.C, P = C * C, W = lanes_per_plane(P), np = w.count * C;
    const uint32_t* tab = ctab + (size_t)w.stream * 2 * s.radius;
    if (s.run_n && lits_ok(P, W)) {
        // literal rounds: each literal's bits (its run's, then its own) placed
        // by a group scan, written into a shared staging copy of the plane's
        // words aligned as in the chunk; then the inner words are stored and
        // the first and last (shared with the neighbouring planes) merged
        __shared__ uint16_t lists[kLaneThreads / 32][kListPerWarp];
        __shared__ uint32_t stage[kLaneThreads / 32][kStagePerWarp];
        const uint32_t gi = (threadIdx.x & 31) / W;
        uint16_t* list = lists[threadIdx.x >> 5] + gi * 32 * W;
        uint32_t* stg = stage[threadIdx.x >> 5] + gi * (24 * W + 2);
        const uint8_t* rb = rbits + (size_t)w.stream * kRunBitsStride;
        uint32_t D, LD;
        const uint32_t J = run_geometry(P, D, LD);
        auto put = [&](uint32_t e, uint32_t& p) {  // e = code << 5 | length, MSB first at bit p
            const uint32_t l = e & 31u, v = e >> 5, o = p & 31u, wi = p >> 5;
            if (!l) return;
            if (o + l <= 32) {
                atomicOr(stg + wi, v << (32 - o - l));
            } else {
                atomicOr(stg + wi, v >> (o + l - 32));
                atomicOr(stg + wi + 1, v << (64 - o - l));
            }
            p += l;
        };
        STZ_GROUP_PLANES(np, W)
        {
            STZ_GROUP_PLANE(np, W);
            const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
            const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
            const LaneSeg g = lane_seg(C, src, W, active);
            const uint32_t L = plane_literals(src, g, s.radius, list);
            const size_t k = s.sub_base + (size_t)c * C + lz;
            const uint32_t b0 = sub_off[k], nb = active ? sub_bits[k] : 0u;
            const uint32_t nw = ((b0 & 31u) + nb + 31u) >> 5;
            for (uint32_t x = g.lane; x < nw; x += W) stg[x] = 0;
            __syncwarp();
            uint32_t at = b0 & 31u;  // the group's next bit in the staging words
            literal_rounds2(list, L, g, [&](bool v0, uint32_t pos0, uint32_t run0, bool v1, uint32_t pos1, uint32_t run1) {
                const uint32_t q0 = v0 ? __ldg(src + pos0) : 0u, q1 = v1 ? __ldg(src + pos1) : 0u;
                uint32_t e0 = 0, e1 = 0, len0 = 0, len1 = 0;
                if (v0) {
                    e0 = __ldg(tab + q0);
                    len0 = __ldg(rb + run0) + (e0 & 31u);
                }
                if (v1) {
                    e1 = __ldg(tab + q1);
                    len1 = __ldg(rb + run1) + (e1 & 31u);
                }
                const uint32_t len = len0 + len1;
                const uint32_t incl = group_scan(len, W, g.lane);
                uint32_t p = at + incl - len;
                at += __shfl_sync(0xffffffffu, incl, W - 1, W);
                auto sym_put = [&](uint32_t sym) { put(__ldg(tab + sym), p); };
                if (v0) {
                    run_symbols(run0, s.radius, s.run_base, J, D, LD, sym_put);
                    put(e0, p);
                }
                if (v1) {
                    run_symbols(run1, s.radius, s.run_base, J, D, LD, sym_put);
                    put(e1, p);
                }
            });
            if (active && g.lane == 0) {
                uint32_t p = at;
                run_symbols(tail_run(list, L, P), s.radius, s.run_base, J, D, LD,
                            [&](uint32_t sym) { put(__ldg(tab + sym), p); });
            }
            __syncwarp();
            if (active && nb) {
                uint32_t* out = payload + s.word_base + chunk_word_off[s.chunk_base + c] + (b0 >> 5);
                for (uint32_t x = g.lane; x < nw; x += W) {
                    const uint32_t v = stg[x];
                    if (x == 0 || x == nw - 1) atomicOr(out + x, v);
                    else out[x] = v;
                }
            }
            __syncwarp();  // list and staging are rewritten for the next plane
        }
        return;
    }
    STZ_GROUP_PLANES(np, W)
    {
        STZ_GROUP_PLANE(np, W);
        const uint32_t c = chunk_ids[w.first + pe / C], lz = pe % C;
        const uint16_t* src = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
        const LaneSeg g = lane_seg(C, src, W, active);
        RunLane rl;
        if (s.run_n) rl.init(src, g, s.radius);
        auto each = [&](auto&& f) {
            if (s.run_n) rl.symbols(src, g, s, f);
            else lane_codes(src, g, f);
        };
        uint32_t bits = 0;
        each([&](uint32_t sym) { bits += __ldg(tab + sym) & 31u; });
        uint32_t off = group_scan(bits, W, g.lane);  // inclusive -> this lane's first bit in the plane
        const uint32_t nb = __shfl_sync(0xffffffffu, off, W - 1, W);
        off -= bits;
        uint32_t* out = payload + s.word_base + chunk_word_off[s.chunk_base + c];
        const uint32_t b0 = sub_off[s.sub_base + (size_t)c * C + lz];
        if (active && nb)
            for (uint32_t x = (b0 >> 5) + 1 + g.lane; x < (b0 + nb - 1) >> 5; x += W) out[x] = 0;
        __syncwarp();
        if (active && bits) {
            const uint32_t pos = b0 + off;
            const uint32_t first_w = pos >> 5, last_w = (pos + bits - 1) >> 5;
            uint32_t wi = first_w;
            uint64_t acc = 0;            // pending bits, right-aligned
            int nacc = (int)(pos & 31);  // leading bits of the first word belong to earlier lanes (zeros here)
            each([&](uint32_t sym) {
                const uint32_t e = __ldg(tab + sym);
                const int l = e & 31;
                acc = (acc << l) | (e >> 5);
                nacc += l;
                if (nacc >= 32) {
                    const uint32_t word = (uint32_t)(acc >> (nacc - 32));
                    nacc -= 32;
                    if (wi == first_w || wi == last_w) atomicOr(out + wi, word);
                    else out[wi] = word;
                    ++wi;
                }
            });
            if (nacc > 0) atomicOr(out + wi, (uint32_t)(acc << (32 - nacc)));
        }
        __syncwarp();
    }
}

// Decode: a warp decodes one plane with a 2^kLutBits-entry table in shared
// memory (symbol | length << 16); longer codes fall back to the canonical
// first-code test per length.
// Symbols of codes longer than kLutBits kept with the tables (the rest of a
// longer tail is read from the codebook).
constexpr int kTailSyms = 4096;

// Decode tables of one stream, built once per prepared stream in device
// memory (k_build_tables) and read by the decoders through L1.
// lut entry: sym | len << 16 for codes of at most kLutBits bits; for a prefix
// of longer codes, l_min << 24 with l_min the shortest code length under that
// prefix (the canonical length search starts there); 0 for a prefix of no code.
struct DecodeTables {
    uint32_t lut[1 << kLutBits];
    uint32_t cnt[kMaxCodeLen + 1];
    uint32_t first_code[kMaxCodeLen + 1];
    uint32_t first_idx[kMaxCodeLen + 1];
    uint16_t tail[kTailSyms];
};

// One CTA per stream.
__global__ void __launch_bounds__(256) k_build_tables(const StreamDesc* __restrict__ sd,
                                                      const uint16_t* __restrict__ cb_sym,
                                                      const uint8_t* __restrict__ cb_len,
                                                      DecodeTables* __restrict__ out)
{
    const StreamDesc s = sd[blockIdx.x];
    DecodeTables& t = out[blockIdx.x];
    __shared__ uint32_t cnt[kMaxCodeLen + 1];
    __shared__ uint32_t first_code[kMaxCodeLen + 1];
    __shared__ uint32_t first_idx[kMaxCodeLen + 1];
    if (threadIdx.x <= kMaxCodeLen) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < s.n_used; i += blockDim.x) atomicAdd(&cnt[cb_len[s.cb_off + i]], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t code = 0, idx = cnt[0];
        first_code[0] = 0;
        first_idx[0] = 0;
        for (int l = 1; l <= kMaxCodeLen; ++l) {
            code = (code + (l > 1 ? cnt[l - 1] : 0)) << 1;
            first_code[l] = code;
            first_idx[l] = idx;
            idx += cnt[l];
        }
    }
    __syncthreads();
    if (threadIdx.x <= kMaxCodeLen) {
        t.cnt[threadIdx.x] = cnt[threadIdx.x];
        t.first_code[threadIdx.x] = first_code[threadIdx.x];
        t.first_idx[threadIdx.x] = first_idx[threadIdx.x];
    }
    // every table entry finds its code: the shortest length whose canonical
    // range holds the entry's prefix; prefixes of longer codes record the
    // shortest such length
    for (uint32_t j = threadIdx.x; j < (1u << kLutBits); j += blockDim.x) {
        uint32_t e = 0;
        for (uint32_t l = 1; l <= (uint32_t)kLutBits; ++l) {
            const uint32_t v = (j >> (kLutBits - l)) - first_code[l];
            if (v < cnt[l]) {
                e = (uint32_t)cb_sym[s.cb_off + first_idx[l] + v] | (l << 16);
                break;
            }
        }
        if (!e) {
            for (uint32_t l = kLutBits + 1; l <= (uint32_t)kMaxCodeLen; ++l) {
                if (!cnt[l]) continue;
                const uint32_t sh = l - kLutBits;
                if (j >= (first_code[l] >> sh) && j <= ((first_code[l] + cnt[l] - 1) >> sh)) {
                    e = l << 24;
                    break;
                }
            }
        }
        t.lut[j] = e;
    }
    const uint32_t t0 = first_idx[kLutBits + 1];
    for (uint32_t i = threadIdx.x; i < (uint32_t)kTailSyms && t0 + i < s.n_used; i += blockDim.x)
        t.tail[i] = cb_sym[s.cb_off + t0 + i];
}

// The symbol whose code starts at the top of `bits` (MSB first, at least
// kMaxCodeLen valid bits); its code length in l (>= 1). A prefix of no code
// (corrupt stream) yields the codebook's first symbol with length 1, so
// every step consumes a bit.
__device__ __forceinline__ uint32_t lookup_symbol(const DecodeTables* __restrict__ t, const StreamDesc& s,
                                                  const uint16_t* __restrict__ cb_sym, uint32_t bits, uint32_t& l)
{
    const uint32_t e = __ldg(&t->lut[bits >> (32 - kLutBits)]);
    uint32_t sym = e & 0xffffu;
    l = (e >> 16) & 0xffu;
    if (!l) {
        // canonical search from the shortest length under this prefix
        l = e >> 24;
        if (!l) l = kLutBits + 1;
        for (; l <= (uint32_t)kMaxCodeLen; ++l) {
            const uint32_t v = bits >> (32 - l), fc = __ldg(&t->first_code[l]);
            if (v - fc < __ldg(&t->cnt[l])) {
                const uint32_t fi = __ldg(&t->first_idx[l]);
                const uint32_t idx = fi + (v - fc);
                const uint32_t ti = idx - __ldg(&t->first_idx[kLutBits + 1]);
                sym = ti < (uint32_t)kTailSyms ? __ldg(&t->tail[ti]) : cb_sym[s.cb_off + idx];
                break;
            }
        }
        if (l > (uint32_t)kMaxCodeLen) {
            sym = cb_sym[s.cb_off];
            l = 1;
        }
    }
    return sym;
}

// Bits of one chunk's payload: 32 bits from any bit position. Plane bit
// ranges are validated against the chunk's words, and every stream keeps at
// least two words of zero padding after its payload, so a read at a position
// below a plane's end stays inside the stream's buffer.
struct ChunkBits {
    const uint32_t* in;
    __device__ __forceinline__ uint32_t peek(uint32_t pos) const
    {
        const uint32_t i = pos >> 5;
        return __funnelshift_l(__ldg(in + i + 1), __ldg(in + i), pos & 31);
    }
};

// Decode every code that starts in [pos, stop): f(sym) for each; returns the
// position after the last one (the first code boundary >= stop, or pos).
template <class F>
__device__ __forceinline__ uint32_t decode_range(const DecodeTables* __restrict__ t, const StreamDesc& s,
                                                 const uint16_t* __restrict__ cb_sym, const ChunkBits& cb,
                                                 uint32_t pos, uint32_t stop, F&& f)
{
    while (pos < stop) {
        uint32_t l;
        const uint32_t sym = lookup_symbol(t, s, cb_sym, cb.peek(pos), l);
        pos += l;
        f(sym);
    }
    return pos;
}

// Decode plane lz of chunk c of stream s (one thread, sequentially): for
// dense streams, where a plane holds many symbols and a warp per plane would
// decode each one about three times.
__device__ void decode_plane_seq(const DecodeTables* __restrict__ t, const StreamDesc& s, uint32_t c, uint32_t lz,
                             const uint16_t* __restrict__ cb_sym, const uint32_t* __restrict__ sub_off,
                             const uint64_t* __restrict__ chunk_word_off, const uint32_t* __restrict__ payload,
                             uint16_t* __restrict__ codes)
{
    const uint32_t* __restrict__ lut = t->lut;
    const uint32_t* __restrict__ cnt = t->cnt;
    const uint32_t* __restrict__ first_code = t->first_code;
    const uint32_t* __restrict__ first_idx = t->first_idx;
    const uint32_t C = s.C;
    const size_t plane = (size_t)C * C;
    uint16_t* dst = codes + s.code_off + (size_t)c * plane * C + (size_t)lz * plane;
    if (s.n_used == 1) {
        // a lone run symbol means the plane is all centre codes
        const uint16_t v0 = cb_sym[s.cb_off];
        const uint16_t v = (uint32_t)v0 - s.run_base < s.run_n ? (uint16_t)s.radius : v0;
        if (plane % 8 == 0 && ((uintptr_t)dst & 15) == 0) {
            const uint32_t v2 = (uint32_t)v | ((uint32_t)v << 16);
            for (size_t j = 0; j < plane / 8; ++j) reinterpret_cast<uint4*>(dst)[j] = make_uint4(v2, v2, v2, v2);
        } else {
            for (size_t j = 0; j < plane; ++j) dst[j] = v;
        }
        return;
    }
    const uint64_t cw = chunk_word_off[s.chunk_base + c];
    const uint32_t* in = payload + s.word_base + cw;
    // words of the stream left from this chunk's start; reads beyond read 0
    const uint64_t lim = s.word_cap > cw ? s.word_cap - cw : 0;
    auto rd = [&](uint64_t i) -> uint32_t { return i < lim ? __ldg(in + i) : 0u; };
    uint32_t pos = sub_off[s.sub_base + (size_t)c * C + lz];  // bit position from the chunk's first word
    // The plane's payload lines are prefetched into L1 up front (its end is
    // the next plane's start, or the chunk's end), so the loads below hit L1.
    {
        const uint64_t cwords = chunk_word_off[s.chunk_base + c + 1] - cw;
        const uint64_t b1 = lz + 1 < C ? (uint64_t)sub_off[s.sub_base + (size_t)c * C + lz + 1] : 32 * cwords;
        const uint64_t w1 = min(min((b1 + 31) >> 5, cwords) + 2, lim);
        for (uint64_t w = (pos >> 5) & ~31u; w < w1; w += 32) asm volatile("prefetch.global.L1 [%0];" ::"l"(in + w));
    }
    // 64-bit bit reservoir, MSB = next bit, `avail` valid bits (>= kLutBits
    // at every symbol start). The dependency chain of a symbol is only
    // table index -> lookup -> length -> shift: the refill word is merged in
    // (below the valid bits, from the length-independent `avail`) while the
    // lookup is in flight, and the next word is loaded one refill ahead.
    uint64_t wi = pos >> 5;
    uint64_t buf = (((uint64_t)rd(wi) << 32) | rd(wi + 1)) << (pos & 31);
    int avail = 64 - (int)(pos & 31);
    uint32_t w = rd(wi + 2);
    wi += 3;
    auto next = [&]() -> uint32_t {
        const uint32_t e = __ldg(lut + (uint32_t)(buf >> (64 - kLutBits)));
        const bool rf = avail < 32;
        const uint64_t b2 = rf ? (buf | ((uint64_t)w << (32 - avail))) : buf;  // >= 32 valid bits
        const int a2 = rf ? avail + 32 : avail;
        if (rf) w = rd(wi++);
        uint32_t sym = e & 0xffffu, l = (e >> 16) & 0xffu;
        if (!l) {
            // canonical search from the shortest length under this prefix; a
            // corrupt stream still yields a symbol of this codebook (never
            // code 0 unless the stream has unpredictable values)
            l = e >> 24;
            if (!l) l = kLutBits + 1;
            for (; l <= (uint32_t)kMaxCodeLen; ++l) {
                const uint32_t v = (uint32_t)(b2 >> (64 - l));
                if (v - first_code[l] < cnt[l]) {
                    const uint32_t idx = first_idx[l] + (v - first_code[l]);
                    const uint32_t ti = idx - first_idx[kLutBits + 1];
                    sym = ti < (uint32_t)kTailSyms ? __ldg(&t->tail[ti]) : cb_sym[s.cb_off + idx];
                    break;
                }
            }
            if (l > (uint32_t)kMaxCodeLen) {
                sym = cb_sym[s.cb_off];
                l = 1;  // corrupt stream: keep going, the result is garbage
            }
        }
        buf = b2 << l;
        avail = a2 - (int)l;
        if (avail < kLutBits) {  // only after a long code taken without a refill
            buf |= (uint64_t)w << (32 - avail);
            avail += 32;
            w = rd(wi++);
        }
        return sym;
    };
    if (s.run_n) {
        // Runs expand to 2^k centre codes, clipped to the plane (a corrupt
        // stream cannot write past it; every symbol yields at least one code,
        // so the loop ends). Vector form: codes collect in a 128-bit shift
        // register and leave as 16-byte stores; long runs store whole
        // 8-code groups directly.
        const uint32_t R = s.radius, base = s.run_base, J = s.run_n;
        uint32_t D, LD;
        run_geometry((uint32_t)plane, D, LD);
        size_t j = 0;
        if (plane % 8 == 0 && ((uintptr_t)dst & 15) == 0) {
            // 8 staged codes in (s0, s1), slot i at bits 16i; n copies of a
            // code enter with one masked OR, a full stage leaves as one store
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            uint64_t s0 = 0, s1 = 0;
            uint32_t ns = 0;
            auto low = [](uint32_t b) -> uint64_t { return b >= 64 ? ~0ull : (1ull << b) - 1; };
            auto flush = [&]() {
                if (ns == 8) {
                    d4[(j >> 3) - 1] =
                        make_uint4((uint32_t)s0, (uint32_t)(s0 >> 32), (uint32_t)s1, (uint32_t)(s1 >> 32));
                    s0 = s1 = 0;
                    ns = 0;
                }
            };
            auto put = [&](uint32_t v, uint32_t n) {  // n <= 8 - ns copies of v
                const uint64_t p = (uint64_t)(v | (v << 16)) * 0x0000000100000001ull;
                const uint32_t a = 16 * ns, b = 16 * (ns + n);
                s0 |= p & (low(min(b, 64u)) & ~low(min(a, 64u)));
                s1 |= p & (low(b > 64 ? b - 64 : 0) & ~low(a > 64 ? a - 64 : 0));
                ns += n;
                j += n;
                flush();
            };
            auto put1 = [&](uint32_t v) {  // one code: a shift into its slot
                if (ns < 4) s0 |= (uint64_t)v << (16 * ns);
                else s1 |= (uint64_t)v << (16 * (ns - 4));
                ++ns;
                ++j;
                flush();
            };
            const uint32_t r2 = R | (R << 16);
            const uint4 rr = make_uint4(r2, r2, r2, r2);
            while (j < plane) {
                const uint32_t sym = next();
                if (sym - base < J) {
                    uint32_t n = (uint32_t)min((size_t)run_length(sym - base, D, LD), plane - j);
                    if (ns) {
                        const uint32_t k = min(n, 8u - ns);
                        put(R, k);
                        n -= k;
                    }
                    for (; n >= 8; n -= 8, j += 8) d4[j >> 3] = rr;
                    if (n) put(R, n);
                } else {
                    put1(sym);
                }
            }
        } else {
            while (j < plane) {
                const uint32_t sym = next();
                if (sym - base < J) {
                    const size_t n = min((size_t)run_length(sym - base, D, LD), plane - j);
                    for (size_t i = 0; i < n; ++i) dst[j++] = (uint16_t)R;
                } else {
                    dst[j++] = (uint16_t)sym;
                }
            }
        }
    } else if (plane % 8 == 0 && ((uintptr_t)dst & 15) == 0) {
        // 8 symbols per 16-byte store; all lanes decode in lockstep
        uint4* d4 = reinterpret_cast<uint4*>(dst);
        for (size_t j = 0; j < plane / 8; ++j) {
            uint4 v;
            v.x = next();
            v.x |= next() << 16;
            v.y = next();
            v.y |= next() << 16;
            v.z = next();
            v.z |= next() << 16;
            v.w = next();
            v.w |= next() << 16;
            d4[j] = v;
        }
    } else {
        for (size_t j = 0; j < plane; ++j) dst[j] = (uint16_t)next();
    }
}

// Decode plane lz of chunk c of stream s (one group of W lanes, see
// lanes_per_plane; Weissenberger & Schmidt, "Massively parallel Huffman
// decoding on GPUs", ICPP 2018: speculative decoding from equal bit slices,
// then resynchronisation). A group without a plane (active false) takes part
// in the shuffles only. The plane's bits [b0, b1) are cut into W slices;
// lane i decodes the codes that start in
// its slice, beginning at the slice start. A lane whose start is not where
// its left neighbour's last code ends decodes again from there, until no
// start moves (lane i is exact after i rounds; codes resynchronise within a
// few symbols, so one or two rounds are usual). An exclusive scan of the
// lanes' code counts (a run symbol counts its run) then places each lane's
// output. With run symbols the plane is first filled with the centre code,
// so a lane writes only its literals. Output past the plane (a corrupt
// stream) is dropped.
__device__ void decode_plane_warp(const DecodeTables* __restrict__ t, const StreamDesc& s, uint32_t W, bool active,
                                  uint32_t c, uint32_t lz,
                                  const uint16_t* __restrict__ cb_sym, const uint32_t* __restrict__ sub_off,
                                  const uint64_t* __restrict__ chunk_word_off, const uint32_t* __restrict__ payload,
                                  uint16_t* __restrict__ codes)
{
    const uint32_t lane = threadIdx.x & (W - 1);
    const uint32_t C = s.C, P = C * C;
    uint16_t* dst = codes + s.code_off + (size_t)c * P * C + (size_t)lz * P;
    const bool vec = P % 8 == 0 && ((uintptr_t)dst & 15) == 0;
    const uint32_t R = s.radius, base = s.run_base, J = s.run_n;
    auto fill = [&](uint16_t v) {
        if (!active) return;
        if (vec) {
            const uint32_t v2 = (uint32_t)v | ((uint32_t)v << 16);
            for (uint32_t j = lane; j < P / 8; j += W) reinterpret_cast<uint4*>(dst)[j] = make_uint4(v2, v2, v2, v2);
        } else {
            for (uint32_t j = lane; j < P; j += W) dst[j] = v;
        }
    };
    if (s.n_used == 1) {
        // a lone run symbol means the plane is all centre codes
        const uint16_t v0 = cb_sym[s.cb_off];
        fill((uint32_t)v0 - base < J ? (uint16_t)R : v0);
        return;
    }
    const uint64_t cw = chunk_word_off[s.chunk_base + c];
    ChunkBits cb;
    cb.in = payload + s.word_base + cw;
    const uint32_t b0 = sub_off[s.sub_base + (size_t)c * C + lz];
    const uint32_t b1 = lz + 1 < C ? sub_off[s.sub_base + (size_t)c * C + lz + 1]
                                   : (uint32_t)(32 * (chunk_word_off[s.chunk_base + c + 1] - cw));
    const uint32_t nb = active && b1 > b0 ? b1 - b0 : 0;
    const uint32_t L = (nb + W - 1) / W;
    const uint32_t stop = b0 + min(nb, (lane + 1) * L);
    uint32_t D, LD;
    run_geometry(P, D, LD);
    uint32_t start = b0 + min(nb, lane * L), cnt = 0;
    auto count = [&](uint32_t sym) { cnt += sym - base < J ? run_length(sym - base, D, LD) : 1u; };
    uint32_t end = decode_range(t, s, cb_sym, cb, start, stop, count);
    for (int round = 0; round < 32; ++round) {
        uint32_t prev = __shfl_up_sync(0xffffffffu, end, 1, W);
        if (lane == 0) prev = b0;
        const bool moved = prev != start;
        if (!__any_sync(0xffffffffu, moved)) break;
        if (moved) {
            start = prev;
            cnt = 0;
            end = decode_range(t, s, cb_sym, cb, start, stop, count);
        }
    }
    uint32_t q = group_scan(cnt, W, lane) - cnt;  // first output position
    if (J) {
        fill((uint16_t)R);
        __syncwarp();
        decode_range(t, s, cb_sym, cb, start, stop, [&](uint32_t sym) {
            if (sym - base < J) {
                q += run_length(sym - base, D, LD);
            } else {
                if (active && q < P) dst[q] = (uint16_t)sym;
                ++q;
            }
        });
    } else {
        decode_range(t, s, cb_sym, cb, start, stop, [&](uint32_t sym) {
            if (active && q < P) dst[q] = (uint16_t)sym;
            ++q;
        });
    }
}

constexpr int kDecodeThreads = 256;  // 8 warps, each one plane
constexpr int kDecodeSlices = 16;    // CTAs per work item (gridDim.y): short CTAs, every warp one plane
constexpr uint32_t kSeqBits = 2048;  // mean payload bits per plane above which a stream decodes one thread per plane

// Lanes decoding one plane: a warp for planes of 1024 codes and more, but
// half a warp where a plane averages fewer than kHalfWarpBits payload bits:
// each lane then takes twice the bits, and the resynchronisation and scans
// cost half as much per symbol (512^3 bench stream, ~600 bits per plane:
// 0.40 -> 0.34 ms; 8 lanes 0.40, 4 lanes 0.59).
constexpr uint32_t kHalfWarpBits = 2048;
__device__ __forceinline__ uint32_t decode_group(const StreamDesc& s)
{
    const uint32_t W = lanes_per_plane(s.C * s.C);
    const uint64_t planes = (uint64_t)s.nchunks * s.C;
    return W == 32 && 32 * (s.word_cap - 4) < (uint64_t)kHalfWarpBits * planes ? 16u : W;
}

// A stream whose planes average more than seq_bits payload bits, with enough
// planes to fill the device one thread per plane, is decoded one thread per
// plane; sparser or smaller streams a lane group per plane (decode_group: the
// group decodes each symbol about three times, a thread once but with the
// full serial chain).
constexpr uint64_t kSeqMinPlanes = 16384;
constexpr int kSeqMinItems = 128;  // smaller launches (single requests) are latency-bound: warps only
__device__ __forceinline__ bool decode_sequential(const StreamDesc& s, uint32_t seq_bits)
{
    const uint64_t planes = (uint64_t)s.nchunks * s.C;
    return planes >= kSeqMinPlanes && 32 * (s.word_cap - 4) > (uint64_t)seq_bits * planes;
}

// Planes of the listed chunks; the tables of stream i at tabs[i]. Warp mode:
// CTA (x, y) takes 8 planes of item x; sequential mode: CTA (x, 0) takes all
// of them, one per thread (at most kDecodeThreads).
__global__ void __launch_bounds__(kDecodeThreads, 5) k_decode(const CtaWork* __restrict__ work,
                                                           const uint32_t* __restrict__ chunk_ids,
                                                           const StreamDesc* __restrict__ sd,
                                                           const DecodeTables* __restrict__ tabs,
                                                           const uint16_t* __restrict__ cb_sym,
                                                           const uint32_t* __restrict__ sub_off,
                                                           const uint64_t* __restrict__ chunk_word_off,
                                                           const uint32_t* __restrict__ payload,
                                                           uint16_t* __restrict__ codes, uint32_t seq_bits)
{
    const CtaWork w = work[blockIdx.x];
    const StreamDesc s = sd[w.stream];
    if (decode_sequential(s, seq_bits)) {
        const uint32_t t = threadIdx.x;
        if (blockIdx.y == 0 && t < w.count * s.C)
            decode_plane_seq(tabs + w.stream, s, chunk_ids[w.first + t / s.C], t % s.C, cb_sym, sub_off,
                             chunk_word_off, payload, codes);
        return;
    }
    const uint32_t W = decode_group(s), np = w.count * s.C;
    STZ_GROUP_PLANES(np, W)
    {
        STZ_GROUP_PLANE(np, W);
        decode_plane_warp(tabs + w.stream, s, W, active, chunk_ids[w.first + pe / s.C], pe % s.C, cb_sym, sub_off,
                          chunk_word_off, payload, codes);
    }
}

// Persistent variant: a fixed grid walks the work list of a batch held in
// device memory (BatchHdr at meta), so one captured launch serves any batch;
// each warp-decoded item is cut into kDecodeSlices slices of 8 planes.
__global__ void __launch_bounds__(kDecodeThreads) k_decode_dyn(const uint8_t* __restrict__ meta,
                                                               const StreamDesc* __restrict__ sd,
                                                               const DecodeTables* __restrict__ tabs,
                                                               const uint16_t* __restrict__ cb_sym,
                                                               const uint32_t* __restrict__ sub_off,
                                                               const uint64_t* __restrict__ chunk_word_off,
                                                               const uint32_t* __restrict__ payload,
                                                               uint16_t* __restrict__ codes, uint32_t seq_bits)
{
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(meta);
    const uint32_t n = h->n_work;
    const CtaWork* __restrict__ work = reinterpret_cast<const CtaWork*>(meta + h->o_work);
    const uint32_t* __restrict__ chunk_ids = reinterpret_cast<const uint32_t*>(meta + h->o_ids);
    const uint32_t nw = blockDim.x >> 5, S = kDecodeSlices;
    // In a batch of at least kSeqMinItems items, dense streams decode one
    // thread per plane (as k_decode does for large launches): a CTA takes
    // whole items, striding over the items so every CTA gets some.
    const uint32_t sb = n >= (uint32_t)kSeqMinItems ? seq_bits : 0xffffffffu;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const CtaWork w = work[i];
        const StreamDesc s = sd[w.stream];
        if (!decode_sequential(s, sb)) continue;  // uniform per block
        const uint32_t t = threadIdx.x;
        if (t < w.count * s.C)
            decode_plane_seq(tabs + w.stream, s, chunk_ids[w.first + t / s.C], t % s.C, cb_sym, sub_off,
                             chunk_word_off, payload, codes);
    }
    // the other items a warp per plane, kDecodeSlices slices per item
    for (uint32_t u = blockIdx.x; u < n * S; u += gridDim.x) {
        const CtaWork w = work[u / S];
        const StreamDesc s = sd[w.stream];
        if (decode_sequential(s, sb)) continue;  // uniform per block
        const uint32_t W = decode_group(s), G = 32 / W, np = w.count * s.C;
        for (uint32_t base = ((u % S) * nw + (threadIdx.x >> 5)) * G; base < np; base += nw * S * G) {
            const uint32_t p = base + (threadIdx.x & 31) / W;
            const bool active = p < np;
            const uint32_t pe = active ? p : base;
            decode_plane_warp(tabs + w.stream, s, W, active, chunk_ids[w.first + pe / s.C], pe % s.C, cb_sym, sub_off,
                              chunk_word_off, payload, codes);
        }
    }
}

// Unpredictable values: for each listed chunk, walk its codes in order and
// move the values between the dense per-position buffer and the chunk's slot
// of the compact list (gather on encode, scatter on decode).
// One pass: every thread owns a contiguous segment of the chunk's codes
// (thread order = code order), counts its zeros, and a block-wide exclusive
// prefix of the counts gives each segment's first rank in the list.
// blockDim.x is a multiple of 32, at most 1024 (wc holds one count per warp).
template <typename T, bool GATHER>
__device__ void unpred_move_one(const UnpredWork& uw, const StreamDesc* __restrict__ sd,
                                const uint16_t* __restrict__ codes, T* __restrict__ dense, T* __restrict__ list,
                                uint32_t* wc)
{
    const StreamDesc s = sd[uw.stream];
    const uint32_t vol = s.C * s.C * s.C;
    const size_t base = s.code_off + (size_t)uw.chunk * vol;
    const uint32_t nt = blockDim.x, seg = (vol + nt - 1) / nt;
    const uint32_t a = min(threadIdx.x * seg, vol), b = min(a + seg, vol);
    uint32_t cnt = 0;
    for (uint32_t i = a; i < b; ++i) cnt += codes[base + i] == 0 ? 1u : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(nt >> 5);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wc[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t v = lane < nw ? wc[lane] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < nw) wc[lane] = x - v;  // exclusive prefix over warps
    }
    __syncthreads();
    uint64_t r = (uint64_t)wc[wid] + incl - cnt;
    if (cnt)
        for (uint32_t i = a; i < b; ++i) {
            if (codes[base + i] != 0) continue;
            if (r < uw.count) {
                if (GATHER) list[uw.list_off + r] = dense[base + i];
                else dense[base + i] = list[uw.list_off + r];
            }
            ++r;
        }
    __syncthreads();  // wc is reused by the block's next item
}

template <typename T, bool GATHER>
__global__ void __launch_bounds__(1024) k_unpred_move(const UnpredWork* __restrict__ work,
                                                      const StreamDesc* __restrict__ sd,
                                                      const uint16_t* __restrict__ codes, T* __restrict__ dense,
                                                      T* __restrict__ list)
{
    __shared__ uint32_t wc[32];
    unpred_move_one<T, GATHER>(work[blockIdx.x], sd, codes, dense, list, wc);
}

// Persistent scatter (decode side) over the unpredictable-value list of a
// batch held in device memory (BatchHdr at meta).
template <typename T>
__global__ void __launch_bounds__(1024) k_unpred_scatter_dyn(const uint8_t* __restrict__ meta,
                                                             const StreamDesc* __restrict__ sd,
                                                             const uint16_t* __restrict__ codes,
                                                             T* __restrict__ dense, T* __restrict__ list)
{
    __shared__ uint32_t wc[32];
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(meta);
    const uint32_t n = h->n_uwork;
    const UnpredWork* __restrict__ work = reinterpret_cast<const UnpredWork*>(meta + h->o_uwork);
    for (uint32_t wi = blockIdx.x; wi < n; wi += gridDim.x)
        unpred_move_one<T, false>(work[wi], sd, codes, dense, list, wc);
}

__global__ void k_pack_streams(const StreamDesc* __restrict__ sd, const uint64_t* __restrict__ stream_words, int s0,
                               const uint32_t* __restrict__ payload, uint32_t* __restrict__ dst)
{
    const int s = s0 + (int)blockIdx.y;
    uint64_t b = 0;  // words of the streams before s in this group
    for (int i = s0; i < s; ++i) b += stream_words[i];
    const uint64_t n = stream_words[s], a = sd[s].word_base;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[b + i] = payload[a + i];
}

}  // namespace

void launch_pack_streams(const StreamDesc* sd, const uint64_t* stream_words, int s0, int s1, const uint32_t* payload,
                         uint32_t* dst, cudaStream_t st)
{
    if (s1 > s0) k_pack_streams<<<dim3(16, s1 - s0), 256, 0, st>>>(sd, stream_words, s0, payload, dst);
}

void launch_expand_codebook(const StreamDesc* sd, int nstreams, const uint16_t* cb_sym, const uint8_t* cb_len,
                            uint32_t* ctab, cudaStream_t st)
{
    if (nstreams) k_expand_codebook<<<nstreams, 256, 0, st>>>(sd, cb_sym, cb_len, ctab);
}

void launch_run_stats(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                      const uint16_t* codes, unsigned long long* stats, cudaStream_t st)
{
    if (nwork > 0) k_run_stats<<<dim3(nwork, kPlaneSlices), kLaneThreads, 0, st>>>(work, chunk_ids, sd, codes, stats);
}

void launch_run_bits(const StreamDesc* sd, int nstreams, const uint32_t* ctab, uint8_t* rbits, cudaStream_t st)
{
    if (nstreams) k_run_bits<<<nstreams, 256, 0, st>>>(sd, ctab, rbits);
}

void launch_sub_bits(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                     const uint16_t* codes, const uint32_t* ctab, const uint8_t* rbits, uint32_t* sub_bits,
                     cudaStream_t st)
{
    if (nwork)
        k_sub_bits<<<dim3(nwork, kPlaneSlices), kLaneThreads, 0, st>>>(work, chunk_ids, sd, codes, ctab, rbits,
                                                                        sub_bits);
}

void launch_scan_streams(const StreamDesc* sd, int nstreams, uint32_t max_chunks, const uint32_t* sub_bits,
                         uint32_t* sub_off, uint64_t* chunk_word_off, uint64_t* stream_words, uint32_t* payload,
                         cudaStream_t st)
{
    if (!nstreams || !max_chunks) return;
    k_plane_offsets<<<dim3(nstreams, (max_chunks + 31) / 32), 1024, 0, st>>>(sd, sub_bits, sub_off, chunk_word_off);
    k_scan_stream<<<nstreams, 1024, 0, st>>>(sd, sub_bits, sub_off, chunk_word_off, stream_words, payload);
}

void launch_encode(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                   const uint16_t* codes, const uint32_t* ctab, const uint8_t* rbits, const uint32_t* sub_bits,
                   const uint32_t* sub_off, const uint64_t* chunk_word_off, uint32_t* payload, cudaStream_t st)
{
    if (nwork)
        k_encode<<<dim3(nwork, kPlaneSlices), kLaneThreads, 0, st>>>(work, chunk_ids, sd, codes, ctab, rbits, sub_bits,
                                                                      sub_off, chunk_word_off, payload);
}

void launch_decode(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                   const uint16_t* cb_sym, const void* tables, const uint32_t* sub_off, const uint64_t* chunk_word_off,
                   const uint32_t* payload, uint16_t* codes, cudaStream_t st)
{
    if (nwork)
        k_decode<<<dim3(nwork, kDecodeSlices), kDecodeThreads, 0, st>>>(
            work, chunk_ids, sd, static_cast<const DecodeTables*>(tables), cb_sym, sub_off, chunk_word_off, payload,
            codes, nwork >= kSeqMinItems ? decode_seq_bits() : 0xffffffffu);
}

size_t decode_tables_bytes() { return sizeof(DecodeTables); }

uint32_t decode_seq_bits()
{
    static const uint32_t v = [] {
        const char* e = std::getenv("STZ_DECODE_SEQ_BITS");
        return e ? (uint32_t)std::strtoul(e, nullptr, 10) : kSeqBits;
    }();
    return v;
}

void launch_build_tables(const StreamDesc* sd, int nstreams, const uint16_t* cb_sym, const uint8_t* cb_len,
                         void* tables, cudaStream_t st)
{
    if (nstreams > 0)
        k_build_tables<<<nstreams, 256, 0, st>>>(sd, cb_sym, cb_len, static_cast<DecodeTables*>(tables));
}

template <typename T>
void launch_unpred_move(bool gather, const UnpredWork* work, int nwork, const StreamDesc* sd, const uint16_t* codes,
                        T* dense, T* list, cudaStream_t st)
{
    if (!nwork) return;
    if (gather) k_unpred_move<T, true><<<nwork, 1024, 0, st>>>(work, sd, codes, dense, list);
    else k_unpred_move<T, false><<<nwork, 1024, 0, st>>>(work, sd, codes, dense, list);
}

template void launch_unpred_move<float>(bool, const UnpredWork*, int, const StreamDesc*, const uint16_t*, float*,
                                        float*, cudaStream_t);
template void launch_unpred_move<double>(bool, const UnpredWork*, int, const StreamDesc*, const uint16_t*, double*,
                                         double*, cudaStream_t);

void launch_decode_dyn(int grid, const uint8_t* meta, const StreamDesc* sd, const uint16_t* cb_sym,
                       const void* tables, const uint32_t* sub_off, const uint64_t* chunk_word_off,
                       const uint32_t* payload, uint16_t* codes, cudaStream_t st)
{
    k_decode_dyn<<<grid, kDecodeThreads, 0, st>>>(meta, sd, static_cast<const DecodeTables*>(tables), cb_sym, sub_off,
                                                  chunk_word_off, payload, codes, decode_seq_bits());
}

template <typename T>
void launch_unpred_scatter_dyn(int grid, const uint8_t* meta, const StreamDesc* sd, const uint16_t* codes, T* dense,
                               T* list, cudaStream_t st)
{
    k_unpred_scatter_dyn<T><<<grid, 1024, 0, st>>>(meta, sd, codes, dense, list);
}

template void launch_unpred_scatter_dyn<float>(int, const uint8_t*, const StreamDesc*, const uint16_t*, float*, float*,
                                               cudaStream_t);
template void launch_unpred_scatter_dyn<double>(int, const uint8_t*, const StreamDesc*, const uint16_t*, double*,
                                                double*, cudaStream_t);

}  // namespace stz
