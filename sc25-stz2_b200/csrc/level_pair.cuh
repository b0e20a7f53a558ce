// Paired f32 level kernels (included by levels.cu inside its anonymous
// namespace, after level_kernels.cuh).
//
// The interior kernels of f32 levels spend most of their issue slots on the
// predictor: ~210 explicitly rounded FP32 adds, subtracts and multiplies per
// coarse point for the 7 blocks (no contraction, the reference's order), plus
// 34 shared-memory taps. sm_100 has packed two-lane FP32 arithmetic
// (add/sub/mul .rn.ftz.f32x2: two independent IEEE operations with the same
// rounding and flushing as the scalar .rn.ftz forms, one instruction). These
// kernels let each thread predict two points of its column at once, (x, y, z)
// and (x, y, z + 1): every predictor operation becomes one f32x2 instruction
// for both points. The coarse halo tile is stored z-doubled in shared memory,
// entry (x, y, t) = (v(x, y, t), v(x, y, t + 1)), so each stencil tap of the
// pair is a single 64-bit shared load at the same offset as in the scalar
// tile. Divisions (the blends) run as two scalar div.rn.ftz.f32. Residuals,
// quantization, codes, histogram and the decoded cell then follow the scalar
// code point by point, so every value written is the scalar kernel's.

// Two f32 lanes in one 64-bit register pair (lo = point z, hi = point z + 1).
struct F2 {
    unsigned long long v;
    F2() = default;
    __device__ __forceinline__ explicit F2(float c) { asm("mov.b64 %0, {%1, %1};" : "=l"(v) : "f"(c)); }
    __device__ __forceinline__ static F2 make(float a, float b)
    {
        F2 r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
        return r;
    }
    __device__ __forceinline__ void split(float& a, float& b) const
    {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    }
};

}  // namespace
template <>
struct Ar<F2> {
    static __device__ __forceinline__ F2 add(F2 a, F2 b)
    {
        F2 r;
        asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
        return r;
    }
    static __device__ __forceinline__ F2 sub(F2 a, F2 b)
    {
        F2 r;
        asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
        return r;
    }
    static __device__ __forceinline__ F2 mul(F2 a, F2 b)
    {
        F2 r;
        asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
        return r;
    }
    static __device__ __forceinline__ F2 div(F2 a, F2 b)
    {
        float a0, a1, b0, b1;
        a.split(a0, a1);
        b.split(b0, b1);
        return F2::make(Ar<float>::div(a0, b0), Ar<float>::div(a1, b1));
    }
};
namespace {

// Accessor on the z-doubled tile: the pair of coarse values at an offset.
struct PairTileAt {
    const unsigned long long* p;
    static constexpr int sx = TSX, sy = TPLANE;
    __device__ __forceinline__ F2 operator()(int off) const
    {
        F2 r;
        r.v = p[off];
        return r;
    }
};

// Pair planes of a ZB-deep brick: plane t holds (v(t), v(t + 1)) of the scalar
// tile's planes t and t + 1, t = 0 .. ZB + 1.
template <int ZB>
constexpr size_t pair_tile_bytes()
{
    return sizeof(unsigned long long) * (size_t)TPLANE * (ZB + 2);
}

// Stage the coarse halo of [x0-1, x0+BX+1] x [y0-1, y0+BY+1] x [z0-1, z0+ZB+1]
// z-doubled (zero outside the grid, as load_tile).
template <int ZB>
__device__ __forceinline__ void load_pair_tile(float* pt, const float* __restrict__ R, int dx, int dy, int dz, int x0,
                                               int y0, int z0)
{
    const int tid = threadIdx.y * BX + threadIdx.x;
    for (int i = tid; i < tile_elems<ZB>(); i += BX * BY) {
        const int tz = i / TPLANE, rem = i - tz * TPLANE;
        const int ty = rem / TSX, tx = rem - ty * TSX;
        const int gx = x0 - 1 + tx, gy = y0 - 1 + ty, gz = z0 - 1 + tz;
        float v = 0.f;
        if (gx >= 0 && gx < dx && gy >= 0 && gy < dy && gz >= 0 && gz < dz)
            v = __ldg(R + ((size_t)gz * dy + gy) * dx + gx);
        if (tz <= ZB + 1) pt[2 * i] = v;            // lo of pair plane tz
        if (tz >= 1) pt[2 * (i - TPLANE) + 1] = v;  // hi of pair plane tz - 1
    }
}

template <int PRED, typename T, class Acc>
__device__ __forceinline__ void predict7_interior(const Acc& r, T (&p)[7])
{
    p[0] = predict_interior_at<PRED, 0, T>(r);
    p[1] = predict_interior_at<PRED, 1, T>(r);
    p[2] = predict_interior_at<PRED, 2, T>(r);
    p[3] = predict_interior_at<PRED, 3, T>(r);
    p[4] = predict_interior_at<PRED, 4, T>(r);
    p[5] = predict_interior_at<PRED, 5, T>(r);
    p[6] = predict_interior_at<PRED, 6, T>(r);
}

// The 7 predictions of points (x, y, z) and (x, y, z + 1), split per point,
// and the two coarse values at the points.
template <int PRED>
__device__ __forceinline__ void predict_pair(const PairTileAt& r, float (&p0)[7], float (&p1)[7], float& r00,
                                             float& r01)
{
    F2 p[7];
    predict7_interior<PRED>(r, p);
#pragma unroll
    for (int b = 0; b < 7; ++b) p[b].split(p0[b], p1[b]);
    r(0).split(r00, r01);
}

// Interior encode of an f32 level, two points per thread per step (see the
// file comment). Same brick, histogram and outputs as k_level_encode.
template <int PRED, bool FINEST, int ZB>
__global__ void __launch_bounds__(BX* BY, 2) k_level_encode_pair(EncodeIO<float> io, const float* __restrict__ R,
                                                                 LevelGeom geo, QuantParams qp, HistArgs hist)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* pt = reinterpret_cast<float*>(smem_raw);
    __shared__ uint32_t sh[7][kSmemBins];
    __shared__ float lut[2 * kRecW];
    const int tid = threadIdx.y * BX + threadIdx.x;
    for (int i = tid; i < 7 * kSmemBins; i += BX * BY) (&sh[0][0])[i] = 0;
    if constexpr (!FINEST) build_recover_lut(lut, qp, tid, BX * BY);
    const int wlo = max(0, qp.radius - kSmemBins / 2);
    const int wn = min(kSmemBins, 2 * qp.radius - wlo);
    const int dx = geo.dx, dy = geo.dy, dz = geo.dz;
    const int x0 = 1 + blockIdx.x * BX, y0 = 1 + blockIdx.y * BY, z0 = 1 + blockIdx.z * ZB;
    load_pair_tile<ZB>(pt, R, dx, dy, dz, x0, y0, z0);
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool valid = x <= dx - 3 && y <= dy - 3;
    ChunkIndex ci;
    ci.init(geo, x, y);
    uint32_t center[7] = {0, 0, 0, 0, 0, 0, 0};
    const int z1 = min(z0 + ZB, dz - 2);
    const unsigned long long* base = reinterpret_cast<const unsigned long long*>(pt);
    for (int z = z0; z < z1; z += 2) {
        int q0[7] = {-1, -1, -1, -1, -1, -1, -1};
        int q1[7] = {-1, -1, -1, -1, -1, -1, -1};
        if (valid) {
            const PairTileAt r{base + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
            float p0[7], p1[7], r00, r01;
            predict_pair<PRED>(r, p0, p1, r00, r01);
            encode_residuals<float, FINEST>(io, geo, qp, lut, ci, x, y, z, p0, r00, q0);
            if (z + 1 < z1) encode_residuals<float, FINEST>(io, geo, qp, lut, ci, x, y, z + 1, p1, r01, q1);
        }
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            hist_code(sh, wlo, wn, hist, b, q0[b], center[b]);
            hist_code(sh, wlo, wn, hist, b, q1[b], center[b]);
        }
    }
    hist_flush_center(sh, wlo, wn, hist, center);
    __syncthreads();
    for (int i = tid; i < 7 * kSmemBins; i += BX * BY) {
        const int b = i / kSmemBins, w = i % kSmemBins;
        const uint32_t c = sh[b][w];
        if (c) atomicAdd(&hist.full[(size_t)b * 2 * hist.radius + wlo + w], c);
    }
}

// Interior decode of an f32 level, two points per thread per step.
template <int PRED, int ZB>
__global__ void __launch_bounds__(BX* BY, 2) k_level_decode_pair(const float* __restrict__ R, LevelGeom geo,
                                                                 QuantParams qp, const uint16_t* __restrict__ codes,
                                                                 const float* __restrict__ unpred_dense,
                                                                 float* __restrict__ G)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* pt = reinterpret_cast<float*>(smem_raw);
    __shared__ float lut[2 * kRecW];
    const int tid = threadIdx.y * BX + threadIdx.x;
    build_recover_lut(lut, qp, tid, BX * BY);
    const int dx = geo.dx, dy = geo.dy, dz = geo.dz;
    const int x0 = 1 + blockIdx.x * BX, y0 = 1 + blockIdx.y * BY, z0 = 1 + blockIdx.z * ZB;
    load_pair_tile<ZB>(pt, R, dx, dy, dz, x0, y0, z0);
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x > dx - 3 || y > dy - 3) return;
    ChunkIndex ci;
    ci.init(geo, x, y);
    const int z1 = min(z0 + ZB, dz - 2);
    const unsigned long long* base = reinterpret_cast<const unsigned long long*>(pt);
    for (int z = z0; z < z1; z += 2) {
        const PairTileAt r{base + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
        float p0[7], p1[7], r00, r01;
        predict_pair<PRED>(r, p0, p1, r00, r01);
        decode_values<float>(geo, qp, lut, codes, unpred_dense, G, ci, x, y, z, p0, r00);
        if (z + 1 < z1) decode_values<float>(geo, qp, lut, codes, unpred_dense, G, ci, x, y, z + 1, p1, r01);
    }
}
