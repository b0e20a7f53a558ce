// Level kernels of the staged predictor (predictor 2, src/dependency.cpp),
// included by levels.cu inside its anonymous namespace after the chunk-index,
// histogram and recover helpers.
//
// The staged predictor makes each level a chain of three dependent steps:
// blocks 0, 1, 3 (one odd axis) are 1-D cubics along that axis of the coarse
// grid; blocks 2, 4, 5 blend two 1-D cubics through the decoded blocks 0, 1,
// 3; block 6 blends three through the decoded blocks 2, 4, 5 (staged_prediction,
// dependency.cpp:258-292). A stage needs its siblings' decoded values at
// -1..+2 along an axis, i.e. from points other threads own, so each stage is
// its own launch over the level's fine grid G: stage 1 writes the coarse copy
// (parity 0) and parities 1, 2, 4; stage 2 reads those and writes 3, 5, 6;
// stage 3 reads 3, 5, 6 and writes 7. No launch reads a position it writes.
// The encoder keeps the decoded values in G (the decoded fine grid the next
// level predicts from, or a scratch grid on the finest level), the decoder
// writes them to its output grid. Codes, unpredictable values, per-chunk
// counts and histograms go where the other predictors' level kernels put
// them, so the entropy coder and the container are the same.
//
// One thread per coarse point and stage; a CTA is a 32 x 8 tile of one
// coarse z plane (grid-strided along z). The taps are plain global loads: the
// mode is off the default path, and its level chain is bound by the three
// launches' passes over G (about 3x the bytes of a one-pass level).

// 1-D cubic along one axis of the coarse grid (interp_axis,
// dependency.cpp:90-118): c the point, st its stride along the axis, pos /
// dim its index and the extent there.
template <typename T>
__device__ __forceinline__ T dep_line(const T* __restrict__ c, long long st, int pos, int dim)
{
    using A = Ar<T>;
    if (pos == dim - 1) return __ldg(c);
    const T b = __ldg(c), cc = __ldg(c + st);
    if (pos == dim - 2 || pos == 0) return A::mul(T(0.5f), A::add(b, cc));
    const T a = __ldg(c - st), d = __ldg(c + 2 * st);
    return A::add(A::add(A::add(A::mul(T(-0.0625f), a), A::mul(T(0.5625f), b)), A::mul(T(0.5625f), cc)),
                  A::mul(T(-0.0625f), d));
}

// The same line with its curvature variance (interp_axis_with_variance,
// dependency.cpp:162-243) on a decoded sibling in G. The reference squares
// |b - a|; squaring b - a gives the same bits.
template <typename T>
__device__ __forceinline__ void dep_line_pv(const T* c, long long st, int pos, int dim, T& p, T& v)
{
    using A = Ar<T>;
    const T eps = T(1e-12f);
    if (pos == dim - 1) {
        p = c[0];
        v = eps;
        return;
    }
    const T b = c[0], cc = c[st];
    if (pos == dim - 2 || pos == 0) {
        const T e = A::sub(cc, b);
        p = A::mul(T(0.5f), A::add(b, cc));
        v = A::add(A::mul(e, e), eps);
        return;
    }
    const T a = c[-st], d = c[2 * st];
    const T c0 = A::add(A::sub(a, A::mul(T(2.0f), b)), cc);
    const T c1 = A::add(A::sub(b, A::mul(T(2.0f), cc)), d);
    p = A::add(A::add(A::add(A::mul(T(-0.0625f), a), A::mul(T(0.5625f), b)), A::mul(T(0.5625f), cc)),
               A::mul(T(-0.0625f), d));
    v = A::add(A::mul(T(0.5f), A::add(A::mul(c0, c0), A::mul(c1, c1))), eps);
}

// inverse_variance_blend2 / blend3 (dependency.cpp:245-256).
template <typename T>
__device__ __forceinline__ T dep_blend2(T p0, T v0, T p1, T v1)
{
    using A = Ar<T>;
    return A::div(A::add(A::mul(p0, v1), A::mul(p1, v0)), A::add(v0, v1));
}
template <typename T>
__device__ __forceinline__ T dep_blend3(T p0, T v0, T p1, T v1, T p2, T v2)
{
    using A = Ar<T>;
    const T w0 = A::mul(v1, v2), w1 = A::mul(v0, v2), w2 = A::mul(v0, v1);
    return A::div(A::add(A::add(A::mul(w0, p0), A::mul(w1, p1)), A::mul(w2, p2)), A::add(A::add(w0, w1), w2));
}

// Level geometry of the staged kernels: coarse strides, fine-grid strides,
// and a sibling's step along each axis (two fine points).
struct StagedGeom {
    int dx, dy, dz;
    long long cy, cz;  // coarse row / plane strides
    long long gy, gz;  // fine row / plane strides (2dx, 4dx*dy)
    __host__ __device__ static StagedGeom make(const LevelGeom& g)
    {
        StagedGeom s;
        s.dx = g.dx, s.dy = g.dy, s.dz = g.dz;
        s.cy = g.dx, s.cz = (long long)g.dx * g.dy;
        s.gy = 2LL * g.dx, s.gz = 4LL * g.dx * g.dy;
        return s;
    }
    // fine-grid index of sub-block s at coarse (x, y, z)
    __device__ __forceinline__ long long fine(int s, int x, int y, int z) const
    {
        return (long long)(2 * z + (s >> 2)) * gz + (long long)(2 * y + ((s >> 1) & 1)) * gy + 2LL * x + (s & 1);
    }
};

// Prediction of block b at coarse (x, y, z) (staged_prediction,
// dependency.cpp:258-292, and interp_axis for blocks 0, 1, 3,
// dependency.cpp:333-383): ref_x, ref_y, ref_z, ref_xy, ref_xz, ref_yz are
// sub-blocks 1, 2, 4, 3, 5, 6 of G.
template <typename T>
__device__ __forceinline__ T staged_predict(int b, const T* __restrict__ R, const T* G, const StagedGeom& s, int x,
                                            int y, int z)
{
    const T* c = R + (long long)z * s.cz + (long long)y * s.cy + x;
    T p0, v0, p1, v1, p2, v2;
    switch (b) {
    case 0: return dep_line<T>(c, 1, x, s.dx);
    case 1: return dep_line<T>(c, s.cy, y, s.dy);
    case 3: return dep_line<T>(c, s.cz, z, s.dz);
    case 2:
        dep_line_pv<T>(G + s.fine(1, x, y, z), 2 * s.gy, y, s.dy, p0, v0);
        dep_line_pv<T>(G + s.fine(2, x, y, z), 2, x, s.dx, p1, v1);
        return dep_blend2(p0, v0, p1, v1);
    case 4:
        dep_line_pv<T>(G + s.fine(1, x, y, z), 2 * s.gz, z, s.dz, p0, v0);
        dep_line_pv<T>(G + s.fine(4, x, y, z), 2, x, s.dx, p1, v1);
        return dep_blend2(p0, v0, p1, v1);
    case 5:
        dep_line_pv<T>(G + s.fine(2, x, y, z), 2 * s.gz, z, s.dz, p0, v0);
        dep_line_pv<T>(G + s.fine(4, x, y, z), 2 * s.gy, y, s.dy, p1, v1);
        return dep_blend2(p0, v0, p1, v1);
    default:
        dep_line_pv<T>(G + s.fine(3, x, y, z), 2 * s.gz, z, s.dz, p0, v0);
        dep_line_pv<T>(G + s.fine(5, x, y, z), 2 * s.gy, y, s.dy, p1, v1);
        dep_line_pv<T>(G + s.fine(6, x, y, z), 2, x, s.dx, p2, v2);
        return dep_blend3(p0, v0, p1, v1, p2, v2);
    }
}

// Blocks of each stage.
__device__ __forceinline__ int staged_block(int stage, int j)
{
    return stage == 1 ? (j == 2 ? 3 : j) : stage == 2 ? (j == 0 ? 2 : j == 1 ? 4 : 5) : 6;
}

constexpr int kStagedTX = 32, kStagedTY = 8;

// Encoder stage: per coarse point and block of the stage, fine value,
// prediction, residual, code (chunk-major), unpredictable value and chunk
// count, histogram, decoded value into G. Stage 1 also copies the coarse
// value into G's parity 0.
template <typename T, int STAGE>
__global__ void __launch_bounds__(kStagedTX* kStagedTY) k_staged_encode(EncodeIO<T> io, T* G, const T* __restrict__ R,
                                                                        LevelGeom geo, QuantParams qp, HistArgs hist)
{
    using A = Ar<T>;
    constexpr int NB = STAGE == 3 ? 1 : 3;
    const StagedGeom s = StagedGeom::make(geo);
    const int x = blockIdx.x * kStagedTX + threadIdx.x, y = blockIdx.y * kStagedTY + threadIdx.y;
    const bool in = x < geo.dx && y < geo.dy;
    ChunkIndex ci;
    if (in) ci.init(geo, x, y);
    uint32_t center[7] = {0, 0, 0, 0, 0, 0, 0};
    const size_t n = geo.n;
    for (int z = blockIdx.z; z < geo.dz; z += gridDim.z) {
        int q[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) q[j] = -1;
        if (in) {
            int chunk;
            const size_t cm = ci.at(z, chunk);
            if (STAGE == 1) G[s.fine(0, x, y, z)] = __ldg(R + (long long)z * s.cz + (long long)y * s.cy + x);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const int b = staged_block(STAGE, j), sb = b + 1;
                const int px = sb & 1, py = (sb >> 1) & 1, pz = sb >> 2;
                const T p = staged_predict<T>(b, R, G, s, x, y, z);
                const T o = __ldg(io.field + (size_t)(io.s * (2 * z + pz)) * io.fsy +
                                  (size_t)(io.s * (2 * y + py)) * io.fsx + (size_t)io.s * (2 * x + px));
                const T d = A::sub(o, p);
                const int code = quantize(d, qp);
                q[j] = code;
                io.codes[(size_t)b * n + cm] = (uint16_t)code;
                if (code == 0) {
                    io.unpred_dense[(size_t)b * n + cm] = d;
                    atomicAdd(&io.unpred_cnt[(size_t)b * (geo.nchunks() + 1) + chunk], 1u);
                }
                G[s.fine(sb, x, y, z)] = A::add(code ? recover<T>(code, qp) : d, p);
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const int b = staged_block(STAGE, j);
            hist_code(nullptr, 0, 0, hist, b, q[j], center[b]);
        }
    }
    hist_flush_center(nullptr, 0, 0, hist, center);
}

// Decoder stage: x' = recover(q) (or the unpredictable value) + prediction,
// into the output grid G; stage 1 also copies the coarse value to parity 0.
template <typename T, int STAGE>
__global__ void __launch_bounds__(kStagedTX* kStagedTY) k_staged_decode(const T* __restrict__ R, LevelGeom geo,
                                                                        QuantParams qp,
                                                                        const uint16_t* __restrict__ codes,
                                                                        const T* __restrict__ unpred_dense, T* G)
{
    using A = Ar<T>;
    constexpr int NB = STAGE == 3 ? 1 : 3;
    const StagedGeom s = StagedGeom::make(geo);
    const int x = blockIdx.x * kStagedTX + threadIdx.x, y = blockIdx.y * kStagedTY + threadIdx.y;
    if (x >= geo.dx || y >= geo.dy) return;
    ChunkIndex ci;
    ci.init(geo, x, y);
    const size_t n = geo.n;
    for (int z = blockIdx.z; z < geo.dz; z += gridDim.z) {
        int chunk;
        const size_t cm = ci.at(z, chunk);
        if (STAGE == 1) G[s.fine(0, x, y, z)] = __ldg(R + (long long)z * s.cz + (long long)y * s.cy + x);
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const int b = staged_block(STAGE, j);
            const int q = __ldg(codes + (size_t)b * n + cm);
            const T dq = q ? recover<T>(q, qp) : __ldg(unpred_dense + (size_t)b * n + cm);
            G[s.fine(b + 1, x, y, z)] = A::add(dq, staged_predict<T>(b, R, G, s, x, y, z));
        }
    }
}

inline dim3 staged_grid(const LevelGeom& g)
{
    return dim3((unsigned)((g.dx + kStagedTX - 1) / kStagedTX), (unsigned)((g.dy + kStagedTY - 1) / kStagedTY),
                (unsigned)std::min(g.dz, 65535));
}

// The reference's per-block stage functions on dense sub-block arrays of
// dx*dy*dz values (mode 0: diff = sub - P, mode 1: out = de + P). Blocks 0, 1,
// 3 read refs.p[0], the coarse sub-block 0 (preprocess_block /
// depreprocess_block, dependency.cpp:333-431); blocks 2, 4, 5, 6 read ref_x,
// ref_y, ref_z, ref_xy, ref_xz, ref_yz = refs.p[0..5]
// (preprocess_block_staged / depreprocess_block_staged,
// dependency.cpp:294-331), each entry only where the block's lines need it.
struct StagedRefs {
    const void* p[6];
};

template <typename T>
__global__ void __launch_bounds__(256) k_block_staged(int mode, int block, const T* __restrict__ src, StagedRefs refs,
                                                      T* __restrict__ dst, int dx, int dy, int dz)
{
    using A = Ar<T>;
    const long long sy = dx, sz = (long long)dx * dy;
    const size_t m = (size_t)sz * dz;
    auto ref = [&](int k, size_t i) { return static_cast<const T*>(refs.p[k]) + i; };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)dx), y = (int)((i / (size_t)dx) % (size_t)dy), z = (int)(i / (size_t)sz);
        T p, p0, v0, p1, v1, p2, v2;
        switch (block) {
        case 0: p = dep_line<T>(ref(0, i), 1, x, dx); break;
        case 1: p = dep_line<T>(ref(0, i), sy, y, dy); break;
        case 3: p = dep_line<T>(ref(0, i), sz, z, dz); break;
        case 2:
            dep_line_pv<T>(ref(0, i), sy, y, dy, p0, v0);
            dep_line_pv<T>(ref(1, i), 1, x, dx, p1, v1);
            p = dep_blend2(p0, v0, p1, v1);
            break;
        case 4:
            dep_line_pv<T>(ref(0, i), sz, z, dz, p0, v0);
            dep_line_pv<T>(ref(2, i), 1, x, dx, p1, v1);
            p = dep_blend2(p0, v0, p1, v1);
            break;
        case 5:
            dep_line_pv<T>(ref(1, i), sz, z, dz, p0, v0);
            dep_line_pv<T>(ref(2, i), sy, y, dy, p1, v1);
            p = dep_blend2(p0, v0, p1, v1);
            break;
        default:
            dep_line_pv<T>(ref(3, i), sz, z, dz, p0, v0);
            dep_line_pv<T>(ref(4, i), sy, y, dy, p1, v1);
            dep_line_pv<T>(ref(5, i), 1, x, dx, p2, v2);
            p = dep_blend3(p0, v0, p1, v1, p2, v2);
            break;
        }
        dst[i] = mode == 0 ? A::sub(src[i], p) : A::add(src[i], p);
    }
}
