// Level kernels of the 12-point truncated bicubic predictor (predictor 3,
// src/stz2.cpp), included by levels.cu inside its anonymous namespace after
// the chunk-index, histogram and recover helpers.
//
// The predictor reads only the coarse grid, so a level is one pass, thread
// per coarse point and all 7 blocks, with the same outputs as the other
// predictors' level kernels (codes chunk-major, unpredictable values, chunk
// counts, histograms, decoded fine grid on the coarser levels). It is the
// plain stencil family of src/float.cpp except in two places:
//   * blocks 2, 4, 5 (two odd axes) take a 12-point truncated bicubic inside:
//     the 4 inner points weighted (9/16)^2, the 8 edge points -(1/16)(9/16),
//     no corners (stz2.cpp:122-155, 170-232);
//   * the one-axis interior cubic has double weights (stz2.cpp:86, 100-118),
//     so the prediction, the residual and the rebuilt value are evaluated in
//     double and rounded to T once.
// Boundaries and block 6 are float.cpp's. Taps are plain global loads
// through L1/L2: the mode is off the default path.

template <typename T>
struct TruncPred {
    T p;        // the prediction in T (unless wide)
    double pd;  // the double prediction (wide)
    bool wide;
};

template <typename T>
__device__ __forceinline__ TruncPred<T> trunc_predict(int b, const Grid<T>& g, int x, int y, int z)
{
    using A = Ar<T>;
    using D = Ar<double>;
    const T* __restrict__ r = g.p + (size_t)z * g.sy + (size_t)y * g.sx + x;
    const long long sx = (long long)g.sx, sy = (long long)g.sy;
    long long st = 0, a1 = 0, a2 = 0;
    int pos = 0, dim = 0;
    bool inner = false;
    switch (b) {
    case 0: st = 1, pos = x, dim = g.dx; break;
    case 1: st = sx, pos = y, dim = g.dy; break;
    case 3: st = sy, pos = z, dim = g.dz; break;
    case 2: a1 = 1, a2 = sx, inner = x >= 1 && x < g.dx - 2 && y >= 1 && y < g.dy - 2; break;
    case 4: a1 = 1, a2 = sy, inner = x >= 1 && x < g.dx - 2 && z >= 1 && z < g.dz - 2; break;
    case 5: a1 = sx, a2 = sy, inner = y >= 1 && y < g.dy - 2 && z >= 1 && z < g.dz - 2; break;
    default: break;
    }
    TruncPred<T> o;
    o.wide = false;
    o.pd = 0.0;
    if (st && pos >= 1 && pos < dim - 2) {
        const double a = A::to_f64(__ldg(r - st)), bb = A::to_f64(__ldg(r)), c = A::to_f64(__ldg(r + st)),
                     d = A::to_f64(__ldg(r + 2 * st));
        o.wide = true;
        o.pd = D::add(D::add(D::add(D::mul(-0.0625, a), D::mul(0.5625, bb)), D::mul(0.5625, c)), D::mul(-0.0625, d));
        o.p = T(0);
        return o;
    }
    if (inner) {
        const T core = A::add(A::add(A::add(__ldg(r), __ldg(r + a1)), __ldg(r + a2)), __ldg(r + a2 + a1));
        T e = A::add(__ldg(r - a1), __ldg(r + 2 * a1));
        e = A::add(e, __ldg(r + a2 - a1));
        e = A::add(e, __ldg(r + a2 + 2 * a1));
        e = A::add(e, __ldg(r - a2));
        e = A::add(e, __ldg(r - a2 + a1));
        e = A::add(e, __ldg(r + 2 * a2));
        e = A::add(e, __ldg(r + 2 * a2 + a1));
        o.p = A::add(A::mul(T(0.31640625f), core), A::mul(T(-0.033203125f), e));
        return o;
    }
    o.p = predict<1>(b, g, x, y, z);
    return o;
}

// residual o - P and rebuilt value dq + P, in double where the prediction is
template <typename T>
__device__ __forceinline__ T trunc_residual(T o, const TruncPred<T>& p)
{
    using A = Ar<T>;
    return p.wide ? A::from_f64(Ar<double>::sub(A::to_f64(o), p.pd)) : A::sub(o, p.p);
}
template <typename T>
__device__ __forceinline__ T trunc_rebuild(T dq, const TruncPred<T>& p)
{
    using A = Ar<T>;
    return p.wide ? A::from_f64(Ar<double>::add(A::to_f64(dq), p.pd)) : A::add(dq, p.p);
}

constexpr int kTruncTX = 32, kTruncTY = 8;

template <typename T>
__global__ void __launch_bounds__(kTruncTX* kTruncTY) k_trunc_encode(EncodeIO<T> io, const T* __restrict__ R,
                                                                     LevelGeom geo, QuantParams qp, HistArgs hist)
{
    const Grid<T> g{R, geo.dx, geo.dy, geo.dz, (size_t)geo.dx, (size_t)geo.dx * geo.dy};
    const int x = blockIdx.x * kTruncTX + threadIdx.x, y = blockIdx.y * kTruncTY + threadIdx.y;
    const bool in = x < geo.dx && y < geo.dy;
    ChunkIndex ci;
    if (in) ci.init(geo, x, y);
    uint32_t center[7] = {0, 0, 0, 0, 0, 0, 0};
    const size_t n = geo.n;
    const long long gy = 2LL * geo.dx, gz = 4LL * geo.dx * geo.dy;
    for (int z = blockIdx.z; z < geo.dz; z += gridDim.z) {
        int q[7] = {-1, -1, -1, -1, -1, -1, -1};
        if (in) {
            int chunk;
            const size_t cm = ci.at(z, chunk);
            if (io.G) io.G[(long long)(2 * z) * gz + (long long)(2 * y) * gy + 2LL * x] = __ldg(R + (size_t)z * g.sy + (size_t)y * g.sx + x);
#pragma unroll
            for (int b = 0; b < 7; ++b) {
                const int sb = b + 1, px = sb & 1, py = (sb >> 1) & 1, pz = sb >> 2;
                const TruncPred<T> p = trunc_predict<T>(b, g, x, y, z);
                const T o = __ldg(io.field + (size_t)(io.s * (2 * z + pz)) * io.fsy +
                                  (size_t)(io.s * (2 * y + py)) * io.fsx + (size_t)io.s * (2 * x + px));
                const T d = trunc_residual(o, p);
                const int code = quantize(d, qp);
                q[b] = code;
                io.codes[(size_t)b * n + cm] = (uint16_t)code;
                if (code == 0) {
                    io.unpred_dense[(size_t)b * n + cm] = d;
                    atomicAdd(&io.unpred_cnt[(size_t)b * (geo.nchunks() + 1) + chunk], 1u);
                }
                if (io.G)
                    io.G[(long long)(2 * z + pz) * gz + (long long)(2 * y + py) * gy + 2LL * x + px] =
                        trunc_rebuild(code ? recover<T>(code, qp) : d, p);
            }
        }
#pragma unroll
        for (int b = 0; b < 7; ++b) hist_code(nullptr, 0, 0, hist, b, q[b], center[b]);
    }
    hist_flush_center(nullptr, 0, 0, hist, center);
}

template <typename T>
__global__ void __launch_bounds__(kTruncTX* kTruncTY) k_trunc_decode(const T* __restrict__ R, LevelGeom geo,
                                                                     QuantParams qp,
                                                                     const uint16_t* __restrict__ codes,
                                                                     const T* __restrict__ unpred_dense, T* G)
{
    const Grid<T> g{R, geo.dx, geo.dy, geo.dz, (size_t)geo.dx, (size_t)geo.dx * geo.dy};
    const int x = blockIdx.x * kTruncTX + threadIdx.x, y = blockIdx.y * kTruncTY + threadIdx.y;
    if (x >= geo.dx || y >= geo.dy) return;
    ChunkIndex ci;
    ci.init(geo, x, y);
    const size_t n = geo.n;
    const long long gy = 2LL * geo.dx, gz = 4LL * geo.dx * geo.dy;
    for (int z = blockIdx.z; z < geo.dz; z += gridDim.z) {
        int chunk;
        const size_t cm = ci.at(z, chunk);
        G[(long long)(2 * z) * gz + (long long)(2 * y) * gy + 2LL * x] = __ldg(R + (size_t)z * g.sy + (size_t)y * g.sx + x);
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            const int sb = b + 1, px = sb & 1, py = (sb >> 1) & 1, pz = sb >> 2;
            const int q = __ldg(codes + (size_t)b * n + cm);
            const T dq = q ? recover<T>(q, qp) : __ldg(unpred_dense + (size_t)b * n + cm);
            G[(long long)(2 * z + pz) * gz + (long long)(2 * y + py) * gy + 2LL * x + px] =
                trunc_rebuild(dq, trunc_predict<T>(b, g, x, y, z));
        }
    }
}

inline dim3 trunc_grid(const LevelGeom& g)
{
    return dim3((unsigned)((g.dx + kTruncTX - 1) / kTruncTX), (unsigned)((g.dy + kTruncTY - 1) / kTruncTY),
                (unsigned)std::min(g.dz, 65535));
}
