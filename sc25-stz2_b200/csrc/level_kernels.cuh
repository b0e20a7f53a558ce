// Level encode / decode kernels (included by levels.cu inside its anonymous
// namespace, after the tile, histogram and chunk-index helpers).
//
// Each level runs as two launches that together cover every coarse point once:
//   * the interior kernel: points with 1 <= x,y,z <= dim-3, where every block
//     uses its interior stencil; 32x8x8 bricks with the coarse halo staged in
//     shared memory, no boundary branches, so no warp ever runs both the
//     interior and the boundary form of the predictor;
//   * the shell kernel: the remaining points (index 0, dim-2, dim-1 on some
//     axis), thread per point, predictor taps read from global memory (L2).

// Shell enumeration: group 1 = boundary z planes (all x, y); group 2 =
// interior z, boundary y rows (all x); group 3 = interior z and y, boundary x.
struct Shell {
    int dx, dy, dz;
    int nbx, nby, nbz, nix, niy, niz;
    uint64_t g1, g2, g3;
    __host__ __device__ static int nb(int d) { return d < 3 ? d : 3; }
    __host__ __device__ static int ni(int d) { return d > 3 ? d - 3 : 0; }
    __host__ static Shell make(int dx, int dy, int dz)
    {
        Shell s;
        s.dx = dx, s.dy = dy, s.dz = dz;
        s.nbx = nb(dx), s.nby = nb(dy), s.nbz = nb(dz);
        s.nix = ni(dx), s.niy = ni(dy), s.niz = ni(dz);
        if (s.nix == 0 || s.niy == 0 || s.niz == 0) {  // no interior: every point is shell
            s.nbz = dz, s.niz = 0;
        }
        s.g1 = (uint64_t)s.nbz * dy * dx;
        s.g2 = (uint64_t)s.niz * s.nby * dx;
        s.g3 = (uint64_t)s.niz * s.niy * s.nbx;
        return s;
    }
    uint64_t total() const { return g1 + g2 + g3; }
    // k-th boundary index of an axis of size d: 0, d-2, d-1 (all when d < 4)
    __device__ static int bval(int k, int d) { return d < 4 ? k : (k == 0 ? 0 : d - 3 + k); }
    // 32-bit index arithmetic when the shell and a plane fit (64-bit
    // division is a long instruction sequence on the GPU)
    __host__ __device__ bool small() const
    {
        return g1 + g2 + g3 < (1ull << 31) && (uint64_t)dx * dy < (1ull << 31);
    }
    __device__ void point32(uint32_t i, int& x, int& y, int& z) const
    {
        const uint32_t G1 = (uint32_t)g1, G2 = (uint32_t)g2, udx = (uint32_t)dx;
        if (i < G1) {
            const uint32_t plane = (uint32_t)dy * udx;
            const uint32_t kz = i / plane, r = i - kz * plane;
            z = nbz == dz ? (int)kz : bval((int)kz, dz);
            y = (int)(r / udx), x = (int)(r - (uint32_t)y * udx);
        } else if (i < G1 + G2) {
            const uint32_t j = i - G1, plane = (uint32_t)nby * udx;
            const uint32_t kz = j / plane, r = j - kz * plane;
            z = 1 + (int)kz;
            y = bval((int)(r / udx), dy), x = (int)(r % udx);
        } else {
            const uint32_t j = i - G1 - G2, plane = (uint32_t)niy * (uint32_t)nbx;
            const uint32_t kz = j / plane, r = j - kz * plane;
            z = 1 + (int)kz;
            y = 1 + (int)(r / (uint32_t)nbx), x = bval((int)(r % (uint32_t)nbx), dx);
        }
    }
    __device__ void point(uint64_t i, int& x, int& y, int& z) const
    {
        if (small()) {
            point32((uint32_t)i, x, y, z);
            return;
        }
        if (i < g1) {
            const uint64_t plane = (uint64_t)dy * dx;
            const int kz = (int)(i / plane);
            z = nbz == dz ? kz : bval(kz, dz);
            const uint64_t r = i - (uint64_t)kz * plane;
            y = (int)(r / dx), x = (int)(r - (uint64_t)y * dx);
        } else if (i < g1 + g2) {
            const uint64_t j = i - g1, plane = (uint64_t)nby * dx;
            z = 1 + (int)(j / plane);
            const uint64_t r = j - (uint64_t)(z - 1) * plane;
            y = bval((int)(r / dx), dy), x = (int)(r % dx);
        } else {
            const uint64_t j = i - g1 - g2, plane = (uint64_t)niy * nbx;
            z = 1 + (int)(j / plane);
            const uint64_t r = j - (uint64_t)(z - 1) * plane;
            y = 1 + (int)(r / nbx), x = bval((int)(r % nbx), dx);
        }
    }
};

// Boundary points owned by an interior CTA (plain decode kernels). Along an axis
// of size d the interior indices [1, d-3] are split into bricks of B; the
// first brick also owns index 0 and the last one indices d-2 and d-1, so a
// CTA owns the contiguous range [a, b) around its interior range [i0, i1).
// Its halo tile covers [i0-1, i0+B+1], which holds every tap of the owned
// boundary points: their boundary rules read the point and its forward
// neighbour, their other axes the usual -1..+2 stencil inside [i0, i1).
struct OwnedAxis {
    int a, i0, i1, b;
    __device__ __forceinline__ static OwnedAxis make(int d, int blk, int nblk, int B)
    {
        OwnedAxis o;
        o.i0 = 1 + blk * B;
        o.i1 = min(o.i0 + B, d - 2);
        o.a = blk == 0 ? 0 : o.i0;
        o.b = blk == nblk - 1 ? d : o.i1;
        return o;
    }
    __device__ __forceinline__ int n() const { return b - a; }
    __device__ __forceinline__ int ni() const { return i1 - i0; }
    __device__ __forceinline__ int nb() const { return (i0 - a) + (b - i1); }
    // k-th owned boundary index (k < nb())
    __device__ __forceinline__ int bnd(int k) const { return k < i0 - a ? a + k : i1 + (k - (i0 - a)); }
};

// The owned boundary points of this CTA as three disjoint boxes: z outside
// the interior range (all owned x, y); z inside, y outside (all owned x); z
// and y inside, x outside. f(x, y, z) for each, spread over the CTA's threads.
// bz / nbz: the CTA's brick index along z and the level's brick count (a
// launch may cover a range of z-bricks). XCOLS: only the third box (the
// x-boundary columns beside the interior; the encoders leave the other two
// to the boundary-shell kernel, whose z-planes and y-rows it reads
// coalesced, while a column point per thread is not).
template <bool XCOLS = false, class F>
__device__ __forceinline__ void for_owned_boundary(const LevelGeom& g, int ZB, int bz, int nbz, int tid, int nthreads,
                                                   F&& f)
{
    const OwnedAxis X = OwnedAxis::make(g.dx, blockIdx.x, gridDim.x, BX);
    const OwnedAxis Y = OwnedAxis::make(g.dy, blockIdx.y, gridDim.y, BY);
    const OwnedAxis Z = OwnedAxis::make(g.dz, bz, nbz, ZB);
    const int ga = XCOLS ? 0 : X.n() * Y.n() * Z.nb();
    const int gb = XCOLS ? 0 : X.n() * Y.nb() * Z.ni();
    const int gc = X.nb() * Y.ni() * Z.ni();
    for (int i = tid; i < ga + gb + gc; i += nthreads) {
        int x, y, z;
        if (i < ga) {
            const int nxy = X.n() * Y.n();
            z = Z.bnd(i / nxy);
            const int r = i % nxy;
            y = Y.a + r / X.n(), x = X.a + r % X.n();
        } else if (i < ga + gb) {
            const int j = i - ga, nxy = X.n() * Y.nb();
            z = Z.i0 + j / nxy;
            const int r = j % nxy;
            y = Y.bnd(r / X.n()), x = X.a + r % X.n();
        } else {
            const int j = i - ga - gb, nxy = X.nb() * Y.ni();
            z = Z.i0 + j / nxy;
            const int r = j % nxy;
            y = Y.i0 + r / X.nb(), x = X.bnd(r % X.nb());
        }
        f(x, y, z);
    }
}

template <typename T>
struct EncodeIO {
    const T* __restrict__ field;
    size_t fsx, fsy;
    int s;  // sampling stride of the fine grid
    uint16_t* __restrict__ codes;
    T* __restrict__ unpred_dense;
    uint32_t* __restrict__ unpred_cnt;
    T* __restrict__ G;  // decoded fine grid (coarser levels only)
};

// Learned correction modes of the level kernels: none, the network per
// thread with dp4a, or block-wide on the tensor cores (the same integers).
constexpr int kLearnNone = 0, kLearnDp4a = 1, kLearnTc = 2;

// p[b] += acc3[b] * so for the blocks la.flags selects.
template <typename T>
__device__ __forceinline__ void apply_corr(const LearnedArgs<T>& la, const int* acc3, T (&p)[7])
{
#pragma unroll
    for (int b = 0; b < 7; ++b)
        if ((la.flags >> b) & 1u) p[b] = Ar<T>::add(p[b], Ar<T>::mul((T)acc3[b], la.so));
}

// Learned correction of the blocks la.flags selects (interior points only;
// la.model in shared memory): LM == kLearnDp4a evaluates the network here,
// kLearnTc takes the accumulators the block computed (acc3).
template <int LM, typename T, class Acc>
__device__ __forceinline__ void apply_learned(const Acc& r, const LearnedArgs<T>& la, const int* acc3, T (&p)[7])
{
    if constexpr (LM == kLearnDp4a) {
        int a[7];
        learned_mlp_int(*la.model, learned_inputs<T>(r, la.rs), a);
        apply_corr(la, a, p);
    } else if constexpr (LM == kLearnTc) {
        apply_corr(la, acc3, p);
    }
}

// Shared-memory state of the block-wide network (instantiated only by the
// kLearnTc kernels, which are the only callers).
__device__ __forceinline__ tc::Net<2>* net_smem()
{
    __shared__ __align__(1024) tc::Net<2> net;
    return &net;
}

// One coarse point of the encoder after its 7 predictions p: fine values,
// residuals, codes, unpredictable values, decoded fine cell (r0 = the coarse
// value at the point, which is the decoded cell's parity-0 value).
template <typename T, bool FINEST>
__device__ __forceinline__ void encode_residuals(const EncodeIO<T>& io, const LevelGeom& geo, const QuantParams& qp,
                                                 const T* lut, const ChunkIndex& ci, int x, int y, int z,
                                                 const T (&p)[7], T r0, int (&q)[7])
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    T o[8];
    if constexpr (FINEST) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int pz = k >> 1, py = k & 1;
            const T2 t = __ldg(reinterpret_cast<const T2*>(io.field + (size_t)(2 * z + pz) * io.fsy +
                                                           (size_t)(2 * y + py) * io.fsx + 2 * (size_t)x));
            o[2 * k] = t.x;
            o[2 * k + 1] = t.y;
        }
    } else {
        const int s = io.s;
#pragma unroll
        for (int si = 1; si < 8; ++si) {
            const int px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
            o[si] = __ldg(io.field + (size_t)(s * (2 * z + pz)) * io.fsy + (size_t)(s * (2 * y + py)) * io.fsx +
                          (size_t)s * (2 * x + px));
        }
    }
    int chunk;
    const size_t cm = ci.at(z, chunk);
    const size_t n = geo.n;
    T v[8];
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const T d = A::sub(o[b + 1], p[b]);
        const int code = quantize(d, qp);
        q[b] = code;
        io.codes[(size_t)b * n + cm] = (uint16_t)code;
        if (code == 0) {
            io.unpred_dense[(size_t)b * n + cm] = d;
            atomicAdd(&io.unpred_cnt[(size_t)b * (geo.nchunks() + 1) + chunk], 1u);
        }
        if constexpr (!FINEST) v[b + 1] = A::add(code ? recover_lut(lut, code, qp) : d, p[b]);
    }
    if constexpr (!FINEST) {
        v[0] = r0;
        const size_t gsx = 2 * (size_t)geo.dx, gsy = 4 * (size_t)geo.dx * geo.dy;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int pz = k >> 1, py = k & 1;
            T2 t;
            t.x = v[2 * k];
            t.y = v[2 * k + 1];
            *reinterpret_cast<T2*>(io.G + (size_t)(2 * z + pz) * gsy + (size_t)(2 * y + py) * gsx + 2 * (size_t)x) = t;
        }
    }
}

// One coarse point of the encoder: fine values, 7 predictions, residuals,
// codes, unpredictable values, decoded fine cell.
template <typename T, int PRED, bool FINEST, bool INTERIOR, int LM = kLearnNone, class Acc>
__device__ __forceinline__ void encode_point(const Acc& r, const EncodeIO<T>& io, const LevelGeom& geo,
                                             const QuantParams& qp, const T* lut, const ChunkIndex& ci, int x, int y,
                                             int z, int (&q)[7], const LearnedArgs<T>& la = LearnedArgs<T>(),
                                             const int* acc3 = nullptr)
{
    T p[7];
    predict7<PRED>(r, INTERIOR, x, y, z, geo.dx, geo.dy, geo.dz, p);
    apply_learned<LM>(r, la, acc3, p);
    encode_residuals<T, FINEST>(io, geo, qp, lut, ci, x, y, z, p, FINEST ? T(0) : r(0), q);
}

// Interior point of the plain encoder (no learned correction), the same
// values as encode_point. A residual under the quantizer's early-exit bound
// is a centre code, counted in a register; only the others run the full
// quantizer, and only they touch the shared histogram or, as code 0, the
// unpredictable list (the histogram counts code 0 too, like hist_code). The
// walk's chunk-major position, field row pointer fp and decoded-grid pointer
// gp move along z with the thread instead of being recomputed per point.
template <typename T, int PRED, bool FINEST, class Acc>
__device__ __forceinline__ void encode_interior(const Acc& r, const EncodeIO<T>& io, const LevelGeom& geo,
                                                const QuantParams& qp, const T* lut, const ZWalk& zw,
                                                const T* __restrict__ fp, T* __restrict__ gp, uint32_t (*sh)[kSmemBins],
                                                int wlo, int wn, const HistArgs& hist, uint32_t (&center)[7],
                                                const float4* qtab, float qr2)
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    T p[7];
    predict7_interior_only<PRED>(r, p);
    T o[8];
    if constexpr (FINEST) {
        const size_t fsx = io.fsx, fsy = io.fsy;
        const T2 t0 = __ldg(reinterpret_cast<const T2*>(fp));
        const T2 t1 = __ldg(reinterpret_cast<const T2*>(fp + fsx));
        const T2 t2 = __ldg(reinterpret_cast<const T2*>(fp + fsy));
        const T2 t3 = __ldg(reinterpret_cast<const T2*>(fp + fsy + fsx));
        o[1] = t0.y, o[2] = t1.x, o[3] = t1.y, o[4] = t2.x, o[5] = t2.y, o[6] = t3.x, o[7] = t3.y;
    } else {
        const size_t s = (size_t)io.s, sx = s * io.fsx, sy = s * io.fsy;
#pragma unroll
        for (int si = 1; si < 8; ++si) {
            const int px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
            o[si] = __ldg(fp + (pz ? sy : 0) + (py ? sx : 0) + (px ? s : 0));
        }
    }
    const size_t n = geo.n;
    uint16_t* __restrict__ cp = io.codes + zw.cm;
    T v[8];
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const T d = A::sub(o[b + 1], p[b]);
        int code = qp.radius;
        if (quantize_is_centre(d, qp)) {
            ++center[b];
        } else {
            if constexpr (sizeof(T) == 4) code = qtab ? quantize_table(d, qp, qtab, qr2) : quantize_full(d, qp);
            else code = quantize_full(d, qp);
            if (code == qp.radius) {
                ++center[b];
            } else {
                hist_add(sh, wlo, wn, hist, b, code, 1u);
                if (code == 0) {
                    io.unpred_dense[(size_t)b * n + zw.cm] = d;
                    atomicAdd(&io.unpred_cnt[(size_t)b * (geo.nchunks() + 1) + zw.chunk], 1u);
                }
            }
        }
        cp[(size_t)b * n] = (uint16_t)code;
        if constexpr (!FINEST) v[b + 1] = A::add(code ? recover_lut(lut, code, qp) : d, p[b]);
    }
    if constexpr (!FINEST) {
        v[0] = r(0);
        const size_t gsx = 2 * (size_t)geo.dx, gsy = 4 * (size_t)geo.dx * geo.dy;
        T2 t;
        t.x = v[0], t.y = v[1];
        *reinterpret_cast<T2*>(gp) = t;
        t.x = v[2], t.y = v[3];
        *reinterpret_cast<T2*>(gp + gsx) = t;
        t.x = v[4], t.y = v[5];
        *reinterpret_cast<T2*>(gp + gsy) = t;
        t.x = v[6], t.y = v[7];
        *reinterpret_cast<T2*>(gp + gsy + gsx) = t;
    }
}

template <typename T, int PRED, bool FINEST, int LM, int ZB = kZSmall>
__global__ void __launch_bounds__(BX* BY, LM == kLearnNone && sizeof(T) == 4 ? (FINEST ? 5 : 4) : 1) k_level_encode(EncodeIO<T> io, const T* __restrict__ R, LevelGeom geo,
                                                         QuantParams qp, HistArgs hist, LearnedArgs<T> la,
                                                         const __grid_constant__ CUtensorMap tmap, int use_tma,
                                                         const __grid_constant__ QuantTable qt)
{
    static_assert(LM == kLearnNone || ZB == kZSmall, "learned kernels use the default tile depth");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* tile = reinterpret_cast<T*>(smem_raw);
    __shared__ uint32_t sh[7][kSmemBins];
    __shared__ T lut[FINEST ? 1 : 2 * kRecW];  // the finest level writes no decoded grid
    const int tid = threadIdx.y * BX + threadIdx.x;
    for (int i = tid; i < 7 * kSmemBins; i += BX * BY) (&sh[0][0])[i] = 0;
    if constexpr (!FINEST) build_recover_lut(lut, qp, tid, BX * BY);
    if constexpr (LM != kLearnNone) {  // the model follows the tile in dynamic shared memory
        LearnedModel* smodel = reinterpret_cast<LearnedModel*>(smem_raw + kTileBytesAligned<T>);
        learned_load(smodel, la.model, tid, BX * BY);
        la.model = smodel;
    }
    const int wlo = max(0, qp.radius - kSmemBins / 2);
    const int wn = min(kSmemBins, 2 * qp.radius - wlo);
    const int dx = geo.dx, dy = geo.dy, dz = geo.dz;
    const int x0 = 1 + blockIdx.x * BX, y0 = 1 + blockIdx.y * BY, z0 = 1 + blockIdx.z * ZB;
    __shared__ __align__(8) uint64_t tile_bar;
    stage_tile<T, ZB>(tile, R, use_tma ? &tmap : nullptr, dx, dy, dz, x0, y0, z0, &tile_bar);
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool valid = x <= dx - 3 && y <= dy - 3;
    ChunkIndex ci;
    ci.init(geo, x, y);
    uint32_t center[7] = {0, 0, 0, 0, 0, 0, 0};
    const int z1 = min(z0 + ZB, dz - 2);
    [[maybe_unused]] uint32_t phase = 0;
    [[maybe_unused]] bool tc_failed = false;
    if constexpr (LM == kLearnTc) tc::net_setup(*net_smem(), *la.model, tid);
    if constexpr (LM == kLearnNone) {
        // the f32 quantizer table in shared memory (read after the tile's
        // barrier below it in the kernel's order: staged before the walk)
        __shared__ float4 qtab[kQuantTableH];
        const bool use_qt = sizeof(T) == 4 && qt.on;
        if (use_qt && tid < kQuantTableH) qtab[tid] = qt.e[tid];
        __syncthreads();
        ZWalk zw;
        zw.init(geo, x, y, z0);
        const size_t s = (size_t)io.s;
        const T* fp = io.field + s * (2 * (size_t)z0) * io.fsy + s * (2 * (size_t)y) * io.fsx + s * 2 * (size_t)x;
        const size_t fstep = 2 * s * io.fsy;
        const size_t gsy = 4 * (size_t)geo.dx * geo.dy;
        T* gp = FINEST ? nullptr : io.G + (2 * (size_t)z0) * gsy + (2 * (size_t)y) * 2 * geo.dx + 2 * (size_t)x;
        for (int z = z0; z < z1; ++z) {
            const TileAt<T, TSX, TPLANE> r{tile + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
            if (valid)
                encode_interior<T, PRED, FINEST>(r, io, geo, qp, lut, zw, fp, gp, sh, wlo, wn, hist, center,
                                                 use_qt ? qtab : nullptr, qt.r2);
            zw.next();
            fp += fstep;
            if constexpr (!FINEST) gp += 2 * gsy;
        }
        // the finest level's x-boundary columns beside this CTA's interior
        // points, from the same tile (first and last CTAs along x; the shell
        // kernel skips them there; on the coarser levels the extra registers
        // and the serial tail cost more than the shell's uncoalesced reads)
        if (FINEST && (blockIdx.x == 0 || blockIdx.x == gridDim.x - 1)) {
            const int bz = blockIdx.z;
            for_owned_boundary<true>(geo, ZB, bz, (int)gridDim.z, tid, BX * BY, [&](int px, int py, int pz) {
                const TileAt<T, TSX, TPLANE> rb{tile + (pz - z0 + 1) * TPLANE + (py - y0 + 1) * TSX + (px - x0 + 1)};
                ChunkIndex bci;
                bci.init(geo, px, py);
                int q[7];
                encode_point<T, PRED, FINEST, false>(rb, io, geo, qp, lut, bci, px, py, pz, q);
#pragma unroll
                for (int b = 0; b < 7; ++b) {
                    if (q[b] == qp.radius) ++center[b];
                    else hist_add(sh, wlo, wn, hist, b, q[b], 1u);
                }
            });
        }
    }
    for (int z = z0; z < z1 && LM != kLearnNone; ++z) {
        int q[7] = {-1, -1, -1, -1, -1, -1, -1};
        const TileAt<T, TSX, TPLANE> r{tile + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
        int acc3[7];
        if constexpr (LM == kLearnTc) {
            const uint4 xin = valid ? learned_inputs<T>(r, la.rs) : make_uint4(0u, 0u, 0u, 0u);
            if (!tc::net_run(*net_smem(), *la.model, xin, phase, tid, acc3)) {
                tc_failed = true;
                break;
            }
        }
        if (valid) encode_point<T, PRED, FINEST, true, LM>(r, io, geo, qp, lut, ci, x, y, z, q, la, acc3);
#pragma unroll
        for (int b = 0; b < 7; ++b) hist_code(sh, wlo, wn, hist, b, q[b], center[b]);
    }
    if constexpr (LM == kLearnTc) {
        tc::net_teardown(*net_smem(), tid);
        if (tc_failed && tid == 0) atomicOr(&g_learned_tc_error, 1u);
    }
    hist_flush_center(sh, wlo, wn, hist, center);
    __syncthreads();
    for (int i = tid; i < 7 * kSmemBins; i += BX * BY) {
        const int b = i / kSmemBins, w = i % kSmemBins;
        const uint32_t c = sh[b][w];
        if (c) atomicAdd(&hist.full[(size_t)b * 2 * hist.radius + wlo + w], c);
    }
}

template <typename T, int PRED, bool FINEST>
__global__ void __launch_bounds__(256) k_level_encode_shell(EncodeIO<T> io, const T* __restrict__ R, LevelGeom geo,
                                                            QuantParams qp, HistArgs hist, Shell sh)
{
    __shared__ T lut[2 * kRecW];
    if constexpr (!FINEST) build_recover_lut(lut, qp, threadIdx.x, blockDim.x);
    __syncthreads();
    uint32_t center[7] = {0, 0, 0, 0, 0, 0, 0};
    const uint64_t total = sh.g1 + sh.g2 + sh.g3;
    const long long sx = geo.dx, sy = (long long)geo.dx * geo.dy;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < total; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        int q[7] = {-1, -1, -1, -1, -1, -1, -1};
        if (i < total) {
            int x, y, z;
            sh.point(i, x, y, z);
            ChunkIndex ci;
            ci.init(geo, x, y);
            const GlobalAt<T> r{R + (size_t)z * sy + (size_t)y * sx + x, sx, sy};
            encode_point<T, PRED, FINEST, false>(r, io, geo, qp, lut, ci, x, y, z, q);
        }
#pragma unroll
        for (int b = 0; b < 7; ++b) hist_code(nullptr, 0, 0, hist, b, q[b], center[b]);
    }
    hist_flush_center(nullptr, 0, 0, hist, center);
}

// One coarse point of the decoder after its 7 predictions p: codes -> dq,
// x' = dq + p, the merged fine cell (r0 = the coarse value at the point).
template <typename T>
__device__ __forceinline__ void decode_values(const LevelGeom& geo, const QuantParams& qp, const T* lut,
                                              const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                                              T* __restrict__ G, const ChunkIndex& ci, int x, int y, int z,
                                              const T (&p)[7], T r0)
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    int chunk;
    const size_t cm = ci.at(z, chunk);
    const size_t n = geo.n;
    int q[7];
#pragma unroll
    for (int b = 0; b < 7; ++b) q[b] = __ldg(codes + (size_t)b * n + cm);
    T v[8];
    v[0] = r0;
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const T dq = q[b] ? recover_lut(lut, q[b], qp) : __ldg(unpred_dense + (size_t)b * n + cm);
        v[b + 1] = A::add(dq, p[b]);
    }
    const size_t gsx = 2 * (size_t)geo.dx, gsy = 4 * (size_t)geo.dx * geo.dy;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int pz = k >> 1, py = k & 1;
        T2 t;
        t.x = v[2 * k];
        t.y = v[2 * k + 1];
        *reinterpret_cast<T2*>(G + (size_t)(2 * z + pz) * gsy + (size_t)(2 * y + py) * gsx + 2 * (size_t)x) = t;
    }
}

// One coarse point of the decoder: codes -> dq, + 7 predictions, merged cell.
template <typename T, int PRED, bool INTERIOR, int LM = kLearnNone, class Acc>
__device__ __forceinline__ void decode_point(const Acc& r, const LevelGeom& geo, const QuantParams& qp, const T* lut,
                                             const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                                             T* __restrict__ G, const ChunkIndex& ci, int x, int y, int z,
                                             const LearnedArgs<T>& la = LearnedArgs<T>(), const int* acc3 = nullptr)
{
    T p[7];
    predict7<PRED>(r, INTERIOR, x, y, z, geo.dx, geo.dy, geo.dz, p);
    apply_learned<LM>(r, la, acc3, p);
    decode_values<T>(geo, qp, lut, codes, unpred_dense, G, ci, x, y, z, p, r(0));
}

// Interior point of the plain decoder (no learned correction), the same
// values as decode_point, with the walk's chunk-major position and the output
// pointer gp (the cell's first fine value) moving along z with the thread.
template <typename T, int PRED, class Acc>
__device__ __forceinline__ void decode_interior(const Acc& r, const LevelGeom& geo, const QuantParams& qp,
                                                const T* lut, const uint16_t* __restrict__ codes,
                                                const T* __restrict__ unpred_dense, const ZWalk& zw,
                                                T* __restrict__ gp)
{
    using A = Ar<T>;
    using T2 = typename V2<T>::type;
    const size_t n = geo.n;
    T p[7];
    predict7_interior_only<PRED>(r, p);
    const uint16_t* __restrict__ cp = codes + zw.cm;
    int q[7];
#pragma unroll
    for (int b = 0; b < 7; ++b) q[b] = __ldg(cp + (size_t)b * n);
    T v[8];
    v[0] = r(0);
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const T dq = q[b] ? recover_lut(lut, q[b], qp) : __ldg(unpred_dense + (size_t)b * n + zw.cm);
        v[b + 1] = A::add(dq, p[b]);
    }
    const size_t gsx = 2 * (size_t)geo.dx, gsy = 4 * (size_t)geo.dx * geo.dy;
    T2 t;
    t.x = v[0], t.y = v[1];
    *reinterpret_cast<T2*>(gp) = t;
    t.x = v[2], t.y = v[3];
    *reinterpret_cast<T2*>(gp + gsx) = t;
    t.x = v[4], t.y = v[5];
    *reinterpret_cast<T2*>(gp + gsy) = t;
    t.x = v[6], t.y = v[7];
    *reinterpret_cast<T2*>(gp + gsy + gsx) = t;
}

template <typename T, int PRED, int LM, int ZB = kZSmall>
__global__ void __launch_bounds__(BX* BY, 4) k_level_decode(const T* __restrict__ R, LevelGeom geo, QuantParams qp,
                                                         const uint16_t* __restrict__ codes,
                                                         const T* __restrict__ unpred_dense, T* __restrict__ G,
                                                         LearnedArgs<T> la, const __grid_constant__ CUtensorMap tmap,
                                                         int use_tma, int zoff, int nzb)
{
    static_assert(LM == kLearnNone || ZB == kZSmall, "learned kernels use the default tile depth");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* tile = reinterpret_cast<T*>(smem_raw);
    __shared__ T lut[2 * kRecW];
    const int tid = threadIdx.y * BX + threadIdx.x;
    build_recover_lut(lut, qp, tid, BX * BY);
    if constexpr (LM != kLearnNone) {  // the model follows the tile in dynamic shared memory
        LearnedModel* smodel = reinterpret_cast<LearnedModel*>(smem_raw + kTileBytesAligned<T>);
        learned_load(smodel, la.model, tid, BX * BY);
        la.model = smodel;
    }
    const int dx = geo.dx, dy = geo.dy, dz = geo.dz;
    const int bz = blockIdx.z + zoff;  // this launch covers z-bricks [zoff, zoff + gridDim.z) of nzb
    const int x0 = 1 + blockIdx.x * BX, y0 = 1 + blockIdx.y * BY, z0 = 1 + bz * ZB;
    __shared__ __align__(8) uint64_t tile_bar;
    stage_tile<T, ZB>(tile, R, use_tma ? &tmap : nullptr, dx, dy, dz, x0, y0, z0, &tile_bar);
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool valid = x <= dx - 3 && y <= dy - 3;
    const int z1 = min(z0 + ZB, dz - 2);
    if constexpr (LM == kLearnNone) {
        if (valid) {
            ZWalk zw;
            zw.init(geo, x, y, z0);
            const size_t gsy = 4 * (size_t)dx * dy;
            T* gp = G + (2 * (size_t)z0) * gsy + (2 * (size_t)y) * 2 * dx + 2 * (size_t)x;
            for (int z = z0; z < z1; ++z) {
                const TileAt<T, TSX, TPLANE> r{tile + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
                decode_interior<T, PRED>(r, geo, qp, lut, codes, unpred_dense, zw, gp);
                zw.next();
                gp += 2 * gsy;
            }
        }
        // the CTA's owned boundary points, predicted from the same tile
        for_owned_boundary(geo, ZB, bz, nzb, tid, BX * BY, [&](int px, int py, int pz) {
            const TileAt<T, TSX, TPLANE> r{tile + (pz - z0 + 1) * TPLANE + (py - y0 + 1) * TSX + (px - x0 + 1)};
            ChunkIndex bci;
            bci.init(geo, px, py);
            decode_point<T, PRED, false>(r, geo, qp, lut, codes, unpred_dense, G, bci, px, py, pz);
        });
        return;
    }
    if constexpr (LM != kLearnTc) {
        if (!valid) return;
    }
    ChunkIndex ci;
    ci.init(geo, x, y);
    [[maybe_unused]] uint32_t phase = 0;
    [[maybe_unused]] bool tc_failed = false;
    if constexpr (LM == kLearnTc) tc::net_setup(*net_smem(), *la.model, tid);
    for (int z = z0; z < z1; ++z) {
        const TileAt<T, TSX, TPLANE> r{tile + (z - z0 + 1) * TPLANE + (threadIdx.y + 1) * TSX + threadIdx.x + 1};
        int acc3[7];
        if constexpr (LM == kLearnTc) {
            const uint4 xin = valid ? learned_inputs<T>(r, la.rs) : make_uint4(0u, 0u, 0u, 0u);
            if (!tc::net_run(*net_smem(), *la.model, xin, phase, tid, acc3)) {
                tc_failed = true;
                break;
            }
        }
        if (valid) decode_point<T, PRED, true, LM>(r, geo, qp, lut, codes, unpred_dense, G, ci, x, y, z, la, acc3);
    }
    if constexpr (LM == kLearnTc) {
        tc::net_teardown(*net_smem(), tid);
        if (tc_failed && tid == 0) atomicOr(&g_learned_tc_error, 1u);
    }
}

template <typename T, int PRED>
__global__ void __launch_bounds__(256) k_level_decode_shell(const T* __restrict__ R, LevelGeom geo, QuantParams qp,
                                                            const uint16_t* __restrict__ codes,
                                                            const T* __restrict__ unpred_dense, T* __restrict__ G,
                                                            Shell sh)
{
    __shared__ T lut[2 * kRecW];
    build_recover_lut(lut, qp, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint64_t total = sh.g1 + sh.g2 + sh.g3;
    const long long sx = geo.dx, sy = (long long)geo.dx * geo.dy;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        sh.point(i, x, y, z);
        ChunkIndex ci;
        ci.init(geo, x, y);
        const GlobalAt<T> r{R + (size_t)z * sy + (size_t)y * sx + x, sx, sy};
        decode_point<T, PRED, false>(r, geo, qp, lut, codes, unpred_dense, G, ci, x, y, z);
    }
}
