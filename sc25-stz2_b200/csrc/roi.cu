// Random-access box / slice reconstruction (the query path of FD5:2460-2640).
//
// After the planner has chosen the marker chunks a box needs and those chunks
// are entropy-decoded, two launches of one kernel finish the query:
//   low level : rebuild the half-resolution ("mid") grid on the bounding box
//               of the high level's reference regions from the decoded base
//               (the reference's low ROI depreprocess FD5:2507-2516 and its
//               reference gather FD5:2520-2538, fused);
//   high level: rebuild the query box from the mid grid (FD5:2573-2605, fused
//               with the desplit).
// A thread rebuilds one coarse cell: the coarse value (parity 0) and the 7
// sub-block values recover(q) + P(coarse) of the 2x2x2 fine points the cell
// predicts, with the same predictor and the same interior/boundary split as
// the full level decode, so a box equals the full decode on the same
// coordinates bit for bit. Cells on the window's edge also evaluate the
// parities outside the window; those values are not written.
#include <cuda_runtime.h>

#include "roi.h"
#include "stz_device.cuh"

namespace stz {

RoiJob cells_job(const int w0[3], const int w1[3], void* out, const int origin[3], uint64_t osx, uint64_t osy,
                 uint64_t start)
{
    RoiJob j{};
    j.cx0 = w0[0] >> 1, j.cy0 = w0[1] >> 1, j.cz0 = w0[2] >> 1;
    j.ncx = (w1[0] >> 1) - j.cx0 + 1, j.ncy = (w1[1] >> 1) - j.cy0 + 1, j.ncz = (w1[2] >> 1) - j.cz0 + 1;
    j.wx0 = w0[0], j.wx1 = w1[0], j.wy0 = w0[1], j.wy1 = w1[1], j.wz0 = w0[2], j.wz1 = w1[2];
    j.ox = origin[0], j.oy = origin[1], j.oz = origin[2];
    j.kind = kJobCells;
    j.osx = osx, j.osy = osy;
    j.start = start;
    j.out = (uint64_t)(uintptr_t)out;
    return j;
}

namespace {

__device__ __forceinline__ size_t cm_index(const LevelGeom& g, int x, int y, int z)
{
    const int C = g.C;
    const int cx = x / C, cy = y / C, cz = z / C;
    const int chunk = (cz * g.ncy + cy) * g.ncx + cx;
    return (size_t)chunk * C * C * C + (size_t)((z - cz * C) * C + (y - cy * C)) * C + (x - cx * C);
}

// Index of the last entry whose start <= t (starts ascending, [0].start == 0).
__device__ __forceinline__ int find_job(const RoiJob* __restrict__ jobs, int n, uint64_t t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int m = (lo + hi + 1) >> 1;
        if (jobs[m].start <= t) lo = m;
        else hi = m - 1;
    }
    return lo;
}

template <typename T, int PRED, bool LEARNED>
__global__ void __launch_bounds__(256) k_roi_cells(const uint8_t* __restrict__ meta, int list, Grid<T> coarse,
                                                   LevelGeom g, Grid<T> base, QuantParams qp,
                                                   const uint16_t* __restrict__ codes,
                                                   const T* __restrict__ unpred_dense, LearnedArgs<T> la)
{
    using A = Ar<T>;
    __shared__ __align__(16) LearnedModel smodel;
    if constexpr (LEARNED) {
        learned_load(&smodel, la.model, threadIdx.x, blockDim.x);
        __syncthreads();
    }
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(meta);
    const int nj = (int)(list ? h->n_req : h->n_mid);
    const uint64_t total = list ? h->req_total : h->mid_total;
    const RoiJob* jobs = reinterpret_cast<const RoiJob*>(meta + (list ? h->o_req : h->o_mid));
    const size_t n = g.n;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const RoiJob J = jobs[find_job(jobs, nj, t)];
        const uint64_t u = t - J.start;
        const int cx = J.cx0 + (int)(u % J.ncx);
        const int cy = J.cy0 + (int)((u / J.ncx) % J.ncy);
        const int cz = J.cz0 + (int)(u / ((uint64_t)J.ncx * J.ncy));
        T* out = reinterpret_cast<T*>(J.out);
        if (J.kind == kJobSample) {
            const int s = J.shift;
            out[(size_t)(cz - J.oz) * J.osy + (size_t)(cy - J.oy) * J.osx + (cx - J.ox)] =
                base.at(((size_t)cz << s) * base.sy + ((size_t)cy << s) * base.sx + ((size_t)cx << s));
            continue;
        }
        const size_t cm = cm_index(g, cx, cy, cz);
        int q[7];
#pragma unroll
        for (int b = 0; b < 7; ++b) q[b] = __ldg(codes + (size_t)b * n + cm);
        const GlobalAt<T> r{coarse.p + (size_t)cz * coarse.sy + (size_t)cy * coarse.sx + cx, (long long)coarse.sx,
                            (long long)coarse.sy};
        const bool interior = cx >= 1 && cx <= g.dx - 3 && cy >= 1 && cy <= g.dy - 3 && cz >= 1 && cz <= g.dz - 3;
        T p[7];
        predict7<PRED>(r, interior, cx, cy, cz, g.dx, g.dy, g.dz, p);
        if constexpr (LEARNED) {
            if (interior) {
                T corr[7];
                learned_corr<T>(smodel, r, la.rs, la.so, corr);
#pragma unroll
                for (int b = 0; b < 7; ++b)
                    if ((la.flags >> b) & 1u) p[b] = A::add(p[b], corr[b]);
            }
        }
        T v[8];
        v[0] = r(0);
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            const T dq = q[b] ? recover<T>(q[b], qp) : __ldg(unpred_dense + (size_t)b * n + cm);
            v[b + 1] = A::add(dq, p[b]);
        }
#pragma unroll
        for (int si = 0; si < 8; ++si) {
            const int X = 2 * cx + (si & 1), Y = 2 * cy + ((si >> 1) & 1), Z = 2 * cz + (si >> 2);
            if (X >= J.wx0 && X <= J.wx1 && Y >= J.wy0 && Y <= J.wy1 && Z >= J.wz0 && Z <= J.wz1)
                out[(size_t)(Z - J.oz) * J.osy + (size_t)(Y - J.oy) * J.osx + (X - J.ox)] = v[si];
        }
    }
}

template <typename T>
Grid<T> grid_of(const T* p, const LevelGeom& g)
{
    Grid<T> G;
    G.p = p;
    G.dx = g.dx, G.dy = g.dy, G.dz = g.dz;
    G.sx = (size_t)g.dx, G.sy = (size_t)g.dx * g.dy;
    return G;
}

}  // namespace

template <typename T>
void launch_roi_cells(int grid, int block, const uint8_t* meta, int list, const T* coarse, const LevelGeom& geo,
                      const T* base, const LevelGeom& base_geo, QuantParams qp, int predictor, const uint16_t* codes,
                      const T* unpred_dense, cudaStream_t st, const LearnedArgs<T>& la)
{
    const Grid<T> gc = grid_of(coarse, geo), gb = grid_of(base, base_geo);
    const bool learned = la.model && la.flags;
    auto kern = predictor == 1 ? (learned ? k_roi_cells<T, 1, true> : k_roi_cells<T, 1, false>)
                               : (learned ? k_roi_cells<T, 0, true> : k_roi_cells<T, 0, false>);
    kern<<<grid, block, 0, st>>>(meta, list, gc, geo, gb, qp, codes, unpred_dense, la);
}

template void launch_roi_cells<float>(int, int, const uint8_t*, int, const float*, const LevelGeom&, const float*,
                                      const LevelGeom&, QuantParams, int, const uint16_t*, const float*,
                                      cudaStream_t, const LearnedArgs<float>&);
template void launch_roi_cells<double>(int, int, const uint8_t*, int, const double*, const LevelGeom&,
                                       const double*, const LevelGeom&, QuantParams, int, const uint16_t*,
                                       const double*, cudaStream_t, const LearnedArgs<double>&);

}  // namespace stz
