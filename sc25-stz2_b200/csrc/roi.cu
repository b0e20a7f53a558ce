// Random-access box / slice reconstruction (the query path of FD5:2460-2640).
//
// After the planner has chosen the marker chunks a box needs and those chunks
// are entropy-decoded, two kernels finish the query:
//   k_roi_mid : rebuild the half-resolution ("mid") grid on the high level's
//               reference regions: sub-block 0 from the decoded base, the other
//               parities as recover(q) + P(base) on the low level (the
//               reference's low ROI depreprocess FD5:2507-2516 and the
//               reference gather FD5:2520-2538, fused);
//   k_roi_box : each box point is either a mid-grid value (even parity) or
//               recover(q) + P(mid) of its high sub-block (FD5:2573-2605,
//               fused with the desplit).
// Every value is computed with the same expression as the full decode, so a
// box equals the full decode on the same coordinates bit for bit.
#include <cuda_runtime.h>

#include "roi.h"
#include "stz_device.cuh"

namespace stz {
namespace {

__device__ __forceinline__ size_t cm_index(const LevelGeom& g, int x, int y, int z)
{
    const int C = g.C;
    const int cx = x / C, cy = y / C, cz = z / C;
    const int chunk = (cz * g.ncy + cy) * g.ncx + cx;
    return (size_t)chunk * C * C * C + (size_t)((z - cz * C) * C + (y - cy * C)) * C + (x - cx * C);
}

template <int PRED, typename T>
__device__ __forceinline__ T predict_rt(int b, const Grid<T>& g, int x, int y, int z)
{
    switch (b) {
    case 0: return predict<PRED>(0, g, x, y, z);
    case 1: return predict<PRED>(1, g, x, y, z);
    case 2: return predict<PRED>(2, g, x, y, z);
    case 3: return predict<PRED>(3, g, x, y, z);
    case 4: return predict<PRED>(4, g, x, y, z);
    case 5: return predict<PRED>(5, g, x, y, z);
    default: return predict<PRED>(6, g, x, y, z);
    }
}

// Value at point (X, Y, Z) of the grid one level finer than `coarse`: the
// coarse value itself at even parity, else recover(q) + P(coarse) of the
// point's sub-block (the level's codes are chunk-major per sub-block).
template <typename T, int PRED>
__device__ __forceinline__ T finer_value(const Grid<T>& coarse, const LevelGeom& g, const QuantParams& qp,
                                         const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                                         int X, int Y, int Z)
{
    const int si = ((Z & 1) << 2) | ((Y & 1) << 1) | (X & 1);
    const int x = X >> 1, y = Y >> 1, z = Z >> 1;
    if (si == 0) return coarse.at((size_t)z * coarse.sy + (size_t)y * coarse.sx + x);
    const size_t k = (size_t)(si - 1) * g.n + cm_index(g, x, y, z);
    const int q = codes[k];
    const T dq = q ? recover<T>(q, qp) : unpred_dense[k];
    return Ar<T>::add(dq, predict_rt<PRED>(si - 1, coarse, x, y, z));
}

// Index of the last box whose start <= t (starts ascending, boxes[0].start == 0).
template <typename B>
__device__ __forceinline__ int find_box(const B* __restrict__ boxes, int n, uint64_t t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int m = (lo + hi + 1) >> 1;
        if (boxes[m].start <= t) lo = m;
        else hi = m - 1;
    }
    return lo;
}

__device__ __forceinline__ void box_point(const RoiBox& bx, uint64_t i, int& X, int& Y, int& Z)
{
    const int ex = bx.x1 - bx.x0 + 1, ey = bx.y1 - bx.y0 + 1;
    X = bx.x0 + (int)(i % ex);
    Y = bx.y0 + (int)((i / ex) % ey);
    Z = bx.z0 + (int)(i / ((uint64_t)ex * ey));
}

// Boxes are given as inclusive ranges; `start` is the prefix sum of box
// volumes so one launch covers all boxes.
template <typename T, int PRED>
__global__ void k_roi_mid(const RoiBox* __restrict__ boxes, int nbox, uint64_t total, Grid<T> base, LevelGeom low,
                          QuantParams qp, const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                          T* __restrict__ mid, size_t msx, size_t msy)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const RoiBox bx = boxes[find_box(boxes, nbox, t)];
        int X, Y, Z;
        box_point(bx, t - bx.start, X, Y, Z);
        mid[(size_t)Z * msy + (size_t)Y * msx + X] = finer_value<T, PRED>(base, low, qp, codes, unpred_dense, X, Y, Z);
    }
}

template <typename T, int PRED>
__global__ void k_roi_box(RoiBox box, Grid<T> mid, LevelGeom high, QuantParams qp, const uint16_t* __restrict__ codes,
                          const T* __restrict__ unpred_dense, T* __restrict__ out)
{
    const int ex = box.x1 - box.x0 + 1, ey = box.y1 - box.y0 + 1;
    const uint64_t total = (uint64_t)ex * ey * (box.z1 - box.z0 + 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        int X, Y, Z;
        box_point(box, i, X, Y, Z);
        out[i] = finer_value<T, PRED>(mid, high, qp, codes, unpred_dense, X, Y, Z);
    }
}

// Batched, device-sized variants (request server): the mid-grid regions and
// the outputs of every request of a batch, counts read from the batch header.
template <typename T, int PRED>
__global__ void k_roi_mid_dyn(const uint8_t* __restrict__ meta, Grid<T> base, LevelGeom low, QuantParams qp,
                              const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                              T* __restrict__ mid, size_t msx, size_t msy)
{
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(meta);
    const uint64_t total = h->mid_total;
    const int nbox = (int)h->n_mid;
    const RoiBox* boxes = reinterpret_cast<const RoiBox*>(meta + h->o_mid);
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const RoiBox bx = boxes[find_box(boxes, nbox, t)];
        int X, Y, Z;
        box_point(bx, t - bx.start, X, Y, Z);
        mid[(size_t)Z * msy + (size_t)Y * msx + X] = finer_value<T, PRED>(base, low, qp, codes, unpred_dense, X, Y, Z);
    }
}

template <typename T, int PRED>
__global__ void k_roi_req_dyn(const uint8_t* __restrict__ meta, Grid<T> mid, Grid<T> base, LevelGeom high,
                              QuantParams qp, const uint16_t* __restrict__ codes,
                              const T* __restrict__ unpred_dense)
{
    const BatchHdr* h = reinterpret_cast<const BatchHdr*>(meta);
    const uint64_t total = h->req_total;
    const int nreq = (int)h->n_req;
    const ReqDesc* reqs = reinterpret_cast<const ReqDesc*>(meta + h->o_req);
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const int ri = find_box(reqs, nreq, t);
        const ReqDesc r = reqs[ri];
        const uint64_t i = t - r.start;
        int X, Y, Z;
        box_point(r.box, i, X, Y, Z);
        T v;
        if (r.kind == kReqBox) {
            v = finer_value<T, PRED>(mid, high, qp, codes, unpred_dense, X, Y, Z);
        } else {
            const int s = r.shift;
            v = base.at(((size_t)Z << s) * base.sy + ((size_t)Y << s) * base.sx + ((size_t)X << s));
        }
        reinterpret_cast<T*>(r.out)[i] = v;
    }
}

int grid_blocks(uint64_t n)
{
    uint64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return (int)(g ? g : 1);
}

}  // namespace

template <typename T>
void launch_roi_mid(const RoiBox* boxes_dev, int nbox, uint64_t total, const T* base, const LevelGeom& low,
                    QuantParams qp, int predictor, const uint16_t* codes, const T* unpred_dense, T* mid,
                    cudaStream_t st)
{
    if (!total) return;
    Grid<T> g;
    g.p = base;
    g.dx = low.dx, g.dy = low.dy, g.dz = low.dz;
    g.sx = (size_t)low.dx, g.sy = (size_t)low.dx * low.dy;
    const size_t msx = 2 * (size_t)low.dx, msy = 4 * (size_t)low.dx * low.dy;
    if (predictor == 1)
        k_roi_mid<T, 1><<<grid_blocks(total), 256, 0, st>>>(boxes_dev, nbox, total, g, low, qp, codes, unpred_dense,
                                                            mid, msx, msy);
    else
        k_roi_mid<T, 0><<<grid_blocks(total), 256, 0, st>>>(boxes_dev, nbox, total, g, low, qp, codes, unpred_dense,
                                                            mid, msx, msy);
}

template <typename T>
void launch_roi_box(const RoiBox& box, const T* mid, const LevelGeom& high, QuantParams qp, int predictor,
                    const uint16_t* codes, const T* unpred_dense, T* out, cudaStream_t st)
{
    const uint64_t total = (uint64_t)(box.x1 - box.x0 + 1) * (box.y1 - box.y0 + 1) * (box.z1 - box.z0 + 1);
    Grid<T> g;
    g.p = mid;
    g.dx = high.dx, g.dy = high.dy, g.dz = high.dz;
    g.sx = (size_t)high.dx, g.sy = (size_t)high.dx * high.dy;
    if (predictor == 1)
        k_roi_box<T, 1><<<grid_blocks(total), 256, 0, st>>>(box, g, high, qp, codes, unpred_dense, out);
    else
        k_roi_box<T, 0><<<grid_blocks(total), 256, 0, st>>>(box, g, high, qp, codes, unpred_dense, out);
}

template <typename T>
void launch_roi_mid_dyn(int grid, int block, const uint8_t* meta, const T* base, const LevelGeom& low, QuantParams qp,
                        int predictor, const uint16_t* codes, const T* unpred_dense, T* mid, cudaStream_t st)
{
    Grid<T> g;
    g.p = base;
    g.dx = low.dx, g.dy = low.dy, g.dz = low.dz;
    g.sx = (size_t)low.dx, g.sy = (size_t)low.dx * low.dy;
    const size_t msx = 2 * (size_t)low.dx, msy = 4 * (size_t)low.dx * low.dy;
    if (predictor == 1)
        k_roi_mid_dyn<T, 1><<<grid, block, 0, st>>>(meta, g, low, qp, codes, unpred_dense, mid, msx, msy);
    else
        k_roi_mid_dyn<T, 0><<<grid, block, 0, st>>>(meta, g, low, qp, codes, unpred_dense, mid, msx, msy);
}

template <typename T>
void launch_roi_req_dyn(int grid, int block, const uint8_t* meta, const T* mid, const T* base, const LevelGeom& low,
                        const LevelGeom& high, QuantParams qp, int predictor, const uint16_t* codes,
                        const T* unpred_dense, cudaStream_t st)
{
    Grid<T> gm;
    gm.p = mid;
    gm.dx = high.dx, gm.dy = high.dy, gm.dz = high.dz;
    gm.sx = (size_t)high.dx, gm.sy = (size_t)high.dx * high.dy;
    Grid<T> gb;
    gb.p = base;
    gb.dx = low.dx, gb.dy = low.dy, gb.dz = low.dz;
    gb.sx = (size_t)low.dx, gb.sy = (size_t)low.dx * low.dy;
    if (predictor == 1)
        k_roi_req_dyn<T, 1><<<grid, block, 0, st>>>(meta, gm, gb, high, qp, codes, unpred_dense);
    else
        k_roi_req_dyn<T, 0><<<grid, block, 0, st>>>(meta, gm, gb, high, qp, codes, unpred_dense);
}

template void launch_roi_mid_dyn<float>(int, int, const uint8_t*, const float*, const LevelGeom&, QuantParams, int,
                                        const uint16_t*, const float*, float*, cudaStream_t);
template void launch_roi_mid_dyn<double>(int, int, const uint8_t*, const double*, const LevelGeom&, QuantParams, int,
                                         const uint16_t*, const double*, double*, cudaStream_t);
template void launch_roi_req_dyn<float>(int, int, const uint8_t*, const float*, const float*, const LevelGeom&,
                                        const LevelGeom&, QuantParams, int, const uint16_t*, const float*,
                                        cudaStream_t);
template void launch_roi_req_dyn<double>(int, int, const uint8_t*, const double*, const double*, const LevelGeom&,
                                         const LevelGeom&, QuantParams, int, const uint16_t*, const double*,
                                         cudaStream_t);

template void launch_roi_mid<float>(const RoiBox*, int, uint64_t, const float*, const LevelGeom&, QuantParams, int,
                                    const uint16_t*, const float*, float*, cudaStream_t);
template void launch_roi_mid<double>(const RoiBox*, int, uint64_t, const double*, const LevelGeom&, QuantParams, int,
                                     const uint16_t*, const double*, double*, cudaStream_t);
template void launch_roi_box<float>(const RoiBox&, const float*, const LevelGeom&, QuantParams, int, const uint16_t*,
                                    const float*, float*, cudaStream_t);
template void launch_roi_box<double>(const RoiBox&, const double*, const LevelGeom&, QuantParams, int,
                                     const uint16_t*, const double*, double*, cudaStream_t);

}  // namespace stz
