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

// Boxes are given as inclusive ranges; `start` is the prefix sum of box
// volumes so one launch covers all boxes.
template <typename T, int PRED>
__global__ void k_roi_mid(const RoiBox* __restrict__ boxes, int nbox, uint64_t total, Grid<T> base, LevelGeom low,
                          QuantParams qp, const uint16_t* __restrict__ codes, const T* __restrict__ unpred_dense,
                          T* __restrict__ mid, size_t msx, size_t msy)
{
    using A = Ar<T>;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        int bi = 0;
        while (bi + 1 < nbox && boxes[bi + 1].start <= t) ++bi;
        const RoiBox bx = boxes[bi];
        const uint64_t i = t - bx.start;
        const int ex = bx.x1 - bx.x0 + 1, ey = bx.y1 - bx.y0 + 1;
        const int X = bx.x0 + (int)(i % ex), Y = bx.y0 + (int)((i / ex) % ey), Z = bx.z0 + (int)(i / ((uint64_t)ex * ey));
        const int si = ((Z & 1) << 2) | ((Y & 1) << 1) | (X & 1);
        const int x = X >> 1, y = Y >> 1, z = Z >> 1;
        T v;
        if (si == 0) {
            v = base.at((size_t)z * base.sy + (size_t)y * base.sx + x);
        } else {
            const size_t k = (size_t)(si - 1) * low.n + cm_index(low, x, y, z);
            const int q = codes[k];
            const T dq = q ? recover<T>(q, qp) : unpred_dense[k];
            v = A::add(dq, predict_rt<PRED>(si - 1, base, x, y, z));
        }
        mid[(size_t)Z * msy + (size_t)Y * msx + X] = v;
    }
}

template <typename T, int PRED>
__global__ void k_roi_box(RoiBox box, Grid<T> mid, LevelGeom high, QuantParams qp, const uint16_t* __restrict__ codes,
                          const T* __restrict__ unpred_dense, T* __restrict__ out)
{
    using A = Ar<T>;
    const int ex = box.x1 - box.x0 + 1, ey = box.y1 - box.y0 + 1;
    const uint64_t total = (uint64_t)ex * ey * (box.z1 - box.z0 + 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const int X = box.x0 + (int)(i % ex), Y = box.y0 + (int)((i / ex) % ey), Z = box.z0 + (int)(i / ((uint64_t)ex * ey));
        const int si = ((Z & 1) << 2) | ((Y & 1) << 1) | (X & 1);
        const int x = X >> 1, y = Y >> 1, z = Z >> 1;
        T v;
        if (si == 0) {
            v = mid.at((size_t)z * mid.sy + (size_t)y * mid.sx + x);
        } else {
            const size_t k = (size_t)(si - 1) * high.n + cm_index(high, x, y, z);
            const int q = codes[k];
            const T dq = q ? recover<T>(q, qp) : unpred_dense[k];
            v = A::add(dq, predict_rt<PRED>(si - 1, mid, x, y, z));
        }
        out[i] = v;
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

template void launch_roi_mid<float>(const RoiBox*, int, uint64_t, const float*, const LevelGeom&, QuantParams, int,
                                    const uint16_t*, const float*, float*, cudaStream_t);
template void launch_roi_mid<double>(const RoiBox*, int, uint64_t, const double*, const LevelGeom&, QuantParams, int,
                                     const uint16_t*, const double*, double*, cudaStream_t);
template void launch_roi_box<float>(const RoiBox&, const float*, const LevelGeom&, QuantParams, int, const uint16_t*,
                                    const float*, float*, cudaStream_t);
template void launch_roi_box<double>(const RoiBox&, const double*, const LevelGeom&, QuantParams, int,
                                     const uint16_t*, const double*, double*, cudaStream_t);

}  // namespace stz
