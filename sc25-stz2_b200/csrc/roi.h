// Host-side launchers of the ROI kernels (roi.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

// Inclusive box in grid coordinates; `start` = sum of the volumes of the
// boxes before it in a batch.
struct RoiBox {
    int x0, x1, y0, y1, z0, z1;
    uint64_t start;
};

// Rebuild the mid grid (dims 2*low) on `boxes` from the decoded base (dims of
// the low level's blocks) and the low level's decoded codes.
template <typename T>
void launch_roi_mid(const RoiBox* boxes_dev, int nbox, uint64_t total, const T* base, const LevelGeom& low,
                    QuantParams qp, int predictor, const uint16_t* codes, const T* unpred_dense, T* mid,
                    cudaStream_t st);
// Reconstruct one full-resolution box from the mid grid and the high level's
// decoded codes into out (row-major over the box).
template <typename T>
void launch_roi_box(const RoiBox& box, const T* mid, const LevelGeom& high, QuantParams qp, int predictor,
                    const uint16_t* codes, const T* unpred_dense, T* out, cudaStream_t st);

}  // namespace stz
