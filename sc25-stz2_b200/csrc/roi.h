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

constexpr int kReqBox = 0;     // box of the full-resolution grid
constexpr int kReqSample = 1;  // progressive level >= 2: every 2^shift-th point of the decoded base

// One output of a batch. box: inclusive output coordinates (full-resolution
// grid for kReqBox, level grid for kReqSample); start: prefix of the output
// volumes of the batch; out: device address of the output (row-major box).
struct ReqDesc {
    RoiBox box;
    uint64_t start;
    uint64_t out;
    int32_t kind, shift;
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

// Batched forms over a device-resident batch (BatchHdr at meta): a fixed
// grid x block walks however many points the header lists, so the launches
// can be captured once and replayed for every batch.
template <typename T>
void launch_roi_mid_dyn(int grid, int block, const uint8_t* meta, const T* base, const LevelGeom& low, QuantParams qp,
                        int predictor, const uint16_t* codes, const T* unpred_dense, T* mid, cudaStream_t st);
template <typename T>
void launch_roi_req_dyn(int grid, int block, const uint8_t* meta, const T* mid, const T* base, const LevelGeom& low,
                        const LevelGeom& high, QuantParams qp, int predictor, const uint16_t* codes,
                        const T* unpred_dense, cudaStream_t st);

}  // namespace stz
