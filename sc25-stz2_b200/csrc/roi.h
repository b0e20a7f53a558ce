// Host-side launchers of the ROI kernels (roi.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

constexpr int kJobCells = 0;   // rebuild the cells of a window of one level
constexpr int kJobSample = 1;  // progressive level >= 2: every 2^shift-th point of the decoded base

// One unit list entry of a ROI launch.
//   kJobCells : the coarse cells (cx0 + [0, ncx), ...) of the level are
//               rebuilt (a cell = the 2x2x2 fine points its coarse point
//               predicts) and the fine points inside the inclusive window
//               [wx0, wx1] x [wy0, wy1] x [wz0, wz1] are written to
//               out + (Z - oz) * osy + (Y - oy) * osx + (X - ox).
//   kJobSample: the points (cx0 + [0, ncx), ...) of a level grid are written
//               as base[(Z << shift), (Y << shift), (X << shift)] at the same
//               output addressing.
// start = units (cells or points) of the entries before this one.
struct RoiJob {
    int cx0, cy0, cz0, ncx, ncy, ncz;
    int wx0, wx1, wy0, wy1, wz0, wz1;
    int ox, oy, oz, kind;
    int shift, pad;
    uint64_t osx, osy;
    uint64_t start;
    uint64_t out;
};

// A kJobCells entry for the fine window [w0, w1] (inclusive, per axis x, y,
// z) of a level, written to out with the given origin and strides.
RoiJob cells_job(const int w0[3], const int w1[3], void* out, const int origin[3], uint64_t osx, uint64_t osy,
                 uint64_t start);
inline uint64_t job_units(const RoiJob& j) { return (uint64_t)j.ncx * j.ncy * j.ncz; }

// One launch over job list `list` of the batch record at meta (BatchHdr:
// list 0 = n_mid / o_mid / mid_total, list 1 = n_req / o_req / req_total).
// coarse: the level's coarse grid (dims geo.dx x geo.dy x geo.dz); base: the
// decoded base (dims base_geo) for kJobSample entries. A fixed grid walks the
// units the header lists, so the launch can be captured once and replayed.
// la: the level's learned correction (applied at interior cells of the
// flagged blocks; the window must hold the -1..+2 stencil of every such cell).
template <typename T>
void launch_roi_cells(int grid, int block, const uint8_t* meta, int list, const T* coarse, const LevelGeom& geo,
                      const T* base, const LevelGeom& base_geo, QuantParams qp, int predictor, const uint16_t* codes,
                      const T* unpred_dense, cudaStream_t st, const LearnedArgs<T>& la = LearnedArgs<T>());

}  // namespace stz
