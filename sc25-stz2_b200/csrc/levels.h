// Host-side launchers of the level kernels (levels.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

template <typename T>
struct LevelEncodeArgs {
    const T* field;     // input field (device)
    size_t fsx, fsy;    // field row / plane strides
    int stride;         // sampling stride of this level's fine grid (1 = finest)
    const T* coarse;    // decoded coarse grid (geo.dx x dy x dz)
    LevelGeom geo;
    int predictor;      // 0 = dynamic lines (FD5), 1 = plain cubic, 2 = staged (dependency.cpp),
                        // 3 = 12-point truncated bicubic (stz2.cpp)
    uint16_t* codes;        // 7 x n, chunk-major per stream
    T* unpred_dense;        // 7 x n, written where the code is 0
    uint32_t* unpred_cnt;   // 7 x (nchunks + 1)
    uint32_t* hist_full;    // 7 x 2*radius
    uint32_t* hist_outside; // 7
    T* decoded;             // decoded fine grid (2dx x 2dy x 2dz) or null on the finest level
                            // (the staged predictor needs one there too: a scratch grid)
    QuantParams qp;
    LearnedArgs<T> learned; // learned correction (model null: none)
    SideStream side;        // boundary-shell kernel placement
};

template <typename T>
struct LevelDecodeArgs {
    const T* coarse;
    LevelGeom geo;
    int predictor;
    QuantParams qp;
    const uint16_t* codes;
    const T* unpred_dense;
    T* out;  // fine grid (2dx x 2dy x 2dz)
    LearnedArgs<T> learned; // learned correction (model null: none)
    SideStream side;        // boundary-shell kernel placement
    // z-bricks [zb_lo, zb_hi) only (zb_hi < 0: the whole level); see
    // level_decode_bricks
    int zb_lo = 0, zb_hi = -1;
};

// The plain decode kernel's z-bricks of a level (0 when a level decode
// cannot be split: learned correction, or no interior). Brick b < n - 1
// reconstructs fine planes from coarse z in [1 + b*ZB, 1 + (b+1)*ZB), the
// first also z = 0 and the last up to dz - 1; *below = the bricks whose
// coarse z stay below zlim (they need only codes of chunk layers under
// zlim / C).
int level_decode_bricks(const LevelGeom& g, bool learned, int zlim, int* below);

template <typename T>
void launch_level_encode(const LevelEncodeArgs<T>& a, cudaStream_t st);
template <typename T>
void launch_level_decode(const LevelDecodeArgs<T>& a, cudaStream_t st);

// Learned-correction choice: on every second interior coarse point per axis
// (1/8 of them) of a level, the codes of each block with the base prediction
// (hist[0][b]) and with the correction a.learned adds (hist[1][b]); bins
// radius-kEvalHalf .. radius+kEvalHalf exactly, every other code (and code 0)
// in the last bin. hist: 2 x 7 x kEvalBins counters, zeroed by the caller.
constexpr int kEvalHalf = 128;
constexpr int kEvalBins = 2 * kEvalHalf + 2;
template <typename T>
void launch_learned_eval(const LevelEncodeArgs<T>& a, uint32_t* hist, cudaStream_t st);
template <typename T>
void launch_subsample(const T* field, int nx, int ny, int nz, int s, T* out, cudaStream_t st);
template <typename T>
void launch_minmax(const T* p, size_t n, double* out2, cudaStream_t st);
double minmax_key_to_double(unsigned long long k);

template <typename T>
void launch_split(const T* full, int nx, int ny, int nz, T* subs, cudaStream_t st);
template <typename T>
void launch_merge(const T* subs, int hx, int hy, int hz, T* full, cudaStream_t st);
// dependency.cpp's per-block stage functions on dense sub-block arrays (mode
// 0 preprocess, 1 depreprocess); refs as stz_preprocess_block_staged_dev.
template <typename T>
void launch_block_staged(int mode, int block, const T* src, const void* const refs[6], T* dst, int dx, int dy, int dz,
                         cudaStream_t st);
template <typename T>
void launch_quantize(const T* d, size_t n, QuantParams qp, int* q, T* unpred, uint32_t* tile_cnt, uint64_t* tile_off,
                     cudaStream_t st);
template <typename T>
void launch_dequantize(const int* q, size_t n, QuantParams qp, const T* unpred, T* out, uint32_t* tile_cnt,
                       uint64_t* tile_off, cudaStream_t st);
template <typename T>
void launch_block_op(int mode, int predictor, int block, const T* src, const T* ref, T* dst, int dx, int dy, int dz,
                     int x0, int x1, int y0, int y1, int z0, int z1, cudaStream_t st);

}  // namespace stz
