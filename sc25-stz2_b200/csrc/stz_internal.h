// Internal shared definitions of the STZ B200 library (host + device).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace stz {

// Message returned by stz_last_error() on the calling thread.
void set_last_error(const std::string& msg);

// Longest canonical Huffman code of the container format.
constexpr int kMaxCodeLen = 24;
// Fast decode table width (bits) of the GPU decoder.
constexpr int kLutBits = 12;
// Histogram window (bins around the radius) kept in shared memory and copied
// to the host for codebook construction; codes outside it take a slow path.
constexpr int kHistWindow = 4096;
// Planes of one coder work item: an item covers max(1, 128 / C) chunks of a
// stream, i.e. up to 128 planes (the coder kernels split an item over
// several CTAs, see huffman.cu).
constexpr int kCoderThreads = 128;

// Learned correction of one level (this project's addition; no reference
// counterpart): an int8 MLP 14 -> 32 -> 32 -> 7 on the 14-point stencil of a
// coarse cell (STZ_LEARNED_STENCIL). Inputs: stencil values minus the mean of
// the 8 cell corners, times rs = 1 / (eb * s_in), rounded to int8 (clamped to
// +-127). Hidden layers: int32 accumulation, ReLU and fixed-point
// requantization a = clamp((acc * m + 2^(sh-1)) >> sh, 0, 127). Output o,
// acc_o * (s_out * eb), is added to the base prediction of block o at interior
// cells (1 <= x,y,z <= dim-3) of the blocks a per-level flag selects. The
// struct is the 2112-byte little-endian record stored in the container.
struct LearnedModel {
    double s_in, s_out;
    int8_t w1[32][16];  // columns 14, 15 are zero
    int32_t b1[32], m1, sh1;
    int8_t w2[32][32];
    int32_t b2[32], m2, sh2;
    int8_t w3[8][32];   // row 7 unused
    int32_t b3[8];
};
static_assert(sizeof(LearnedModel) == 2112, "LearnedModel is a fixed on-disk record");

// Stencil of the learned correction around coarse point (x, y, z): the 8
// corners of the cell, then (-1,0,0), (0,-1,0), (0,0,-1), (2,1,1), (1,2,1),
// (1,1,2) (x, y, z offsets).
#define STZ_LEARNED_STENCIL                                                                                       \
    {                                                                                                             \
        {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}, {-1, 0, 0},       \
            {0, -1, 0}, {0, 0, -1}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}                                               \
    }

// What a level kernel needs to apply a learned correction (model == nullptr:
// none). rs and so in the level's value type, computed on the host as
// (T)(1 / (eb * s_in)) and (T)(s_out * eb).
template <typename T>
struct LearnedArgs {
    const LearnedModel* model = nullptr;  // device memory
    uint32_t flags = 0;                    // blocks (bit b) that use it
    T rs = T(0), so = T(0);
    // Level kernels: evaluate the network block-wide on the tensor cores
    // (tcgen05 kind::i8) instead of per thread with dp4a (same integers).
    bool tensor_cores = true;
};

// Nonzero when a tensor-core MMA of the learned network did not complete in
// time (a bounded wait gave up); read and cleared by learned_tc_error_take.
uint32_t learned_tc_error_take(cudaStream_t st);

// The level kernels' TMA tile-load error word: level_error_init maps it for
// the current device (once per context); level_error_take returns whether a
// tile load gave up waiting since the last call, and clears it.
cudaError_t level_error_init();
bool level_error_take();

// Quantizer constants of one level (FD5:1208-1210): eb, 1/eb computed once on
// the host (recip = 1.0 / eb), radius.
struct QuantParams {
    double eb;
    double recip;
    int radius;
    // |d| < tlo (in the residual's own type) guarantees code == radius: tlo is
    // the largest value <= eb with fl(tlo * recip) < 1. Zero disables the
    // shortcut (it is only an early exit; the full path gives the same code).
    float tlo32 = 0.f;
    double tlo64 = 0.0;
};

// Quantizer constants with the fast-path thresholds filled in.
QuantParams make_quant_params(double eb, int radius);

// Exact f32 quantizer table of one eb (the plain level encoders): for half
// index h < kQuantTableH, entry h = {S_h, S_{h+1}, lo_h, hi_h} on |d|: the
// residuals with S_h <= |d| < S_{h+1} are the ones quantize_full puts at
// half h (S_h = the least float with trunc(|d| / eb) >= 2h - 1, S_0 = 0), and
// of those exactly lo_h <= |d| <= hi_h pass its error check (code radius +- h;
// the others are unpredictable, code 0). Every threshold is found on the
// host with the device's own operations (IEEE double products, float
// subtraction flushed to zero), so the table reproduces quantize_full bit for
// bit; |d| outside an entry's interval, or beyond the table, takes
// quantize_full itself. r2 (~ 0.5 / eb in float) only estimates h.
constexpr int kQuantTableH = 64;
struct QuantTable {
    float4 e[kQuantTableH];
    float r2;
    int on;  // 0: every residual takes quantize_full (eb out of the table's range)
};
QuantTable make_quant_table(const QuantParams& qp);

// One refinement level: the 7 residual sub-blocks of size (dx,dy,dz) predicted
// from the decoded coarse grid of the same size.
struct LevelGeom {
    int dx, dy, dz;
    int C;              // marker chunk edge
    int ncx, ncy, ncz;  // chunks per axis
    size_t n;           // dx*dy*dz
    __host__ __device__ int nchunks() const { return ncx * ncy * ncz; }
};

// One residual stream (level k, block b) as the entropy coder sees it.
struct StreamDesc {
    uint64_t code_off;    // element offset of the stream's codes / unpred_dense
    uint64_t chunk_base;  // offset into per-chunk arrays (unpred counts, word offsets: +stream index)
    uint64_t sub_base;    // offset into per-sub-chunk arrays (nchunks * C)
    uint64_t word_base;   // payload word offset of the stream
    uint64_t word_cap;    // payload words reserved for the stream
    uint32_t C, ncx, ncy, ncz;
    uint32_t nchunks;
    uint32_t cb_off;      // offset of the canonical list (sym/len) in the codebook arrays
    uint32_t n_used;      // symbols in the codebook
    uint32_t radius;      // also the centre code
    uint32_t run_base;    // run symbols in code values [run_base, run_base + run_n)
    uint32_t run_n;       // (0: no runs); see run_geometry
};

// Run symbols of a plane of `plane` codes (container version 3): J =
// min(14, floor(log2 plane)), D = min(32, 2^J), LD = log2 D. Slot i < D - 1
// stands for a run of i + 2 centre codes, slot D - 1 + m for 2^(LD + 1 + m)
// (m < J - LD); run_n = D - 1 + J - LD slots. Returns J (0: no runs).
__host__ __device__ inline uint32_t run_geometry(uint32_t plane, uint32_t& D, uint32_t& LD)
{
    uint32_t J = 0;
    while (J < 14 && (2ull << J) <= plane) ++J;
    LD = J < 5 ? J : 5;
    D = 1u << LD;
    return J;
}
__host__ __device__ inline uint32_t run_slot_count(uint32_t plane)
{
    uint32_t D, LD;
    const uint32_t J = run_geometry(plane, D, LD);
    return J ? D - 1 + J - LD : 0;
}
__host__ __device__ inline uint32_t run_length(uint32_t slot, uint32_t D, uint32_t LD)
{
    return slot < D - 1 ? slot + 2 : 1u << (slot - (D - 1) + LD + 1);
}

// Where a level launch runs its boundary-shell kernel: on `st`, concurrently
// with the interior kernel (forked from and joined back to the caller's
// stream with the two events); st null: after the interior kernel on the
// caller's stream. The two kernels write disjoint points.
struct SideStream {
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

// One CTA of the chunk coders: `count` chunks of stream `stream` whose ids are
// chunk_ids[first .. first + count).
struct CtaWork {
    uint32_t stream;
    uint32_t first;
    uint32_t count;
    uint32_t pad;
};

// Header of a request batch in device memory (request server). The arrays
// (CtaWork, chunk ids, UnpredWork, low-level and high-level ROI job lists)
// follow at the given byte offsets from the header's start.
struct BatchHdr {
    uint32_t n_work, n_uwork, n_mid, n_req;
    uint64_t mid_total, req_total;  // points of all mid regions / all outputs
    uint32_t o_work, o_ids, o_uwork, o_mid, o_req, pad;
};

}  // namespace stz
