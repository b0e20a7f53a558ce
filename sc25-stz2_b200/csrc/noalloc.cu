// Quantizer entry point that allocates no memory.
//
// stz_quantize_dev (the quantize_range_nodec equivalent) needs a few hundred
// KB of scratch for per-tile counts and offsets, which it takes from its
// context's cudaMalloc'ed buffers. Some callers cannot allocate at all: code
// that runs inside another framework's memory pool or arena (which forbids
// foreign cudaMalloc/cudaFree because those synchronize the device and
// fragment the pool), code that must not stall on an implicit device-wide
// synchronization in a latency-critical loop, and hosts that pre-reserve all
// GPU memory up front. For them, stz_quantize_noalloc_dev uses a fixed scratch
// array that lives in the library image itself (a file-scope __device__
// array, loaded with the module on every GPU that uses the library and held
// until the process exits) and takes the CUDA stream from the caller, so it
// needs no context either.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "levels.h"
#include "stz/stz.h"
#include "stz_internal.h"

namespace {

// One tile of the quantizer is 1024 values; the scratch holds the per-tile
// unpredictable counts (uint32) and their exclusive prefix sums (uint64, one
// extra entry for the total).
constexpr size_t kTile = 1024;
constexpr size_t kMaxTiles = 65536;
constexpr size_t kCntBytes = (kMaxTiles * sizeof(uint32_t) + 255) & ~size_t(255);
constexpr size_t kScratchBytes = kCntBytes + (kMaxTiles + 1) * sizeof(uint64_t);
static_assert(STZ_NOALLOC_MAX_VALUES == kMaxTiles * kTile, "header limit and scratch size disagree");

// The scratch itself. In host code this name is only a host-side stand-in:
// the device address comes from cudaGetSymbolAddress in the current context.
static __device__ __align__(256) unsigned char g_quantize_scratch[kScratchBytes];

// Device address of the scratch in the current context. Looked up on every
// call: the lookup is a host-side table read once the module is loaded, and a
// cached address would go stale after cudaDeviceReset (the module reloads,
// possibly elsewhere) or belong to another context on the same device.
cudaError_t scratch_address(void** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_quantize_scratch);
    if (e != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}

}  // namespace

extern "C" stz_status stz_quantize_noalloc_dev(stz_dtype dtype, const void* data, size_t n, double eb, int radius,
                                              int32_t* q, void* unpred, size_t* n_unpred, void* stream)
{
    stz::set_last_error("");
    if (!n_unpred || (n && (!data || !q || !unpred))) {
        stz::set_last_error("null pointer");
        return STZ_ERR_ARG;
    }
    if (dtype != STZ_F32 && dtype != STZ_F64) {
        stz::set_last_error("bad dtype");
        return STZ_ERR_ARG;
    }
    if (!(eb > 0) || radius < 1 || radius > (1 << 30)) {
        stz::set_last_error("bad eb or radius");
        return STZ_ERR_ARG;
    }
    if (n > STZ_NOALLOC_MAX_VALUES) {
        stz::set_last_error("stz_quantize_noalloc_dev handles at most " + std::to_string(STZ_NOALLOC_MAX_VALUES) +
                            " values per call (its fixed scratch), got " + std::to_string(n) +
                            "; split the data or use stz_quantize_dev");
        return STZ_ERR_RANGE;
    }
    *n_unpred = 0;
    if (n == 0) return STZ_OK;
    void* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) {
        stz::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return STZ_ERR_CUDA;
    }
    // Every scratch word the kernels read was written earlier in this call
    // (each tile writes its count, the scan writes every offset), so nothing
    // needs clearing between calls.
    uint32_t* cnt = static_cast<uint32_t*>(base);
    uint64_t* off = reinterpret_cast<uint64_t*>(static_cast<unsigned char*>(base) + kCntBytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const stz::QuantParams qp = stz::make_quant_params(eb, radius);
    if (dtype == STZ_F64)
        stz::launch_quantize<double>(static_cast<const double*>(data), n, qp, q, static_cast<double*>(unpred), cnt, off, st);
    else
        stz::launch_quantize<float>(static_cast<const float*>(data), n, qp, q, static_cast<float*>(unpred), cnt, off, st);
    e = cudaGetLastError();
    uint64_t total = 0;
    const size_t tiles = (n + kTile - 1) / kTile;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, off + tiles, sizeof(total), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        stz::set_last_error(std::string("quantize: ") + cudaGetErrorString(e));
        return STZ_ERR_CUDA;
    }
    *n_unpred = (size_t)total;
    return STZ_OK;
}
