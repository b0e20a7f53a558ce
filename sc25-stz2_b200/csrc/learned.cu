// Batch inference of the learned correction's int8 network on rows of int8
// inputs: the tcgen05 kind::i8 form (three MMAs per 128-row tile, int32
// accumulators in TMEM) and the per-thread dp4a form the level kernels use.
// Both return the integer output accumulators, so the two agree bit for bit
// (stz_debug_learned_infer; the tensor-core form also runs the training
// module's int8 evaluation).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "learned.h"
#include "learned_tc.cuh"
#include "runtime.h"
#include "stz/stz.h"
#include "stz_device.cuh"
#include "stz_internal.h"

namespace stz {
namespace {

// 128 threads; thread t owns row t of each 128-row tile (tc::net_run).
__global__ void __launch_bounds__(128) k_learned_infer_tc(const int8_t* __restrict__ xq, uint64_t n,
                                                          const LearnedModel* __restrict__ M,
                                                          int32_t* __restrict__ out, uint32_t* __restrict__ err)
{
    __shared__ __align__(1024) tc::Net<1> net;
    __shared__ __align__(16) LearnedModel sm;
    const int tid = threadIdx.x;
    learned_load(&sm, M, tid, 128);
    __syncthreads();
    tc::net_setup(net, sm, tid);
    uint32_t phase = 0;
    bool failed = false;
    for (uint64_t tile = blockIdx.x; tile * 128 < n; tile += gridDim.x) {
        const uint64_t s = tile * 128 + tid;
        const bool valid = s < n;
        const uint4 x = valid ? *reinterpret_cast<const uint4*>(xq + s * 16) : make_uint4(0u, 0u, 0u, 0u);
        int acc3[7];
        if (!tc::net_run(net, sm, x, phase, tid, acc3)) {
            failed = true;
            break;
        }
        if (valid) {
            int4* o = reinterpret_cast<int4*>(out + s * 8);
            o[0] = make_int4(acc3[0], acc3[1], acc3[2], acc3[3]);
            o[1] = make_int4(acc3[4], acc3[5], acc3[6], 0);
        }
    }
    tc::net_teardown(net, tid);
    if (failed && tid == 0) atomicOr(err, 1u);
}

// The same network, thread per row, dp4a (the level kernels' form).
__global__ void __launch_bounds__(256) k_learned_infer_dp4a(const int8_t* __restrict__ xq, uint64_t n,
                                                            const LearnedModel* __restrict__ M,
                                                            int32_t* __restrict__ out)
{
    __shared__ __align__(16) LearnedModel sm;
    learned_load(&sm, M, threadIdx.x, blockDim.x);
    __syncthreads();
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n; s += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 x = *reinterpret_cast<const uint4*>(xq + s * 16);
        int acc3[7];
        learned_mlp_int(sm, x, acc3);
        int4* o = reinterpret_cast<int4*>(out + s * 8);
        o[0] = make_int4(acc3[0], acc3[1], acc3[2], acc3[3]);
        o[1] = make_int4(acc3[4], acc3[5], acc3[6], 0);
    }
}

}  // namespace

void launch_learned_infer(bool tensor_cores, const int8_t* xq, uint64_t n, const LearnedModel* M, int32_t* out,
                          uint32_t* err, cudaStream_t st)
{
    if (!n) return;
    if (tensor_cores) {
        const uint64_t tiles = (n + 127) / 128;
        k_learned_infer_tc<<<(unsigned)std::min<uint64_t>(tiles, 148 * 8), 128, 0, st>>>(xq, n, M, out, err);
    } else {
        k_learned_infer_dp4a<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(xq, n, M, out);
    }
}

}  // namespace stz

using namespace stz;

extern "C" stz_status stz_debug_learned_infer(stz_context* ctx, const int8_t* xq, size_t n, const void* record,
                                              int tensor_cores, int32_t* out)
{
    if (!ctx || !xq || !record || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (n == 0) return STZ_OK;
    LearnedModel m;
    std::memcpy(&m, record, sizeof m);
    if (!learned_model_valid(m)) STZ_FAIL(STZ_ERR_ARG, "bad learned model record");
    STZ_TRY(enter(ctx));
    cudaStream_t st = ctx->st;
    DevBuf dx, dout, dm, derr;
    STZ_CUDA(dx.ensure(n * 16));
    STZ_CUDA(dout.ensure(n * 32));
    STZ_CUDA(dm.ensure(sizeof m));
    STZ_CUDA(derr.ensure(4));
    STZ_CUDA(cudaMemcpyAsync(dx.p, xq, n * 16, cudaMemcpyHostToDevice, st));
    STZ_CUDA(cudaMemcpyAsync(dm.p, &m, sizeof m, cudaMemcpyHostToDevice, st));
    STZ_CUDA(cudaMemsetAsync(derr.p, 0, 4, st));
    launch_learned_infer(tensor_cores != 0, (const int8_t*)dx.p, n, dm.as<LearnedModel>(), dout.as<int32_t>(),
                         derr.as<uint32_t>(), st);
    STZ_CUDA(cudaGetLastError());
    uint32_t e = 0;
    STZ_CUDA(cudaMemcpyAsync(out, dout.p, n * 32, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaMemcpyAsync(&e, derr.p, 4, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaStreamSynchronize(st));
    if (e) STZ_FAIL(STZ_ERR_CUDA, "tensor-core inference: an MMA did not complete in time");
    return STZ_OK;
}
