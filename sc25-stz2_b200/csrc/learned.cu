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

constexpr uint32_t kIdescN32 = tc::idesc_i8_m128(32);
// Layer 3 (7 outputs) runs as N = 16, the smallest N every M = 128 form takes.
constexpr uint32_t kIdescN16 = tc::idesc_i8_m128(16);

// 128 threads; thread t owns row t of each 128-row tile. Per tile and layer:
// the A rows are written to shared memory, one thread issues the MMA and
// commits it to an mbarrier, all wait (bounded), each warp loads its 32
// rows' accumulators from TMEM, adds the bias and requantizes (layers 1, 2)
// into the next layer's A rows, or writes the output accumulators (layer 3).
__global__ void __launch_bounds__(128) k_learned_infer_tc(const int8_t* __restrict__ xq, uint64_t n,
                                                          const LearnedModel* __restrict__ M,
                                                          int32_t* __restrict__ out, uint32_t* __restrict__ err)
{
    __shared__ __align__(1024) uint8_t sA[4096];
    __shared__ __align__(1024) uint8_t sB1[1024];
    __shared__ __align__(1024) uint8_t sB2[1024];
    __shared__ __align__(1024) uint8_t sB3[512];
    __shared__ __align__(16) LearnedModel sm;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tbase_s;
    const int tid = threadIdx.x, warp = tid >> 5;
    learned_load(&sm, M, tid, 128);
    __syncthreads();
    for (int i = tid; i < 32 * 32; i += 128) {
        const int r = i >> 5, k = i & 31;
        sB1[tc::kmajor_off(r, k)] = (uint8_t)(k < 16 ? sm.w1[r][k] : 0);
        sB2[tc::kmajor_off(r, k)] = (uint8_t)sm.w2[r][k];
        if (r < 16) sB3[tc::kmajor_off(r, k)] = (uint8_t)(r < 8 ? sm.w3[r][k] : 0);
    }
    if (tid == 0) {
        tc::mbar_init(tc::smem_addr(&mbar), 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tbase_s), 32);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tbase_s;
    const uint32_t my_lanes = tbase + ((uint32_t)(warp * 32) << 16);
    const uint32_t mb = tc::smem_addr(&mbar);
    const uint64_t adesc = tc::kmajor_desc(tc::smem_addr(sA));
    const uint64_t bdesc[3] = {tc::kmajor_desc(tc::smem_addr(sB1)), tc::kmajor_desc(tc::smem_addr(sB2)),
                               tc::kmajor_desc(tc::smem_addr(sB3))};
    uint32_t phase = 0;
    bool failed = false;
    for (uint64_t tile = blockIdx.x; tile * 128 < n && !failed; tile += gridDim.x) {
        const uint64_t s = tile * 128 + tid;
        const bool valid = s < n;
        const uint4 x = valid ? *reinterpret_cast<const uint4*>(xq + s * 16) : make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 0)) = x;
        *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 16)) = make_uint4(0u, 0u, 0u, 0u);
        for (int layer = 0; layer < 3; ++layer) {
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if (tid == 0) {
                tc::mma_i8(tbase, adesc, bdesc[layer], layer < 2 ? kIdescN32 : kIdescN16, 0u);
                tc::mma_commit(mb);
            }
            const bool ok = tc::mbar_wait(mb, phase);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            tc::fence_after_sync();
            if (layer < 2) {
                uint32_t acc[32];
                tc::tmem_ld32(my_lanes, acc);
                tc::tmem_wait_ld();
                const int32_t* b = layer == 0 ? sm.b1 : sm.b2;
                const int m = layer == 0 ? sm.m1 : sm.m2, sh = layer == 0 ? sm.sh1 : sm.sh2;
                uint32_t w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
                for (int j = 0; j < 32; ++j) w[j >> 2] |= learned_requant((int)acc[j] + b[j], m, sh) << (8 * (j & 3));
                *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 16)) = make_uint4(w[4], w[5], w[6], w[7]);
            } else {
                uint32_t acc[8];
                tc::tmem_ld8(my_lanes, acc);
                tc::tmem_wait_ld();
                if (valid) {
                    int4* o = reinterpret_cast<int4*>(out + s * 8);
                    o[0] = make_int4((int)acc[0] + sm.b3[0], (int)acc[1] + sm.b3[1], (int)acc[2] + sm.b3[2],
                                     (int)acc[3] + sm.b3[3]);
                    o[1] = make_int4((int)acc[4] + sm.b3[4], (int)acc[5] + sm.b3[5], (int)acc[6] + sm.b3[6], 0);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (failed && tid == 0) atomicOr(err, 1u);
    if (warp == 0) tc::tmem_dealloc(tbase, 32);
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
