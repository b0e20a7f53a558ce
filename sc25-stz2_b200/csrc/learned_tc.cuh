// 5th-generation tensor-core (tcgen05, kind::i8) primitives for the learned
// correction's int8 network: operand layout in shared memory, instruction
// and matrix descriptors, TMEM allocation, MMA issue / commit / bounded
// mbarrier wait, and TMEM loads.
//
// Operands are K-major without swizzling: a tile of R rows x 32 int8 (K)
// is stored as groups of 8 rows, each group two 128-byte core matrices (8
// rows x 16 bytes: K bytes 0-15, then 16-31). In the matrix descriptor the
// leading byte offset (between the two K halves) is 128 and the stride byte
// offset (between 8-row groups) 256.
//
// D (int32, M = 128 rows) lives in TMEM: row m in lane m, column n in column
// base + n; warp w of the CTA reads lanes 32w .. 32w + 31.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "stz_device.cuh"
#include "stz_internal.h"

namespace stz {
namespace tc {

// Bounded waits: about a second at most before a kernel gives up and
// reports an error (the MMAs here complete in well under a microsecond).
constexpr int kMbarSpin = 1 << 20;

// Instruction descriptor: D s32, A and B signed 8-bit, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_i8_m128(int n)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of (row, k) in a K-major no-swizzle operand tile with 32 K bytes.
__host__ __device__ __forceinline__ int kmajor_off(int row, int k)
{
    return (row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15);
}

// Shared-memory matrix descriptor of such a tile (start 16-byte aligned).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Whole warp: allocate ncols (power of two >= 32) TMEM columns, address to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// One thread: D[tmem] (+)= A * B^T.
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The issuing thread: arrive on the mbarrier once its MMAs have completed.
__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
// The initialized mbarrier visible to the tensor core's arrivals.
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    return ok != 0;
}
// false when the phase did not complete within kMbarSpin tries.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase)
{
    for (int i = 0; i < kMbarSpin; ++i)
        if (mbar_try(mbar, phase)) return true;
    return false;
}

// This warp's 32 lanes, 32 consecutive 32-bit columns from taddr.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
// 8 consecutive columns.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- the int8 network for a block of NT x 128 threads ------------------------------
// Thread t owns row t & 127 of tile t >> 7. Layers 1 and 2 are M = 128,
// N = 32, K = 32 MMAs (inputs padded from 14 to 32), layer 3 N = 16 (7
// outputs); tile t's accumulators use TMEM columns 32t .. 32t + 31.
constexpr uint32_t kIdescN32 = idesc_i8_m128(32);
constexpr uint32_t kIdescN16 = idesc_i8_m128(16);

template <int NT>
struct Net {
    uint8_t A[NT][4096];  // this layer's inputs, K-major
    uint8_t B1[1024], B2[1024], B3[512];
    uint64_t mbar;
    uint32_t tbase;
};

// Whole block (NT x 128 threads), after M is readable: weights into the B
// operands, the mbarrier, TMEM columns. Ends with a block barrier.
template <int NT>
__device__ __forceinline__ void net_setup(Net<NT>& s, const LearnedModel& M, int tid)
{
    for (int i = tid; i < 32 * 32; i += NT * 128) {
        const int r = i >> 5, k = i & 31;
        s.B1[kmajor_off(r, k)] = (uint8_t)(k < 16 ? M.w1[r][k] : 0);
        s.B2[kmajor_off(r, k)] = (uint8_t)M.w2[r][k];
        if (r < 16) s.B3[kmajor_off(r, k)] = (uint8_t)(r < 8 ? M.w3[r][k] : 0);
    }
    if (tid == 0) {
        mbar_init(smem_addr(&s.mbar), 1);
        fence_mbar_init();
    }
    if (tid < 32) tmem_alloc(smem_addr(&s.tbase), 32 * NT);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

// Whole block: the network on this thread's packed inputs x. acc3 gets the
// 7 output accumulators. false (on every thread) when an MMA did not
// complete in time; the block must then stop issuing and tear down.
template <int NT>
__device__ __forceinline__ bool net_run(Net<NT>& s, const LearnedModel& M, const uint4& x, uint32_t& phase, int tid,
                                        int (&acc3)[7])
{
    const int tile = tid >> 7, row = tid & 127;
    uint8_t* A = s.A[tile];
    const uint32_t taddr = s.tbase + ((uint32_t)(((tid >> 5) & 3) * 32) << 16) + (uint32_t)(32 * tile);
    const uint32_t mb = smem_addr(&s.mbar);
    *reinterpret_cast<uint4*>(A + kmajor_off(row, 0)) = x;
    *reinterpret_cast<uint4*>(A + kmajor_off(row, 16)) = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll 1
    for (int layer = 0; layer < 3; ++layer) {
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (tid == 0) {
            const uint64_t bd = kmajor_desc(smem_addr(layer == 0 ? s.B1 : layer == 1 ? s.B2 : s.B3));
#pragma unroll
            for (int t = 0; t < NT; ++t)
                mma_i8(s.tbase + 32u * t, kmajor_desc(smem_addr(s.A[t])), bd, layer < 2 ? kIdescN32 : kIdescN16, 0u);
            mma_commit(mb);
        }
        const bool ok = mbar_wait(mb, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) return false;
        fence_after_sync();
        if (layer < 2) {
            uint32_t acc[32];
            tmem_ld32(taddr, acc);
            tmem_wait_ld();
            const int32_t* b = layer == 0 ? M.b1 : M.b2;
            const int m = layer == 0 ? M.m1 : M.m2, sh = layer == 0 ? M.sh1 : M.sh2;
            uint32_t w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
            for (int j = 0; j < 32; ++j) w[j >> 2] |= learned_requant((int)acc[j] + b[j], m, sh) << (8 * (j & 3));
            *reinterpret_cast<uint4*>(A + kmajor_off(row, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(A + kmajor_off(row, 16)) = make_uint4(w[4], w[5], w[6], w[7]);
        } else {
            uint32_t acc[8];
            tmem_ld8(taddr, acc);
            tmem_wait_ld();
#pragma unroll
            for (int o = 0; o < 7; ++o) acc3[o] = (int)acc[o] + M.b3[o];
        }
    }
    return true;
}

// Whole block: release the TMEM columns (after the last net_run).
template <int NT>
__device__ __forceinline__ void net_teardown(Net<NT>& s, int tid)
{
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (tid < 32) tmem_dealloc(s.tbase, 32 * NT);
}

}  // namespace tc
}  // namespace stz
