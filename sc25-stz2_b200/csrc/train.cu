// GPU training of the learned correction (stz_trainer_*): pairs from the
// compressor's own decoded grids, a BF16-operand / FP32-accumulate MLP
// forward + backward, Adam, quantization-aware training and the int8 export
// the level kernels run.
//
// Float network of one level (trained per level; one trunk, one output per
// sub-block):
//   u  = clamp(x / s_in, -127, 127) / 127        x: 14 stencil features in eb
//   h1 = relu(W1 u + b1)          32             (BF16 operands, FP32 sums)
//   h2 = relu(W2 h1 + b2)         32
//   y  = W3 h2 + b3               7              correction = y * s_t (eb)
// Loss: Huber (delta in eb) of y * s_t - t, t = fine value minus the plain
// prediction in eb. Quantization-aware training rounds u to the int8 grid,
// each weight tensor to max|W| / 127 steps and each activation to the int8
// grid of its calibrated scale (straight-through gradients inside the
// clamp ranges), which is exactly what the exported integer network does up
// to the fixed-point requantization.
//
// A training step is two launches: k_mlp_step (one CTA per 128 samples:
// forward, backward and per-CTA partial gradients, no atomics) and k_adam
// (one CTA: the partials summed in CTA order, so a run is deterministic). A
// device-side step counter drives the epoch shuffles and the learning-rate
// schedule, so a whole phase is one captured CUDA graph of step pairs,
// replayed until the counter reaches the phase's step count.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "levels.h"
#include "runtime.h"
#include "stz/stz.h"
#include "stz_device.cuh"
#include "stz_internal.h"

namespace stz {
namespace {

// Parameter layout (floats): W1[32][16] (columns 14, 15 stay zero), b1[32],
// W2[32][32], b2[32], W3[8][32] (row 7 stays zero), b3[8].
constexpr int kPW1 = 0, kPB1 = 512, kPW2 = 544, kPB2 = 1568, kPW3 = 1600, kPB3 = 1856, kNP = 1864;
constexpr int kTile = 128;         // samples per step CTA
constexpr int kStepThreads = 256;  // two threads per sample
constexpr int kMaxEpochs = 256;
constexpr int kCalib = 65536;      // samples used for scale calibration

// Strides of the step kernel's shared arrays (floats; odd to spread banks).
constexpr int kSX = 17, kSH = 33, kSD = 9;
constexpr size_t kStepSmem = sizeof(float) * (kNP + kTile * (kSX + 4 * kSH + kSD)) + sizeof(uint32_t) * 4 * kTile;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ bool structural_zero(int p)
{
    return (p < kPB1 && (p & 15) >= 14) || (p >= kPW3 + 7 * 32 && p < kPB3) || p == kPB3 + 7;
}

__device__ __forceinline__ bool is_weight(int p) { return p < kPB1 || (p >= kPW2 && p < kPB2) || (p >= kPW3 && p < kPB3); }

// ---- pairs -------------------------------------------------------------------------
// Features and targets at the interior coarse cells x = 1 + step * i (and the
// same on y, z) of one level: features (v - mean of the 8 corners) / eb of
// the 14-point stencil on the decoded coarse grid R (BF16, 16 per pair, the
// last two zero), targets (fine - plain prediction) / eb of the 7 sub-blocks
// (FP32, 8 per pair, the last zero). Pair o = first + i; stops at cap.
template <typename T, int PRED>
__global__ void __launch_bounds__(256) k_train_pairs(const T* __restrict__ field, size_t fsx, size_t fsy, int s,
                                                     const T* __restrict__ R, LevelGeom geo, double inv_eb, int step,
                                                     int sx, int sy, int sz, uint64_t first, uint64_t cap,
                                                     __nv_bfloat16* __restrict__ X, float* __restrict__ Y)
{
    using A = Ar<T>;
    const uint64_t total = (uint64_t)sx * sy * sz;
    const long long gx = geo.dx, gy = (long long)geo.dx * geo.dy;
    constexpr int st[14][3] = STZ_LEARNED_STENCIL;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t o = first + i;
        if (o >= cap) break;
        const int ix = (int)(i % sx), iy = (int)((i / sx) % sy), iz = (int)(i / ((uint64_t)sx * sy));
        const int x = 1 + step * ix, y = 1 + step * iy, z = 1 + step * iz;
        const GlobalAt<T> r{R + (size_t)z * gy + (size_t)y * gx + x, gx, gy};
        T p[7];
        predict7<PRED>(r, true, x, y, z, geo.dx, geo.dy, geo.dz, p);
        T v[14];
#pragma unroll
        for (int k = 0; k < 14; ++k) v[k] = r(st[k][2] * gy + st[k][1] * gx + st[k][0]);
        T m = v[0];
#pragma unroll
        for (int k = 1; k < 8; ++k) m = A::add(m, v[k]);
        m = A::mul(m, T(0.125));
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int a = 2 * k, b = 2 * k + 1;
            const float fa = a < 14 ? (float)((double)A::sub(v[a], m) * inv_eb) : 0.f;
            const float fb = b < 14 ? (float)((double)A::sub(v[b], m) * inv_eb) : 0.f;
            const __nv_bfloat162 h = __floats2bfloat162_rn(fa, fb);
            w[k] = *reinterpret_cast<const uint32_t*>(&h);
        }
        uint4* xo = reinterpret_cast<uint4*>(X + o * 16);
        xo[0] = make_uint4(w[0], w[1], w[2], w[3]);
        xo[1] = make_uint4(w[4], w[5], w[6], w[7]);
        float t[8];
#pragma unroll
        for (int b = 0; b < 7; ++b) {
            const int si = b + 1, px = si & 1, py = (si >> 1) & 1, pz = si >> 2;
            const T f = __ldg(field + (size_t)s * (2 * z + pz) * fsy + (size_t)s * (2 * y + py) * fsx +
                              (size_t)s * (2 * x + px));
            t[b] = (float)(((double)f - (double)p[b]) * inv_eb);
        }
        t[7] = 0.f;
        float4* yo = reinterpret_cast<float4*>(Y + o * 8);
        yo[0] = make_float4(t[0], t[1], t[2], t[3]);
        yo[1] = make_float4(t[4], t[5], t[6], t[7]);
    }
}

// ---- one training step ---------------------------------------------------------------
struct StepArgs {
    const __nv_bfloat16* X;
    const float* Y;
    uint64_t n;               // pairs
    const uint64_t* perm;     // per epoch (a, c): sample g of the epoch is pair (a * g + c) mod n
    const float* Wf;          // forward weights (kNP)
    float* part;              // [CTA][kNP + 1]: partial gradients, then the partial loss sum
    const uint32_t* counter;  // steps done in this phase
    uint32_t steps_per_epoch, total_steps, batch;
    float inv_s_in, inv_s_t, delta;  // delta: Huber delta in units of s_t
    int qat;
    float sa1, sa2;
};

// Input feature u of the network from a stored feature (eb units).
__device__ __forceinline__ float input_u(float x, float inv_s_in, int qat)
{
    const float q = fminf(fmaxf(qat ? rintf(x * inv_s_in) : x * inv_s_in, -127.f), 127.f);
    return qat ? q * (1.f / 127.f) : bf16r(q * (1.f / 127.f));
}

// Activation of a hidden unit: float mode relu + BF16 rounding; QAT the int8
// grid of scale sa. Sets *pass when the gradient flows through.
__device__ __forceinline__ float act(float pre, int qat, float sa, bool* pass)
{
    if (!qat) {
        *pass = pre > 0.f;
        return pre > 0.f ? bf16r(pre) : 0.f;
    }
    *pass = pre > 0.f && pre < 127.f * sa;
    return fminf(fmaxf(rintf(pre / sa), 0.f), 127.f) * sa;
}

__global__ void __launch_bounds__(kStepThreads) k_mlp_step(StepArgs P)
{
    extern __shared__ __align__(16) float sm[];
    float* sW = sm;
    float* xs = sW + kNP;
    float* h1 = xs + kTile * kSX;
    float* h2 = h1 + kTile * kSH;
    float* dh2 = h2 + kTile * kSH;
    float* dh1 = dh2 + kTile * kSH;
    float* dy = dh1 + kTile * kSH;
    uint32_t* mask = reinterpret_cast<uint32_t*>(dy + kTile * kSD);  // [2 layers][2 halves][kTile] (16 bits used)
    __shared__ float red[kStepThreads / 32];

    const uint32_t step = *P.counter;
    if (step >= P.total_steps) return;
    const int tid = threadIdx.x, j = tid & (kTile - 1), half = tid >> 7;
    const uint32_t epoch = step / P.steps_per_epoch, sie = step % P.steps_per_epoch;
    const uint64_t a = P.perm[2 * epoch], c = P.perm[2 * epoch + 1];
    const uint64_t base = (uint64_t)sie * P.batch;
    const uint64_t nb = min((uint64_t)P.batch, P.n - base);
    const float inv_norm = 1.f / (float)(nb * 7);
    for (int i = tid; i < kNP; i += kStepThreads) sW[i] = P.Wf[i];
    const uint64_t local = (uint64_t)blockIdx.x * kTile + j;
    const bool valid = local < nb;
    const uint64_t idx = valid ? (a * (base + local) + c) % P.n : 0;
    // features: each half loads 8 of the 16
    {
        const uint4 w = reinterpret_cast<const uint4*>(P.X + idx * 16)[half];
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&w);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(h[k]);
            xs[j * kSX + 8 * half + 2 * k] = valid ? input_u(f.x, P.inv_s_in, P.qat) : 0.f;
            xs[j * kSX + 8 * half + 2 * k + 1] = valid ? input_u(f.y, P.inv_s_in, P.qat) : 0.f;
        }
    }
    const float4 tv = valid ? reinterpret_cast<const float4*>(P.Y + idx * 8)[half] : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    // layer 1: this half's 16 units
    {
        uint32_t mk = 0;
        const float* x = xs + j * kSX;
        for (int u = 0; u < 16; ++u) {
            const int n = 16 * half + u;
            float acc = sW[kPB1 + n];
#pragma unroll
            for (int k = 0; k < 14; ++k) acc = __fmaf_rn(sW[kPW1 + n * 16 + k], x[k], acc);
            bool pass;
            h1[j * kSH + n] = act(acc, P.qat, P.sa1, &pass);
            mk |= (uint32_t)pass << u;
        }
        mask[(0 * 2 + half) * kTile + j] = mk;
    }
    __syncthreads();
    // layer 2
    {
        uint32_t mk = 0;
        const float* x = h1 + j * kSH;
        for (int u = 0; u < 16; ++u) {
            const int n = 16 * half + u;
            float acc = sW[kPB2 + n];
#pragma unroll
            for (int k = 0; k < 32; ++k) acc = __fmaf_rn(sW[kPW2 + n * 32 + k], x[k], acc);
            bool pass;
            h2[j * kSH + n] = act(acc, P.qat, P.sa2, &pass);
            mk |= (uint32_t)pass << u;
        }
        mask[(1 * 2 + half) * kTile + j] = mk;
    }
    __syncthreads();
    // outputs 4*half .. 4*half+3 (output 7 does not exist), loss and dL/dy
    float loss = 0.f;
    {
        const float* x = h2 + j * kSH;
        const float tt[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int b = 4 * half + q;
            float d = 0.f;
            if (b < 7 && valid) {
                float y = sW[kPB3 + b];
#pragma unroll
                for (int k = 0; k < 32; ++k) y = __fmaf_rn(sW[kPW3 + b * 32 + k], x[k], y);
                const float e = y - tt[q] * P.inv_s_t;
                const float ae = fabsf(e);
                loss += ae <= P.delta ? 0.5f * e * e : P.delta * (ae - 0.5f * P.delta);
                d = fminf(fmaxf(e, -P.delta), P.delta) * inv_norm;
            }
            dy[j * kSD + b] = d;
        }
    }
    __syncthreads();
    // dL/dh2 for this half's units
    {
        const uint32_t mk = mask[(1 * 2 + half) * kTile + j];
        for (int u = 0; u < 16; ++u) {
            const int n = 16 * half + u;
            float g = 0.f;
#pragma unroll
            for (int b = 0; b < 7; ++b) g = __fmaf_rn(sW[kPW3 + b * 32 + n], dy[j * kSD + b], g);
            dh2[j * kSH + n] = (mk >> u & 1u) ? g : 0.f;
        }
    }
    __syncthreads();
    // dL/dh1
    {
        const uint32_t mk = mask[(0 * 2 + half) * kTile + j];
        for (int u = 0; u < 16; ++u) {
            const int i = 16 * half + u;
            float g = 0.f;
#pragma unroll 8
            for (int n = 0; n < 32; ++n) g = __fmaf_rn(sW[kPW2 + n * 32 + i], dh2[j * kSH + n], g);
            dh1[j * kSH + i] = (mk >> u & 1u) ? g : 0.f;
        }
    }
    __syncthreads();
    // partial gradients of this CTA's samples, summed in sample order
    float* out = P.part + (size_t)blockIdx.x * (kNP + 1);
    for (int p = tid; p < kNP; p += kStepThreads) {
        float g = 0.f;
        if (p < kPB1) {
            const int n = p >> 4, k = p & 15;
            if (k < 14)
                for (int s = 0; s < kTile; ++s) g = __fmaf_rn(dh1[s * kSH + n], xs[s * kSX + k], g);
        } else if (p < kPW2) {
            const int n = p - kPB1;
            for (int s = 0; s < kTile; ++s) g += dh1[s * kSH + n];
        } else if (p < kPB2) {
            const int q = p - kPW2, n = q >> 5, i = q & 31;
            for (int s = 0; s < kTile; ++s) g = __fmaf_rn(dh2[s * kSH + n], h1[s * kSH + i], g);
        } else if (p < kPW3) {
            const int n = p - kPB2;
            for (int s = 0; s < kTile; ++s) g += dh2[s * kSH + n];
        } else if (p < kPB3) {
            const int q = p - kPW3, b = q >> 5, n = q & 31;
            if (b < 7)
                for (int s = 0; s < kTile; ++s) g = __fmaf_rn(dy[s * kSD + b], h2[s * kSH + n], g);
        } else {
            const int b = p - kPB3;
            if (b < 7)
                for (int s = 0; s < kTile; ++s) g += dy[s * kSD + b];
        }
        out[p] = g;
    }
    // loss: warp sums, then warps in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((tid & 31) == 0) red[tid >> 5] = loss;
    __syncthreads();
    if (tid == 0) {
        float s = 0.f;
        for (int w = 0; w < kStepThreads / 32; ++w) s += red[w];
        out[kNP] = s;
    }
}

// Forward weights from the master weights: BF16-rounded weights (float
// phase) or each weight tensor on the int8 grid of max|W| / 127 (QAT);
// biases stay FP32. Whole block; `red` holds 3 floats.
__device__ void write_forward_weights(const float* W, float* Wf, int qat, float* red)
{
    if (qat) {
        if (threadIdx.x < 3) red[threadIdx.x] = 0.f;
        __syncthreads();
        float mx[3] = {0.f, 0.f, 0.f};
        for (int p = threadIdx.x; p < kNP; p += blockDim.x) {
            const int t = p < kPB1 ? 0 : (p >= kPW2 && p < kPB2) ? 1 : (p >= kPW3 && p < kPB3) ? 2 : -1;
            if (t >= 0) mx[t] = fmaxf(mx[t], fabsf(W[p]));
        }
        for (int t = 0; t < 3; ++t) {
            float v = mx[t];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            // max is order-independent: the atomics give the same value every run
            if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(&red[t]), __float_as_int(v));
        }
        __syncthreads();
    }
    for (int p = threadIdx.x; p < kNP; p += blockDim.x) {
        float w = W[p];
        if (is_weight(p)) {
            if (qat) {
                const int t = p < kPB1 ? 0 : p < kPB2 ? 1 : 2;
                const float stp = red[t] / 127.f;
                w = stp > 0.f ? rintf(w / stp) * stp : 0.f;
            } else {
                w = bf16r(w);
            }
        }
        Wf[p] = w;
    }
}

struct AdamArgs {
    float* W;
    float* m;
    float* v;
    float* Wf;
    const float* part;
    int ctas;
    uint32_t* counter;
    uint32_t steps_per_epoch, total_steps, batch;
    uint64_t n;
    float lr, lr_min;
    int qat;
    double* loss;  // [epoch][2]: loss sum, residual count
};

__global__ void __launch_bounds__(1024) k_adam(AdamArgs A)
{
    __shared__ float red[4];
    const uint32_t step = *A.counter;
    if (step >= A.total_steps) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float t = (float)(step + 1);
    const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
    const float lr = A.lr_min + 0.5f * (A.lr - A.lr_min) * (1.f + cospif((float)step / (float)A.total_steps));
    for (int p = threadIdx.x; p < kNP; p += blockDim.x) {
        if (structural_zero(p)) continue;
        float g = 0.f;
        for (int c = 0; c < A.ctas; ++c) g += A.part[(size_t)c * (kNP + 1) + p];
        const float m = b1 * A.m[p] + (1.f - b1) * g;
        const float v = b2 * A.v[p] + (1.f - b2) * g * g;
        A.m[p] = m;
        A.v[p] = v;
        A.W[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
    __syncthreads();
    write_forward_weights(A.W, A.Wf, A.qat, red);
    if (threadIdx.x == 0) {
        const uint32_t epoch = step / A.steps_per_epoch;
        const uint64_t nb = min((uint64_t)A.batch, A.n - (uint64_t)(step % A.steps_per_epoch) * A.batch);
        double s = 0.0;
        for (int c = 0; c < A.ctas; ++c) s += A.part[(size_t)c * (kNP + 1) + kNP];
        A.loss[2 * epoch] += s;
        A.loss[2 * epoch + 1] += (double)(nb * 7);
    }
    __syncthreads();
    if (threadIdx.x == 0) *A.counter = step + 1;
}

__global__ void __launch_bounds__(1024) k_refresh_forward(const float* W, float* Wf, int qat)
{
    __shared__ float red[4];
    write_forward_weights(W, Wf, qat, red);
}

// Float-mode activations of samples 0..n-1 (calibration of the int8 scales).
__global__ void __launch_bounds__(256) k_mlp_calib(const __nv_bfloat16* __restrict__ X, uint64_t n,
                                                   const float* __restrict__ Wf, float inv_s_in, float* __restrict__ H)
{
    __shared__ float sW[kNP];
    for (int i = threadIdx.x; i < kNP; i += blockDim.x) sW[i] = Wf[i];
    __syncthreads();
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n; s += (uint64_t)gridDim.x * blockDim.x) {
        float u[14], a1[32];
#pragma unroll
        for (int k = 0; k < 14; ++k) u[k] = input_u(__bfloat162float(X[s * 16 + k]), inv_s_in, 0);
        for (int n1 = 0; n1 < 32; ++n1) {
            float acc = sW[kPB1 + n1];
#pragma unroll
            for (int k = 0; k < 14; ++k) acc = __fmaf_rn(sW[kPW1 + n1 * 16 + k], u[k], acc);
            a1[n1] = acc > 0.f ? bf16r(acc) : 0.f;
            H[s * 64 + n1] = a1[n1];
        }
        for (int n2 = 0; n2 < 32; ++n2) {
            float acc = sW[kPB2 + n2];
#pragma unroll 8
            for (int k = 0; k < 32; ++k) acc = __fmaf_rn(sW[kPW2 + n2 * 32 + k], a1[k], acc);
            H[s * 64 + 32 + n2] = acc > 0.f ? bf16r(acc) : 0.f;
        }
    }
}

// Huber loss (eb units) of the exported int8 network on the stored features
// and of no correction at all; per-block partial sums [block][2].
__global__ void __launch_bounds__(256) k_int8_loss(const __nv_bfloat16* __restrict__ X, const float* __restrict__ Y,
                                                   uint64_t n, const LearnedModel* __restrict__ M, double delta,
                                                   double* __restrict__ part)
{
    __shared__ __align__(16) LearnedModel sm;
    __shared__ double red[2][8];
    learned_load(&sm, M, threadIdx.x, blockDim.x);
    __syncthreads();
    const float inv_s_in = (float)(1.0 / sm.s_in);
    double l_int = 0.0, l_zero = 0.0;
    auto huber = [delta](double e) {
        const double ae = fabs(e);
        return ae <= delta ? 0.5 * e * e : delta * (ae - 0.5 * delta);
    };
    const int* w1 = reinterpret_cast<const int*>(&sm.w1[0][0]);
    const int* w2 = reinterpret_cast<const int*>(&sm.w2[0][0]);
    const int* w3 = reinterpret_cast<const int*>(&sm.w3[0][0]);
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n; s += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t xw[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < 14; ++k) {
            const float q = fminf(fmaxf(rintf(__bfloat162float(X[s * 16 + k]) * inv_s_in), -127.f), 127.f);
            xw[k >> 2] |= ((uint32_t)(int)q & 0xffu) << (8 * (k & 3));
        }
        uint32_t a1[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u}, a2[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        for (int jj = 0; jj < 32; ++jj) {
            int acc = sm.b1[jj];
#pragma unroll
            for (int w = 0; w < 4; ++w) acc = __dp4a(w1[jj * 4 + w], (int)xw[w], acc);
            a1[jj >> 2] |= learned_requant(acc, sm.m1, sm.sh1) << (8 * (jj & 3));
        }
        for (int jj = 0; jj < 32; ++jj) {
            int acc = sm.b2[jj];
#pragma unroll
            for (int w = 0; w < 8; ++w) acc = __dp4a(w2[jj * 8 + w], (int)a1[w], acc);
            a2[jj >> 2] |= learned_requant(acc, sm.m2, sm.sh2) << (8 * (jj & 3));
        }
        for (int o = 0; o < 7; ++o) {
            int acc = sm.b3[o];
#pragma unroll
            for (int w = 0; w < 8; ++w) acc = __dp4a(w3[o * 8 + w], (int)a2[w], acc);
            const double t = Y[s * 8 + o];
            l_int += huber((double)acc * sm.s_out - t);
            l_zero += huber(-t);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l_int += __shfl_xor_sync(0xffffffffu, l_int, o);
        l_zero += __shfl_xor_sync(0xffffffffu, l_zero, o);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = l_int, red[1][threadIdx.x >> 5] = l_zero;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += red[0][w], b += red[1][w];
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

template <typename T>
void launch_train_pairs(const T* field, int nx, int ny, int s, const T* coarse, const LevelGeom& g, int predictor,
                        double eb, int step, uint64_t first, uint64_t cap, __nv_bfloat16* X, float* Y,
                        uint64_t* added, cudaStream_t st)
{
    auto cnt = [step](int d) { return d >= 4 ? (d - 4) / step + 1 : 0; };
    const int sx = cnt(g.dx), sy = cnt(g.dy), sz = cnt(g.dz);
    const uint64_t total = (uint64_t)sx * sy * sz;
    *added = first >= cap ? 0 : std::min<uint64_t>(total, cap - first);
    if (!*added) return;
    const int gs = (int)std::min<uint64_t>((total + 255) / 256, 148 * 8);
    if (predictor == 1)
        k_train_pairs<T, 1><<<gs, 256, 0, st>>>(field, (size_t)nx, (size_t)nx * ny, s, coarse, g, 1.0 / eb, step, sx,
                                                 sy, sz, first, cap, X, Y);
    else
        k_train_pairs<T, 0><<<gs, 256, 0, st>>>(field, (size_t)nx, (size_t)nx * ny, s, coarse, g, 1.0 / eb, step, sx,
                                                 sy, sz, first, cap, X, Y);
}

// ---- host helpers ------------------------------------------------------------------
float bf16_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}
uint16_t bf16_bits(float x)
{
    const float r = bf16_host(x);
    uint32_t u;
    std::memcpy(&u, &r, 4);
    return (uint16_t)(u >> 16);
}
float bf16_to_float(uint16_t b)
{
    const uint32_t u = (uint32_t)b << 16;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

double quantile(std::vector<float>& v, double q)
{
    if (v.empty()) return 0.0;
    const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1)));
    std::nth_element(v.begin(), v.begin() + (long)k, v.end());
    return v[k];
}

// Fixed-point multiplier m / 2^sh ~ M with m in [2^14, 2^15) where possible.
void fixed_point(double M, int32_t& m, int32_t& sh)
{
    if (!(M > 0) || !std::isfinite(M)) {
        m = 0, sh = 1;
        return;
    }
    int s = 14 - (int)std::floor(std::log2(M));
    s = std::max(1, std::min(62, s));
    const double mm = std::nearbyint(std::ldexp(M, s));
    m = (int32_t)std::min(mm, 2147483647.0);
    sh = s;
}

int32_t sat32(double v)
{
    v = std::nearbyint(v);
    return (int32_t)std::max(-1073741824.0, std::min(1073741824.0, v));
}

// The int8 record of a QAT-trained float network (weights on the grid the
// last QAT step used).
LearnedModel export_model(const float* W, double s_in, double s_t, double sa1, double sa2)
{
    LearnedModel m{};
    auto tmax = [&](int b, int e) {
        double x = 0;
        for (int p = b; p < e; ++p) x = std::max(x, (double)std::fabs(W[p]));
        return x;
    };
    const double st1 = (double)((float)tmax(kPW1, kPB1) / 127.f), st2 = (double)((float)tmax(kPW2, kPB2) / 127.f),
                 st3 = (double)((float)tmax(kPW3, kPB3) / 127.f);
    auto q = [](float w, double stp) { return stp > 0 ? (int8_t)std::max(-127.0, std::min(127.0, (double)rintf(w / (float)stp))) : (int8_t)0; };
    for (int n = 0; n < 32; ++n)
        for (int k = 0; k < 16; ++k) m.w1[n][k] = k < 14 ? q(W[kPW1 + n * 16 + k], st1) : 0;
    for (int n = 0; n < 32; ++n)
        for (int k = 0; k < 32; ++k) m.w2[n][k] = q(W[kPW2 + n * 32 + k], st2);
    for (int b = 0; b < 8; ++b)
        for (int k = 0; k < 32; ++k) m.w3[b][k] = b < 7 ? q(W[kPW3 + b * 32 + k], st3) : 0;
    const double e1 = st1 > 0 ? st1 / 127.0 : 1.0, e2 = st2 > 0 ? st2 * sa1 : 1.0, e3 = st3 > 0 ? st3 * sa2 : 1.0;
    for (int n = 0; n < 32; ++n) m.b1[n] = sat32(W[kPB1 + n] / e1);
    for (int n = 0; n < 32; ++n) m.b2[n] = sat32(W[kPB2 + n] / e2);
    for (int b = 0; b < 8; ++b) m.b3[b] = b < 7 ? sat32(W[kPB3 + b] / e3) : 0;
    fixed_point(e1 / sa1, m.m1, m.sh1);
    fixed_point(e2 / sa2, m.m2, m.sh2);
    m.s_in = s_in;
    m.s_out = e3 * s_t;
    if (!(m.s_out > 0)) m.s_out = 1e-300;
    return m;
}

}  // namespace
}  // namespace stz

using namespace stz;

struct stz_trainer {
    stz_context* ctx = nullptr;
    stz_opts o{};
    stz_train_opts t{};
    struct Slot {
        DevBuf X, Y;
        uint64_t n = 0;
    } lv[2];
    DevBuf grid[2], codes, unpred, ucnt, hist, hist_out, state, part, perm, calib, lossbuf, model;
    stz_train_stats stats{};
};

namespace {

// One phase (float or QAT) of one level: `epochs` passes over the pairs.
stz_status run_phase(stz_trainer* tr, int slot, int epochs, int qat, float lr, float lr_min, float inv_s_in,
                     float inv_s_t, float delta, float sa1, float sa2, double* loss_last)
{
    stz_context* ctx = tr->ctx;
    cudaStream_t st = ctx->st;
    const uint64_t n = tr->lv[slot].n;
    const uint32_t batch = (uint32_t)tr->t.batch;
    const uint32_t spe = (uint32_t)((n + batch - 1) / batch);
    const uint32_t total = spe * (uint32_t)epochs;
    const int ctas = (int)(batch / kTile);
    // per-epoch affine shuffles
    std::mt19937_64 rng(tr->t.seed * 0x9E3779B97F4A7C15ull + (uint64_t)slot * 131 + (uint64_t)qat * 7);
    std::vector<uint64_t> perm(2 * (size_t)epochs);
    for (int e = 0; e < epochs; ++e) {
        uint64_t a = 1;
        if (n > 2)
            do a = 1 + rng() % (n - 1);
            while (std::gcd(a, n) != 1);
        perm[2 * e] = a;
        perm[2 * e + 1] = n ? rng() % n : 0;
    }
    STZ_CUDA(tr->perm.ensure(perm.size() * 8));
    STZ_CUDA(cudaMemcpyAsync(tr->perm.p, perm.data(), perm.size() * 8, cudaMemcpyHostToDevice, st));
    STZ_CUDA(tr->part.ensure((size_t)ctas * (kNP + 1) * 4));
    STZ_CUDA(tr->lossbuf.ensure(2 * kMaxEpochs * 8));
    STZ_CUDA(cudaMemsetAsync(tr->lossbuf.p, 0, 2 * kMaxEpochs * 8, st));
    float* S = tr->state.as<float>();
    float *W = S, *m = S + kNP, *v = S + 2 * kNP, *Wf = S + 3 * kNP;
    uint32_t* counter = reinterpret_cast<uint32_t*>(S + 4 * kNP);
    STZ_CUDA(cudaMemsetAsync(m, 0, 2 * kNP * 4, st));  // m, v
    STZ_CUDA(cudaMemsetAsync(counter, 0, 4, st));
    k_refresh_forward<<<1, 1024, 0, st>>>(W, Wf, qat);
    StepArgs P{};
    P.X = reinterpret_cast<const __nv_bfloat16*>(tr->lv[slot].X.p);
    P.Y = tr->lv[slot].Y.as<float>();
    P.n = n;
    P.perm = tr->perm.as<uint64_t>();
    P.Wf = Wf;
    P.part = tr->part.as<float>();
    P.counter = counter;
    P.steps_per_epoch = spe, P.total_steps = total, P.batch = batch;
    P.inv_s_in = inv_s_in, P.inv_s_t = inv_s_t, P.delta = delta;
    P.qat = qat, P.sa1 = sa1, P.sa2 = sa2;
    AdamArgs A{};
    A.W = W, A.m = m, A.v = v, A.Wf = Wf, A.part = P.part, A.ctas = ctas, A.counter = counter;
    A.steps_per_epoch = spe, A.total_steps = total, A.batch = batch, A.n = n;
    A.lr = lr, A.lr_min = lr_min, A.qat = qat;
    A.loss = tr->lossbuf.as<double>();
    STZ_CUDA(cudaFuncSetAttribute(k_mlp_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStepSmem));
    // one graph of G step pairs, replayed until the counter reaches `total`
    const uint32_t G = std::min<uint32_t>(total, 64);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    STZ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (uint32_t i = 0; i < G; ++i) {
        k_mlp_step<<<ctas, kStepThreads, kStepSmem, st>>>(P);
        k_adam<<<1, 1024, 0, st>>>(A);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        STZ_CUDA(ce);
    }
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    STZ_CUDA(ie);
    const uint32_t replays = (total + G - 1) / G;
    cudaError_t le = cudaSuccess;
    for (uint32_t r = 0; r < replays && le == cudaSuccess; ++r) le = cudaGraphLaunch(exec, st);
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    STZ_CUDA(le);
    STZ_CUDA(se);
    std::vector<double> L(2 * (size_t)epochs);
    STZ_CUDA(cudaMemcpy(L.data(), tr->lossbuf.p, L.size() * 8, cudaMemcpyDeviceToHost));
    const int e = epochs - 1;
    *loss_last = L[2 * e + 1] > 0 ? L[2 * e] / L[2 * e + 1] : 0.0;
    return STZ_OK;
}

template <typename T>
stz_status add_field(stz_trainer* tr, const T* field, int nx, int ny, int nz)
{
    stz_context* ctx = tr->ctx;
    cudaStream_t st = ctx->st;
    const stz_opts& o = tr->o;
    const Geometry g = make_geometry(nx, ny, nz, o.chunk_high, o.chunk_low, o.radius);
    const int K = g.K;
    if (K < 2) STZ_FAIL(STZ_ERR_DIMS, "training needs at least two refinement levels");
    double eb = 0;
    std::vector<double> ebk;
    STZ_TRY(level_error_bounds<T>(ctx, field, (size_t)nx * ny * nz, o, K, eb, ebk));
    const size_t elem = sizeof(T);
    STZ_CUDA(tr->grid[0].ensure(g.n_fine_max * elem));
    STZ_CUDA(tr->grid[1].ensure(g.n_fine_max * elem));
    size_t nmax = 0, cmax = 0;
    for (int k = 1; k < K; ++k) nmax = std::max(nmax, g.lv[k].n), cmax = std::max<size_t>(cmax, g.lv[k].nchunks());
    STZ_CUDA(tr->codes.ensure(7 * nmax * 2));
    STZ_CUDA(tr->unpred.ensure(7 * nmax * elem));
    STZ_CUDA(tr->ucnt.ensure(7 * (cmax + 1) * 4));
    STZ_CUDA(tr->hist.ensure(7 * 2 * (size_t)o.radius * 4));
    STZ_CUDA(tr->hist_out.ensure(7 * 4));
    const uint64_t cap = tr->t.max_pairs;
    for (int i = 0; i < 2; ++i) {
        STZ_CUDA(tr->lv[i].X.ensure(cap * 16 * 2));
        STZ_CUDA(tr->lv[i].Y.ensure(cap * 8 * 4));
    }
    int cur = 0;
    launch_subsample<T>(field, nx, ny, nz, 1 << K, tr->grid[cur].as<T>(), st);
    for (int k = 1; k <= K; ++k) {
        const T* coarse = tr->grid[cur].as<T>();
        if (k >= K - 1) {
            auto& S = tr->lv[k - (K - 1)];
            uint64_t added = 0;
            launch_train_pairs<T>(field, nx, ny, 1 << (K - k), coarse, g.lv[k], o.predictor, ebk[k],
                                  tr->t.sample_step, S.n, cap, reinterpret_cast<__nv_bfloat16*>(S.X.p),
                                  S.Y.as<float>(), &added, st);
            S.n += added;
        }
        if (k == K) break;
        const LevelGeom& L = g.lv[k];
        STZ_CUDA(cudaMemsetAsync(tr->hist.p, 0, 7 * 2 * (size_t)o.radius * 4, st));
        STZ_CUDA(cudaMemsetAsync(tr->hist_out.p, 0, 7 * 4, st));
        STZ_CUDA(cudaMemsetAsync(tr->ucnt.p, 0, 7 * ((size_t)L.nchunks() + 1) * 4, st));
        LevelEncodeArgs<T> a;
        a.field = field;
        a.fsx = (size_t)nx;
        a.fsy = (size_t)nx * ny;
        a.stride = 1 << (K - k);
        a.coarse = coarse;
        a.geo = L;
        a.predictor = o.predictor;
        // streams of this level laid out as in the compressor (per block n codes, nchunks + 1 counters)
        a.codes = tr->codes.as<uint16_t>();
        a.unpred_dense = tr->unpred.as<T>();
        a.unpred_cnt = tr->ucnt.as<uint32_t>();
        a.hist_full = tr->hist.as<uint32_t>();
        a.hist_outside = tr->hist_out.as<uint32_t>();
        a.decoded = tr->grid[1 - cur].as<T>();
        a.qp = make_quant_params(ebk[k], o.radius);
        launch_level_encode<T>(a, st);
        cur = 1 - cur;
    }
    STZ_CUDA(cudaGetLastError());
    STZ_CUDA(cudaStreamSynchronize(st));
    return STZ_OK;
}

stz_status fit_level(stz_trainer* tr, int slot, LearnedModel& out)
{
    stz_context* ctx = tr->ctx;
    cudaStream_t st = ctx->st;
    const uint64_t n = tr->lv[slot].n;
    const stz_train_opts& T = tr->t;
    // scales: inputs from the stored features, targets from the stored residuals
    const uint64_t nc = std::min<uint64_t>(n, kCalib);
    std::vector<uint16_t> xb(nc * 16);
    std::vector<float> yb(nc * 8);
    STZ_CUDA(cudaMemcpy(xb.data(), tr->lv[slot].X.p, xb.size() * 2, cudaMemcpyDeviceToHost));
    STZ_CUDA(cudaMemcpy(yb.data(), tr->lv[slot].Y.p, yb.size() * 4, cudaMemcpyDeviceToHost));
    std::vector<float> ax, at;
    ax.reserve(nc * 14);
    at.reserve(nc * 7);
    for (uint64_t s = 0; s < nc; ++s) {
        for (int k = 0; k < 14; ++k) ax.push_back(std::fabs(bf16_to_float(xb[s * 16 + k])));
        for (int b = 0; b < 7; ++b) at.push_back(std::fabs(yb[s * 8 + b]));
    }
    double s_in = quantile(ax, 0.999) / 127.0;
    if (!(s_in > 0) || !std::isfinite(s_in)) s_in = 1.0 / 127.0;
    const double tclip = quantile(at, 0.999);
    double ss = 0;
    for (float v : at) ss += std::min<double>(v, tclip) * std::min<double>(v, tclip);
    double s_t = std::sqrt(ss / std::max<size_t>(1, at.size()));
    if (!(s_t > 0.25) || !std::isfinite(s_t)) s_t = std::max(0.25, std::isfinite(s_t) ? s_t : 0.25);
    tr->stats.s_in[slot] = s_in;
    tr->stats.s_t[slot] = s_t;
    // initial weights: uniform(+-sqrt(6 / fan_in)) hidden layers, zero output layer
    std::vector<float> W(kNP, 0.f);
    std::mt19937_64 rng(T.seed * 0x2545F4914F6CDD1Dull + (uint64_t)slot);
    std::uniform_real_distribution<float> u1(-std::sqrt(6.f / 14.f), std::sqrt(6.f / 14.f));
    std::uniform_real_distribution<float> u2(-std::sqrt(6.f / 32.f), std::sqrt(6.f / 32.f));
    for (int nn = 0; nn < 32; ++nn)
        for (int k = 0; k < 14; ++k) W[kPW1 + nn * 16 + k] = u1(rng);
    for (int p = kPW2; p < kPB2; ++p) W[p] = u2(rng);
    for (int nn = 0; nn < 32; ++nn) W[kPB1 + nn] = 0.01f, W[kPB2 + nn] = 0.01f;
    STZ_CUDA(tr->state.ensure(4 * kNP * 4 + 16));
    STZ_CUDA(cudaMemcpyAsync(tr->state.p, W.data(), kNP * 4, cudaMemcpyHostToDevice, st));
    const float inv_s_in = (float)(1.0 / s_in), inv_s_t = (float)(1.0 / s_t);
    const float delta = (float)(T.huber_delta / s_t);
    double lf = 0, lq = 0;
    STZ_TRY(run_phase(tr, slot, T.epochs, 0, (float)T.lr, (float)T.lr * 0.1f, inv_s_in, inv_s_t, delta, 1.f, 1.f, &lf));
    tr->stats.loss_float[slot] = lf * s_t * s_t;
    // activation scales from the float network
    float* S = tr->state.as<float>();
    STZ_CUDA(tr->calib.ensure(nc * 64 * 4));
    k_mlp_calib<<<(unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nc + 255) / 256, 148 * 4)), 256, 0, st>>>(
        reinterpret_cast<const __nv_bfloat16*>(tr->lv[slot].X.p), nc, S + 3 * kNP, inv_s_in, tr->calib.as<float>());
    STZ_CUDA(cudaGetLastError());
    std::vector<float> H(nc * 64);
    STZ_CUDA(cudaMemcpyAsync(H.data(), tr->calib.p, H.size() * 4, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaStreamSynchronize(st));
    std::vector<float> a1, a2;
    for (uint64_t s = 0; s < nc; ++s)
        for (int k = 0; k < 32; ++k) {
            if (H[s * 64 + k] > 0) a1.push_back(H[s * 64 + k]);
            if (H[s * 64 + 32 + k] > 0) a2.push_back(H[s * 64 + 32 + k]);
        }
    double sa1 = quantile(a1, 0.999) / 127.0, sa2 = quantile(a2, 0.999) / 127.0;
    if (!(sa1 > 0)) sa1 = 1.0 / 127.0;
    if (!(sa2 > 0)) sa2 = 1.0 / 127.0;
    if (T.qat_epochs > 0) {
        STZ_TRY(run_phase(tr, slot, T.qat_epochs, 1, (float)T.lr / 8.f, (float)T.lr / 80.f, inv_s_in, inv_s_t, delta,
                          (float)sa1, (float)sa2, &lq));
        tr->stats.loss_qat[slot] = lq * s_t * s_t;
    }
    std::vector<float> Wm(kNP);
    STZ_CUDA(cudaMemcpy(Wm.data(), tr->state.p, kNP * 4, cudaMemcpyDeviceToHost));
    out = export_model(Wm.data(), s_in, s_t, sa1, sa2);
    // the exported network on every pair, and the plain prediction
    STZ_CUDA(tr->model.ensure(sizeof(LearnedModel)));
    STZ_CUDA(cudaMemcpyAsync(tr->model.p, &out, sizeof(LearnedModel), cudaMemcpyHostToDevice, st));
    const int gb = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 4));
    STZ_CUDA(tr->calib.ensure((size_t)gb * 16));
    k_int8_loss<<<gb, 256, 0, st>>>(reinterpret_cast<const __nv_bfloat16*>(tr->lv[slot].X.p), tr->lv[slot].Y.as<float>(),
                                    n, tr->model.as<LearnedModel>(), T.huber_delta, tr->calib.as<double>());
    STZ_CUDA(cudaGetLastError());
    std::vector<double> pl(2 * (size_t)gb);
    STZ_CUDA(cudaMemcpyAsync(pl.data(), tr->calib.p, pl.size() * 8, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaStreamSynchronize(st));
    double li = 0, lz = 0;
    for (int b = 0; b < gb; ++b) li += pl[2 * b], lz += pl[2 * b + 1];
    tr->stats.loss_int8[slot] = li / (double)(n * 7);
    tr->stats.loss_zero[slot] = lz / (double)(n * 7);
    return STZ_OK;
}

}  // namespace

extern "C" {

void stz_default_train_opts(stz_train_opts* t)
{
    if (!t) return;
    t->epochs = 8;
    t->qat_epochs = 3;
    t->batch = 4096;
    t->lr = 2e-3;
    t->huber_delta = 2.0;
    t->sample_step = 2;
    t->max_pairs = (size_t)1 << 23;
    t->seed = 1;
}

stz_status stz_trainer_create(stz_context* ctx, const stz_opts* opts, const stz_train_opts* topts, stz_trainer** out)
{
    if (!ctx || !opts || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *out = nullptr;
    STZ_TRY(check_opts(opts));
    if (opts->predictor >= STZ_PRED_STAGED)
        STZ_FAIL(STZ_ERR_UNSUPPORTED, "no learned correction for the staged and truncated predictors");
    stz_train_opts t;
    stz_default_train_opts(&t);
    if (topts) t = *topts;
    if (t.epochs < 1 || t.epochs > kMaxEpochs || t.qat_epochs < 0 || t.qat_epochs > kMaxEpochs)
        STZ_FAIL(STZ_ERR_ARG, "epochs must be in [1, 256] and qat_epochs in [0, 256]");
    if (t.batch < kTile || t.batch % kTile || t.batch > kTile * 148 * 8)
        STZ_FAIL(STZ_ERR_ARG, "batch must be a positive multiple of 128, at most 151552");
    if (!(t.lr > 0) || !std::isfinite(t.lr) || !(t.huber_delta > 0) || !std::isfinite(t.huber_delta))
        STZ_FAIL(STZ_ERR_ARG, "lr and huber_delta must be positive");
    if (t.sample_step < 1 || t.sample_step > 64) STZ_FAIL(STZ_ERR_ARG, "sample_step must be in [1, 64]");
    if (t.max_pairs < 1 || t.max_pairs > ((size_t)1 << 31)) STZ_FAIL(STZ_ERR_ARG, "max_pairs must be in [1, 2^31]");
    auto* tr = new (std::nothrow) stz_trainer();
    if (!tr) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    tr->ctx = ctx;
    tr->o = *opts;
    tr->o.model = nullptr;
    tr->t = t;
    *out = tr;
    return STZ_OK;
}

stz_status stz_trainer_add_field_dev(stz_trainer* t, const void* field_dev, stz_dtype dtype, size_t nx, size_t ny,
                                     size_t nz)
{
    if (!t || !field_dev) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    STZ_TRY(enter(t->ctx));
    const std::string dm = validate_dims((long long)nx, (long long)ny, (long long)nz, t->o.chunk_high, t->o.chunk_low);
    if (!dm.empty()) STZ_FAIL(STZ_ERR_DIMS, dm);
    if (dtype == STZ_F64) return add_field<double>(t, (const double*)field_dev, (int)nx, (int)ny, (int)nz);
    if (dtype == STZ_F32) return add_field<float>(t, (const float*)field_dev, (int)nx, (int)ny, (int)nz);
    STZ_FAIL(STZ_ERR_ARG, "bad dtype");
}

stz_status stz_trainer_fit(stz_trainer* t, stz_model** out)
{
    if (!t || !out) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *out = nullptr;
    STZ_TRY(enter(t->ctx));
    if (!t->lv[0].n && !t->lv[1].n) STZ_FAIL(STZ_ERR_ARG, "no training pairs: add fields first");
    auto* m = new (std::nothrow) stz_model();
    if (!m) STZ_FAIL(STZ_ERR_NOMEM, "out of host memory");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, t->ctx->st);
    for (int i = 0; i < 2; ++i) {
        t->stats.pairs[i] = t->lv[i].n;
        if (t->lv[i].n < kTile) continue;
        const stz_status s = fit_level(t, i, m->lv[i]);
        if (s != STZ_OK) {
            delete m;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return s;
        }
        m->mask |= 1u << i;
    }
    cudaEventRecord(e1, t->ctx->st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    t->stats.train_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!m->mask) {
        delete m;
        STZ_FAIL(STZ_ERR_ARG, "too few training pairs");
    }
    for (int i = 0; i < 2; ++i)
        if ((m->mask >> i & 1u) && !learned_model_valid(m->lv[i])) {
            delete m;
            STZ_FAIL(STZ_ERR_ARG, "training produced an unusable model (degenerate scales)");
        }
    m->serialize();
    *out = m;
    return STZ_OK;
}

stz_status stz_trainer_stats(const stz_trainer* t, stz_train_stats* st)
{
    if (!t || !st) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    *st = t->stats;
    st->pairs[0] = t->lv[0].n;
    st->pairs[1] = t->lv[1].n;
    return STZ_OK;
}

void stz_trainer_free(stz_trainer* t) { delete t; }

stz_status stz_debug_mlp_grad(stz_context* ctx, const float* params, const float* x, const float* t, size_t n,
                              double s_in, double s_t, double huber_delta, int qat, const double sa[2], float* grad,
                              double* loss)
{
    if (!ctx || !params || !x || !t || !grad || !loss || (qat && !sa)) STZ_FAIL(STZ_ERR_ARG, "null pointer");
    if (n == 0 || n > (size_t)kTile * 148 * 8) STZ_FAIL(STZ_ERR_ARG, "n must be in [1, 151552]");
    if (!(s_in > 0) || !(s_t > 0) || !(huber_delta > 0)) STZ_FAIL(STZ_ERR_ARG, "scales must be positive");
    STZ_TRY(enter(ctx));
    cudaStream_t st = ctx->st;
    const int ctas = (int)((n + kTile - 1) / kTile);
    std::vector<uint16_t> xb(n * 16);
    for (size_t i = 0; i < n * 16; ++i) xb[i] = bf16_bits(x[i]);
    DevBuf dx, dy, ds, dp, dperm;
    STZ_CUDA(dx.ensure(n * 32));
    STZ_CUDA(dy.ensure(n * 32));
    STZ_CUDA(ds.ensure(4 * kNP * 4 + 16));
    STZ_CUDA(dp.ensure((size_t)ctas * (kNP + 1) * 4));
    STZ_CUDA(dperm.ensure(16));
    const uint64_t perm[2] = {1, 0};
    STZ_CUDA(cudaMemcpyAsync(dx.p, xb.data(), n * 32, cudaMemcpyHostToDevice, st));
    STZ_CUDA(cudaMemcpyAsync(dy.p, t, n * 32, cudaMemcpyHostToDevice, st));
    STZ_CUDA(cudaMemcpyAsync(ds.p, params, kNP * 4, cudaMemcpyHostToDevice, st));
    STZ_CUDA(cudaMemcpyAsync(dperm.p, perm, 16, cudaMemcpyHostToDevice, st));
    float* S = ds.as<float>();
    uint32_t* counter = reinterpret_cast<uint32_t*>(S + 4 * kNP);
    STZ_CUDA(cudaMemsetAsync(counter, 0, 4, st));
    k_refresh_forward<<<1, 1024, 0, st>>>(S, S + 3 * kNP, qat);
    StepArgs P{};
    P.X = reinterpret_cast<const __nv_bfloat16*>(dx.p);
    P.Y = dy.as<float>();
    P.n = n;
    P.perm = dperm.as<uint64_t>();
    P.Wf = S + 3 * kNP;
    P.part = dp.as<float>();
    P.counter = counter;
    P.steps_per_epoch = 1, P.total_steps = 1, P.batch = (uint32_t)(ctas * kTile);
    P.inv_s_in = (float)(1.0 / s_in), P.inv_s_t = (float)(1.0 / s_t), P.delta = (float)(huber_delta / s_t);
    P.qat = qat;
    P.sa1 = qat ? (float)sa[0] : 1.f, P.sa2 = qat ? (float)sa[1] : 1.f;
    STZ_CUDA(cudaFuncSetAttribute(k_mlp_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStepSmem));
    k_mlp_step<<<ctas, kStepThreads, kStepSmem, st>>>(P);
    STZ_CUDA(cudaGetLastError());
    std::vector<float> part((size_t)ctas * (kNP + 1));
    STZ_CUDA(cudaMemcpyAsync(part.data(), dp.p, part.size() * 4, cudaMemcpyDeviceToHost, st));
    STZ_CUDA(cudaStreamSynchronize(st));
    double l = 0;
    for (int p = 0; p < kNP; ++p) {
        float g = 0.f;
        for (int c = 0; c < ctas; ++c) g += part[(size_t)c * (kNP + 1) + p];
        grad[p] = g;
    }
    for (int c = 0; c < ctas; ++c) l += part[(size_t)c * (kNP + 1) + kNP];
    *loss = l / (double)(n * 7);
    return STZ_OK;
}

}  // extern "C"
