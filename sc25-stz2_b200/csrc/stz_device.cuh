// Device-side arithmetic of the STZ hot path: the level predictors and the
// linear quantizer, evaluated with the reference's operation order.
//
// Bit-exactness with the reference CPU build (g++ -O3, SSE2 scalar float/double,
// no FMA contraction, FTZ+DAZ enabled in main, FD5:3046-3047) is obtained by
// issuing every floating-point operation as explicit round-to-nearest PTX:
// f32 ops carry .ftz (flush subnormal inputs and results, as FTZ/DAZ do on the
// host), and nothing can be contracted into an FMA or reassociated.
//
// Predictors read the coarse grid through an accessor `a(off)` relative to the
// predicted point, with row / plane strides a.sx / a.sy: SmemTile has
// compile-time strides (every tap is one shared-memory load with an immediate
// offset), GlobalGrid runtime strides.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

template <typename T>
struct Ar;

template <>
struct Ar<float> {
    static __device__ __forceinline__ float add(float a, float b)
    {
        float r;
        asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    static __device__ __forceinline__ float sub(float a, float b)
    {
        float r;
        asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    static __device__ __forceinline__ float mul(float a, float b)
    {
        float r;
        asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    static __device__ __forceinline__ float div(float a, float b)
    {
        float r;
        asm("div.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    // (double)x on the host with DAZ set: subnormal inputs read as zero.
    static __device__ __forceinline__ double to_f64(float a)
    {
        double r;
        asm("cvt.ftz.f64.f32 %0, %1;" : "=d"(r) : "f"(a));
        return r;
    }
    // (float)x on the host: round to nearest, then FTZ.
    static __device__ __forceinline__ float from_f64(double a)
    {
        float r;
        asm("cvt.rn.ftz.f32.f64 %0, %1;" : "=f"(r) : "d"(a));
        return r;
    }
    // Exact sign flip (the host negates with a sign-mask xor, no flush).
    static __device__ __forceinline__ float neg(float a) { return __int_as_float(__float_as_int(a) ^ 0x80000000); }
    static __device__ __forceinline__ bool is_neg(float a)
    {
        unsigned r;
        asm("{ .reg .pred p; setp.lt.ftz.f32 p, %1, 0f00000000; selp.u32 %0, 1, 0, p; }" : "=r"(r) : "f"(a));
        return r != 0;
    }
};

template <>
struct Ar<double> {
    static __device__ __forceinline__ double add(double a, double b)
    {
        double r;
        asm("add.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
        return r;
    }
    static __device__ __forceinline__ double sub(double a, double b)
    {
        double r;
        asm("sub.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
        return r;
    }
    static __device__ __forceinline__ double mul(double a, double b)
    {
        double r;
        asm("mul.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
        return r;
    }
    static __device__ __forceinline__ double div(double a, double b)
    {
        double r;
        asm("div.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
        return r;
    }
    static __device__ __forceinline__ double to_f64(double a) { return a; }
    static __device__ __forceinline__ double from_f64(double a) { return a; }
    static __device__ __forceinline__ double neg(double a)
    {
        return __longlong_as_double(__double_as_longlong(a) ^ 0x8000000000000000ull);
    }
    static __device__ __forceinline__ bool is_neg(double a) { return a < 0.0; }
};

__device__ __forceinline__ double d_mul(double a, double b)
{
    double r;
    asm("mul.rn.f64 %0, %1, %2;" : "=d"(r) : "d"(a), "d"(b));
    return r;
}

// Strided view of a coarse (decoded) grid in global memory.
template <typename T>
struct Grid {
    const T* __restrict__ p;
    int dx, dy, dz;
    size_t sx, sy;  // row and plane strides (elements)
    __device__ __forceinline__ T at(size_t i) const { return __ldg(p + i); }
};

// Accessor on a global grid, positioned at one point.
template <typename T>
struct GlobalAt {
    const T* __restrict__ p;
    long long sx, sy;
    __device__ __forceinline__ T operator()(long long off) const { return __ldg(p + off); }
};

// Accessor on a shared-memory tile with compile-time strides.
template <typename T, int SX, int SY>
struct TileAt {
    const T* p;
    static constexpr int sx = SX, sy = SY;
    __device__ __forceinline__ T operator()(int off) const { return p[off]; }
};

// cubic_line_pred (FD5:141-146): -(1/16)a + (9/16)b + (9/16)c - (1/16)d.
template <typename T>
__device__ __forceinline__ T cubic(T a, T b, T c, T d)
{
    using A = Ar<T>;
    return A::sub(A::add(A::add(A::mul(T(-0.0625f), a), A::mul(T(0.5625f), b)), A::mul(T(0.5625f), c)),
                  A::mul(T(0.0625f), d));
}

// cubic_line_pv_cse (FD5:163-175): shared second differences.
template <typename T>
__device__ __forceinline__ void line_pv(T a, T b, T c, T d, T& p, T& v)
{
    using A = Ar<T>;
    const T eps = T(1e-12f);
    const T c0 = A::add(A::sub(a, A::mul(T(2.0f), b)), c);
    const T c1 = A::add(A::sub(b, A::mul(T(2.0f), c)), d);
    v = A::add(A::mul(T(0.5f), A::add(A::mul(c0, c0), A::mul(c1, c1))), eps);
    p = A::sub(A::mul(T(0.5f), A::add(b, c)), A::mul(T(0.0625f), A::add(c0, c1)));
}

// blend2 (FD5:178-186).
template <typename T>
__device__ __forceinline__ T blend2(T p0, T v0, T p1, T v1)
{
    using A = Ar<T>;
    return A::div(A::add(A::mul(p0, v1), A::mul(p1, v0)), A::add(v0, v1));
}

// blend4 (FD5:188-203).
template <typename T>
__device__ __forceinline__ T blend4(T p0, T v0, T p1, T v1, T p2, T v2, T p3, T v3)
{
    using A = Ar<T>;
    const T w0 = A::mul(A::mul(v1, v2), v3);
    const T w1 = A::mul(A::mul(v0, v2), v3);
    const T w2 = A::mul(A::mul(v0, v1), v3);
    const T w3 = A::mul(A::mul(v0, v1), v2);
    const T num = A::add(A::add(A::add(A::mul(w0, p0), A::mul(w1, p1)), A::mul(w2, p2)), A::mul(w3, p3));
    const T den = A::add(A::add(A::add(w0, w1), w2), w3);
    return A::div(num, den);
}

// Interior form of the FD5 "dynamic lines" predictor (predict_interior_const,
// FD5:828-840, with predict_dynamic_lines_const FD5:624-688). BLOCK = sub_index-1.
template <int BLOCK, typename T, class Acc>
__device__ __forceinline__ T dynamic_interior(const Acc& r)
{
    const auto sx = r.sx, sy = r.sy;
    T p0, v0, p1, v1, p2, v2, p3, v3;
    if constexpr (BLOCK == 0) {
        return cubic(r(-1), r(0), r(1), r(2));
    } else if constexpr (BLOCK == 1) {
        return cubic(r(-sx), r(0), r(sx), r(2 * sx));
    } else if constexpr (BLOCK == 3) {
        return cubic(r(-sy), r(0), r(sy), r(2 * sy));
    } else if constexpr (BLOCK == 2) {
        line_pv(r(-sx - 1), r(0), r(sx + 1), r(2 * sx + 2), p0, v0);
        line_pv(r(-sx + 2), r(1), r(sx), r(2 * sx - 1), p1, v1);
        return blend2(p0, v0, p1, v1);
    } else if constexpr (BLOCK == 4) {
        line_pv(r(-sy - 1), r(0), r(sy + 1), r(2 * sy + 2), p0, v0);
        line_pv(r(-sy + 2), r(1), r(sy), r(2 * sy - 1), p1, v1);
        return blend2(p0, v0, p1, v1);
    } else if constexpr (BLOCK == 5) {
        line_pv(r(-sy - sx), r(0), r(sy + sx), r(2 * sy + 2 * sx), p0, v0);
        line_pv(r(-sy + 2 * sx), r(sx), r(sy), r(2 * sy - sx), p1, v1);
        return blend2(p0, v0, p1, v1);
    } else {
        line_pv(r(-sy - sx - 1), r(0), r(sy + sx + 1), r(2 * sy + 2 * sx + 2), p0, v0);
        line_pv(r(-sy - sx + 2), r(1), r(sy + sx), r(2 * sy + 2 * sx - 1), p1, v1);
        line_pv(r(-sy + 2 * sx - 1), r(sx), r(sy + 1), r(2 * sy - sx + 2), p2, v2);
        line_pv(r(2 * sy - sx - 1), r(sy), r(sx + 1), r(-sy + 2 * sx + 2), p3, v3);
        return blend4(p0, v0, p1, v1, p2, v2, p3, v3);
    }
}

// Full FD5 predictor with its boundary rules (predict_block_const,
// FD5:690-748): last index copies the reference, index 0 / dim-2 average the
// 2 / 4 / 8 forward neighbours, the rest is the interior form.
template <int BLOCK, typename T, class Acc>
__device__ __forceinline__ T dynamic_block(const Acc& r, int x, int y, int z, int dx, int dy, int dz)
{
    using A = Ar<T>;
    const auto sx = r.sx, sy = r.sy;
    if constexpr (BLOCK == 0) {
        if (x == dx - 1) return r(0);
        if (x == dx - 2 || x == 0) return A::mul(T(0.5f), A::add(r(0), r(1)));
    } else if constexpr (BLOCK == 1) {
        if (y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0) return A::mul(T(0.5f), A::add(r(0), r(sx)));
    } else if constexpr (BLOCK == 3) {
        if (z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0) return A::mul(T(0.5f), A::add(r(0), r(sy)));
    } else if constexpr (BLOCK == 2) {
        if (x == dx - 1 || y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(r(0), r(sx + 1)), r(sx)), r(1)));
    } else if constexpr (BLOCK == 4) {
        if (x == dx - 1 || z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(r(0), r(sy + 1)), r(1)), r(sy)));
    } else if constexpr (BLOCK == 5) {
        if (z == dz - 1 || y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(r(0), r(sy + sx)), r(sy)), r(sx)));
    } else {
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(r(0), r(sy + sx + 1));
            s = A::add(s, r(sy + sx));
            s = A::add(s, r(sy + 1));
            s = A::add(s, r(sx + 1));
            s = A::add(s, r(1));
            s = A::add(s, r(sx));
            s = A::add(s, r(sy));
            return A::mul(T(0.125f), s);
        }
    }
    return dynamic_interior<BLOCK, T>(r);
}

// Sum of w*tap over four taps, then minus v*tap for four more: the fixed
// stencil expressions of src/float.cpp keep that order.
template <typename T, class Acc, class O>
__device__ __forceinline__ T plain2(const Acc& r, T wp, O a0, O a1, O a2, O a3, T wn, O b0, O b1, O b2, O b3)
{
    using A = Ar<T>;
    T s = A::add(A::mul(wp, r(a0)), A::mul(wp, r(a1)));
    s = A::add(s, A::mul(wp, r(a2)));
    s = A::add(s, A::mul(wp, r(a3)));
    s = A::sub(s, A::mul(wn, r(b0)));
    s = A::sub(s, A::mul(wn, r(b1)));
    s = A::sub(s, A::mul(wn, r(b2)));
    s = A::sub(s, A::mul(wn, r(b3)));
    return s;
}

// Plain tricubic-family predictor of src/float.cpp:84-273 (templated copy in
// src/stz-rd.cpp): fixed weights, boundary averages as sums of scaled taps.
template <int BLOCK, typename T, class Acc>
__device__ __forceinline__ T plain_block(const Acc& r, int x, int y, int z, int dx, int dy, int dz)
{
    using A = Ar<T>;
    const auto sx = r.sx, sy = r.sy;
    using O = decltype(sx + 0);
    if constexpr (BLOCK == 0) {
        if (x == dx - 1) return r(0);
        if (x == dx - 2 || x == 0) return A::add(A::mul(T(0.5f), r(0)), A::mul(T(0.5f), r(1)));
        return cubic(r(-1), r(0), r(1), r(2));
    } else if constexpr (BLOCK == 1) {
        if (y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0) return A::add(A::mul(T(0.5f), r(0)), A::mul(T(0.5f), r(sx)));
        return cubic(r(-sx), r(0), r(sx), r(2 * sx));
    } else if constexpr (BLOCK == 3) {
        if (z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0) return A::add(A::mul(T(0.5f), r(0)), A::mul(T(0.5f), r(sy)));
        return cubic(r(-sy), r(0), r(sy), r(2 * sy));
    } else if constexpr (BLOCK == 2) {
        if (x == dx - 1 || y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.25f), r(0)), A::mul(T(0.25f), r(sx + 1)));
            s = A::add(s, A::mul(T(0.25f), r(sx)));
            return A::add(s, A::mul(T(0.25f), r(1)));
        }
        return plain2<T>(r, T(0.28125f), O(0), O(sx + 1), O(sx), O(1), T(0.03125f), O(-sx - 1), O(2 * sx + 2),
                         O(2 * sx - 1), O(-sx + 2));
    } else if constexpr (BLOCK == 4) {
        if (x == dx - 1 || z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.25f), r(0)), A::mul(T(0.25f), r(sy + 1)));
            s = A::add(s, A::mul(T(0.25f), r(1)));
            return A::add(s, A::mul(T(0.25f), r(sy)));
        }
        return plain2<T>(r, T(0.28125f), O(0), O(sy + 1), O(1), O(sy), T(0.03125f), O(-sy - 1), O(2 - sy),
                         O(2 * sy - 1), O(2 * sy + 2));
    } else if constexpr (BLOCK == 5) {
        if (z == dz - 1 || y == dy - 1) return r(0);
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0) {
            T s = A::add(A::mul(T(0.25f), r(0)), A::mul(T(0.25f), r(sy + sx)));
            s = A::add(s, A::mul(T(0.25f), r(sy)));
            return A::add(s, A::mul(T(0.25f), r(sx)));
        }
        return plain2<T>(r, T(0.28125f), O(0), O(sy + sx), O(sy), O(sx), T(0.03125f), O(-sy - sx), O(2 * sy + 2 * sx),
                         O(2 * sy - sx), O(2 * sx - sy));
    } else {
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return r(0);
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.125f), r(0)), A::mul(T(0.125f), r(sy + sx + 1)));
            s = A::add(s, A::mul(T(0.125f), r(sy + sx)));
            s = A::add(s, A::mul(T(0.125f), r(sy + 1)));
            s = A::add(s, A::mul(T(0.125f), r(sx + 1)));
            s = A::add(s, A::mul(T(0.125f), r(1)));
            s = A::add(s, A::mul(T(0.125f), r(sx)));
            return A::add(s, A::mul(T(0.125f), r(sy)));
        }
        T s = A::add(A::mul(T(0.140625f), r(0)), A::mul(T(0.140625f), r(sy + sx + 1)));
        s = A::add(s, A::mul(T(0.140625f), r(sy + sx)));
        s = A::add(s, A::mul(T(0.140625f), r(sy + 1)));
        s = A::add(s, A::mul(T(0.140625f), r(sx + 1)));
        s = A::add(s, A::mul(T(0.140625f), r(1)));
        s = A::add(s, A::mul(T(0.140625f), r(sx)));
        s = A::add(s, A::mul(T(0.140625f), r(sy)));
        s = A::sub(s, A::mul(T(0.015625f), r(-sy - sx - 1)));
        s = A::sub(s, A::mul(T(0.015625f), r(2 * sy + 2 * sx + 2)));
        s = A::sub(s, A::mul(T(0.015625f), r(2 * sy - sx + 2)));
        s = A::sub(s, A::mul(T(0.015625f), r(2 * sy + 2 * sx - 1)));
        s = A::sub(s, A::mul(T(0.015625f), r(-sy + 2 * sx + 2)));
        s = A::sub(s, A::mul(T(0.015625f), r(2 * sy - sx - 1)));
        s = A::sub(s, A::mul(T(0.015625f), r(-sy + 2 * sx - 1)));
        return A::sub(s, A::mul(T(0.015625f), r(-sy - sx + 2)));
    }
}

// Predictor dispatch: PRED 0 = FD5 dynamic lines, 1 = plain tricubic.
template <int PRED, int BLOCK, typename T, class Acc>
__device__ __forceinline__ T predict_at(const Acc& r, int x, int y, int z, int dx, int dy, int dz)
{
    if constexpr (PRED == 1) return plain_block<BLOCK, T>(r, x, y, z, dx, dy, dz);
    else return dynamic_block<BLOCK, T>(r, x, y, z, dx, dy, dz);
}

// Interior-only form (caller guarantees 1 <= x,y,z <= dim-3 on every axis).
template <int PRED, int BLOCK, typename T, class Acc>
__device__ __forceinline__ T predict_interior_at(const Acc& r)
{
    if constexpr (PRED == 1) return plain_block<BLOCK, T>(r, 1, 1, 1, 1 << 30, 1 << 30, 1 << 30);
    else return dynamic_interior<BLOCK, T>(r);
}

// The 7 interior predictions of one coarse point (1 <= x,y,z <= dim-3).
template <int PRED, typename T, class Acc>
__device__ __forceinline__ void predict7_interior_only(const Acc& r, T (&p)[7])
{
    p[0] = predict_interior_at<PRED, 0, T>(r);
    p[1] = predict_interior_at<PRED, 1, T>(r);
    p[2] = predict_interior_at<PRED, 2, T>(r);
    p[3] = predict_interior_at<PRED, 3, T>(r);
    p[4] = predict_interior_at<PRED, 4, T>(r);
    p[5] = predict_interior_at<PRED, 5, T>(r);
    p[6] = predict_interior_at<PRED, 6, T>(r);
}

// The 7 predictions of one coarse point (interior: 1 <= x,y,z <= dim-3).
template <int PRED, typename T, class Acc>
__device__ __forceinline__ void predict7(const Acc& r, bool interior, int x, int y, int z, int dx, int dy, int dz,
                                         T (&p)[7])
{
    if (interior) {
        p[0] = predict_interior_at<PRED, 0, T>(r);
        p[1] = predict_interior_at<PRED, 1, T>(r);
        p[2] = predict_interior_at<PRED, 2, T>(r);
        p[3] = predict_interior_at<PRED, 3, T>(r);
        p[4] = predict_interior_at<PRED, 4, T>(r);
        p[5] = predict_interior_at<PRED, 5, T>(r);
        p[6] = predict_interior_at<PRED, 6, T>(r);
    } else {
        p[0] = predict_at<PRED, 0, T>(r, x, y, z, dx, dy, dz);
        p[1] = predict_at<PRED, 1, T>(r, x, y, z, dx, dy, dz);
        p[2] = predict_at<PRED, 2, T>(r, x, y, z, dx, dy, dz);
        p[3] = predict_at<PRED, 3, T>(r, x, y, z, dx, dy, dz);
        p[4] = predict_at<PRED, 4, T>(r, x, y, z, dx, dy, dz);
        p[5] = predict_at<PRED, 5, T>(r, x, y, z, dx, dy, dz);
        p[6] = predict_at<PRED, 6, T>(r, x, y, z, dx, dy, dz);
    }
}

// ---- learned correction (LearnedModel in stz_internal.h) -------------------
// Exact integer inference: the encoder, the decoder and the ROI path compute
// the same 7 corrections bit for bit.
__device__ __forceinline__ int learned_to_i8(float t)
{
    if (!(t == t)) return 0;
    if (t >= 127.f) return 127;
    if (t <= -127.f) return -127;
    return __float2int_rn(t);
}
__device__ __forceinline__ int learned_to_i8(double t)
{
    if (!(t == t)) return 0;
    if (t >= 127.0) return 127;
    if (t <= -127.0) return -127;
    return __double2int_rn(t);
}
__device__ __forceinline__ uint32_t learned_requant(int acc, int m, int sh)
{
    const long long p = ((long long)acc * m + (1ll << (sh - 1))) >> sh;
    return p < 0 ? 0u : (p > 127 ? 127u : (uint32_t)p);
}

// The integer network on packed int8 inputs (16 bytes, the last two zero):
// the output accumulators of the 7 blocks.
__device__ __forceinline__ void learned_mlp_int(const LearnedModel& M, const uint4& x, int (&acc3)[7])
{
    const uint32_t xw[4] = {x.x, x.y, x.z, x.w};
    const int* w1 = reinterpret_cast<const int*>(&M.w1[0][0]);
    const int* w2 = reinterpret_cast<const int*>(&M.w2[0][0]);
    const int* w3 = reinterpret_cast<const int*>(&M.w3[0][0]);
    uint32_t a1[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        int acc = M.b1[j];
#pragma unroll
        for (int w = 0; w < 4; ++w) acc = __dp4a(w1[j * 4 + w], (int)xw[w], acc);
        a1[j >> 2] |= learned_requant(acc, M.m1, M.sh1) << (8 * (j & 3));
    }
    uint32_t a2[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        int acc = M.b2[j];
#pragma unroll
        for (int w = 0; w < 8; ++w) acc = __dp4a(w2[j * 8 + w], (int)a1[w], acc);
        a2[j >> 2] |= learned_requant(acc, M.m2, M.sh2) << (8 * (j & 3));
    }
#pragma unroll
    for (int o = 0; o < 7; ++o) {
        int acc = M.b3[o];
#pragma unroll
        for (int w = 0; w < 8; ++w) acc = __dp4a(w3[o * 8 + w], (int)a2[w], acc);
        acc3[o] = acc;
    }
}

// The network's int8 inputs at a coarse point (accessor r positioned on it;
// the stencil reaches -1..+2 on each axis): stencil values minus the mean of
// the 8 cell corners, times rs, rounded and clamped, packed 4 per word.
template <typename T, class Acc>
__device__ __forceinline__ uint4 learned_inputs(const Acc& r, T rs)
{
    using A = Ar<T>;
    constexpr int st[14][3] = STZ_LEARNED_STENCIL;
    T v[14];
#pragma unroll
    for (int i = 0; i < 14; ++i) v[i] = r(st[i][2] * (long long)r.sy + st[i][1] * (long long)r.sx + st[i][0]);
    T m = v[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) m = A::add(m, v[i]);
    m = A::mul(m, T(0.125));
    uint32_t xw[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int i = 0; i < 14; ++i)
        xw[i >> 2] |= ((uint32_t)learned_to_i8(A::mul(A::sub(v[i], m), rs)) & 0xffu) << (8 * (i & 3));
    return make_uint4(xw[0], xw[1], xw[2], xw[3]);
}

// The 7 corrections at a coarse point. M is usually in shared memory.
template <typename T, class Acc>
__device__ __forceinline__ void learned_corr(const LearnedModel& M, const Acc& r, T rs, T so, T (&corr)[7])
{
    int acc3[7];
    learned_mlp_int(M, learned_inputs<T>(r, rs), acc3);
#pragma unroll
    for (int o = 0; o < 7; ++o) corr[o] = Ar<T>::mul((T)acc3[o], so);
}

// Copy a model into shared memory (all threads of the block; caller syncs).
__device__ __forceinline__ void learned_load(LearnedModel* dst, const LearnedModel* src, int tid, int nthreads)
{
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = tid; i < (int)(sizeof(LearnedModel) / 16); i += nthreads) d[i] = s[i];
}

// Runtime-block predictor on a global grid (boundary-kernel and ROI paths).
template <int PRED, typename T>
__device__ __forceinline__ T predict(int block, const Grid<T>& g, int x, int y, int z)
{
    const GlobalAt<T> r{g.p + (size_t)z * g.sy + (size_t)y * g.sx + x, (long long)g.sx, (long long)g.sy};
    switch (block) {
    case 0: return predict_at<PRED, 0, T>(r, x, y, z, g.dx, g.dy, g.dz);
    case 1: return predict_at<PRED, 1, T>(r, x, y, z, g.dx, g.dy, g.dz);
    case 2: return predict_at<PRED, 2, T>(r, x, y, z, g.dx, g.dy, g.dz);
    case 3: return predict_at<PRED, 3, T>(r, x, y, z, g.dx, g.dy, g.dz);
    case 4: return predict_at<PRED, 4, T>(r, x, y, z, g.dx, g.dy, g.dz);
    case 5: return predict_at<PRED, 5, T>(r, x, y, z, g.dx, g.dy, g.dz);
    default: return predict_at<PRED, 6, T>(r, x, y, z, g.dx, g.dy, g.dz);
    }
}

// quantize_range_nodec for one residual (FD5:1216-1229). Returns the shifted
// code, 0 when unpredictable. quantize_is_centre is the early exit: |d| below
// the precomputed threshold tlo guarantees the centre code (QuantParams).
// quantize_full is the whole computation; its half == 0 case (|d|/eb < 1) is
// taken first: there the decompressed value is +-0 and the check reduces to
// |d| <= eb.
template <typename T>
__device__ __forceinline__ bool quantize_is_centre(T d, const QuantParams& qp)
{
    if constexpr (sizeof(T) == 4) return fabsf(d) < qp.tlo32;
    else return fabs(d) < qp.tlo64;
}

template <typename T>
__device__ __forceinline__ int quantize_full(T d, const QuantParams& qp);

template <typename T>
__device__ __forceinline__ int quantize(T d, const QuantParams& qp)
{
    if (quantize_is_centre(d, qp)) return qp.radius;
    return quantize_full(d, qp);
}

template <typename T>
__device__ __forceinline__ int quantize_full(T d, const QuantParams& qp)
{
    using A = Ar<T>;
    const double dd = fabs(A::to_f64(d));
    const double ad = d_mul(dd, qp.recip);
    if (ad < 1.0) return dd <= qp.eb ? qp.radius : 0;
    const bool in_range = ad < (double)(2 * qp.radius - 1);
    const double adc = in_range ? ad : 0.0;
    const int half = (__double2int_rz(adc) + 1) >> 1;
    const T mag = A::from_f64(d_mul((double)(2 * half), qp.eb));
    const bool neg = A::is_neg(d);
    const T dk = neg ? A::neg(mag) : mag;
    const T derr = A::sub(dk, d);
    const bool ok = in_range && (fabs(A::to_f64(derr)) <= qp.eb);
    if (!ok) return 0;
    return neg ? qp.radius - half : qp.radius + half;
}

// quantize_full of an f32 residual through the level's QuantTable (tab in
// shared memory, r2 = 0.5 / eb in float): the table entry of the estimated
// half index decides when |d| lies inside its interval, else quantize_full
// itself does (interval edges, values beyond the table, NaN, inf).
__device__ __forceinline__ int quantize_table(float d, const QuantParams& qp, const float4* tab, float r2)
{
    const float a = fabsf(d);
    const int h = min(max(__float2int_rn(a * r2), 0), kQuantTableH - 1);
    const float4 e = tab[h];
    if (!(a >= e.x && a < e.y)) return quantize_full(d, qp);
    const bool pass = a >= e.z && a <= e.w;
    return pass ? (Ar<float>::is_neg(d) ? qp.radius - h : qp.radius + h) : 0;
}

// recover LUT entry (FD5:1531-1535): (T)(2*(q - radius)*eb).
template <typename T>
__device__ __forceinline__ T recover(int q, const QuantParams& qp)
{
    return Ar<T>::from_f64(d_mul((double)(2 * (q - qp.radius)), qp.eb));
}

}  // namespace stz
