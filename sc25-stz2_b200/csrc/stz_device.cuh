// Device-side arithmetic of the STZ hot path: the level predictors and the
// linear quantizer, evaluated with the reference's operation order.
//
// Bit-exactness with the reference CPU build (g++ -O3, SSE2 scalar float/double,
// no FMA contraction, FTZ+DAZ enabled in main, FD5:3046-3047) is obtained by
// issuing every floating-point operation as explicit round-to-nearest PTX:
// f32 ops carry .ftz (flush subnormal inputs and results, as FTZ/DAZ do on the
// host), and nothing can be contracted into an FMA or reassociated.
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

// Strided view of the coarse (decoded) grid a level predicts from.
template <typename T>
struct Grid {
    const T* __restrict__ p;
    int dx, dy, dz;
    size_t sx, sy;  // row and plane strides (elements)
    __device__ __forceinline__ T at(size_t i) const { return __ldg(p + i); }
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

// FD5 "dynamic lines" predictor for sub-block `block` (= sub_index - 1) at
// coarse point (x,y,z): predict_block_const<Block> (FD5:690-748) with
// predict_dynamic_lines_const (FD5:624-688) in the interior.
template <typename T>
__device__ __forceinline__ T predict_dynamic(int block, const Grid<T>& g, int x, int y, int z)
{
    using A = Ar<T>;
    const size_t sx = g.sx, sy = g.sy;
    const size_t i = (size_t)z * sy + (size_t)y * sx + x;
    const int dx = g.dx, dy = g.dy, dz = g.dz;
    T p0, v0, p1, v1, p2, v2, p3, v3;
    switch (block) {
    case 0:
        if (x == dx - 1) return g.at(i);
        if (x == dx - 2 || x == 0) return A::mul(T(0.5f), A::add(g.at(i), g.at(i + 1)));
        return cubic(g.at(i - 1), g.at(i), g.at(i + 1), g.at(i + 2));
    case 1:
        if (y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0) return A::mul(T(0.5f), A::add(g.at(i), g.at(i + sx)));
        return cubic(g.at(i - sx), g.at(i), g.at(i + sx), g.at(i + 2 * sx));
    case 2:
        if (x == dx - 1 || y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(g.at(i), g.at(i + sx + 1)), g.at(i + sx)), g.at(i + 1)));
        line_pv(g.at(i - sx - 1), g.at(i), g.at(i + sx + 1), g.at(i + 2 * sx + 2), p0, v0);
        line_pv(g.at(i - sx + 2), g.at(i + 1), g.at(i + sx), g.at(i + 2 * sx - 1), p1, v1);
        return blend2(p0, v0, p1, v1);
    case 3:
        if (z == dz - 1) return g.at(i);
        if (z == dz - 2 || z == 0) return A::mul(T(0.5f), A::add(g.at(i), g.at(i + sy)));
        return cubic(g.at(i - sy), g.at(i), g.at(i + sy), g.at(i + 2 * sy));
    case 4:
        if (x == dx - 1 || z == dz - 1) return g.at(i);
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(g.at(i), g.at(i + sy + 1)), g.at(i + 1)), g.at(i + sy)));
        line_pv(g.at(i - sy - 1), g.at(i), g.at(i + sy + 1), g.at(i + 2 * sy + 2), p0, v0);
        line_pv(g.at(i - sy + 2), g.at(i + 1), g.at(i + sy), g.at(i + 2 * sy - 1), p1, v1);
        return blend2(p0, v0, p1, v1);
    case 5:
        if (z == dz - 1 || y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0)
            return A::mul(T(0.25f), A::add(A::add(A::add(g.at(i), g.at(i + sy + sx)), g.at(i + sy)), g.at(i + sx)));
        line_pv(g.at(i - sy - sx), g.at(i), g.at(i + sy + sx), g.at(i + 2 * sy + 2 * sx), p0, v0);
        line_pv(g.at(i - sy + 2 * sx), g.at(i + sx), g.at(i + sy), g.at(i + 2 * sy - sx), p1, v1);
        return blend2(p0, v0, p1, v1);
    default:
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return g.at(i);
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(g.at(i), g.at(i + sy + sx + 1));
            s = A::add(s, g.at(i + sy + sx));
            s = A::add(s, g.at(i + sy + 1));
            s = A::add(s, g.at(i + sx + 1));
            s = A::add(s, g.at(i + 1));
            s = A::add(s, g.at(i + sx));
            s = A::add(s, g.at(i + sy));
            return A::mul(T(0.125f), s);
        }
        line_pv(g.at(i - sy - sx - 1), g.at(i), g.at(i + sy + sx + 1), g.at(i + 2 * sy + 2 * sx + 2), p0, v0);
        line_pv(g.at(i - sy - sx + 2), g.at(i + 1), g.at(i + sy + sx), g.at(i + 2 * sy + 2 * sx - 1), p1, v1);
        line_pv(g.at(i - sy + 2 * sx - 1), g.at(i + sx), g.at(i + sy + 1), g.at(i + 2 * sy - sx + 2), p2, v2);
        line_pv(g.at(i + 2 * sy - sx - 1), g.at(i + sy), g.at(i + sx + 1), g.at(i - sy + 2 * sx + 2), p3, v3);
        return blend4(p0, v0, p1, v1, p2, v2, p3, v3);
    }
}

// Sum of w*tap over a tap list, left to right, then minus v*tap for the rest:
// the fixed-stencil expressions of src/float.cpp keep that order.
template <typename T>
__device__ __forceinline__ T plain2(const Grid<T>& g, size_t i, T wp, size_t a0, size_t a1, size_t a2, size_t a3,
                                    T wn, size_t b0, size_t b1, size_t b2, size_t b3)
{
    using A = Ar<T>;
    T s = A::add(A::mul(wp, g.at(a0)), A::mul(wp, g.at(a1)));
    s = A::add(s, A::mul(wp, g.at(a2)));
    s = A::add(s, A::mul(wp, g.at(a3)));
    s = A::sub(s, A::mul(wn, g.at(b0)));
    s = A::sub(s, A::mul(wn, g.at(b1)));
    s = A::sub(s, A::mul(wn, g.at(b2)));
    s = A::sub(s, A::mul(wn, g.at(b3)));
    return s;
}

// Plain tricubic-family predictor of src/float.cpp:84-273 (src/stz-rd.cpp
// templated copy): fixed weights, boundary averages as sums of scaled taps.
template <typename T>
__device__ __forceinline__ T predict_plain(int block, const Grid<T>& g, int x, int y, int z)
{
    using A = Ar<T>;
    const size_t sx = g.sx, sy = g.sy;
    const size_t i = (size_t)z * sy + (size_t)y * sx + x;
    const int dx = g.dx, dy = g.dy, dz = g.dz;
    switch (block) {
    case 0:
        if (x == dx - 1) return g.at(i);
        if (x == dx - 2 || x == 0) return A::add(A::mul(T(0.5f), g.at(i)), A::mul(T(0.5f), g.at(i + 1)));
        return cubic(g.at(i - 1), g.at(i), g.at(i + 1), g.at(i + 2));
    case 1:
        if (y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0) return A::add(A::mul(T(0.5f), g.at(i)), A::mul(T(0.5f), g.at(i + sx)));
        return cubic(g.at(i - sx), g.at(i), g.at(i + sx), g.at(i + 2 * sx));
    case 2:
        if (x == dx - 1 || y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.25f), g.at(i)), A::mul(T(0.25f), g.at(i + sx + 1)));
            s = A::add(s, A::mul(T(0.25f), g.at(i + sx)));
            return A::add(s, A::mul(T(0.25f), g.at(i + 1)));
        }
        return plain2(g, i, T(0.28125f), i, i + sx + 1, i + sx, i + 1, T(0.03125f), i - sx - 1, i + 2 * sx + 2,
                      i + 2 * sx - 1, i - sx + 2);
    case 3:
        if (z == dz - 1) return g.at(i);
        if (z == dz - 2 || z == 0) return A::add(A::mul(T(0.5f), g.at(i)), A::mul(T(0.5f), g.at(i + sy)));
        return cubic(g.at(i - sy), g.at(i), g.at(i + sy), g.at(i + 2 * sy));
    case 4:
        if (x == dx - 1 || z == dz - 1) return g.at(i);
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.25f), g.at(i)), A::mul(T(0.25f), g.at(i + sy + 1)));
            s = A::add(s, A::mul(T(0.25f), g.at(i + 1)));
            return A::add(s, A::mul(T(0.25f), g.at(i + sy)));
        }
        return plain2(g, i, T(0.28125f), i, i + sy + 1, i + 1, i + sy, T(0.03125f), i - sy - 1, i + 2 - sy,
                      i + 2 * sy - 1, i + 2 * sy + 2);
    case 5:
        if (z == dz - 1 || y == dy - 1) return g.at(i);
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0) {
            T s = A::add(A::mul(T(0.25f), g.at(i)), A::mul(T(0.25f), g.at(i + sy + sx)));
            s = A::add(s, A::mul(T(0.25f), g.at(i + sy)));
            return A::add(s, A::mul(T(0.25f), g.at(i + sx)));
        }
        return plain2(g, i, T(0.28125f), i, i + sy + sx, i + sy, i + sx, T(0.03125f), i - sy - sx,
                      i + 2 * sy + 2 * sx, i + 2 * sy - sx, i + 2 * sx - sy);
    default: {
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return g.at(i);
        const size_t t[8] = {i, i + sy + sx + 1, i + sy + sx, i + sy + 1, i + sx + 1, i + 1, i + sx, i + sy};
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0) {
            T s = A::add(A::mul(T(0.125f), g.at(t[0])), A::mul(T(0.125f), g.at(t[1])));
#pragma unroll
            for (int k = 2; k < 8; ++k) s = A::add(s, A::mul(T(0.125f), g.at(t[k])));
            return s;
        }
        T s = A::add(A::mul(T(0.140625f), g.at(t[0])), A::mul(T(0.140625f), g.at(t[1])));
#pragma unroll
        for (int k = 2; k < 8; ++k) s = A::add(s, A::mul(T(0.140625f), g.at(t[k])));
        const size_t u[8] = {i - sy - sx - 1,     i + 2 * sy + 2 * sx + 2, i + 2 * sy - sx + 2, i + 2 * sy + 2 * sx - 1,
                             i - sy + 2 * sx + 2, i + 2 * sy - sx - 1,     i - sy + 2 * sx - 1, i - sy - sx + 2};
#pragma unroll
        for (int k = 0; k < 8; ++k) s = A::sub(s, A::mul(T(0.015625f), g.at(u[k])));
        return s;
    }
    }
}

template <int PRED, typename T>
__device__ __forceinline__ T predict(int block, const Grid<T>& g, int x, int y, int z)
{
    if constexpr (PRED == 1) return predict_plain(block, g, x, y, z);
    else return predict_dynamic(block, g, x, y, z);
}

// quantize_range_nodec for one residual (FD5:1216-1229). Returns the shifted
// code, 0 when unpredictable. dec receives the decompressed residual.
template <typename T>
__device__ __forceinline__ int quantize(T d, const QuantParams& qp, T& dec)
{
    using A = Ar<T>;
    const double ad = d_mul(fabs(A::to_f64(d)), qp.recip);
    const bool in_range = ad < (double)(2 * qp.radius - 1);
    const double adc = in_range ? ad : 0.0;
    const int half = (__double2int_rz(adc) + 1) >> 1;
    const T mag = A::from_f64(d_mul((double)(2 * half), qp.eb));
    const bool neg = A::is_neg(d);
    const T dk = neg ? A::neg(mag) : mag;
    const T derr = A::sub(dk, d);
    const bool ok = in_range && (fabs(A::to_f64(derr)) <= qp.eb);
    dec = dk;
    if (!ok) return 0;
    return neg ? qp.radius - half : qp.radius + half;
}

// recover LUT entry (FD5:1531-1535): (T)(2*(q - radius)*eb).
template <typename T>
__device__ __forceinline__ T recover(int q, const QuantParams& qp)
{
    return Ar<T>::from_f64(d_mul((double)(2 * (q - qp.radius)), qp.eb));
}

}  // namespace stz
