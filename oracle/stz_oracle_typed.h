/*
 * Typed half of the CPU oracle, included twice by stz_oracle.c with
 * T = float / SUF = f32 and T = double / SUF = f64 (the reference's
 * run_typed<float> / run_typed<double>, FD5:1954, 3070-3076).
 *
 * Test infrastructure only (see stz_oracle.h). Every arithmetic expression
 * keeps the reference's operand order; the build disables FMA contraction and
 * the entry points enable FTZ/DAZ as the reference main() does (FD5:3046-3047).
 */
#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUF)

/* cubic_line_pred, FD5:141-146: -(1/16)a + (9/16)b + (9/16)c - (1/16)d, left to right. */
static inline T FN(cubic)(T a, T b, T c, T d)
{
    return -(1.0f / 16.0f) * a + (9.0f / 16.0f) * b + (9.0f / 16.0f) * c - (1.0f / 16.0f) * d;
}

/* cubic_line_pv_cse, FD5:163-175 (default build, PRED_NO_CSE unset). The
 * epsilon is a float literal converted to T, as in the reference. */
static inline void FN(line_pv)(T a, T b, T c, T d, T* p, T* v)
{
    const T eps = (T)1e-12f;
    const T c0 = a - 2.0f * b + c;
    const T c1 = b - 2.0f * c + d;
    *v = 0.5f * (c0 * c0 + c1 * c1) + eps;
    *p = 0.5f * (b + c) - (1.0f / 16.0f) * (c0 + c1);
}

/* blend2, FD5:178-186 (PRED_WPOW2 unset). */
static inline T FN(blend2)(T p0, T v0, T p1, T v1)
{
    return (p0 * v1 + p1 * v0) / (v0 + v1);
}

/* blend4, FD5:188-203: product weights and one division. */
static inline T FN(blend4)(T p0, T v0, T p1, T v1, T p2, T v2, T p3, T v3)
{
    const T w0 = v1 * v2 * v3;
    const T w1 = v0 * v2 * v3;
    const T w2 = v0 * v1 * v3;
    const T w3 = v0 * v1 * v2;
    return (w0 * p0 + w1 * p1 + w2 * p2 + w3 * p3) / (w0 + w1 + w2 + w3);
}

/* predict_dynamic_lines_const<Block>, FD5:624-688 (no PRED_PLANE_AXIS /
 * PRED_CUBE_AXIS): diagonal cubic lines blended by inverse variance. */
static inline T FN(dyn_lines)(int block, const T* r, size_t i, size_t sx, size_t sy)
{
    T p0, v0, p1, v1, p2, v2, p3, v3;
    if (block == 2) {
        FN(line_pv)(r[i - sx - 1], r[i], r[i + sx + 1], r[i + 2 * sx + 2], &p0, &v0);
        FN(line_pv)(r[i - sx + 2], r[i + 1], r[i + sx], r[i + 2 * sx - 1], &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    }
    if (block == 4) {
        FN(line_pv)(r[i - sy - 1], r[i], r[i + sy + 1], r[i + 2 * sy + 2], &p0, &v0);
        FN(line_pv)(r[i - sy + 2], r[i + 1], r[i + sy], r[i + 2 * sy - 1], &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    }
    if (block == 5) {
        FN(line_pv)(r[i - sy - sx], r[i], r[i + sy + sx], r[i + 2 * sy + 2 * sx], &p0, &v0);
        FN(line_pv)(r[i - sy + 2 * sx], r[i + sx], r[i + sy], r[i + 2 * sy - sx], &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    }
    FN(line_pv)(r[i - sy - sx - 1], r[i], r[i + sy + sx + 1], r[i + 2 * sy + 2 * sx + 2], &p0, &v0);
    FN(line_pv)(r[i - sy - sx + 2], r[i + 1], r[i + sy + sx], r[i + 2 * sy + 2 * sx - 1], &p1, &v1);
    FN(line_pv)(r[i - sy + 2 * sx - 1], r[i + sx], r[i + sy + 1], r[i + 2 * sy - sx + 2], &p2, &v2);
    FN(line_pv)(r[i + 2 * sy - sx - 1], r[i + sy], r[i + sx + 1], r[i - sy + 2 * sx + 2], &p3, &v3);
    return FN(blend4)(p0, v0, p1, v1, p2, v2, p3, v3);
}

/* predict_block_const<Block>, FD5:690-748. The split kernels of FD5 use this
 * on the boundary shells and predict_interior_const (FD5:828-840) inside; both
 * give the same value at every point, so the oracle evaluates it pointwise. */
static T FN(t_predict)(int block, const T* r, int x, int y, int z, int dx, int dy, int dz)
{
    const size_t sx = (size_t)dx, sy = (size_t)dx * (size_t)dy;
    const size_t i = ((size_t)z * dy + y) * dx + x;
    switch (block) {
    case 0:
        if (x == dx - 1) return r[i];
        if (x == dx - 2 || x == 0) return (T)0.5f * (r[i] + r[i + 1]);
        return FN(cubic)(r[i - 1], r[i], r[i + 1], r[i + 2]);
    case 1:
        if (y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0) return (T)0.5f * (r[i] + r[i + sx]);
        return FN(cubic)(r[i - sx], r[i], r[i + sx], r[i + 2 * sx]);
    case 2:
        if (x == dx - 1 || y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return (T)0.25f * (r[i] + r[i + sx + 1] + r[i + sx] + r[i + 1]);
        return FN(dyn_lines)(2, r, i, sx, sy);
    case 3:
        if (z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0) return (T)0.5f * (r[i] + r[i + sy]);
        return FN(cubic)(r[i - sy], r[i], r[i + sy], r[i + 2 * sy]);
    case 4:
        if (x == dx - 1 || z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0)
            return (T)0.25f * (r[i] + r[i + sy + 1] + r[i + 1] + r[i + sy]);
        return FN(dyn_lines)(4, r, i, sx, sy);
    case 5:
        if (z == dz - 1 || y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0)
            return (T)0.25f * (r[i] + r[i + sy + sx] + r[i + sy] + r[i + sx]);
        return FN(dyn_lines)(5, r, i, sx, sy);
    default:
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return (T)0.125f * (r[i] + r[i + sy + sx + 1] + r[i + sy + sx] + r[i + sy + 1] +
                                r[i + sx + 1] + r[i + 1] + r[i + sx] + r[i + sy]);
        return FN(dyn_lines)(6, r, i, sx, sy);
    }
}

/* Plain tricubic-family predictor, src/float.cpp:84-273 (templated copy in
 * src/stz-rd.cpp:114-300): fixed stencils, boundary averages written as sums
 * of scaled taps (0.5a + 0.5b) in that file's operand order. */
static T FN(t_predict_plain)(int block, const T* r, int x, int y, int z, int dx, int dy, int dz)
{
    const size_t sx = (size_t)dx, sy = (size_t)dx * (size_t)dy;
    const size_t i = ((size_t)z * dy + y) * dx + x;
    switch (block) {
    case 0:
        if (x == dx - 1) return r[i];
        if (x == dx - 2 || x == 0) return 0.5f * r[i] + 0.5f * r[i + 1];
        return -(1.0f / 16.0f) * r[i - 1] + (9.0f / 16.0f) * r[i] + (9.0f / 16.0f) * r[i + 1] -
               (1.0f / 16.0f) * r[i + 2];
    case 1:
        if (y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0) return 0.5f * r[i] + 0.5f * r[i + sx];
        return -(1.0f / 16.0f) * r[i - sx] + (9.0f / 16.0f) * r[i] + (9.0f / 16.0f) * r[i + sx] -
               (1.0f / 16.0f) * r[i + 2 * sx];
    case 2:
        if (x == dx - 1 || y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return 0.25f * r[i] + 0.25f * r[i + sx + 1] + 0.25f * r[i + sx] + 0.25f * r[i + 1];
        return 0.28125f * r[i] + 0.28125f * r[i + sx + 1] + 0.28125f * r[i + sx] + 0.28125f * r[i + 1] -
               0.03125f * r[i - sx - 1] - 0.03125f * r[i + 2 * sx + 2] - 0.03125f * r[i + 2 * sx - 1] -
               0.03125f * r[i - sx + 2];
    case 3:
        if (z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0) return 0.5f * r[i] + 0.5f * r[i + sy];
        return -(1.0f / 16.0f) * r[i - sy] + (9.0f / 16.0f) * r[i] + (9.0f / 16.0f) * r[i + sy] -
               (1.0f / 16.0f) * r[i + 2 * sy];
    case 4:
        if (x == dx - 1 || z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0 || x == dx - 2 || x == 0)
            return 0.25f * r[i] + 0.25f * r[i + sy + 1] + 0.25f * r[i + 1] + 0.25f * r[i + sy];
        return 0.28125f * r[i] + 0.28125f * r[i + sy + 1] + 0.28125f * r[i + 1] + 0.28125f * r[i + sy] -
               0.03125f * r[i - sy - 1] - 0.03125f * r[i + 2 - sy] - 0.03125f * r[i + 2 * sy - 1] -
               0.03125f * r[i + 2 * sy + 2];
    case 5:
        if (z == dz - 1 || y == dy - 1) return r[i];
        if (y == dy - 2 || y == 0 || z == dz - 2 || z == 0)
            return 0.25f * r[i] + 0.25f * r[i + sy + sx] + 0.25f * r[i + sy] + 0.25f * r[i + sx];
        return 0.28125f * r[i] + 0.28125f * r[i + sy + sx] + 0.28125f * r[i + sy] + 0.28125f * r[i + sx] -
               0.03125f * r[i - sy - sx] - 0.03125f * r[i + 2 * sy + 2 * sx] -
               0.03125f * r[i + 2 * sy - sx] - 0.03125f * r[i + 2 * sx - sy];
    default:
        if (x == dx - 1 || y == dy - 1 || z == dz - 1) return r[i];
        if (z == dz - 2 || z == 0 || y == dy - 2 || y == 0 || x == dx - 2 || x == 0)
            return 0.125f * r[i] + 0.125f * r[i + sy + sx + 1] + 0.125f * r[i + sy + sx] +
                   0.125f * r[i + sy + 1] + 0.125f * r[i + sx + 1] + 0.125f * r[i + 1] +
                   0.125f * r[i + sx] + 0.125f * r[i + sy];
        return 0.140625f * r[i] + 0.140625f * r[i + sy + sx + 1] + 0.140625f * r[i + sy + sx] +
               0.140625f * r[i + sy + 1] + 0.140625f * r[i + sx + 1] + 0.140625f * r[i + 1] +
               0.140625f * r[i + sx] + 0.140625f * r[i + sy] -
               0.015625f * r[i - sy - sx - 1] - 0.015625f * r[i + 2 * sy + 2 * sx + 2] -
               0.015625f * r[i + 2 * sy - sx + 2] - 0.015625f * r[i + 2 * sy + 2 * sx - 1] -
               0.015625f * r[i - sy + 2 * sx + 2] - 0.015625f * r[i + 2 * sy - sx - 1] -
               0.015625f * r[i - sy + 2 * sx - 1] - 0.015625f * r[i - sy - sx + 2];
    }
}

/* Staged predictor of src/dependency.cpp (predictor 2). Blocks 0, 1, 3 (one
 * odd axis) take a 1-D cubic along that axis of the coarse grid; blocks 2, 4, 5
 * blend two 1-D cubics through the decoded blocks 0, 1, 3 by inverse
 * variance; block 6 blends three through the decoded blocks 2, 4, 5. A line
 * is addressed by the point c, its stride st along the axis, and the point's
 * index pos on an axis of extent dim. */

/* interp_axis, dependency.cpp:90-118 (W0..W3 = -1/16, 9/16, 9/16, -1/16). */
static inline T FN(dep_line)(const T* c, ptrdiff_t st, int pos, int dim)
{
    if (pos == dim - 1) return c[0];
    if (pos == dim - 2 || pos == 0) return 0.5f * (c[0] + c[st]);
    return -0.0625f * c[-st] + 0.5625f * c[0] + 0.5625f * c[st] + -0.0625f * c[2 * st];
}

/* interp_axis_with_variance, dependency.cpp:162-243. The reference squares
 * |b - a|; squaring b - a gives the same bits. */
static inline void FN(dep_line_pv)(const T* c, ptrdiff_t st, int pos, int dim, T* p, T* v)
{
    const T eps = (T)1e-12f;
    if (pos == dim - 1) {
        *p = c[0];
        *v = eps;
        return;
    }
    if (pos == dim - 2 || pos == 0) {
        const T a = c[0], b = c[st];
        const T e = b - a;
        *p = 0.5f * (a + b);
        *v = e * e + eps;
        return;
    }
    const T a = c[-st], b = c[0], cc = c[st], d = c[2 * st];
    const T c0 = a - 2.0f * b + cc;
    const T c1 = b - 2.0f * cc + d;
    *p = -0.0625f * a + 0.5625f * b + 0.5625f * cc + -0.0625f * d;
    *v = 0.5f * (c0 * c0 + c1 * c1) + eps;
}

/* inverse_variance_blend3, dependency.cpp:250-256 (blend2 above is
 * inverse_variance_blend2, dependency.cpp:245-248, the same expression). */
static inline T FN(blend3)(T p0, T v0, T p1, T v1, T p2, T v2)
{
    const T w0 = v1 * v2;
    const T w1 = v0 * v2;
    const T w2 = v0 * v1;
    return (w0 * p0 + w1 * p1 + w2 * p2) / (w0 + w1 + w2);
}

/* Prediction of block b at coarse (x, y, z): stage-1 blocks from the coarse
 * grid r (interp_axis on sub-block 0, preprocess_block dependency.cpp:333-383), the others
 * from the decoded fine grid F of this level (2dx x 2dy x 2dz), in which
 * sub-block s sits at parity (s & 1, s >> 1 & 1, s >> 2) and a step along an
 * axis of a sub-block is two fine points (staged_prediction,
 * dependency.cpp:258-292: ref_x, ref_y, ref_z, ref_xy, ref_xz, ref_yz are
 * sub-blocks 1, 2, 4, 3, 5, 6). */
static T FN(staged_pred)(int b, const T* r, const T* F, int x, int y, int z, int dx, int dy, int dz)
{
    const size_t cx = 1, cy = (size_t)dx, cz = (size_t)dx * dy;
    const size_t i = (size_t)z * cz + (size_t)y * cy + x;
    const ptrdiff_t fx = 2, fy = 4 * (ptrdiff_t)dx, fz = 8 * (ptrdiff_t)dx * dy;
#define SIB(s) (F + (size_t)(2 * z + ((s) >> 2)) * (4 * (size_t)dx * dy) + (size_t)(2 * y + (((s) >> 1) & 1)) * (2 * (size_t)dx) + 2 * (size_t)x + ((s) & 1))
    T p0, v0, p1, v1, p2, v2;
    switch (b) {
    case 0: return FN(dep_line)(r + i, (ptrdiff_t)cx, x, dx);
    case 1: return FN(dep_line)(r + i, (ptrdiff_t)cy, y, dy);
    case 3: return FN(dep_line)(r + i, (ptrdiff_t)cz, z, dz);
    case 2:
        FN(dep_line_pv)(SIB(1), fy, y, dy, &p0, &v0);
        FN(dep_line_pv)(SIB(2), fx, x, dx, &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    case 4:
        FN(dep_line_pv)(SIB(1), fz, z, dz, &p0, &v0);
        FN(dep_line_pv)(SIB(4), fx, x, dx, &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    case 5:
        FN(dep_line_pv)(SIB(2), fz, z, dz, &p0, &v0);
        FN(dep_line_pv)(SIB(4), fy, y, dy, &p1, &v1);
        return FN(blend2)(p0, v0, p1, v1);
    default:
        FN(dep_line_pv)(SIB(3), fz, z, dz, &p0, &v0);
        FN(dep_line_pv)(SIB(5), fy, y, dy, &p1, &v1);
        FN(dep_line_pv)(SIB(6), fx, x, dx, &p2, &v2);
        return FN(blend3)(p0, v0, p1, v1, p2, v2);
    }
#undef SIB
}

/* Predictor of src/stz2.cpp (predictor 3): the plain stencils above, except
 * that the two-axis blocks 2, 4, 5 take a 12-point truncated bicubic inside
 * (the 4 inner points at (9/16)^2, the 8 edge points at -(1/16)(9/16), no
 * corners; stz2.cpp:122-155, 170-232) and that the one-axis interior cubic
 * has double weights (stz2.cpp:86, 100-118), so the reference evaluates it,
 * the residual and the rebuilt value in double and rounds once. Returns the
 * prediction as a double; *wide = 1 for that double-evaluated case. */
static double FN(t_predict_trunc)(int block, const T* r, int x, int y, int z, int dx, int dy, int dz, int* wide)
{
    const size_t sx = (size_t)dx, sy = (size_t)dx * (size_t)dy;
    const size_t i = ((size_t)z * dy + y) * dx + x;
    *wide = 0;
    size_t st = 0, a1 = 0, a2 = 0; /* cubic stride; the 12-point form's two axes */
    int pos = 0, dim = 0, inner = 0;
    switch (block) {
    case 0: st = 1, pos = x, dim = dx; break;
    case 1: st = sx, pos = y, dim = dy; break;
    case 3: st = sy, pos = z, dim = dz; break;
    case 2: a1 = 1, a2 = sx, inner = x >= 1 && x < dx - 2 && y >= 1 && y < dy - 2; break;
    case 4: a1 = 1, a2 = sy, inner = x >= 1 && x < dx - 2 && z >= 1 && z < dz - 2; break;
    case 5: a1 = sx, a2 = sy, inner = y >= 1 && y < dy - 2 && z >= 1 && z < dz - 2; break;
    default: break;
    }
    if (st && pos >= 1 && pos < dim - 2) {
        *wide = 1;
        return -0.0625 * (double)r[i - st] + 0.5625 * (double)r[i] + 0.5625 * (double)r[i + st] +
               -0.0625 * (double)r[i + 2 * st];
    }
    if (inner) {
        const T core = r[i] + r[i + a1] + r[i + a2] + r[i + a2 + a1];
        const T edge = r[i - a1] + r[i + 2 * a1] + r[i + a2 - a1] + r[i + a2 + 2 * a1] + r[i - a2] + r[i - a2 + a1] +
                       r[i + 2 * a2] + r[i + 2 * a2 + a1];
        return (double)(T)(0.31640625f * core + -0.033203125f * edge);
    }
    return (double)FN(t_predict_plain)(block, r, x, y, z, dx, dy, dz);
}

static inline T FN(predict_any)(int predictor, int block, const T* r, int x, int y, int z, int dx, int dy,
                                int dz)
{
    return predictor == 1 ? FN(t_predict_plain)(block, r, x, y, z, dx, dy, dz)
                          : FN(t_predict)(block, r, x, y, z, dx, dy, dz);
}

/* Learned correction of one interior coarse cell (stzo_model in
 * stz_oracle.h; this project's addition). rs = (T)(1/(eb*s_in)),
 * so = (T)(s_out*eb). */
static inline int FN(to_i8)(T v)
{
    if (!(v == v)) return 0;
    if (v >= (T)127) return 127;
    if (v <= (T)-127) return -127;
    return (int)rint((double)v);
}

static void FN(mlp_corr)(const stzo_model* M, const T* r, int x, int y, int z, int dx, int dy, T rs, T so, T corr[7])
{
    const size_t sy = (size_t)dx, sz = (size_t)dx * dy;
    T v[14];
    for (int i = 0; i < 14; ++i)
        v[i] = r[(size_t)(z + kStencil[i][2]) * sz + (size_t)(y + kStencil[i][1]) * sy + (size_t)(x + kStencil[i][0])];
    T m = v[0];
    for (int i = 1; i < 8; ++i) m = m + v[i];
    m = m * (T)0.125;
    int xin[16] = {0};
    for (int i = 0; i < 14; ++i) xin[i] = FN(to_i8)((v[i] - m) * rs);
    int a1[32], a2[32];
    for (int j = 0; j < 32; ++j) {
        int32_t acc = M->b1[j];
        for (int i = 0; i < 16; ++i) acc += (int32_t)M->w1[j][i] * xin[i];
        a1[j] = requant(acc, M->m1, M->sh1);
    }
    for (int j = 0; j < 32; ++j) {
        int32_t acc = M->b2[j];
        for (int i = 0; i < 32; ++i) acc += (int32_t)M->w2[j][i] * a1[i];
        a2[j] = requant(acc, M->m2, M->sh2);
    }
    for (int o = 0; o < 7; ++o) {
        int32_t acc = M->b3[o];
        for (int i = 0; i < 32; ++i) acc += (int32_t)M->w3[o][i] * a2[i];
        corr[o] = (T)acc * so;
    }
}

static inline int FN(learned_at)(const stzo_model* M, uint32_t flags, int b, int x, int y, int z, int dx, int dy,
                                 int dz)
{
    return M && ((flags >> b) & 1u) && x >= 1 && x <= dx - 3 && y >= 1 && y <= dy - 3 && z >= 1 && z <= dz - 3;
}

/* One value of quantize_range_nodec, FD5:1216-1229 (the fallback loop
 * FD5:1232-1249 yields the same code for every input). Returns the shifted
 * code, 0 when unpredictable; *dec gets the decompressed residual. */
static inline int FN(quant1)(T d, double eb, double recip, int radius, T* dec)
{
    const double ad = fabs((double)d) * recip;
    const int in_range = ad < (double)(2 * radius - 1);
    const double adc = in_range ? ad : 0.0;
    const int half = ((int)adc + 1) >> 1;
    const T dec_mag = (T)(2 * half * eb);
    const T dec_k = (d < 0) ? -dec_mag : dec_mag;
    const T derr = dec_k - d;
    const int ok = in_range && (fabs((double)derr) <= eb);
    if (!ok) return 0;
    *dec = dec_k;
    return (d < 0) ? radius - half : radius + half;
}

/* recover LUT entry, FD5:1531-1535. */
static inline T FN(recover)(int q, double eb, int radius)
{
    return (T)(2 * (q - radius) * eb);
}

static long long FN(t_quantize)(const T* d, size_t n, double eb, int radius, int* q, T* unpred, size_t cap)
{
    ftz_on();
    const double recip = 1.0 / eb;
    size_t nu = 0;
    for (size_t i = 0; i < n; ++i) {
        T dec;
        q[i] = FN(quant1)(d[i], eb, recip, radius, &dec);
        if (q[i] == 0) {
            if (nu >= cap) return -1;
            unpred[nu++] = d[i];
        }
    }
    return (long long)nu;
}

/* Level step of predictor 3: as t_level_encode / t_level_decode, with the
 * residual and the rebuilt value in double where the prediction is. */
static int FN(t_level_encode_trunc)(const T* fine, const T* coarse, int dx, int dy, int dz, double eb, int radius,
                                    int* q, T* unpred, size_t cap, size_t* counts, T* decoded)
{
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    const double recip = 1.0 / eb;
    size_t nu = 0;
    for (int b = 0; b < 7; ++b) {
        const int s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        size_t nb = 0;
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const size_t i = ((size_t)z * dy + y) * dx + x;
                    const size_t fi = (2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px;
                    int wide;
                    const double pd = FN(t_predict_trunc)(b, coarse, x, y, z, dx, dy, dz, &wide);
                    const T p = (T)pd;
                    const T d = wide ? (T)((double)fine[fi] - pd) : fine[fi] - p;
                    T dec = 0;
                    const int code = FN(quant1)(d, eb, recip, radius, &dec);
                    q[(size_t)b * n + i] = code;
                    if (code == 0) {
                        if (nu >= cap) return -1;
                        unpred[nu++] = d;
                        ++nb;
                    }
                    if (decoded) {
                        const T dq = code ? FN(recover)(code, eb, radius) : d;
                        decoded[fi] = wide ? (T)((double)dq + pd) : dq + p;
                    }
                }
        counts[b] = nb;
    }
    if (decoded) {
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x)
                    decoded[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] =
                        coarse[((size_t)z * dy + y) * dx + x];
    }
    return 0;
}

static void FN(t_level_decode_trunc)(const int* q, const T* unpred, const T* coarse, int dx, int dy, int dz,
                                     double eb, int radius, T* out)
{
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    size_t u = 0;
    for (int b = 0; b < 7; ++b) {
        const int s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const int code = q[(size_t)b * n + ((size_t)z * dy + y) * dx + x];
                    const T dq = code ? FN(recover)(code, eb, radius) : unpred[u++];
                    int wide;
                    const double pd = FN(t_predict_trunc)(b, coarse, x, y, z, dx, dy, dz, &wide);
                    out[(2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px] =
                        wide ? (T)((double)dq + pd) : dq + (T)pd;
                }
    }
    for (int z = 0; z < dz; ++z)
        for (int y = 0; y < dy; ++y)
            for (int x = 0; x < dx; ++x)
                out[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] = coarse[((size_t)z * dy + y) * dx + x];
}

/* Level step of the staged predictor: the blocks in the reference's stage
 * order (compress dependency.cpp:659-704 and 591-634 for the
 * second level, decompress 755-772): 0, 1, 3, then
 * 2, 4, 5, then 6, each predicted from the decoded values of the stages
 * before it (the encoder quantizes every residual and rebuilds the decoded
 * value before the next stage reads it, as SZ_compress hands back the
 * decoded residuals there). Codes and unpredictable values come out in block
 * order, like the other predictors. decoded null: a scratch fine grid. */
static const int FN(staged_order)[7] = {0, 1, 3, 2, 4, 5, 6};

static int FN(t_level_encode_staged)(const T* fine, const T* coarse, int dx, int dy, int dz, double eb, int radius,
                                     int* q, T* unpred, size_t cap, size_t* counts, T* decoded)
{
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    const double recip = 1.0 / eb;
    T* F = decoded ? decoded : (T*)malloc(8 * n * sizeof(T) + 1);
    T* dres = (T*)malloc(7 * n * sizeof(T) + 1);
    int rc = 0;
    if (!F || !dres) {
        rc = -1;
        goto done;
    }
    for (int z = 0; z < dz; ++z)
        for (int y = 0; y < dy; ++y)
            for (int x = 0; x < dx; ++x)
                F[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] = coarse[((size_t)z * dy + y) * dx + x];
    for (int o = 0; o < 7; ++o) {
        const int b = FN(staged_order)[o], s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const size_t i = ((size_t)z * dy + y) * dx + x;
                    const size_t fi = (2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px;
                    const T p = FN(staged_pred)(b, coarse, F, x, y, z, dx, dy, dz);
                    const T d = fine[fi] - p;
                    T dec = 0;
                    const int code = FN(quant1)(d, eb, recip, radius, &dec);
                    q[(size_t)b * n + i] = code;
                    dres[(size_t)b * n + i] = d;
                    F[fi] = (code ? FN(recover)(code, eb, radius) : d) + p;
                }
    }
    {
        size_t nu = 0;
        for (int b = 0; b < 7 && !rc; ++b) {
            size_t nb = 0;
            for (size_t i = 0; i < n; ++i)
                if (q[(size_t)b * n + i] == 0) {
                    if (nu >= cap) {
                        rc = -1;
                        break;
                    }
                    unpred[nu++] = dres[(size_t)b * n + i];
                    ++nb;
                }
            counts[b] = nb;
        }
    }
done:
    if (F != decoded) free(F);
    free(dres);
    return rc;
}

static void FN(t_level_decode_staged)(const int* q, const T* unpred, const T* coarse, int dx, int dy, int dz,
                                      double eb, int radius, T* out)
{
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    size_t first[7], u = 0;  /* each block's first unpredictable value */
    for (int b = 0; b < 7; ++b) {
        first[b] = u;
        for (size_t i = 0; i < n; ++i) u += q[(size_t)b * n + i] == 0;
    }
    for (int z = 0; z < dz; ++z)
        for (int y = 0; y < dy; ++y)
            for (int x = 0; x < dx; ++x)
                out[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] = coarse[((size_t)z * dy + y) * dx + x];
    for (int o = 0; o < 7; ++o) {
        const int b = FN(staged_order)[o], s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        size_t ub = first[b];
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const int code = q[(size_t)b * n + ((size_t)z * dy + y) * dx + x];
                    const T dq = code ? FN(recover)(code, eb, radius) : unpred[ub++];
                    const T p = FN(staged_pred)(b, coarse, out, x, y, z, dx, dy, dz);
                    out[(2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px] = dq + p;
                }
    }
}

/* Level encode: residual of sub-block (block+1) against the predictor on the
 * decoded coarse grid (FD5 preprocess + quantize, see the fd5ref shim for the
 * reference's call sequence). The decoded fine grid uses the decoder's
 * recover values, so it equals what the decompressor rebuilds. */
static int FN(t_level_encode)(const T* fine, const T* coarse, int dx, int dy, int dz, int predictor, double eb,
                          int radius, int* q, T* unpred, size_t cap, size_t* counts, T* decoded,
                          const stzo_model* M, uint32_t flags)
{
    ftz_on();
    if (predictor == 2)
        return FN(t_level_encode_staged)(fine, coarse, dx, dy, dz, eb, radius, q, unpred, cap, counts, decoded);
    if (predictor == 3)
        return FN(t_level_encode_trunc)(fine, coarse, dx, dy, dz, eb, radius, q, unpred, cap, counts, decoded);
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    const double recip = 1.0 / eb;
    const T rs = M ? (T)(1.0 / (eb * M->s_in)) : (T)0, so = M ? (T)(M->s_out * eb) : (T)0;
    size_t nu = 0;
    for (int b = 0; b < 7; ++b) {
        const int s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        size_t nb = 0;
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const size_t i = ((size_t)z * dy + y) * dx + x;
                    const size_t fi = (2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px;
                    T p = FN(predict_any)(predictor, b, coarse, x, y, z, dx, dy, dz);
                    if (FN(learned_at)(M, flags, b, x, y, z, dx, dy, dz)) {
                        T corr[7];
                        FN(mlp_corr)(M, coarse, x, y, z, dx, dy, rs, so, corr);
                        p = p + corr[b];
                    }
                    const T d = fine[fi] - p;
                    T dec = 0;
                    const int code = FN(quant1)(d, eb, recip, radius, &dec);
                    q[(size_t)b * n + i] = code;
                    if (code == 0) {
                        if (nu >= cap) return -1;
                        unpred[nu++] = d;
                        ++nb;
                    }
                    if (decoded) {
                        const T dq = code ? FN(recover)(code, eb, radius) : d;
                        decoded[fi] = dq + p;
                    }
                }
        counts[b] = nb;
    }
    if (decoded) {
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x)
                    decoded[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] =
                        coarse[((size_t)z * dy + y) * dx + x];
    }
    return 0;
}

/* Level decode: x' = dq + P (FD5:1049-1143), merged into the fine grid. */
static void FN(t_level_decode)(const int* q, const T* unpred, const size_t* counts, const T* coarse, int dx, int dy,
                           int dz, int predictor, double eb, int radius, T* out, const stzo_model* M, uint32_t flags)
{
    ftz_on();
    if (predictor == 2) {
        FN(t_level_decode_staged)(q, unpred, coarse, dx, dy, dz, eb, radius, out);
        return;
    }
    if (predictor == 3) {
        FN(t_level_decode_trunc)(q, unpred, coarse, dx, dy, dz, eb, radius, out);
        return;
    }
    const size_t n = (size_t)dx * dy * dz;
    const size_t fx = 2 * (size_t)dx, fxy = 4 * (size_t)dx * dy;
    const T rs = M ? (T)(1.0 / (eb * M->s_in)) : (T)0, so = M ? (T)(M->s_out * eb) : (T)0;
    size_t u = 0;
    for (int b = 0; b < 7; ++b) {
        const int s = b + 1, px = s & 1, py = (s >> 1) & 1, pz = (s >> 2) & 1;
        for (int z = 0; z < dz; ++z)
            for (int y = 0; y < dy; ++y)
                for (int x = 0; x < dx; ++x) {
                    const size_t i = ((size_t)z * dy + y) * dx + x;
                    const int code = q[(size_t)b * n + i];
                    const T dq = code ? FN(recover)(code, eb, radius) : unpred[u++];
                    T p = FN(predict_any)(predictor, b, coarse, x, y, z, dx, dy, dz);
                    if (FN(learned_at)(M, flags, b, x, y, z, dx, dy, dz)) {
                        T corr[7];
                        FN(mlp_corr)(M, coarse, x, y, z, dx, dy, rs, so, corr);
                        p = p + corr[b];
                    }
                    out[(2 * (size_t)z + pz) * fxy + (2 * (size_t)y + py) * fx + 2 * (size_t)x + px] = dq + p;
                }
        (void)counts;
    }
    for (int z = 0; z < dz; ++z)
        for (int y = 0; y < dy; ++y)
            for (int x = 0; x < dx; ++x)
                out[(2 * (size_t)z) * fxy + (2 * (size_t)y) * fx + 2 * (size_t)x] = coarse[((size_t)z * dy + y) * dx + x];
}

/* Subsample the field to the fine grid of one level: every s-th point. */
static void FN(subsample)(const T* field, int nx, int ny, int nz, int s, T* out)
{
    const int ox = nx / s, oy = ny / s, oz = nz / s;
    size_t o = 0;
    for (int z = 0; z < oz; ++z)
        for (int y = 0; y < oy; ++y)
            for (int x = 0; x < ox; ++x)
                out[o++] = field[((size_t)z * s * ny + (size_t)y * s) * nx + (size_t)x * s];
}

#undef FN
#undef CAT
#undef CAT_
