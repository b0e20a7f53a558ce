// Test-infrastructure shim for the reference's plain tricubic STZ variant,
// src/stz-rd.cpp (fixed stencils, templated on T; the same predictor as the
// SC'25 artifact programs src/float.cpp / src/double.cpp). The file is compiled
// unmodified from where it lies (path passed as STZ_RD_SOURCE) against the
// oracle's SZ3-ncp stand-in declarations, and its preprocess_block /
// depreprocess_block templates are exported for float and double.
//
// Output goes to oracle/_ref/ only. FTZ/DAZ as in the reference programs'
// FP environment of the FD5 build (set per call on every OpenMP thread).
#include <xmmintrin.h>
#include <pmmintrin.h>

#define main stz_rd_reference_main_unused
#include STZ_RD_SOURCE
#undef main

namespace {
struct FtzGuard {
    FtzGuard()
    {
        _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
        _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
#pragma omp parallel
        {
            _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
            _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
        }
    }
};
}  // namespace

#define RD_TYPED(SUF, T)                                                                                         \
    extern "C" void rdref_preprocess_block_##SUF(int block, const T* sub, const T* ref, T* diff, int dx, int dy,  \
                                                  int dz)                                                        \
    {                                                                                                            \
        FtzGuard g;                                                                                              \
        preprocess_block<T>(block, sub, ref, diff, dx, dy, dz);                                                  \
    }                                                                                                            \
    extern "C" void rdref_depreprocess_block_##SUF(int block, const T* de, const T* ref, T* out, int dx, int dy,  \
                                                    int dz, int ex, int ey, int ez, int sx, int sy, int sz)      \
    {                                                                                                            \
        FtzGuard g;                                                                                              \
        depreprocess_block<T>(block, de, ref, out, dx, dy, dz, ex, ey, ez, sx, sy, sz);                          \
    }

RD_TYPED(f32, float)
RD_TYPED(f64, double)
