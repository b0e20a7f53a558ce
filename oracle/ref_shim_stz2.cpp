// Test-infrastructure shim for the reference's 12-point truncated bicubic
// experiment, src/stz2.cpp (float only). The file is compiled unmodified from
// where it lies (path passed as STZ_STZ2_SOURCE) against the oracle's SZ3-ncp
// stand-in declarations, and its preprocess_block / depreprocess_block
// (stz2.cpp:82-309, 311-526) are exported.
//
// Output goes to oracle/_ref/ only. FTZ/DAZ set per call on every OpenMP
// thread, the FP environment of the library's codec (FD5's main). <cmath>
// comes first: the file calls log10 and gets <cmath> through the real SZ3
// headers, which the stand-in declarations do not include.
#include <cmath>
#include <xmmintrin.h>
#include <pmmintrin.h>

#define main stz2_reference_main_unused
#include STZ_STZ2_SOURCE
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

extern "C" void stz2ref_preprocess_block(int block, const float* sub, const float* ref, float* diff, int dx, int dy,
                                         int dz)
{
    FtzGuard g;
    preprocess_block(block, sub, ref, diff, dx, dy, dz);
}

extern "C" void stz2ref_depreprocess_block(int block, const float* de, const float* ref, float* out, int dx, int dy,
                                           int dz)
{
    FtzGuard g;
    depreprocess_block(block, de, ref, out, dx, dy, dz);
}
