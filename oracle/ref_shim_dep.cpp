// Test-infrastructure shim for the reference's staged-predictor experiment,
// src/dependency.cpp (float only). The file is compiled unmodified from where
// it lies (path passed as STZ_DEP_SOURCE) against the oracle's SZ3-ncp
// stand-in declarations, and its four stage functions are exported:
// preprocess_block / depreprocess_block (blocks 0, 1, 3 from the coarse
// sub-block 0, dependency.cpp:333-431) and preprocess_block_staged /
// depreprocess_block_staged (blocks 2, 4, 5, 6 from decoded siblings,
// dependency.cpp:294-331). refs[0..5] are ref_x, ref_y, ref_z, ref_xy,
// ref_xz, ref_yz (the decoded sub-blocks 1, 2, 4, 3, 5, 6).
//
// Output goes to oracle/_ref/ only. FTZ/DAZ set per call on every OpenMP
// thread, the FP environment of the library's codec (FD5's main).
#include <xmmintrin.h>
#include <pmmintrin.h>

#define main dependency_reference_main_unused
#include STZ_DEP_SOURCE
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

extern "C" void depref_preprocess_block(int block, const float* sub, const float* ref, float* diff, int dx, int dy,
                                        int dz)
{
    FtzGuard g;
    preprocess_block(block, sub, ref, diff, dx, dy, dz);
}

extern "C" void depref_depreprocess_block(int block, const float* de, const float* ref, float* out, int dx, int dy,
                                          int dz)
{
    FtzGuard g;
    depreprocess_block(block, de, ref, out, dx, dy, dz);
}

extern "C" void depref_preprocess_block_staged(int block, const float* sub, const float* const* refs, float* diff,
                                               int dx, int dy, int dz)
{
    FtzGuard g;
    preprocess_block_staged(block, sub, refs[0], refs[1], refs[2], refs[3], refs[4], refs[5], diff, dx, dy, dz);
}

extern "C" void depref_depreprocess_block_staged(int block, const float* de, const float* const* refs, float* out,
                                                 int dx, int dy, int dz)
{
    FtzGuard g;
    depreprocess_block_staged(block, de, refs[0], refs[1], refs[2], refs[3], refs[4], refs[5], out, dx, dy, dz);
}
