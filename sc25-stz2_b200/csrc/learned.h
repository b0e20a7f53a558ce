// Batch inference of the learned correction's int8 network (learned.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

// out[s][0..6] = the network's output accumulators for input row s
// (xq: n rows of 16 int8, the last two zero; out[s][7] = 0). tensor_cores:
// tcgen05 kind::i8 MMAs (err set nonzero when an MMA does not complete in
// time), else per-thread dp4a.
void launch_learned_infer(bool tensor_cores, const int8_t* xq, uint64_t n, const LearnedModel* M, int32_t* out,
                          uint32_t* err, cudaStream_t st);

}  // namespace stz
