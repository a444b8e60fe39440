// The dycore kernels and step orchestration built as namespace hexdyn_strict.
// Compiled with -fmad=false: bit-identical FP32 arithmetic.
#include "dycore_geo.cuh"
#include "hexdyn_ctx.h"
#include "powf_gnu.cuh"

namespace hexdyn_strict {
#include "dycore_kernels.cuh"
#include "dycore_kernels_vec.cuh"
#include "dycore_step.cuh"
}  // namespace hexdyn_strict
