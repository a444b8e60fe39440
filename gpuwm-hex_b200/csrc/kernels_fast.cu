// The dycore kernels and step orchestration built as namespace hexdyn_fast.
// Compiled with -fmad=true: multiply-adds contracted (fast numerics).
#include "dycore_geo.cuh"
#include "hexdyn_ctx.h"
#include "powf_gnu.cuh"

namespace hexdyn_fast {
#include "dycore_kernels.cuh"
#include "dycore_kernels_vec.cuh"
#include "dycore_step.cuh"
}  // namespace hexdyn_fast
