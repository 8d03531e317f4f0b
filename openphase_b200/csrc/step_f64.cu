// FP64 form of the fused step (the parity drop-in).  This translation unit is compiled with
// --fmad=false so that no multiply-add is contracted, as in the reference's x86-64 release build.
#include "tile_kernel.cuh"

namespace opgpu {
int launch_step_f64(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream)
{
    return launch_step<double>(p, a, k_slots, variant, stream);
}
}  // namespace opgpu
