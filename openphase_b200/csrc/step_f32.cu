// FP32 form of the fused step: field values, increments and stencil arithmetic in FP32; the
// simplex sums (limiter sums, finalize total) and the grain-volume reduction stay in FP64.  This
// translation unit is compiled with --fmad=false: the adjoint recomputes the per-voxel FP32
// arithmetic operation by operation and must round exactly as the forward did.
#include "tile_kernel.cuh"

namespace opgpu {
int launch_step_f32(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                    LaunchInfo* info)
{
    return launch_step<float>(p, a, k_slots, variant, stream, info);
}

int launch_classify_f32(const StepParams& p, const StepArrays& a, int k_slots, void* stream)
{
    return launch_classify<float>(p, a, k_slots, stream);
}
}  // namespace opgpu
