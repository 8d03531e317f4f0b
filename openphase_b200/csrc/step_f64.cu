// FP64 form of the fused step (the parity drop-in).  This translation unit is compiled with
// --fmad=false so that no multiply-add is contracted, as in the reference's x86-64 release build.
#include "tile_kernel.cuh"

namespace opgpu {

int launch_step_f64(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                    LaunchInfo* info)
{
    return launch_step<double>(p, a, k_slots, variant, stream, info);
}

int launch_classify_f64(const StepParams& p, const StepArrays& a, int k_slots, void* stream)
{
    return launch_classify<double>(p, a, k_slots, stream);
}

// Grain volumes of the window planes of a state (slab decomposition: before the first step).
__global__ void volume_recount_kernel(const __grid_constant__ StepParams p, const uint8_t* __restrict__ cnt,
                                      const int16_t* __restrict__ idx, const void* __restrict__ val, int fp32,
                                      double* __restrict__ vol_acc)
{
    __shared__ int s_key[kVolSlots];
    __shared__ double s_sum[kVolSlots];
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    __syncthreads();
    const long long N = p.n;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N && in_volume_window(p, v))
    {
        const int c = cnt[v];
        for (int s = 0; s < c; s++)
        {
            const double w = fp32 ? (double)static_cast<const float*>(val)[s * N + v]
                                  : static_cast<const double*>(val)[s * N + v];
            vol_insert_n(s_key, s_sum, kVolSlots, vol_acc, idx[s * N + v], w);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x)
        if (s_key[i] >= 0) atomicAdd(&vol_acc[s_key[i]], s_sum[i]);
}

int launch_volume_recount(const StepParams& p, const uint8_t* cnt, const int16_t* idx, const void* val, int fp32,
                          double* vol_acc, void* stream)
{
    volume_recount_kernel<<<(unsigned)((p.n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, cnt, idx, val, fp32, vol_acc);
    return (int)cudaGetLastError();
}

}  // namespace opgpu
