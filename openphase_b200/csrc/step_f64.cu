// FP64 form of the fused step (the parity drop-in).  This translation unit is compiled with
// --fmad=false so that no multiply-add is contracted, as in the reference's x86-64 release build.
#include "tile_kernel.cuh"

namespace opgpu {

int launch_step_f64(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                    LaunchInfo* info)
{
    return launch_step<double>(p, a, k_slots, variant, stream, info);
}

__global__ void dg_pair_kernel(const __grid_constant__ StepParams p, const double* __restrict__ dg,
                               const int16_t* __restrict__ gphase, double* __restrict__ out)
{
    const long long G = p.ngrains;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G * G) return;
    const int ga = (int)(i / G), gb = (int)(i % G);
    double locdG = dg[gb] - dg[ga];
    if (p.limiting)
    {
        const double allowed = p.allowed_p[gphase[ga] * p.nphases + gphase[gb]];
        locdG = allowed * tanh(locdG / allowed);
    }
    out[i] = locdG;
}

int launch_dg_pair(const StepParams& p, const double* dg, const int16_t* gphase, double* out, void* stream)
{
    const long long GG = (long long)p.ngrains * p.ngrains;
    dg_pair_kernel<<<(unsigned)((GG + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, dg, gphase, out);
    return (int)cudaGetLastError();
}

}  // namespace opgpu
