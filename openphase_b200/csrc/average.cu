// Driving-force averaging: DrivingForce::Average with $Average Yes (src/DrivingForce.cpp:242-256),
// the reference default.  For the per-grain driving force, every interface voxel's pair (A, B)
// carries raw = dG_B - dG_A (A before B in the voxel's list) and weight sqrt(phi_A phi_B)
// (SetWeights, :276-291).  Two passes over a sphere of radius Range around each interface voxel:
//   collect    (CollectAverage, :293-383): for a pair whose weight exceeds Threshold' * VR_A VR_B,
//              tmp = sum(w_u raw) / sum(w_u) over the sphere's voxels holding the pair (w_u > 0);
//   distribute (DistributeAverage, :384-478): for every pair of positive fields, average =
//              sum(w_u tmp_u) / sum(w_u) over the sphere's voxels where the pair's weight exceeds
//              the threshold, or the voxel's own tmp (0 when the pair is not above the threshold
//              there: such a pair gets no driving force), then the tanh limiter of
//              MergePhaseFieldIncrementsSR (:548-583).
// Weights: PHASEFIELDS (the default, :59, :137); Threshold' = sqrt(t (1 - t)).  A step with
// averaging runs the per-voxel generic kernel, which reads the averaged force (pair_force).  The
// sphere offsets with Range - |d| > 0 are enumerated on the host in the reference's (x, y, z) loop
// order, so every sum is formed in its order.  Compiled with --fmad=false.  The limiter's tanh is
// CUDA's here (the averaged value differs per voxel), which can differ from the C library's in the
// last bit.
//
// Storage: every stored pair (a < b < c) of an interface voxel has a slot
// off[v] + pair_pos(a, b, c) for tmp and for the limited average (compact, an exclusive scan per
// step); a voxel whose slots would pass the capacity keeps the raw per-pair force and raises
// OPGPU_E_AVERAGE_SKIPPED.
#include <cfloat>
#include <cstdint>

#include <cub/device/device_scan.cuh>

#include "opgpu_device.h"
#include "step_kernel.cuh"

namespace opgpu {

namespace {

__device__ __forceinline__ long long wrap_voxel(const StepParams& p, int x, int y, int z)
{
    x = x < 0 ? x + p.nx : (x >= p.nx ? x - p.nx : x);
    y = y < 0 ? y + p.ny : (y >= p.ny ? y - p.ny : y);
    z = z < 0 ? z + p.nz : (z >= p.nz ? z - p.nz : z);
    return ((long long)x * p.ny + y) * p.nz + z;
}

// Force(u).get_weight(A, B): sqrt(phi_A phi_B) at an interface voxel u holding both, else 0; the
// list positions of A and B in sa, sb.
template <class R>
__device__ __forceinline__ double pair_weight(const uint8_t* __restrict__ cnt, const int16_t* __restrict__ idx,
                                              const R* __restrict__ val, long long N, long long u, int A, int B,
                                              int& sa, int& sb)
{
    sa = -1;
    sb = -1;
    const int c = cnt[u];
    if (c < 2) return 0.0;
    for (int k = 0; k < c; k++)
    {
        const int g = idx[k * N + u];
        if (g == A) sa = k;
        if (g == B) sb = k;
    }
    if (sa < 0 || sb < 0) return 0.0;
    return sqrt((double)val[sa * N + u] * (double)val[sb * N + u]);
}

__global__ void df_count_kernel(long long N, const uint8_t* __restrict__ cnt, unsigned* __restrict__ npairs)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const unsigned c = cnt[v];
    npairs[v] = c > 1 ? c * (c - 1) / 2 : 0u;
}

__device__ __forceinline__ bool fits(const AvgArrays& aa, long long u, int c)
{
    return (unsigned long long)aa.off[u] + (unsigned)(c * (c - 1) / 2) <= aa.cap;
}

template <class R>
__global__ void __launch_bounds__(128) df_collect_kernel(const __grid_constant__ StepParams p, AvgArrays aa,
                                                          const uint8_t* __restrict__ cnt,
                                                          const int16_t* __restrict__ idx, const R* __restrict__ val,
                                                          const double* __restrict__ vr, const double* __restrict__ dg)
{
    const long long N = p.n;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int c = cnt[v];
    if (c < 2 || !fits(aa, v, c)) return;
    const int x = (int)(v / ((long long)p.ny * p.nz)), y = (int)((v / p.nz) % p.ny), z = (int)(v % p.nz);
    const unsigned o = aa.off[v];
    for (int a = 0; a < c; a++)
        for (int b = a + 1; b < c; b++)
        {
            const int A = idx[a * N + v], B = idx[b * N + v];
            const double raw = dg[B] - dg[A];
            const double weight = sqrt((double)val[a * N + v] * (double)val[b * N + v]);
            const double scale = vr[A] * vr[B];
            double tmp = 0.0;
            if (weight > aa.weight_threshold * scale)
            {
                double value = 0.0, sum_weights = 0.0;
                for (int q = 0; q < aa.noff; q++)
                {
                    const signed char* d = aa.off3 + 3 * q;
                    int sa, sb;
                    const double wphi = pair_weight(cnt, idx, val, N, wrap_voxel(p, x + d[0], y + d[1], z + d[2]),
                                                    A, B, sa, sb);
                    if (wphi > 0.0)
                    {
                        sum_weights += wphi;
                        value += wphi * raw;
                    }
                }
                tmp = sum_weights > 0.0 ? value / sum_weights : raw;
            }
            aa.tmp[o + pair_pos(a, b, c)] = tmp;
        }
}

template <class R>
__global__ void __launch_bounds__(128) df_distribute_kernel(const __grid_constant__ StepParams p, AvgArrays aa,
                                                             const uint8_t* __restrict__ cnt,
                                                             const int16_t* __restrict__ idx, const R* __restrict__ val,
                                                             const double* __restrict__ vr,
                                                             const int16_t* __restrict__ gphase, uint32_t* status)
{
    const long long N = p.n;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int c = cnt[v];
    if (c < 2) return;
    if (!fits(aa, v, c))
    {
        atomicOr(status, kStAverageSkipped);
        return;
    }
    const int x = (int)(v / ((long long)p.ny * p.nz)), y = (int)((v / p.nz) % p.ny), z = (int)(v % p.nz);
    const unsigned o = aa.off[v];
    uint32_t st = 0;
    for (int a = 0; a < c; a++)
        for (int b = a + 1; b < c; b++)
        {
            const int A = idx[a * N + v], B = idx[b * N + v];
            const double scale = vr[A] * vr[B];
            const double thr = aa.weight_threshold * scale;
            double value = 0.0, sum_weights = 0.0;
            for (int q = 0; q < aa.noff; q++)
            {
                const signed char* d = aa.off3 + 3 * q;
                const long long u = wrap_voxel(p, x + d[0], y + d[1], z + d[2]);
                int sa, sb;
                const double wphi = pair_weight(cnt, idx, val, N, u, A, B, sa, sb);
                if (wphi > thr)
                {
                    sum_weights += wphi;
                    const int cu = cnt[u];
                    double t;
                    if (fits(aa, u, cu))
                    {
                        // get_tmp(A, B): the neighbour's tmp, negated when it lists B before A
                        const double tu = aa.tmp[aa.off[u] + (sa < sb ? pair_pos(sa, sb, cu) : pair_pos(sb, sa, cu))];
                        t = sa < sb ? tu : -tu;
                    }
                    else
                    {
                        t = 0.0;
                        st |= kStAverageSkipped;
                    }
                    value += wphi * t;
                }
            }
            double avg = sum_weights > 0.0 ? value / sum_weights : aa.tmp[o + pair_pos(a, b, c)];
            if (p.limiting)
            {
                const double allowed = p.allowed_p[gphase[A] * p.nphases + gphase[B]];
                avg = allowed * tanh(avg / allowed);
            }
            aa.lim[o + pair_pos(a, b, c)] = avg;
        }
    if (st) atomicOr(status, st);
}

}  // namespace

// Scratch bytes of the pair-slot scan over n voxels.
size_t average_scan_bytes(long long n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const unsigned*)nullptr, (unsigned*)nullptr, (int)n);
    return bytes;
}

__global__ void df_total_kernel(long long N, const unsigned* __restrict__ npairs, const unsigned* __restrict__ off,
                                unsigned long long* __restrict__ total)
{
    *total = (unsigned long long)off[N - 1] + npairs[N - 1];
}

int launch_average_scan(long long n, const AvgArrays& aa, const uint8_t* cnt, unsigned long long* d_total, void* stream)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    df_count_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(n, cnt, aa.npairs);
    size_t bytes = aa.scan_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(aa.scan_tmp, bytes, aa.npairs, aa.off, (int)n, s);
    if (e != cudaSuccess) return (int)e;
    df_total_kernel<<<1, 1, 0, s>>>(n, aa.npairs, aa.off, d_total);
    return (int)cudaGetLastError();
}

int launch_average(const StepParams& p, const AvgArrays& aa, const uint8_t* cnt, const int16_t* idx,
                   const void* val, bool fp32, const double* vr, const double* dg, const int16_t* gphase,
                   uint32_t* status, void* stream)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((p.n + 127) / 128);
    if (fp32)
    {
        df_collect_kernel<float><<<blocks, 128, 0, s>>>(p, aa, cnt, idx, static_cast<const float*>(val), vr, dg);
        df_distribute_kernel<float><<<blocks, 128, 0, s>>>(p, aa, cnt, idx, static_cast<const float*>(val), vr,
                                                           gphase, status);
    }
    else
    {
        df_collect_kernel<double><<<blocks, 128, 0, s>>>(p, aa, cnt, idx, static_cast<const double*>(val), vr, dg);
        df_distribute_kernel<double><<<blocks, 128, 0, s>>>(p, aa, cnt, idx, static_cast<const double*>(val), vr,
                                                            gphase, status);
    }
    return (int)cudaGetLastError();
}

}  // namespace opgpu
