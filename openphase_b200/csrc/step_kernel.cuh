// The fused multiphase-field time step for sm_100a: one thread per voxel, one launch per step.
//
// For every voxel the kernel performs, in registers/local memory, what the reference spreads over
// five grid passes:
//   1. derivatives + candidates   PhaseField::CalculateDerivativesSR  (src/PhaseField.cpp:566-615)
//   2. pairwise kinetics          DoubleObstacle::CalculatePhaseFieldIncrementsSR
//                                 (src/DoubleObstacle.cpp:502-571)
//   3. driving-force merge        DrivingForce::MergePhaseFieldIncrementsSR (src/DrivingForce.cpp:497-602)
//   4. simplex projection         PhaseField::NormalizeIncrementsSR (src/PhaseField.cpp:1351-1561)
//   5. merge + finalize           PhaseField::MergeIncrementsSR (:1268-1299), NodePF::finalize
//                                 (include/Containers/NodePF.h:214-255)
// and it accumulates the grain volumes of the new state (PhaseField::CalculateGrainsVolume,
// src/PhaseField.cpp:812-951) through a per-block shared-memory table.  The flags of
// PhaseField::SetFlagsSR are derived from neighbour counts on the fly, the periodic boundary
// copies (BoundaryConditions::SetX/Y/Z) become index wrap-around.
//
// Exactness: in the FP64 form (this header compiled with --fmad=false) every floating-point
// expression is evaluated in the reference's order, so results are bit-identical to the
// reference except for tanh (CUDA vs. libm, a few ulp) and the grain-volume summation order.
#pragma once
#include <cfloat>
#include <cstdint>

#include "opgpu_device.h"
#include "opgpu_rng.h"

namespace opgpu {

__device__ __forceinline__ int pair_pos(int a, int b, int n)
{
    return a * (2 * n - a - 1) / 2 + (b - a - 1);
}

__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; }  // std::min

__device__ __forceinline__ double pair_energy(const StepParams& p, const StepArrays& a, int ga, int gb)
{
    if (p.pair_mode == 1 && a.pair_sigma) return a.pair_sigma[(long long)ga * p.ngrains + gb];
    if (p.pair_mode == 2)
    {
        const unsigned long long lo = ga < gb ? ga : gb, hi = ga < gb ? gb : ga;
        return p.hash_lo + p.hash_span * uniform01(p.hash_seed, kStreamSigma, lo, hi);
    }
    return p.sigma_p[a.gphase[ga] * p.nphases + a.gphase[gb]];
}

__device__ __forceinline__ double pair_mobility(const StepParams& p, const StepArrays& a, int ga, int gb)
{
    if (p.pair_mode == 1 && a.pair_mu) return a.pair_mu[(long long)ga * p.ngrains + gb];
    return p.mu_p[a.gphase[ga] * p.nphases + a.gphase[gb]];
}

// Per-block grain-volume table in shared memory.
constexpr int kVolSlots = 1024;

__device__ __forceinline__ void vol_insert(int* keys, double* sums, double* global_acc, int g, double v)
{
    unsigned h = ((unsigned)g * 2654435761u) & (kVolSlots - 1);
    for (int probe = 0; probe < kVolSlots; probe++)
    {
        const int k = atomicCAS(&keys[h], -1, g);
        if (k == -1 || k == g)
        {
            atomicAdd(&sums[h], v);
            return;
        }
        h = (h + 1) & (kVolSlots - 1);
    }
    atomicAdd(&global_acc[g], v);
}

// One voxel of the step, reading its 3x3x3 neighbourhood straight from global memory, with the
// field+candidate list and the pair increments in local memory (capacity KL entries).  This is
// the general path: the full-grid reference kernel below and the overflow kernel of the tiled step
// (voxels whose lists exceed the tiled kernel's register capacity) both run it.
template <class R, int KS, int KL>
__device__ __forceinline__ void voxel_step_generic(const StepParams& p, const StepArrays& a, long long v,
                                                   int* s_key, double* s_sum, unsigned& wide, unsigned& ein,
                                                   unsigned& eout, uint32_t& st, bool count_in)
{
    const long long N = p.n;
    {
        const uint8_t* __restrict__ cnt = a.cnt_in;
        const int16_t* __restrict__ gin = a.idx_in;
        const R* __restrict__ vin = static_cast<const R*>(a.val_in);
        R* __restrict__ vout = static_cast<R*>(a.val_out);

        const int nx = p.nx, ny = p.ny, nz = p.nz;
        const int z = (int)(v % nz);
        const long long t = v / nz;
        const int y = (int)(t % ny);
        const int x = (int)(t / ny);
        const long long plane = (long long)ny * nz;
        long long X[3], Y[3], Z[3];
        X[0] = (long long)(x == 0 ? nx - 1 : x - 1) * plane; X[1] = (long long)x * plane;
        X[2] = (long long)(x == nx - 1 ? 0 : x + 1) * plane;
        Y[0] = (long long)(y == 0 ? ny - 1 : y - 1) * nz; Y[1] = (long long)y * nz;
        Y[2] = (long long)(y == ny - 1 ? 0 : y + 1) * nz;
        Z[0] = (z == 0 ? nz - 1 : z - 1); Z[1] = z; Z[2] = (z == nz - 1 ? 0 : z + 1);

        const int c = cnt[v];
        ein = c;
        int flag = c > 1 ? 2 : 0;
        if (flag == 0)
        {
            for (int q = 0; q < 27 && flag == 0; q++)
            {
                const long long u = X[q / 9] + Y[(q / 3) % 3] + Z[q % 3];
                if (cnt[u] > 1) flag = 1;
            }
        }

        if (flag == 0)
        {
            // bulk voxel: the state is carried over unchanged (it is not touched by any stage)
            a.cnt_out[v] = (uint8_t)c;
            for (int s = 0; s < c; s++)
            {
                const int g = gin[s * N + v];
                const R phi = vin[s * N + v];
                a.idx_out[s * N + v] = (int16_t)g;
                vout[s * N + v] = phi;
                vol_insert(s_key, s_sum, a.vol_acc, g, (double)phi);
            }
            eout = c;
        }
        else
        {
            wide = 1;
            // ---- 1. own entries, then candidates, with Laplacians (stencil order) -----------
            int n = 0;
            int gL[KL];
            R val[KL];
            R lap[KL];
            for (int s = 0; s < c; s++)
            {
                gL[n] = gin[s * N + v];
                val[n] = vin[s * N + v];
                lap[n] = R(0);
                n++;
            }
            for (int q = 0; q < p.ns; q++)
            {
                const long long u = X[p.lap_d[q][0] + 1] + Y[p.lap_d[q][1] + 1] + Z[p.lap_d[q][2] + 1];
                const R w = (R)p.lap_w[q];
                const int cu = cnt[u];
                for (int s = 0; s < cu; s++)
                {
                    const R phi = vin[s * N + u];
                    if (phi != R(0))
                    {
                        const int g = gin[s * N + u];
                        const R l = w * phi;
                        int f = 0;
                        while (f < n && gL[f] != g) f++;
                        if (f < n) lap[f] += l;
                        else if (n < KL) { gL[n] = g; val[n] = R(0); lap[n] = l; n++; }
                        else st |= kStOverflowList;
                    }
                }
            }
            // the gradient pass of CalculateDerivativesSR appends indices it meets first
            for (int q = 0; q < p.ng; q++)
            {
                const long long u = X[p.grad_d[q][0] + 1] + Y[p.grad_d[q][1] + 1] + Z[p.grad_d[q][2] + 1];
                const int cu = cnt[u];
                for (int s = 0; s < cu; s++)
                {
                    const R phi = vin[s * N + u];
                    if (phi != R(0))
                    {
                        const int g = gin[s * N + u];
                        int f = 0;
                        while (f < n && gL[f] != g) f++;
                        if (f == n)
                        {
                            if (n < KL) { gL[n] = g; val[n] = R(0); lap[n] = R(0); n++; }
                            else st |= kStOverflowList;
                        }
                    }
                }
            }

            // ---- 2. double-obstacle pair kinetics -------------------------------------------
            constexpr int KP = KL * (KL - 1) / 2;
            // pair increments are kept in FP64 from here on (the FP32 form widens the kinetics'
            // result so that the projection's sums and limiter run as in the FP64 form)
            double pv[KP];
            R sg[KP];
            R mg[KP];
            double localN;
            if (p.consider_nucleus_volume)
            {
                localN = 0.0;
                for (int q = 0; q < n; q++) localN += a.vr[gL[q]];
            }
            else
            {
                localN = (double)n;
            }
            const R norm_1 = (R)(1.0 / localN);
            for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const int q = pair_pos(i, j, n);
                sg[q] = (R)pair_energy(p, a, gL[i], gL[j]);
                mg[q] = (R)pair_mobility(p, a, gL[i], gL[j]);
            }
            const R pref = (R)p.pref_do;
            for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const int q = pair_pos(i, j, n);
                const R scale = (R)sqrt(a.vr[gL[i]] * a.vr[gL[j]]);
                const R h = R(0.5) * (R(1) + scale) * pref;
                R dphi = sg[q] * ((lap[i] + h * val[i]) - (lap[j] + h * val[j]));
                if (n > 2)
                {
                    for (int k = 0; k < n; k++)
                    {
                        if (k == i || k == j) continue;
                        const R sbk = sg[j < k ? pair_pos(j, k, n) : pair_pos(k, j, n)];
                        const R sak = sg[i < k ? pair_pos(i, k, n) : pair_pos(k, i, n)];
                        dphi += (sbk - sak) * (lap[k] + h * val[k]);
                        if (p.tj_factor != 0.0 || scale < R(1))
                        {
                            const int pA = a.gphase[gL[i]], pB = a.gphase[gL[j]], pG = a.gphase[gL[k]];
                            const int P = p.nphases;
                            const R tj = (R)dmax_ref(p.tj_factor, (double)(R(1) - scale));
                            dphi += tj * pref
                                  * (((R)p.sigma_p[pA * P + pB] + (R)p.sigma_p[pB * P + pG]) + (R)p.sigma_p[pA * P + pG])
                                  * (val[i] * val[k] - val[j] * val[k]);
                        }
                    }
                }
                dphi *= mg[q] * norm_1 * scale;
                pv[q] = (double)dphi;
            }

            // ---- 3. driving force (interface voxels only) -----------------------------------
            if (p.use_dg && flag == 2)
            {
                const int P = p.nphases;
                for (int i = 0; i < n; i++)
                for (int j = i + 1; j < n; j++)
                {
                    const int q = pair_pos(i, j, n);
                    const int gi = gL[i], gj = gL[j];
                    double locdG = a.dg[gj] - a.dg[gi];
                    double norm = sqrt((double)val[i] * (double)val[j]);
                    if (a.gstage[gi] == 1 || a.gstage[gj] == 1) norm += 1.0e-6;
                    if (p.limiting)
                    {
                        const double allowed = p.allowed_p[a.gphase[gi] * P + a.gphase[gj]];
                        locdG = allowed * tanh(locdG / allowed);
                    }
                    const double dpsi = locdG * (double)mg[q] * norm * p.pref_df;
                    pv[q] += dpsi;
                }
            }

            // ---- 4. projection of the increments (NormalizeIncrementsSR) --------------------
            const double dt = p.dt;
            const int np = n * (n - 1) / 2;
            if (np == 1)
            {
                const double valueA = ((double)pv[0] + 0.0) * dt;
                const double old_value = (double)val[0];
                if ((old_value == 0.0 && valueA < 0.0) || (old_value == 1.0 && valueA > 0.0))
                {
                    pv[0] = 0.0;
                }
                else
                {
                    const double new_value = old_value + valueA;
                    double norm = 1.0;
                    if (new_value < 0.0) norm *= -old_value / valueA;
                    else if (new_value > 1.0) norm *= (1.0 - old_value) / valueA;
                    if (norm > DBL_EPSILON) pv[0] *= norm;
                    else pv[0] = 0.0;
                }
            }
            else if (np > 1)
            {
                for (int i = 0; i < n; i++)
                {
                    double dpsi = 0.0;
                    for (int j = 0; j < n; j++)
                    {
                        if (j == i) continue;
                        dpsi += (i < j) ? (double)pv[pair_pos(i, j, n)] : (double)pv[pair_pos(j, i, n)] * (-1.0);
                    }
                    if (((double)val[i] == 0.0 && dpsi < 0.0) || ((double)val[i] == 1.0 && dpsi > 0.0))
                    {
                        for (int j = 0; j < n; j++)
                        {
                            if (j == i) continue;
                            pv[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = 0.0;
                        }
                    }
                }
                bool any = false;
                for (int q = 0; q < np; q++) any |= (pv[q] != 0.0);
                if (any)
                {
                    double pos[KL], neg[KL], limP[KL], limN[KL];
                    int iterations = 0;
                    bool needed = true;
                    while (needed)
                    {
                        iterations++;
                        needed = false;
                        for (int i = 0; i < n; i++) { pos[i] = 0.0; neg[i] = 0.0; }
                        for (int i = 0; i < n; i++)
                        for (int j = i + 1; j < n; j++)
                        {
                            const double w = (double)pv[pair_pos(i, j, n)];
                            if (w < 0.0) { neg[i] += w; pos[j] += -w; }
                            if (w > 0.0) { pos[i] += w; neg[j] += -w; }
                        }
                        for (int i = 0; i < n; i++)
                        {
                            const double vi = (double)val[i];
                            const double newPF = vi + (pos[i] + neg[i]) * dt;
                            limN[i] = 1.0;
                            limP[i] = 1.0;
                            if (newPF < 0.0) limN[i] = dmin_ref(1.0, -(vi + pos[i] * dt) / (neg[i] * dt));
                            if (newPF > 1.0) limP[i] = dmin_ref(1.0, (1.0 - (vi + neg[i] * dt)) / (pos[i] * dt));
                        }
                        for (int i = 0; i < n; i++)
                        for (int j = i + 1; j < n; j++)
                        {
                            const int q = pair_pos(i, j, n);
                            if (pv[q] < 0.0)
                            {
                                const double lim = dmin_ref(limN[i], limP[j]);
                                pv[q] *= lim;
                                if (lim < 1.0) needed = true;
                            }
                            if (pv[q] > 0.0)
                            {
                                const double lim = dmin_ref(limP[i], limN[j]);
                                pv[q] *= lim;
                                if (lim < 1.0) needed = true;
                            }
                        }
                        if (iterations > 24)
                        {
                            if (needed) st |= kStLimiterCap;
                            needed = false;
                        }
                    }
                    for (int q = 0; q < np; q++)
                        if (fabs(pv[q] * dt) < DBL_EPSILON) pv[q] = 0.0;
                    // plausibility check (a warning in the reference)
                    for (int i = 0; i < n; i++) pos[i] = (double)val[i];
                    for (int i = 0; i < n; i++)
                    for (int j = i + 1; j < n; j++)
                    {
                        const double w = (double)pv[pair_pos(i, j, n)];
                        if (w != 0.0) { pos[i] += w * dt; pos[j] += -w * dt; }
                    }
                    for (int i = 0; i < n; i++)
                        if (pos[i] < -(double)FLT_EPSILON || pos[i] > 1.0 + (double)FLT_EPSILON) st |= kStNormalizeWarn;
                }
            }

            // ---- 5. merge (volume conserving, pair by pair) ---------------------------------
            // accumulated in FP64; the FP32 form rounds only when the record is stored
            double vd[KL];
            for (int i = 0; i < n; i++) vd[i] = (double)val[i];
            for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const double w = pv[pair_pos(i, j, n)];
                const double value = 1.0 * (w + 0.0) * dt;
                if (fabs(value) >= DBL_EPSILON)
                {
                    vd[i] += value;
                    vd[j] += -value;
                }
            }

            // ---- 6. finalize: snap, erase, renormalise --------------------------------------
            double total = 0.0;
            int m = 0;
            const double hi_snap = 1.0 - p.eps_snap;
            const double lo_snap = 0.0 + p.eps_snap;
            for (int i = 0; i < n; i++)
            {
                double w = vd[i];
                bool erase = false;
                if (w >= hi_snap) w = 1.0;
                if (w <= lo_snap) { w = 0.0; erase = true; }
                total += w;
                if (!erase) { gL[m] = gL[i]; vd[m] = w; m++; }
            }
            if (m > 1)
            {
                const double norm = 1.0 / total;
                for (int i = 0; i < m; i++) val[i] = (R)(vd[i] * norm);
            }
            else if (m == 1)
            {
                val[0] = R(1);
            }
            else
            {
                st |= kStEmptyVoxel;
            }
            if (m > KS) { st |= kStOverflowK; m = KS; }
            a.cnt_out[v] = (uint8_t)m;
            for (int i = 0; i < m; i++)
            {
                if (!isfinite((double)val[i])) st |= kStNonFinite;
                a.idx_out[i * N + v] = (int16_t)gL[i];
                vout[i * N + v] = val[i];
                vol_insert(s_key, s_sum, a.vol_acc, gL[i], (double)val[i]);
            }
            eout = m;
        }
    }
    if (!count_in) { ein = 0; }
}

template <class R, int KS, int KL>
__global__ void __launch_bounds__(256) step_kernel(const __grid_constant__ StepParams p, const StepArrays a)
{
    __shared__ int s_key[kVolSlots];
    __shared__ double s_sum[kVolSlots];
    __shared__ unsigned long long s_cnt[3];
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0ull;
    __syncthreads();

    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned wide = 0, ein = 0, eout = 0;
    uint32_t st = 0;
    if (v < p.n) voxel_step_generic<R, KS, KL>(p, a, v, s_key, s_sum, wide, ein, eout, st, true);

    if (st) atomicOr(a.status, st);
    // block totals of the counters
    unsigned w = wide, ei = ein, eo = eout;
    for (int o = 16; o > 0; o >>= 1)
    {
        w += __shfl_down_sync(0xffffffffu, w, o);
        ei += __shfl_down_sync(0xffffffffu, ei, o);
        eo += __shfl_down_sync(0xffffffffu, eo, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        if (w) atomicAdd(&s_cnt[0], (unsigned long long)w);
        if (ei) atomicAdd(&s_cnt[1], (unsigned long long)ei);
        if (eo) atomicAdd(&s_cnt[2], (unsigned long long)eo);
    }
    if (st & (kStOverflowK | kStOverflowList)) atomicAdd(&a.counters[kCntOverflowVoxels], 1ull);
    __syncthreads();
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x)
        if (s_key[i] >= 0) atomicAdd(&a.vol_acc[s_key[i]], s_sum[i]);
    if (threadIdx.x < 3 && s_cnt[threadIdx.x])
        atomicAdd(&a.counters[threadIdx.x == 0 ? kCntWide : (threadIdx.x == 1 ? kCntEntriesIn : kCntEntriesOut)],
                  s_cnt[threadIdx.x]);
}

template <class R>
int launch_step_generic(const StepParams& p, const StepArrays& a, int k_slots, void* stream)
{
    const int threads = 256;
    const long long blocks = (p.n + threads - 1) / threads;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (k_slots)
    {
        case 8:  step_kernel<R, 8, 16><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 12: step_kernel<R, 12, 20><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 16: step_kernel<R, 16, 24><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        default: return -1;
    }
    return (int)cudaGetLastError();
}

}  // namespace opgpu
