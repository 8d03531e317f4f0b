// General path of the tiled step, one warp per voxel: the voxels whose list is too long for the
// per-length kernels (or whose window had a grain without a slot) are stepped by a whole warp.
//
// Same arithmetic as list_step (step_kernel.cuh) in the same operation order, spread over lanes
// where the reference's order allows it:
//   - the 27 neighbours are staged in shared memory by 27 lanes at once;
//   - the candidate passes walk the stencil in order; the entries of one neighbour are matched by
//     lanes in parallel (a list holds distinct grains, so each field gets at most one term per
//     stencil element and the Laplacian sums keep their stencil order);
//   - pair energies, pair kinetics (each with its own sequential sum over the third field), driving
//     force and the limiter's pair updates run one pair per lane;
//   - every per-field sum (limiter sums, plausibility check, merge) runs one field per lane, adding
//     its pairs in the lexicographic pair order of the reference loops: first the pairs (i, f) with
//     i < f, then (f, j) with j > f;
//   - the order-dependent serial parts (the bound check that zeroes a field's pairs, the finalize
//     total) run on lane 0.
#pragma once
#include "step_kernel.cuh"

namespace opgpu {

template <class R, int KL>
struct WarpScratch {
    static constexpr int KP = KL * (KL - 1) / 2;
    static constexpr int KN = 27 * 16;     // staged neighbour entries (K <= 16)
    double pv[KP];
    R sg[KP];
    double pos[KL], neg[KL], nv[KL];
    R val[KL], lap[KL];
    int16_t g[KL];
    int16_t ng[KN];
    R nval[KN];
    int noff[28];
};

// (i, j) of pair position q in a list of n fields (i < j, lexicographic order)
__device__ __forceinline__ void pair_of(int q, int n, int& i, int& j)
{
    int a = 0;
    while (q >= n - 1 - a) { q -= n - 1 - a; a++; }
    i = a;
    j = a + 1 + q;
}

template <class R, int KS, int KL>
__device__ void warp_voxel_step(const StepParams& p, const StepArrays& a, long long v, WarpScratch<R, KL>& W,
                                int* s_key, double* s_sum, uint32_t& st, unsigned& eout)
{
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long N = p.n;
    const uint8_t* __restrict__ cnt = a.cnt_in;
    const int16_t* __restrict__ gin = a.idx_in;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    R* __restrict__ vout = static_cast<R*>(a.val_out);
    const Neighbourhood nb(p, v);
    const int c = cnt[v];

    // ---- stage the 3x3x3 neighbourhood (lane l: offsets (l/9-1, (l/3)%3-1, l%3-1)) --------------
    long long u = 0;
    int cu = 0;
    if (lane < 27)
    {
        u = nb.at(lane / 9 - 1, (lane / 3) % 3 - 1, lane % 3 - 1);
        cu = cnt[u];
    }
    int incl = cu;
    for (int o = 1; o < 32; o <<= 1)
    {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    const int excl = incl - cu;
    if (lane < 27) W.noff[lane] = excl;
    if (lane == 26) W.noff[27] = incl;
    if (lane < 27)
        for (int s = 0; s < cu; s++)
        {
            W.ng[excl + s] = gin[s * N + u];
            W.nval[excl + s] = vin[s * N + u];
        }
    const int flag = c > 1 ? 2 : (__any_sync(FULL, lane < 27 && cu > 1) ? 1 : 0);
    __syncwarp();
    const int own0 = W.noff[13];
    if (flag == 0)
    {
        // bulk voxel: carried over unchanged
        if (lane < c)
        {
            const int g = W.ng[own0 + lane];
            const R phi = W.nval[own0 + lane];
            a.idx_out[lane * N + v] = (int16_t)g;
            vout[lane * N + v] = phi;
            if (in_volume_window(p, v)) vol_insert_n(s_key, s_sum, kVolSlots, a.vol_acc, g, (double)phi);
        }
        if (lane == 0)
        {
            a.cnt_out[v] = (uint8_t)c;
            eout += c;
        }
        return;
    }
    // ---- 1. own fields, then the candidates, with their Laplacians --------------------------------
    if (lane < c)
    {
        W.g[lane] = W.ng[own0 + lane];
        W.val[lane] = W.nval[own0 + lane];
        W.lap[lane] = R(0);
    }
    int n = c;
    bool overflow = false;
    __syncwarp();
    const int npass = p.ns + p.ng;
    for (int qq = 0; qq < npass; qq++)
    {
        const bool lapl = qq < p.ns;
        const signed char* d = lapl ? p.lap_d[qq] : p.grad_d[qq - p.ns];
        const int l27 = (d[0] + 1) * 9 + (d[1] + 1) * 3 + (d[2] + 1);
        const int o = W.noff[l27], cq = W.noff[l27 + 1] - o;
        const R w = lapl ? (R)p.lap_w[qq] : R(0);
        int f = -1, g = -1;
        R term = R(0);
        bool fresh = false;
        if (lane < cq)
        {
            const R phi = W.nval[o + lane];
            if (phi != R(0))
            {
                g = W.ng[o + lane];
                term = w * phi;
                f = 0;
                while (f < n && W.g[f] != g) f++;
                fresh = f == n;
            }
        }
        const unsigned fm = __ballot_sync(FULL, fresh);
        __syncwarp();
        if (f >= 0 && !fresh && lapl) W.lap[f] += term;
        if (fresh)
        {
            const int k = n + __popc(fm & ((1u << lane) - 1u));
            if (k < KL)
            {
                W.g[k] = (int16_t)g;
                W.val[k] = R(0);
                W.lap[k] = lapl ? term : R(0);
            }
        }
        n += __popc(fm);
        if (n > KL) { overflow = true; n = KL; }
        __syncwarp();
    }
    if (overflow) st |= kStOverflowList;
    const int np = n * (n - 1) / 2;
    // ---- 2. pair kinetics ---------------------------------------------------------------------------
    double localN = 0.0;
    if (lane == 0)
    {
        if (p.consider_nucleus_volume)
            for (int k = 0; k < n; k++) localN += a.vr[W.g[k]];
        else
            localN = (double)n;
    }
    localN = __shfl_sync(FULL, localN, 0);
    const R norm_1 = (R)(1.0 / localN);
    for (int q = lane; q < np; q += 32)
    {
        int i, j;
        pair_of(q, n, i, j);
        W.sg[q] = (R)pair_energy(p, a, W.g[i], W.g[j]);
    }
    __syncwarp();
    const R pref = (R)p.pref_do;
    for (int q = lane; q < np; q += 32)
    {
        int i, j;
        pair_of(q, n, i, j);
        const int gi = W.g[i], gj = W.g[j];
        const double vri = a.vr[gi], vrj = a.vr[gj];
        const R scale = (vri == 1.0 && vrj == 1.0) ? R(1) : (R)sqrt(vri * vrj);
        const R h = R(0.5) * (R(1) + scale) * pref;
        const R vali = W.val[i], valj = W.val[j];
        R dphi = W.sg[q] * ((W.lap[i] + h * vali) - (W.lap[j] + h * valj));
        if (n > 2)
        {
            for (int k = 0; k < n; k++)
            {
                if (k == i || k == j) continue;
                const R sbk = W.sg[j < k ? pair_pos(j, k, n) : pair_pos(k, j, n)];
                const R sak = W.sg[i < k ? pair_pos(i, k, n) : pair_pos(k, i, n)];
                const R valk = W.val[k];
                dphi += (sbk - sak) * (W.lap[k] + h * valk);
                if (p.tj_factor != 0.0 || scale < R(1))
                {
                    const int pA = a.gphase[gi], pB = a.gphase[gj], pG = a.gphase[W.g[k]];
                    const int P = p.nphases;
                    const R tj = (R)dmax_ref(p.tj_factor, (double)(R(1) - scale));
                    dphi += tj * pref
                          * (((R)p.sigma_p[pA * P + pB] + (R)p.sigma_p[pB * P + pG]) + (R)p.sigma_p[pA * P + pG])
                          * (vali * valk - valj * valk);
                }
            }
        }
        dphi *= (R)pair_mobility(p, a, gi, gj) * norm_1 * scale;
        double pvq = (double)dphi;
        // ---- 3. driving force (interface voxels only) ----
        if (p.use_dg && flag == 2)
        {
            const double locdG = limited_force(p, a, gi, gj);
            double norm = sqrt((double)vali * (double)valj);
            if (a.gstage[gi] == 1 || a.gstage[gj] == 1) norm += 1.0e-6;
            const double dpsi = locdG * (double)(R)pair_mobility(p, a, gi, gj) * norm * p.pref_df;
            pvq += dpsi;
        }
        W.pv[q] = pvq;
    }
    __syncwarp();
    // ---- 4. projection ----------------------------------------------------------------------------
    const double dt = p.dt;
    if (np == 1)
    {
        if (lane == 0)
        {
            const double valueA = (W.pv[0] + 0.0) * dt;
            const double old_value = (double)W.val[0];
            if ((old_value == 0.0 && valueA < 0.0) || (old_value == 1.0 && valueA > 0.0))
            {
                W.pv[0] = 0.0;
            }
            else
            {
                const double new_value = old_value + valueA;
                double norm = 1.0;
                if (new_value < 0.0) norm *= -old_value / valueA;
                else if (new_value > 1.0) norm *= (1.0 - old_value) / valueA;
                if (norm > DBL_EPSILON) W.pv[0] *= norm;
                else W.pv[0] = 0.0;
            }
        }
        __syncwarp();
    }
    else if (np > 1)
    {
        if (lane == 0)
        {
            // the bound check in field order: a field's test sees the pairs earlier fields zeroed
            for (int i = 0; i < n; i++)
            {
                double dpsi = 0.0;
                for (int j = 0; j < n; j++)
                {
                    if (j == i) continue;
                    dpsi += (i < j) ? W.pv[pair_pos(i, j, n)] : W.pv[pair_pos(j, i, n)] * (-1.0);
                }
                const double vi = (double)W.val[i];
                if ((vi == 0.0 && dpsi < 0.0) || (vi == 1.0 && dpsi > 0.0))
                    for (int j = 0; j < n; j++)
                        if (j != i) W.pv[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = 0.0;
            }
        }
        __syncwarp();
        bool nz = false;
        for (int q = lane; q < np; q += 32) nz |= W.pv[q] != 0.0;
        if (__any_sync(FULL, nz))
        {
            for (int it = 1; it <= 25; it++)
            {
                if (lane < n)
                {
                    const int f = lane;
                    double ps = 0.0, ng = 0.0;
                    for (int i = 0; i < f; i++)
                    {
                        const double w = W.pv[pair_pos(i, f, n)];
                        if (w < 0.0) ps += -w;
                        if (w > 0.0) ng += -w;
                    }
                    for (int j = f + 1; j < n; j++)
                    {
                        const double w = W.pv[pair_pos(f, j, n)];
                        if (w < 0.0) ng += w;
                        if (w > 0.0) ps += w;
                    }
                    const double vi = (double)W.val[f];
                    const double newPF = vi + (ps + ng) * dt;
                    double limN = 1.0, limP = 1.0;
                    if (newPF < 0.0) limN = dmin_ref(1.0, -(vi + ps * dt) / (ng * dt));
                    if (newPF > 1.0) limP = dmin_ref(1.0, (1.0 - (vi + ng * dt)) / (ps * dt));
                    W.neg[f] = limN;
                    W.pos[f] = limP;
                }
                __syncwarp();
                bool needed = false;
                for (int q = lane; q < np; q += 32)
                {
                    int i, j;
                    pair_of(q, n, i, j);
                    double w = W.pv[q];
                    if (w < 0.0)
                    {
                        const double lim = dmin_ref(W.neg[i], W.pos[j]);
                        w *= lim;
                        if (lim < 1.0) needed = true;
                    }
                    if (w > 0.0)
                    {
                        const double lim = dmin_ref(W.pos[i], W.neg[j]);
                        w *= lim;
                        if (lim < 1.0) needed = true;
                    }
                    W.pv[q] = w;
                }
                const bool any_needed = __any_sync(FULL, needed);
                __syncwarp();
                if (!any_needed) break;
                if (it == 25) st |= kStLimiterCap;
            }
            for (int q = lane; q < np; q += 32)
                if (fabs(W.pv[q] * dt) < DBL_EPSILON) W.pv[q] = 0.0;
            __syncwarp();
            // plausibility check (a warning in the reference)
            if (lane < n)
            {
                const int f = lane;
                double chk = (double)W.val[f];
                for (int i = 0; i < f; i++)
                {
                    const double w = W.pv[pair_pos(i, f, n)];
                    if (w != 0.0) chk += -w * dt;
                }
                for (int j = f + 1; j < n; j++)
                {
                    const double w = W.pv[pair_pos(f, j, n)];
                    if (w != 0.0) chk += w * dt;
                }
                if (chk < -(double)FLT_EPSILON || chk > 1.0 + (double)FLT_EPSILON) st |= kStNormalizeWarn;
            }
        }
    }
    // ---- 5. merge (FP64) and finalize -------------------------------------------------------------
    const double hi_snap = 1.0 - p.eps_snap;
    const double lo_snap = 0.0 + p.eps_snap;
    bool keep = false;
    if (lane < n)
    {
        const int f = lane;
        double nvf = (double)W.val[f];
        for (int i = 0; i < f; i++)
        {
            const double value = 1.0 * (W.pv[pair_pos(i, f, n)] + 0.0) * dt;
            if (fabs(value) >= DBL_EPSILON) nvf += -value;
        }
        for (int j = f + 1; j < n; j++)
        {
            const double value = 1.0 * (W.pv[pair_pos(f, j, n)] + 0.0) * dt;
            if (fabs(value) >= DBL_EPSILON) nvf += value;
        }
        double w = nvf;
        keep = true;
        if (w >= hi_snap) w = 1.0;
        if (w <= lo_snap) { w = 0.0; keep = false; }
        W.nv[f] = w;
    }
    const unsigned km = __ballot_sync(FULL, keep);
    __syncwarp();
    double total = 0.0;
    if (lane == 0)
        for (int i = 0; i < n; i++) total += W.nv[i];
    total = __shfl_sync(FULL, total, 0);
    const int m = __popc(km);
    if (keep)
    {
        const int pos = __popc(km & ((1u << lane) - 1u));
        if (pos < KS)
        {
            const R w = (m > 1) ? (R)(W.nv[lane] * (1.0 / total)) : R(1);
            if (!isfinite((double)w)) st |= kStNonFinite;
            a.idx_out[pos * N + v] = W.g[lane];
            vout[pos * N + v] = w;
            if (in_volume_window(p, v)) vol_insert_n(s_key, s_sum, kVolSlots, a.vol_acc, W.g[lane], (double)w);
        }
    }
    if (lane == 0)
    {
        if (m == 0) st |= kStEmptyVoxel;
        if (m > KS) st |= kStOverflowK;
        const int mm = m > KS ? KS : m;
        a.cnt_out[v] = (uint8_t)mm;
        eout += mm;
    }
    __syncwarp();
}

// The general-path worklist, one warp per voxel.
template <class R, int KS, int KL>
__global__ void __launch_bounds__(128) warp_general_kernel(const __grid_constant__ StepParams p, const StepArrays a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_key[kVolSlots];
    __shared__ double s_sum[kVolSlots];
    __shared__ unsigned long long s_cnt[3];
    WarpScratch<R, KL>* scratch = reinterpret_cast<WarpScratch<R, KL>*>(smem_raw);
    WarpScratch<R, KL>& W = scratch[threadIdx.x >> 5];
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0ull;
    __syncthreads();
    const unsigned total = min(*a.slow_count, a.slow_cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.counters[kCntGeneralLast], (unsigned long long)total);
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    uint32_t st = 0;
    unsigned eo = 0;
    for (unsigned i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < total; i += warps)
        warp_voxel_step<R, KS, KL>(p, a, a.slow_list[i], W, s_key, s_sum, st, eo);
    flush_block(a, 0u, 0u, eo, st, s_cnt, s_key, s_sum, kVolSlots, threadIdx.x, blockDim.x);
}

}  // namespace opgpu
