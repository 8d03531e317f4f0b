// Tangent-linear and adjoint of the fused step (no counterpart in the reference).
//
// The step maps the stored fields of a voxel's neighbourhood at t to the stored fields of the voxel
// at t+1.  Its discrete decisions -- which fields form the voxel's list (own fields and
// candidates), which increments the projection zeroes, which limits it applies, which increments
// the merge drops, which fields finalize snaps or erases -- are taken from the forward state and
// held fixed; the derivatives are those of the smooth map between the decisions (obstacle
// clipping as subgradient masks).  The grain volume ratios (VolumeRatio, LocalN with
// ConsiderNucleusVolume) and the limiter's cap (Limit*Pi/Eta*MaxEnergy) are held fixed as well.
//
// Parameters: the per-grain-pair interface energy sigma(a,b) and mobility mu(a,b) (symmetric, as
// the step reads them: table, hash or phase pair) and the per-grain driving force dG(g).
//
// Kernels
//   tlm_step_kernel      one forward step of the FP64 form with dual numbers: new state + tangent
//   adjoint_core         per wide voxel: recompute the step's arithmetic (same operation order as
//                        the forward), reverse it: adjoint of the voxel's own input values, of the
//                        Laplacians of its list, and the parameter gradients; driven by
//   adjoint_list_kernel  the classify kernel's work records of one list length (the forward's own
//                        lists, values and Laplacians), and by
//   adjoint_worklist_kernel the voxels of the general-path worklist (general gather);
//   adjoint_bulk_kernel  bulk voxels: the adjoint passes through
//   adjoint_gather_kernel adjoint of the stored values at t: own part plus the transposed stencil
//                        over the neighbours' Laplacian adjoints (tiled like the classify kernel)
// Compiled with --fmad=false so that the recomputed FP64 arithmetic repeats the forward's.
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "adjoint.h"
#include "step_kernel.cuh"
#include "tile_kernel.cuh"

namespace opgpu {

// ---- dual numbers (value, tangent) ------------------------------------------------------------
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual mkd(double v, double d = 0.0) { return Dual{v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual dsqrt(Dual a)
{
    const double s = sqrt(a.v);
    return {s, s > 0.0 ? a.d / (2.0 * s) : 0.0};
}
__device__ __forceinline__ Dual dmin_d(Dual a, Dual b) { return (b.v < a.v) ? b : a; }   // std::min

// ---- parameters ---------------------------------------------------------------------------------
__device__ __forceinline__ long long pair_key(int ga, int gb, int G)
{
    return ga < gb ? (long long)ga * G + gb : (long long)gb * G + ga;
}

// d F / d dG_b of F(a,b) = allowed*tanh((dG_b - dG_a)/allowed) (or dG_b - dG_a without limiting):
// 1 - tanh^2, with tanh = F/allowed from the tabulated limited force F (0 where allowed = 0)
__device__ __forceinline__ double force_slope(const StepParams& p, const StepArrays& a, int ga, int gb, double F)
{
    if (!p.limiting) return 1.0;
    const double allowed = p.allowed_p[a.gphase[ga] * p.nphases + a.gphase[gb]];
    if (allowed == 0.0) return 0.0;
    const double t = F / allowed;
    return 1.0 - t * t;
}

// ---- tangent-linear step (FP64 form) --------------------------------------------------------------
// Stages 2-5 of list_step<double> on dual numbers, operation by operation in the same order, so the
// value parts are the forward's bit for bit and every decision is the forward's.
template <int KL>
__device__ int stages_dual(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int n, int flag,
                           int16_t* g, Dual* val, const Dual* lap, Dual* sg, Dual* pv, Dual* pos, Dual* neg,
                           uint32_t& st)
{
    const int G = p.ngrains;
    double localN;
    if (p.consider_nucleus_volume)
    {
        localN = 0.0;
        for (int k = 0; k < n; k++) localN += a.vr[g[k]];
    }
    else
    {
        localN = (double)n;
    }
    const double norm_1 = 1.0 / localN;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            sg[pair_pos(i, j, n)] = mkd(pair_energy(p, a, g[i], g[j]), aa.tsig ? aa.tsig[pair_key(g[i], g[j], G)] : 0.0);
    const double pref = p.pref_do;
    for (int i = 0; i < n; i++)
    {
        const double vri = a.vr[g[i]];
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            const double vrj = a.vr[g[j]];
            const double scale = (vri == 1.0 && vrj == 1.0) ? 1.0 : sqrt(vri * vrj);
            const double h = 0.5 * (1.0 + scale) * pref;
            Dual dphi = sg[q] * ((lap[i] + h * val[i]) - (lap[j] + h * val[j]));
            if (n > 2)
            {
                for (int k = 0; k < n; k++)
                {
                    if (k == i || k == j) continue;
                    const Dual sbk = sg[j < k ? pair_pos(j, k, n) : pair_pos(k, j, n)];
                    const Dual sak = sg[i < k ? pair_pos(i, k, n) : pair_pos(k, i, n)];
                    dphi = dphi + (sbk - sak) * (lap[k] + h * val[k]);
                    if (p.tj_factor != 0.0 || scale < 1.0)
                    {
                        const int pA = a.gphase[g[i]], pB = a.gphase[g[j]], pG = a.gphase[g[k]];
                        const int P = p.nphases;
                        const double tj = dmax_ref(p.tj_factor, 1.0 - scale);
                        dphi = dphi + tj * pref * ((p.sigma_p[pA * P + pB] + p.sigma_p[pB * P + pG]) + p.sigma_p[pA * P + pG])
                                    * (val[i] * val[k] - val[j] * val[k]);
                    }
                }
            }
            const Dual mob = mkd(pair_mobility(p, a, g[i], g[j]), aa.tmu ? aa.tmu[pair_key(g[i], g[j], G)] : 0.0);
            dphi = dphi * ((mob * norm_1) * scale);
            pv[q] = dphi;
        }
    }
    if (p.use_dg && flag == 2)
    {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const double F = limited_force(p, a, g[i], g[j]);
                const double slope = force_slope(p, a, g[i], g[j], F);
                const double dF = aa.tdg ? slope * (aa.tdg[g[j]] - aa.tdg[g[i]]) : 0.0;
                const Dual locdG = mkd(F, dF);
                Dual norm = dsqrt(val[i] * val[j]);
                if (a.gstage[g[i]] == 1 || a.gstage[g[j]] == 1) norm = norm + 1.0e-6;
                const Dual mob = mkd(pair_mobility(p, a, g[i], g[j]), aa.tmu ? aa.tmu[pair_key(g[i], g[j], G)] : 0.0);
                const Dual dpsi = ((locdG * mob) * norm) * p.pref_df;
                pv[pair_pos(i, j, n)] = pv[pair_pos(i, j, n)] + dpsi;
            }
    }
    const double dt = p.dt;
    const int np = n * (n - 1) / 2;
    if (np == 1)
    {
        const Dual valueA = (pv[0] + 0.0) * dt;
        const Dual old_value = val[0];
        if ((old_value.v == 0.0 && valueA.v < 0.0) || (old_value.v == 1.0 && valueA.v > 0.0))
        {
            pv[0] = mkd(0.0);
        }
        else
        {
            const Dual new_value = old_value + valueA;
            Dual norm = mkd(1.0);
            if (new_value.v < 0.0) norm = norm * (-old_value / valueA);
            else if (new_value.v > 1.0) norm = norm * ((1.0 - old_value) / valueA);
            if (norm.v > DBL_EPSILON) pv[0] = pv[0] * norm;
            else pv[0] = mkd(0.0);
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
                dpsi += (i < j) ? pv[pair_pos(i, j, n)].v : pv[pair_pos(j, i, n)].v * (-1.0);
            }
            if ((val[i].v == 0.0 && dpsi < 0.0) || (val[i].v == 1.0 && dpsi > 0.0))
                for (int j = 0; j < n; j++)
                    if (j != i) pv[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = mkd(0.0);
        }
        bool any = false;
        for (int q = 0; q < np; q++) any |= (pv[q].v != 0.0);
        if (any)
        {
            for (int it = 1; it <= 25; it++)
            {
                for (int i = 0; i < n; i++) { pos[i] = mkd(0.0); neg[i] = mkd(0.0); }
                for (int i = 0; i < n; i++)
                    for (int j = i + 1; j < n; j++)
                    {
                        const Dual w = pv[pair_pos(i, j, n)];
                        if (w.v < 0.0) { neg[i] = neg[i] + w; pos[j] = pos[j] + (-w); }
                        if (w.v > 0.0) { pos[i] = pos[i] + w; neg[j] = neg[j] + (-w); }
                    }
                for (int i = 0; i < n; i++)
                {
                    const Dual vi = val[i], pi = pos[i], ni = neg[i];
                    const Dual newPF = vi + (pi + ni) * dt;
                    Dual limN = mkd(1.0), limP = mkd(1.0);
                    if (newPF.v < 0.0) limN = dmin_d(mkd(1.0), -(vi + pi * dt) / (ni * dt));
                    if (newPF.v > 1.0) limP = dmin_d(mkd(1.0), (1.0 - (vi + ni * dt)) / (pi * dt));
                    neg[i] = limN;
                    pos[i] = limP;
                }
                bool needed = false;
                for (int i = 0; i < n; i++)
                    for (int j = i + 1; j < n; j++)
                    {
                        const int q = pair_pos(i, j, n);
                        Dual w = pv[q];
                        if (w.v < 0.0)
                        {
                            const Dual lim = dmin_d(neg[i], pos[j]);
                            w = w * lim;
                            if (lim.v < 1.0) needed = true;
                        }
                        if (w.v > 0.0)
                        {
                            const Dual lim = dmin_d(pos[i], neg[j]);
                            w = w * lim;
                            if (lim.v < 1.0) needed = true;
                        }
                        pv[q] = w;
                    }
                if (!needed) break;
                if (it == 25) st |= kStLimiterCap;
            }
            for (int q = 0; q < np; q++)
                if (fabs(pv[q].v * dt) < DBL_EPSILON) pv[q] = mkd(0.0);
        }
    }
    for (int i = 0; i < n; i++) neg[i] = val[i];
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const Dual value = (1.0 * (pv[pair_pos(i, j, n)] + 0.0)) * dt;
            if (fabs(value.v) >= DBL_EPSILON)
            {
                neg[i] = neg[i] + value;
                neg[j] = neg[j] + (-value);
            }
        }
    const double hi_snap = 1.0 - p.eps_snap;
    const double lo_snap = 0.0 + p.eps_snap;
    Dual total = mkd(0.0);
    int m = 0;
    for (int i = 0; i < n; i++)
    {
        Dual w = neg[i];
        bool erase = false;
        if (w.v >= hi_snap) w = mkd(1.0);
        if (w.v <= lo_snap) { w = mkd(0.0); erase = true; }
        total = total + w;
        if (!erase)
        {
            g[m] = g[i];
            neg[m] = w;
            m++;
        }
    }
    if (m > 1)
    {
        const Dual norm = 1.0 / total;
        for (int i = 0; i < m; i++) val[i] = neg[i] * norm;
    }
    else if (m == 1)
    {
        val[0] = mkd(1.0);
    }
    else
    {
        st |= kStEmptyVoxel;
    }
    return m;
}

// Position of grain g in voxel u's stored list (-1 if absent).
__device__ __forceinline__ int find_entry(const uint8_t* cnt, const int16_t* idx, long long N, long long u, int g)
{
    const int c = cnt[u];
    for (int s = 0; s < c; s++)
        if (idx[s * N + u] == g) return s;
    return -1;
}

template <int KS, int KL>
__global__ void __launch_bounds__(128) tlm_step_kernel(const __grid_constant__ StepParams p, const StepArrays a,
                                                        const AdjArrays aa)
{
    __shared__ int s_key[kVolSlots];
    __shared__ double s_sum[kVolSlots];
    __shared__ unsigned long long s_cnt[3];
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0ull;
    __syncthreads();
    const long long N = p.n;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t st = 0;
    unsigned wide = 0, ein = 0, eout = 0;
    if (v < N)
    {
        const uint8_t* cnt = a.cnt_in;
        const int16_t* gin = a.idx_in;
        const double* vin = static_cast<const double*>(a.val_in);
        double* vout = static_cast<double*>(a.val_out);
        const Neighbourhood nb(p, v);
        const int c = cnt[v];
        ein = c;
        const int flag = voxel_flag(cnt, nb, v);
        if (flag == 0)
        {
            a.cnt_out[v] = (uint8_t)c;
            for (int s = 0; s < c; s++)
            {
                const int g = gin[s * N + v];
                a.idx_out[s * N + v] = (int16_t)g;
                vout[s * N + v] = vin[s * N + v];
                aa.dphi_out[s * N + v] = aa.dphi_in[s * N + v];
                vol_insert_n(s_key, s_sum, kVolSlots, a.vol_acc, g, vin[s * N + v]);
                atomicAdd(&aa.tvol[g], aa.dphi_in[s * N + v]);
            }
            eout = c;
        }
        else
        {
            wide = 1;
            constexpr int KP = KL * (KL - 1) / 2;
            int16_t gL[KL];
            double vr[KL], lr[KL];
            const int n = gather_list<double, KL>(p, cnt, gin, vin, nb, v, gL, vr, lr, nullptr, st);
            Dual val[KL], lap[KL], sg[KP], pv[KP], pos[KL], neg[KL];
            for (int k = 0; k < n; k++)
            {
                val[k] = mkd(vr[k], k < c ? aa.dphi_in[k * N + v] : 0.0);
                lap[k] = mkd(lr[k], 0.0);
            }
            // tangent of the Laplacians: the same stencil over the neighbours' tangents
            for (int q = 0; q < p.ns; q++)
            {
                const long long u = nb.at(p.lap_d[q][0], p.lap_d[q][1], p.lap_d[q][2]);
                const int cu = cnt[u];
                for (int s = 0; s < cu; s++)
                {
                    const int g = gin[s * N + u];
                    for (int k = 0; k < n; k++)
                        if (gL[k] == g) { lap[k].d += p.lap_w[q] * aa.dphi_in[s * N + u]; break; }
                }
            }
            int m = stages_dual<KL>(p, a, aa, n, flag, gL, val, lap, sg, pv, pos, neg, st);
            if (m > KS) { st |= kStOverflowK; m = KS; }
            a.cnt_out[v] = (uint8_t)m;
            for (int i = 0; i < m; i++)
            {
                a.idx_out[i * N + v] = gL[i];
                vout[i * N + v] = val[i].v;
                aa.dphi_out[i * N + v] = val[i].d;
                vol_insert_n(s_key, s_sum, kVolSlots, a.vol_acc, gL[i], val[i].v);
                atomicAdd(&aa.tvol[gL[i]], val[i].d);
            }
            eout = m;
        }
    }
    flush_block(a, wide, ein, eout, st, s_cnt, s_key, s_sum, kVolSlots, threadIdx.x, blockDim.x);
}

// ---- adjoint -------------------------------------------------------------------------------------
// One limiter iteration of NormalizeIncrementsSR (src/PhaseField.cpp:1447-1519) on pv (in place).
// Records the per-field sums and limits the reverse sweep needs.  Returns whether a limit < 1 acted.
__device__ __forceinline__ bool limiter_iteration(int n, const double* val, double dt, double* pv, double* pos,
                                                  double* neg, double* limN, double* limP)
{
    for (int i = 0; i < n; i++) { pos[i] = 0.0; neg[i] = 0.0; }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const double w = pv[pair_pos(i, j, n)];
            if (w < 0.0) { neg[i] += w; pos[j] += -w; }
            if (w > 0.0) { pos[i] += w; neg[j] += -w; }
        }
    for (int i = 0; i < n; i++)
    {
        const double vi = val[i], pi = pos[i], ni = neg[i];
        const double newPF = vi + (pi + ni) * dt;
        limN[i] = 1.0;
        limP[i] = 1.0;
        if (newPF < 0.0) limN[i] = dmin_ref(1.0, -(vi + pi * dt) / (ni * dt));
        if (newPF > 1.0) limP[i] = dmin_ref(1.0, (1.0 - (vi + ni * dt)) / (pi * dt));
    }
    bool needed = false;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            double w = pv[q];
            if (w < 0.0)
            {
                const double lim = dmin_ref(limN[i], limP[j]);
                w *= lim;
                if (lim < 1.0) needed = true;
            }
            if (w > 0.0)
            {
                const double lim = dmin_ref(limP[i], limN[j]);
                w *= lim;
                if (lim < 1.0) needed = true;
            }
            pv[q] = w;
        }
    return needed;
}

// Sums and limits of one limiter iteration for the increments pv (pv itself is not changed).
__device__ __forceinline__ void limiter_limits(int n, const double* val, double dt, const double* pv, double* pos,
                                               double* neg, double* limN, double* limP)
{
    for (int i = 0; i < n; i++) { pos[i] = 0.0; neg[i] = 0.0; }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const double w = pv[pair_pos(i, j, n)];
            if (w < 0.0) { neg[i] += w; pos[j] += -w; }
            if (w > 0.0) { pos[i] += w; neg[j] += -w; }
        }
    for (int i = 0; i < n; i++)
    {
        const double vi = val[i], pi = pos[i], ni = neg[i];
        const double newPF = vi + (pi + ni) * dt;
        limN[i] = 1.0;
        limP[i] = 1.0;
        if (newPF < 0.0) limN[i] = dmin_ref(1.0, -(vi + pi * dt) / (ni * dt));
        if (newPF > 1.0) limP[i] = dmin_ref(1.0, (1.0 - (vi + ni * dt)) / (pi * dt));
    }
}

// Reverse of one limiter iteration: pv_in is the input of the iteration (restored), lout the adjoint
// of its output; returns the adjoint of its input in lin and adds to lval.
__device__ void limiter_iteration_reverse(int n, const double* val, double dt, const double* pv_in,
                                          const double* lout, double* lin, double* lval, double* pos, double* neg,
                                          double* limN, double* limP, double* lpos, double* lneg)
{
    // forward quantities of this iteration
    limiter_limits(n, val, dt, pv_in, pos, neg, limN, limP);
    double llimN[KAdjList], llimP[KAdjList];
    for (int i = 0; i < n; i++) { llimN[i] = 0.0; llimP[i] = 0.0; lpos[i] = 0.0; lneg[i] = 0.0; }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            const double w = pv_in[q];
            if (w < 0.0)
            {
                const bool useP = limP[j] < limN[i];
                const double lim = useP ? limP[j] : limN[i];
                lin[q] = lout[q] * lim;
                if (useP) llimP[j] += lout[q] * w;
                else llimN[i] += lout[q] * w;
            }
            else if (w > 0.0)
            {
                const bool useN = limN[j] < limP[i];
                const double lim = useN ? limN[j] : limP[i];
                lin[q] = lout[q] * lim;
                if (useN) llimN[j] += lout[q] * w;
                else llimP[i] += lout[q] * w;
            }
            else
            {
                lin[q] = lout[q];
            }
        }
    for (int i = 0; i < n; i++)
    {
        const double vi = val[i], pi = pos[i], ni = neg[i];
        const double newPF = vi + (pi + ni) * dt;
        if (newPF < 0.0)
        {
            const double ratio = -(vi + pi * dt) / (ni * dt);
            if (ratio < 1.0 && llimN[i] != 0.0)
            {
                lval[i] += llimN[i] * (-1.0 / (ni * dt));
                lpos[i] += llimN[i] * (-1.0 / ni);
                lneg[i] += llimN[i] * ((vi + pi * dt) / (ni * ni * dt));
            }
        }
        if (newPF > 1.0)
        {
            const double ratio = (1.0 - (vi + ni * dt)) / (pi * dt);
            if (ratio < 1.0 && llimP[i] != 0.0)
            {
                lval[i] += llimP[i] * (-1.0 / (pi * dt));
                lneg[i] += llimP[i] * (-1.0 / pi);
                lpos[i] += llimP[i] * (-(1.0 - (vi + ni * dt)) / (pi * pi * dt));
            }
        }
    }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            const double w = pv_in[q];
            if (w < 0.0) lin[q] += lneg[i] - lpos[j];
            if (w > 0.0) lin[q] += lpos[i] - lneg[j];
        }
}

// The adjoint of one wide voxel's step, from its list (own fields first, then candidates) with the
// values and Laplacians the step used.  KL: capacity of the working arrays (the list-length
// kernels pass their exact length, so that every loop has a fixed trip count).
// R: the precision of the forward step's per-voxel arithmetic (the state's); the pair kinetics are
// recomputed in it, operation by operation as the forward kernels do (every unit compiled without
// contraction), so that the recomputed increments and every decision after them are the forward's.
template <int KL, int KS, class R = double>
__device__ __forceinline__ void adjoint_core(const StepParams& p, const StepArrays& a, const AdjArrays& aa,
                                             long long v, int flag, int n, int c, const int16_t* g0,
                                             const double* val_in, const double* lap_in, uint32_t st)
{
    constexpr int KP = KL * (KL - 1) / 2;
    const long long N = p.n;
    int16_t g[KL];
    double val[KL], lap[KL], lval[KL], llap[KL];
    for (int k = 0; k < n; k++)
    {
        g[k] = g0[k];
        val[k] = val_in[k];
        lap[k] = lap_in[k];
        lval[k] = 0.0;
        llap[k] = 0.0;
    }
    const int G = p.ngrains;
    const int np = n * (n - 1) / 2;
    const double dt = p.dt;
    // ---- forward recompute: pair kinetics (list_step order) ----
    double localN;
    if (p.consider_nucleus_volume)
    {
        localN = 0.0;
        for (int k = 0; k < n; k++) localN += a.vr[g[k]];
    }
    else
    {
        localN = (double)n;
    }
    const double norm_1 = 1.0 / localN;
    const double pref = p.pref_do;
    double psi[KP], pv0[KP], pv[KP], lpv[KP], lpw[KP];
    {
        // the forward's arithmetic in R (list_compute_kernel / warp_general_kernel / list_step)
        const R norm_1r = (R)(1.0 / localN);
        const R prefr = (R)p.pref_do;
        for (int i = 0; i < n; i++)
        {
            const double vri = a.vr[g[i]];
            const R vi = (R)val[i], li = (R)lap[i];
            for (int j = i + 1; j < n; j++)
            {
                const int q = pair_pos(i, j, n);
                const double vrj = a.vr[g[j]];
                const R scale = (vri == 1.0 && vrj == 1.0) ? R(1) : (R)sqrt(vri * vrj);
                const R h = R(0.5) * (R(1) + scale) * prefr;
                const R vj = (R)val[j];
                R dphi = (R)pair_energy(p, a, g[i], g[j]) * ((li + h * vi) - ((R)lap[j] + h * vj));
                if (n > 2)
                {
                    for (int k = 0; k < n; k++)
                    {
                        if (k == i || k == j) continue;
                        const R sbk = (R)pair_energy(p, a, g[j], g[k]);
                        const R sak = (R)pair_energy(p, a, g[i], g[k]);
                        const R vk = (R)val[k];
                        dphi += (sbk - sak) * ((R)lap[k] + h * vk);
                        if (p.tj_factor != 0.0 || scale < R(1))
                        {
                            const int pA = a.gphase[g[i]], pB = a.gphase[g[j]], pG = a.gphase[g[k]];
                            const int P = p.nphases;
                            const R tj = (R)dmax_ref(p.tj_factor, (double)(R(1) - scale));
                            dphi += tj * prefr
                                  * (((R)p.sigma_p[pA * P + pB] + (R)p.sigma_p[pB * P + pG]) + (R)p.sigma_p[pA * P + pG])
                                  * (vi * vk - vj * vk);
                        }
                    }
                }
                psi[q] = (double)dphi;
                dphi *= (R)pair_mobility(p, a, g[i], g[j]) * norm_1r * scale;
                pv0[q] = (double)dphi;
            }
        }
    }
    const bool with_dg = p.use_dg && flag == 2;
    if (with_dg)
    {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const double locdG = limited_force(p, a, g[i], g[j]);
                double norm = sqrt(val[i] * val[j]);
                if (a.gstage[g[i]] == 1 || a.gstage[g[j]] == 1) norm += 1.0e-6;
                pv0[pair_pos(i, j, n)] += locdG * (double)(R)pair_mobility(p, a, g[i], g[j]) * norm * p.pref_df;
            }
    }
    // ---- forward recompute: projection ----
    uint32_t zeroed = 0;       // fields whose increments the bound check zeroed
    int iters = 0;             // limiter iterations run
    bool single_clip = false;  // one pair: the increment was scaled onto the bound
    bool single_zero = false;
    double pos[KL], neg[KL], limN[KL], limP[KL], lpos[KL], lneg[KL];
    for (int q = 0; q < np; q++) pv[q] = pv0[q];
    if (np == 1)
    {
        const double valueA = (pv[0] + 0.0) * dt;
        const double old_value = val[0];
        if ((old_value == 0.0 && valueA < 0.0) || (old_value == 1.0 && valueA > 0.0))
        {
            pv[0] = 0.0;
            single_zero = true;
        }
        else
        {
            const double new_value = old_value + valueA;
            double norm = 1.0;
            if (new_value < 0.0) norm *= -old_value / valueA;
            else if (new_value > 1.0) norm *= (1.0 - old_value) / valueA;
            if (norm > DBL_EPSILON) { pv[0] *= norm; single_clip = norm != 1.0; }
            else { pv[0] = 0.0; single_zero = true; }
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
                dpsi += (i < j) ? pv[pair_pos(i, j, n)] : pv[pair_pos(j, i, n)] * (-1.0);
            }
            if ((val[i] == 0.0 && dpsi < 0.0) || (val[i] == 1.0 && dpsi > 0.0))
            {
                zeroed |= 1u << i;
                for (int j = 0; j < n; j++)
                    if (j != i) pv[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = 0.0;
            }
        }
        bool any = false;
        for (int q = 0; q < np; q++) any |= (pv[q] != 0.0);
        if (any)
        {
            for (int it = 1; it <= 25; it++)
            {
                iters = it;
                if (!limiter_iteration(n, val, dt, pv, pos, neg, limN, limP)) break;
            }
        }
    }
    uint64_t epsmask0 = 0, epsmask1 = 0;   // pairs dropped by |pv*dt| < DBL_EPSILON (after the limiter)
    if (np > 1 && iters > 0)
        for (int q = 0; q < np; q++)
            if (fabs(pv[q] * dt) < DBL_EPSILON)
            {
                pv[q] = 0.0;
                if (q < 64) epsmask0 |= 1ull << q; else epsmask1 |= 1ull << (q - 64);
            }
    // ---- forward recompute: merge and finalize ----
    double nv[KL];
    for (int i = 0; i < n; i++) nv[i] = val[i];
    uint64_t mm0 = 0, mm1 = 0;   // pairs the merge applied (|value| >= DBL_EPSILON)
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            const double value = 1.0 * (pv[q] + 0.0) * dt;
            if (fabs(value) >= DBL_EPSILON)
            {
                nv[i] += value;
                nv[j] += -value;
                if (q < 64) mm0 |= 1ull << q; else mm1 |= 1ull << (q - 64);
            }
        }
    const double hi_snap = 1.0 - p.eps_snap, lo_snap = 0.0 + p.eps_snap;
    double w[KL], total = 0.0;
    bool keep[KL], snap[KL];
    int m = 0;
    for (int i = 0; i < n; i++)
    {
        w[i] = nv[i];
        snap[i] = false;
        keep[i] = true;
        if (w[i] >= hi_snap) { w[i] = 1.0; snap[i] = true; }
        if (w[i] <= lo_snap) { w[i] = 0.0; keep[i] = false; snap[i] = true; }
        total += w[i];
        m += keep[i];
    }
    // ---- reverse: finalize (lambda of the kept outputs, in list order) ----
    double lnv[KL];
    for (int i = 0; i < n; i++) lnv[i] = 0.0;
    {
        // the adjoint of each kept field, found by grain in the stored next state (the lists agree
        // entry by entry when the recomputed step reproduces the stored one).  Finalize stores the
        // kept fields in list order, so the k-th kept field is looked up at entry k first and
        // searched for only when that entry holds another grain.
        const int c1 = aa.cnt1[v];
        double lout[KL];
        int kept = 0;
        for (int i = 0; i < n; i++)
        {
            lout[i] = 0.0;
            if (!keep[i]) continue;
            int s1 = (kept < c1 && aa.idx1[kept * N + v] == g[i]) ? kept : -1;
            if (s1 < 0) s1 = find_entry(aa.cnt1, aa.idx1, N, v, g[i]);
            kept++;
            if (s1 >= 0) lout[i] = aa.lam1[s1 * N + v];
            else st |= kStAdjointMismatch;
        }
        if (m != c1 && !(m > KS && c1 == KS)) st |= kStAdjointMismatch;
        if (m > 1)
        {
            double s = 0.0;
            for (int k = 0; k < n; k++)
                if (keep[k]) s += lout[k] * w[k];
            const double it = 1.0 / total;
            for (int i = 0; i < n; i++)
                if (keep[i] && !snap[i]) lnv[i] = lout[i] * it - s * it * it;
        }
    }
    // ---- reverse: merge ----
    for (int i = 0; i < n; i++) lval[i] += lnv[i];
    for (int q = 0; q < np; q++) lpv[q] = 0.0;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            const bool applied = q < 64 ? ((mm0 >> q) & 1ull) : ((mm1 >> (q - 64)) & 1ull);
            if (applied) lpv[q] = (lnv[i] - lnv[j]) * dt;
        }
    // ---- reverse: projection ----
    if (np == 1)
    {
        if (single_zero) lpv[0] = 0.0;
        else if (single_clip)
        {
            // pv*norm = -old/dt (lower bound) or (1-old)/dt (upper bound): depends on the old value only
            lval[0] += lpv[0] * (-1.0 / dt);
            lpv[0] = 0.0;
        }
    }
    else if (np > 1)
    {
        for (int q = 0; q < np; q++)
        {
            const bool dropped = q < 64 ? ((epsmask0 >> q) & 1ull) : ((epsmask1 >> (q - 64)) & 1ull);
            if (dropped) lpv[q] = 0.0;
        }
        // limiter iterations in reverse; the input of iteration r is rebuilt from the zeroed increments
        double* pin = pv;   // the forward's increments are no longer needed
        for (int r = iters; r >= 1; r--)
        {
            for (int q = 0; q < np; q++) pin[q] = pv0[q];
            for (int i = 0; i < n; i++)
                if ((zeroed >> i) & 1u)
                    for (int j = 0; j < n; j++)
                        if (j != i) pin[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = 0.0;
            for (int s = 1; s < r; s++) limiter_iteration(n, val, dt, pin, pos, neg, limN, limP);
            limiter_iteration_reverse(n, val, dt, pin, lpv, lpw, lval, pos, neg, limN, limP, lpos, lneg);
            for (int q = 0; q < np; q++) lpv[q] = lpw[q];
        }
        for (int i = 0; i < n; i++)
            if ((zeroed >> i) & 1u)
                for (int j = 0; j < n; j++)
                    if (j != i) lpv[i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)] = 0.0;
    }
    // ---- reverse: driving force ----
    if (with_dg)
    {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
            {
                const int q = pair_pos(i, j, n);
                if (lpv[q] == 0.0) continue;
                const double F = limited_force(p, a, g[i], g[j]);
                const double mob = pair_mobility(p, a, g[i], g[j]);
                const double s = sqrt(val[i] * val[j]);
                double norm = s;
                if (a.gstage[g[i]] == 1 || a.gstage[g[j]] == 1) norm += 1.0e-6;
                const long long key = pair_key(g[i], g[j], G);
                atomicAdd(&aa.gmu[key], lpv[q] * F * norm * p.pref_df);
                const double lF = lpv[q] * mob * norm * p.pref_df;
                const double dFb = lF * force_slope(p, a, g[i], g[j], F);
                atomicAdd(&aa.gdg[g[j]], dFb);
                atomicAdd(&aa.gdg[g[i]], -dFb);
                if (s > 0.0)
                {
                    const double ln = lpv[q] * F * mob * p.pref_df;
                    lval[i] += ln * val[j] / (2.0 * s);
                    lval[j] += ln * val[i] / (2.0 * s);
                }
            }
    }
    // ---- reverse: pair kinetics ----
    for (int i = 0; i < n; i++)
    {
        const double vri = a.vr[g[i]];
        for (int j = i + 1; j < n; j++)
        {
            const int q = pair_pos(i, j, n);
            if (lpv[q] == 0.0) continue;
            const double vrj = a.vr[g[j]];
            const double scale = (vri == 1.0 && vrj == 1.0) ? 1.0 : sqrt(vri * vrj);
            const double h = 0.5 * (1.0 + scale) * pref;
            const double mob = pair_mobility(p, a, g[i], g[j]);
            const long long key = pair_key(g[i], g[j], G);
            atomicAdd(&aa.gmu[key], lpv[q] * psi[q] * norm_1 * scale);
            const double lpsi = lpv[q] * mob * norm_1 * scale;
            const double sij = pair_energy(p, a, g[i], g[j]);
            atomicAdd(&aa.gsig[key], lpsi * ((lap[i] + h * val[i]) - (lap[j] + h * val[j])));
            llap[i] += lpsi * sij; lval[i] += lpsi * sij * h;
            llap[j] -= lpsi * sij; lval[j] -= lpsi * sij * h;
            if (n > 2)
            {
                for (int k = 0; k < n; k++)
                {
                    if (k == i || k == j) continue;
                    const double sbk = pair_energy(p, a, g[j], g[k]);
                    const double sak = pair_energy(p, a, g[i], g[k]);
                    const double Sk = lap[k] + h * val[k];
                    atomicAdd(&aa.gsig[pair_key(g[j], g[k], G)], lpsi * Sk);
                    atomicAdd(&aa.gsig[pair_key(g[i], g[k], G)], -lpsi * Sk);
                    llap[k] += lpsi * (sbk - sak);
                    lval[k] += lpsi * (sbk - sak) * h;
                    if (p.tj_factor != 0.0 || scale < 1.0)
                    {
                        const int pA = a.gphase[g[i]], pB = a.gphase[g[j]], pG = a.gphase[g[k]];
                        const int P = p.nphases;
                        const double tj = dmax_ref(p.tj_factor, 1.0 - scale);
                        const double ck = tj * pref * ((p.sigma_p[pA * P + pB] + p.sigma_p[pB * P + pG]) + p.sigma_p[pA * P + pG]);
                        lval[i] += lpsi * ck * val[k];
                        lval[j] -= lpsi * ck * val[k];
                        lval[k] += lpsi * ck * (val[i] - val[j]);
                    }
                }
            }
        }
    }
    // ---- outputs ----
    for (int s = 0; s < c; s++) aa.lam_local[s * N + v] = lval[s];
    aa.lcnt[v] = (uint8_t)n;
    for (int k = 0; k < n; k++)
    {
        aa.lidx[k * N + v] = g0[k];
        aa.llam[k * N + v] = llap[k];
    }
    if (st) atomicOr(a.status, st);
}


// Bulk voxels of the state before the step are carried over unchanged: identity adjoint.  (The
// wide voxels are left to the list-length kernels and the worklist kernel.)
__global__ void adjoint_bulk_kernel(const __grid_constant__ StepParams p, const uint8_t* __restrict__ cnt,
                                    const AdjArrays aa)
{
    const long long N = p.n;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const Neighbourhood nb(p, v);
    if (voxel_flag(cnt, nb, v) != 0) return;
    const int c = cnt[v];
    for (int s = 0; s < c; s++) aa.lam_local[s * N + v] = aa.lam1[s * N + v];
    aa.lcnt[v] = 0;
}

// Wide voxels whose list has N fields, from the classify kernel's work records (the lists, values
// and Laplacians the forward step used; own fields are the leading nonzero values).
template <class R, int N, int KS>
__global__ void __launch_bounds__(128) adjoint_list_kernel(const __grid_constant__ StepParams p, const StepArrays a,
                                                            const AdjArrays aa, int nslices)
{
    // the entries of length N from all classify slices form one index range, split evenly in whole
    // multiples of the block size (every thread of a block that has work gets some)
    const unsigned* __restrict__ off = a.bucket_off + (long long)N * (nslices + 1);
    const unsigned total = off[nslices];
    const unsigned per = ((total + gridDim.x * blockDim.x - 1u) / (gridDim.x * blockDim.x)) * blockDim.x;
    const unsigned r0 = blockIdx.x * per;
    if (r0 >= total) return;
    const unsigned r1 = min(total, r0 + per);
    const int2* __restrict__ buck = a.bucket + (long long)N * a.bucket_cap;
    constexpr int kPad = ((2 * N + 7) / 8) * 8;
    for (unsigned e = r0 + threadIdx.x; e < r1; e += blockDim.x)
    {
        const int sl = slice_of(off, nslices, e);
        const int2 ent = buck[(long long)sl * a.slice + (e - off[sl])];
        const unsigned char* __restrict__ wbase = a.wl + (long long)sl * a.wl_slice;
        const long long v = ent.x & 0x7fffffff;
        const int flag = (ent.x >> 31) ? 2 : 1;
        const int16_t* __restrict__ rg = reinterpret_cast<const int16_t*>(wbase + ent.y);
        const R* __restrict__ rv = reinterpret_cast<const R*>(wbase + ent.y + kPad);
        int16_t g[N];
        double val[N], lap[N];
        int c = 0;
        bool own = true;
#pragma unroll
        for (int k = 0; k < N; k++)
        {
            g[k] = rg[k];
            val[k] = (double)rv[k];
            lap[k] = (double)rv[N + k];
            own = own && val[k] != 0.0;
            c += own ? 1 : 0;
        }
        adjoint_core<N, KS, R>(p, a, aa, v, flag, N, c, g, val, lap, 0u);
    }
}

// Wide voxels of the classify kernel's general-path worklist: the general gather, then the core.
template <class R, int KS>
__global__ void __launch_bounds__(64) adjoint_worklist_kernel(const __grid_constant__ StepParams p, const StepArrays a,
                                                               const AdjArrays aa)
{
    constexpr int KL = KAdjList;
    const unsigned total = min(*a.slow_count, a.slow_cap);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
    {
        const long long v = a.slow_list[i];
        const Neighbourhood nb(p, v);
        const int c = a.cnt_in[v];
        const int flag = voxel_flag(a.cnt_in, nb, v);
        uint32_t st = 0;
        int16_t g[KL];
        R vr[KL], lr[KL];
        const int n = gather_list<R, KL>(p, a.cnt_in, a.idx_in, static_cast<const R*>(a.val_in), nb, v, g, vr, lr,
                                         nullptr, st);
        double val[KL], lap[KL];
        for (int k = 0; k < n; k++) { val[k] = (double)vr[k]; lap[k] = (double)lr[k]; }
        adjoint_core<KL, KS, R>(p, a, aa, v, flag, n, c, g, val, lap, st);
    }
}

// lambda_t(u, s) = own part + sum_q w_q * (adjoint of the Laplacian of grain g_s at u - d_q)
//
// The adjoints of the Laplacians form ragged lists (lcnt, lidx, llam) in the slot-planar layout of
// a state, so the transposed stencil is evaluated like the forward Laplacians: the classify
// kernel's plane loader brings three x-planes of those lists into dense per-slot planes, and every
// entry of the centre voxel sums w_q * dense[slot(g_s)][u - d_q] in stencil order (absent grains
// read zeros, which leave the sum unchanged).  Voxels next to a list grain without a window slot
// take the same sum from global memory.

// Neighbour u - d without indexing the offset arrays by a runtime value (selects only).
__device__ __forceinline__ long long nb_back(const Neighbourhood& nb, const signed char* d)
{
    const long long x = d[0] > 0 ? nb.X[0] : (d[0] < 0 ? nb.X[2] : nb.X[1]);
    const long long y = d[1] > 0 ? nb.Y[0] : (d[1] < 0 ? nb.Y[2] : nb.Y[1]);
    const long long z = d[2] > 0 ? nb.Z[0] : (d[2] < 0 ? nb.Z[2] : nb.Z[1]);
    return x + y + z;
}

__device__ __forceinline__ double gather_global(const StepParams& p, const AdjArrays& aa, const Neighbourhood& nb,
                                                int g, double l)
{
    const long long N = p.n;
    for (int q = 0; q < p.ns; q++)
    {
        const long long v = nb_back(nb, p.lap_d[q]);
        const int lc = aa.lcnt[v];
        for (int k = 0; k < lc; k++)
            if (aa.lidx[k * N + v] == g) { l += p.lap_w[q] * aa.llam[k * N + v]; break; }
    }
    return l;
}

template <int KS, int NS>
__global__ void __launch_bounds__(kTileZ * kTileTY)
adjoint_gather_kernel(const __grid_constant__ StepParams p, const StepArrays la, const uint8_t* __restrict__ cnt,
                      const int16_t* __restrict__ idx, const AdjArrays aa, double* __restrict__ lam0, int xchunk)
{
    constexpr int TY = kTileTY;
    using Geo = TileGeom<TY>;
    using Smem = TileSmem<double, KS, TY>;
    constexpr int NT = Geo::NT;
    constexpr int kC = Geo::kCols;
    constexpr int kSlots = WindowSlots<double>::value;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);

    const int tz = threadIdx.x, ty = threadIdx.y, t = ty * kTileZ + tz;
    const int z0 = blockIdx.x * kTileZ, y0 = blockIdx.y * TY, x0 = blockIdx.z * xchunk;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x1 = min(x0 + xchunk, nx);
    const long long N = p.n;
    const long long plane = (long long)ny * nz;
    const int z = z0 + tz, y = y0 + ty;
    const bool inside = (z < nz) && (y < ny);

    for (int i = t; i < kSlots * 3 * Geo::kRecs; i += NT) (&S.dense[0][0][0])[i] = 0.0;
    for (int i = t; i < 3 * Geo::kRecs; i += NT) (&S.word[0][0])[i] = 0u;
    if (t < kSlots) { S.grain_of[t] = -1; S.lastpos[t] = -1000; }
    if (t < kSlotHash) S.hkey[t] = -1;
    if (t < 32) S.pending[t] = -1;
    if (t == 0) S.tomb = 0;
    int cr[PlaneRegs<TY>::kPer];
    prefetch_counts<TY>(p, la, x0 == 0 ? nx - 1 : x0 - 1, y0, z0, t, cr);
    __syncthreads();

    const int rec0 = (ty + 1) * kC + (tz + 1);
    const int nj = (x1 - x0) + 2;
    for (int j = 0; j < nj; j++)
    {
        int xp = x0 - 1 + j;
        xp = xp < 0 ? xp + nx : (xp >= nx ? xp - nx : xp);
        if (j > 0) __syncthreads();
        load_plane(p, la, S, j % 3, xp, j - 1, y0, z0, t, cr);
        __syncthreads();
        if (j < 2 || !inside) continue;
        const int x = x0 + j - 2;
        const int sl0 = (j - 2) % 3, sl1 = (j - 1) % 3, sl2 = j % 3;
        const long long u = (long long)x * plane + (long long)y * nz + z;
        // a list grain of a stencil neighbour without a window slot: the global sum
        bool crowded = false;
#pragma unroll
        for (int q = 0; q < NS; q++)
        {
            const int dx = stencil_dx<NS>(q);
            const int pl = dx > 0 ? sl0 : (dx < 0 ? sl2 : sl1);
            const int r = rec0 - stencil_dy<NS>(q) * kC - stencil_dz<NS>(q);
            crowded |= ((S.word[pl][r] >> 30) & 1u) != 0u;
        }
        const int c = cnt[u];
        for (int s = 0; s < c; s++)
        {
            const int g = idx[s * N + u];
            double l = aa.lam_local[s * N + u];
            if (crowded)
            {
                const Neighbourhood nb(p, u);
                l = gather_global(p, aa, nb, g, l);
            }
            else
            {
                const int k = find_slot(S.hkey, S.hslot, g);
                if (k >= 0)
                {
#pragma unroll
                    for (int q = 0; q < NS; q++)
                    {
                        const int dx = stencil_dx<NS>(q);
                        const int pl = dx > 0 ? sl0 : (dx < 0 ? sl2 : sl1);
                        const int r = rec0 - stencil_dy<NS>(q) * kC - stencil_dz<NS>(q);
                        l += p.lap_w[q] * S.dense[k][pl][r];
                    }
                }
            }
            lam0[s * N + u] = l;
        }
    }
}

template <int KS, int NS>
static int launch_gather_ns(const StepParams& p, const StepArrays& a, const AdjArrays& aa, double* lam0, cudaStream_t s)
{
    using Smem = TileSmem<double, KS, kTileTY>;
    int xchunk = 0, gz = 0, gy = 0, gx = 0;
    tiled_geometry(p.nx, p.ny, p.nz, &xchunk, &gz, &gy, &gx);
    StepArrays la = a;   // the plane loader reads the lists of the Laplacian adjoints
    la.cnt_in = aa.lcnt;
    la.idx_in = aa.lidx;
    la.val_in = aa.llam;
    auto kern = adjoint_gather_kernel<KS, NS>;
    const size_t smem = sizeof(Smem);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    kern<<<dim3(gz, gy, gx), dim3(kTileZ, kTileTY), smem, s>>>(p, la, a.cnt_in, a.idx_in, aa, lam0, xchunk);
    return (int)cudaGetLastError();
}

template <int KS>
static int launch_gather(const StepParams& p, const StepArrays& a, const AdjArrays& aa, double* lam0, cudaStream_t s)
{
    if (p.ns == 27) return launch_gather_ns<KS, 27>(p, a, aa, lam0, s);
    if (p.ns == 7) return launch_gather_ns<KS, 7>(p, a, aa, lam0, s);
    return -1;
}

__global__ void lambda_init_kernel(long long N, const uint8_t* __restrict__ cnt, const int16_t* __restrict__ idx,
                                   const double* __restrict__ dLdV, double* __restrict__ lam)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int c = cnt[v];
    for (int s = 0; s < c; s++) lam[s * N + v] = dLdV[idx[s * N + v]];
}

static unsigned grid_of(long long n, int t) { return (unsigned)((n + t - 1) / t); }

int launch_tlm_step(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int k_slots, void* stream)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (k_slots)
    {
        case 8:  tlm_step_kernel<8, KAdjList><<<grid_of(p.n, 128), 128, 0, s>>>(p, a, aa); break;
        case 12: tlm_step_kernel<12, KAdjList><<<grid_of(p.n, 128), 128, 0, s>>>(p, a, aa); break;
        case 16: tlm_step_kernel<16, KAdjList><<<grid_of(p.n, 128), 128, 0, s>>>(p, a, aa); break;
        default: return -1;
    }
    return (int)cudaGetLastError();
}

constexpr int kAdjListBlocks = 148 * 32;   // blocks of each per-length adjoint kernel

// The worklist kernel (few voxels, each a long serial chain) runs on the side stream, launched
// first, so that it overlaps the list-length kernels instead of adding its latency after them.
template <class R, int KS>
static void adjoint_kernels(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int nblocks, cudaStream_t s,
                            cudaStream_t side)
{
    adjoint_worklist_kernel<R, KS><<<148 * 4, 64, 0, side>>>(p, a, aa);
    adjoint_list_kernel<R, 2, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 3, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 4, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 5, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 6, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 7, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
    adjoint_list_kernel<R, 8, KS><<<kAdjListBlocks, 128, 0, s>>>(p, a, aa, nblocks);
}

int launch_adjoint_step(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int k_slots, bool fp32,
                        int nblocks, double* lam0, void* stream, const AdjStreams& fork)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStream_t side = fork.side ? static_cast<cudaStream_t>(fork.side) : s;
    adjoint_bulk_kernel<<<grid_of(p.n, 256), 256, 0, s>>>(p, a.cnt_in, aa);
    cudaError_t e;
    if (side != s)
    {
        if ((e = cudaEventRecord(static_cast<cudaEvent_t>(fork.ev_fork), s)) != cudaSuccess) return (int)e;
        if ((e = cudaStreamWaitEvent(side, static_cast<cudaEvent_t>(fork.ev_fork), 0)) != cudaSuccess) return (int)e;
    }
    switch (k_slots * 2 + (fp32 ? 1 : 0))
    {
        case 16: adjoint_kernels<double, 8>(p, a, aa, nblocks, s, side); break;
        case 17: adjoint_kernels<float, 8>(p, a, aa, nblocks, s, side); break;
        case 24: adjoint_kernels<double, 12>(p, a, aa, nblocks, s, side); break;
        case 25: adjoint_kernels<float, 12>(p, a, aa, nblocks, s, side); break;
        case 32: adjoint_kernels<double, 16>(p, a, aa, nblocks, s, side); break;
        case 33: adjoint_kernels<float, 16>(p, a, aa, nblocks, s, side); break;
        default: return -1;
    }
    if (side != s)
    {
        if ((e = cudaEventRecord(static_cast<cudaEvent_t>(fork.ev_join), side)) != cudaSuccess) return (int)e;
        if ((e = cudaStreamWaitEvent(s, static_cast<cudaEvent_t>(fork.ev_join), 0)) != cudaSuccess) return (int)e;
    }
    int rc = -1;
    switch (k_slots)
    {
        case 8:  rc = launch_gather<8>(p, a, aa, lam0, s); break;
        case 12: rc = launch_gather<12>(p, a, aa, lam0, s); break;
        case 16: rc = launch_gather<16>(p, a, aa, lam0, s); break;
        default: return -1;
    }
    if (rc != 0) return rc;
    return (int)cudaGetLastError();
}

int launch_lambda_init(long long n, const uint8_t* cnt, const int16_t* idx, const double* dLdV, double* lam,
                       void* stream)
{
    lambda_init_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, cnt, idx, dLdV, lam);
    return (int)cudaGetLastError();
}

}  // namespace opgpu
