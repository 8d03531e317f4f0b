// Tiled form of the fused step (the production path).
//
// A block owns a (y, z) tile of TY x 32 voxels and marches along x over `xchunk` planes.  The 3x3x3
// neighbourhoods come from a ring of three x-planes held in shared memory (tile plus a one-voxel
// halo in y and z, periodic wrap by index arithmetic); only the first KT stored slots of a record
// are staged, the rare deeper slots are read from global memory.  Every plane goes through
//
//   A  (thread per voxel)   flag from the 27 neighbour counts; bulk voxels are copied straight to
//                           the output; interface voxels build their field + candidate list with
//                           Laplacians in registers (capacity NF) and park it in shared memory.
//                           Lists longer than NF go to the overflow worklist (generic kernel).
//   B  (thread per list)    lists are bucketed by length so that each warp runs one
//                           length-specialised, fully unrolled path for the pair kinetics,
//                           driving force, projection, merge and finalize (registers only).
//   C  (thread per voxel)   the new records are written back coalesced and the grain volumes
//                           are accumulated in a per-block shared-memory table.
//
// The per-voxel arithmetic and its operation order are those of voxel_step_generic (and of the
// reference), so both kernels give bit-identical FP64 results.
#pragma once
#include "step_kernel.cuh"

namespace opgpu {

constexpr int kTileZ = 32;
constexpr int kTileVolSlots = 512;

template <class R, int KT, int TY>
struct TileRing {
    static constexpr int kRows = TY + 2;
    static constexpr int kCols = kTileZ + 2;
    static constexpr int kRecs = kRows * kCols;
    R phi[3][KT][kRecs];
    int16_t g[3][KT][kRecs];
    uint8_t cnt[3][kRecs];
};

template <class R, int NF, int NT>
struct TileLists {
    R val[NF][NT];
    R lap[NF][NT];
    int16_t g[NF][NT];
    uint16_t perm[NT];
    uint8_t n[NT];      // 0 = bulk / outside, 1..NF = list length, 255 = overflow worklist
    uint8_t flag[NT];
    uint8_t m[NT];      // entries of the new record
};

template <class R, int KT, int NF, int TY>
struct TileSmem {
    TileRing<R, KT, TY> ring;
    TileLists<R, NF, 32 * TY> lists;
    double vol_sum[kTileVolSlots];
    int vol_key[kTileVolSlots];
    unsigned bucket[NF + 2];
    unsigned base[NF + 2];
    unsigned long long cnt[3];
};

__device__ __forceinline__ void tile_vol_insert(int* keys, double* sums, double* global_acc, int g, double v)
{
    unsigned h = ((unsigned)g * 2654435761u) & (kTileVolSlots - 1);
    for (int probe = 0; probe < kTileVolSlots; probe++)
    {
        const int k = atomicCAS(&keys[h], -1, g);
        if (k == -1 || k == g)
        {
            atomicAdd(&sums[h], v);
            return;
        }
        h = (h + 1) & (kTileVolSlots - 1);
    }
    atomicAdd(&global_acc[g], v);
}

// Stages 2-6 for a list of exactly N entries (compile-time), all arrays in registers.  Writes the
// new record (m entries, in list order) into the shared-memory list of the voxel; returns m.
template <class R, int N, int NF, int NT>
__device__ __forceinline__ int process_list(const StepParams& p, const StepArrays& a, TileLists<R, NF, NT>& L,
                                            int t, int flag, uint32_t& st)
{
    constexpr int NP = N * (N - 1) / 2;
    int g[N];
    R val[N], lap[N];
#pragma unroll
    for (int k = 0; k < N; k++)
    {
        g[k] = L.g[k][t];
        val[k] = L.val[k][t];
        lap[k] = L.lap[k][t];
    }
    // ---- pair kinetics (DoubleObstacle::CalculatePhaseFieldIncrementsSR) ----------------------
    double localN;
    if (p.consider_nucleus_volume)
    {
        localN = 0.0;
#pragma unroll
        for (int k = 0; k < N; k++) localN += a.vr[g[k]];
    }
    else
    {
        localN = (double)N;
    }
    const R norm_1 = (R)(1.0 / localN);
    R sg[NP > 0 ? NP : 1];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i + 1; j < N; j++) sg[pair_pos(i, j, N)] = (R)pair_energy(p, a, g[i], g[j]);
    const R pref = (R)p.pref_do;
    double pv[NP > 0 ? NP : 1];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i + 1; j < N; j++)
        {
            const int q = pair_pos(i, j, N);
            const R scale = (R)sqrt(a.vr[g[i]] * a.vr[g[j]]);
            const R h = R(0.5) * (R(1) + scale) * pref;
            R dphi = sg[q] * ((lap[i] + h * val[i]) - (lap[j] + h * val[j]));
            if (N > 2)
            {
#pragma unroll
                for (int k = 0; k < N; k++)
                {
                    if (k == i || k == j) continue;
                    const R sbk = sg[j < k ? pair_pos(j, k, N) : pair_pos(k, j, N)];
                    const R sak = sg[i < k ? pair_pos(i, k, N) : pair_pos(k, i, N)];
                    dphi += (sbk - sak) * (lap[k] + h * val[k]);
                    if (p.tj_factor != 0.0 || scale < R(1))
                    {
                        const int pA = a.gphase[g[i]], pB = a.gphase[g[j]], pG = a.gphase[g[k]];
                        const int P = p.nphases;
                        const R tj = (R)dmax_ref(p.tj_factor, (double)(R(1) - scale));
                        dphi += tj * pref
                              * (((R)p.sigma_p[pA * P + pB] + (R)p.sigma_p[pB * P + pG]) + (R)p.sigma_p[pA * P + pG])
                              * (val[i] * val[k] - val[j] * val[k]);
                    }
                }
            }
            dphi *= (R)pair_mobility(p, a, g[i], g[j]) * norm_1 * scale;
            pv[q] = (double)dphi;
        }
    // ---- driving force (DrivingForce::MergePhaseFieldIncrementsSR), interface voxels ---------
    if (p.use_dg && flag == 2)
    {
        const int P = p.nphases;
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i + 1; j < N; j++)
            {
                const int q = pair_pos(i, j, N);
                double locdG = a.dg[g[j]] - a.dg[g[i]];
                double norm = sqrt((double)val[i] * (double)val[j]);
                if (a.gstage[g[i]] == 1 || a.gstage[g[j]] == 1) norm += 1.0e-6;
                if (p.limiting)
                {
                    const double allowed = p.allowed_p[a.gphase[g[i]] * P + a.gphase[g[j]]];
                    locdG = allowed * tanh(locdG / allowed);
                }
                const double dpsi = locdG * (double)(R)pair_mobility(p, a, g[i], g[j]) * norm * p.pref_df;
                pv[q] += dpsi;
            }
    }
    // ---- projection (PhaseField::NormalizeIncrementsSR) ---------------------------------------
    const double dt = p.dt;
    if (NP == 1)
    {
        const double valueA = (pv[0] + 0.0) * dt;
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
    else if (NP > 1)
    {
#pragma unroll
        for (int i = 0; i < N; i++)
        {
            double dpsi = 0.0;
#pragma unroll
            for (int j = 0; j < N; j++)
            {
                if (j == i) continue;
                dpsi += (i < j) ? pv[pair_pos(i, j, N)] : pv[pair_pos(j, i, N)] * (-1.0);
            }
            if (((double)val[i] == 0.0 && dpsi < 0.0) || ((double)val[i] == 1.0 && dpsi > 0.0))
            {
#pragma unroll
                for (int j = 0; j < N; j++)
                {
                    if (j == i) continue;
                    pv[i < j ? pair_pos(i, j, N) : pair_pos(j, i, N)] = 0.0;
                }
            }
        }
        bool any = false;
#pragma unroll
        for (int q = 0; q < NP; q++) any |= (pv[q] != 0.0);
        if (any)
        {
            for (int it = 1; it <= 25; it++)
            {
                double pos[N], neg[N];
#pragma unroll
                for (int i = 0; i < N; i++) { pos[i] = 0.0; neg[i] = 0.0; }
#pragma unroll
                for (int i = 0; i < N; i++)
#pragma unroll
                    for (int j = i + 1; j < N; j++)
                    {
                        const double w = pv[pair_pos(i, j, N)];
                        if (w < 0.0) { neg[i] += w; pos[j] += -w; }
                        if (w > 0.0) { pos[i] += w; neg[j] += -w; }
                    }
                // limits (pos/neg reused as the positive / negative limit of each field)
#pragma unroll
                for (int i = 0; i < N; i++)
                {
                    const double vi = (double)val[i];
                    const double newPF = vi + (pos[i] + neg[i]) * dt;
                    double limN = 1.0, limP = 1.0;
                    if (newPF < 0.0) limN = dmin_ref(1.0, -(vi + pos[i] * dt) / (neg[i] * dt));
                    if (newPF > 1.0) limP = dmin_ref(1.0, (1.0 - (vi + neg[i] * dt)) / (pos[i] * dt));
                    neg[i] = limN;
                    pos[i] = limP;
                }
                bool needed = false;
#pragma unroll
                for (int i = 0; i < N; i++)
#pragma unroll
                    for (int j = i + 1; j < N; j++)
                    {
                        const int q = pair_pos(i, j, N);
                        if (pv[q] < 0.0)
                        {
                            const double lim = dmin_ref(neg[i], pos[j]);
                            pv[q] *= lim;
                            if (lim < 1.0) needed = true;
                        }
                        if (pv[q] > 0.0)
                        {
                            const double lim = dmin_ref(pos[i], neg[j]);
                            pv[q] *= lim;
                            if (lim < 1.0) needed = true;
                        }
                    }
                if (!needed) break;
                if (it == 25) st |= kStLimiterCap;
            }
#pragma unroll
            for (int q = 0; q < NP; q++)
                if (fabs(pv[q] * dt) < DBL_EPSILON) pv[q] = 0.0;
            // plausibility check (a warning in the reference)
            double chk[N];
#pragma unroll
            for (int i = 0; i < N; i++) chk[i] = (double)val[i];
#pragma unroll
            for (int i = 0; i < N; i++)
#pragma unroll
                for (int j = i + 1; j < N; j++)
                {
                    const double w = pv[pair_pos(i, j, N)];
                    if (w != 0.0) { chk[i] += w * dt; chk[j] += -w * dt; }
                }
#pragma unroll
            for (int i = 0; i < N; i++)
                if (chk[i] < -(double)FLT_EPSILON || chk[i] > 1.0 + (double)FLT_EPSILON) st |= kStNormalizeWarn;
        }
    }
    // ---- merge (accumulated in FP64; the FP32 form rounds only when the record is stored) ---------
    double vd[N];
#pragma unroll
    for (int i = 0; i < N; i++) vd[i] = (double)val[i];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i + 1; j < N; j++)
        {
            const double value = 1.0 * (pv[pair_pos(i, j, N)] + 0.0) * dt;
            if (fabs(value) >= DBL_EPSILON)
            {
                vd[i] += value;
                vd[j] += -value;
            }
        }
    // ---- finalize (NodePF::finalize) -----------------------------------------------------------
    const double hi_snap = 1.0 - p.eps_snap;
    const double lo_snap = 0.0 + p.eps_snap;
    double total = 0.0;
    int m = 0;
    bool keep[N];
#pragma unroll
    for (int i = 0; i < N; i++)
    {
        double w = vd[i];
        keep[i] = true;
        if (w >= hi_snap) w = 1.0;
        if (w <= lo_snap) { w = 0.0; keep[i] = false; }
        total += w;
        vd[i] = w;
        m += keep[i];
    }
    const double norm = 1.0 / total;
    int pos = 0;
#pragma unroll
    for (int i = 0; i < N; i++)
    {
        if (keep[i])
        {
            const R w = (m > 1) ? (R)(vd[i] * norm) : R(1);
            if (!isfinite((double)w)) st |= kStNonFinite;
            L.g[pos][t] = (int16_t)g[i];
            L.val[pos][t] = w;
            pos++;
        }
    }
    if (m == 0) st |= kStEmptyVoxel;
    return m;
}

template <class R, int KT, int TY>
__device__ __forceinline__ void load_plane(const StepParams& p, const StepArrays& a, TileRing<R, KT, TY>& ring,
                                           int slot, int xp, int y0, int z0, int t, int nt)
{
    using Ring = TileRing<R, KT, TY>;
    const long long N = p.n;
    const long long base = (long long)xp * p.ny * p.nz;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    for (int r = t; r < Ring::kRecs; r += nt)
    {
        const int row = r / Ring::kCols, col = r - (r / Ring::kCols) * Ring::kCols;
        int yy = y0 - 1 + row; yy = yy < 0 ? yy + p.ny : (yy >= p.ny ? yy % p.ny : yy);
        int zz = z0 - 1 + col; zz = zz < 0 ? zz + p.nz : (zz >= p.nz ? zz % p.nz : zz);
        const long long v = base + (long long)yy * p.nz + zz;
        const int c = a.cnt_in[v];
        ring.cnt[slot][r] = (uint8_t)c;
#pragma unroll
        for (int s = 0; s < KT; s++)
        {
            if (s < c)
            {
                ring.g[slot][s][r] = a.idx_in[s * N + v];
                ring.phi[slot][s][r] = vin[s * N + v];
            }
        }
    }
}

// Append-or-accumulate into a register list of capacity NF (dynamic length n).
template <class R, int NF>
__device__ __forceinline__ void list_add(int (&gl)[NF], R (&vl)[NF], R (&ll)[NF], int& n, bool& over, int g, R l,
                                         bool with_lap)
{
    bool found = false;
#pragma unroll
    for (int k = 0; k < NF; k++)
    {
        if (k < n && gl[k] == g)
        {
            if (with_lap) ll[k] += l;
            found = true;
        }
    }
    if (!found)
    {
        if (n < NF)
        {
#pragma unroll
            for (int k = 0; k < NF; k++)
            {
                if (k == n)
                {
                    gl[k] = g;
                    vl[k] = R(0);
                    ll[k] = with_lap ? l : R(0);
                }
            }
            n++;
        }
        else
        {
            over = true;
        }
    }
}

template <class R, int KS, int KT, int NF, int TY>
__global__ void __launch_bounds__(32 * TY)
tile_step_kernel(const __grid_constant__ StepParams p, const StepArrays a, int xchunk, int* __restrict__ slow_list,
                 unsigned* __restrict__ slow_count, unsigned slow_cap)
{
    constexpr int NT = 32 * TY;
    using Smem = TileSmem<R, KT, NF, TY>;
    using Ring = TileRing<R, KT, TY>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    auto& ring = S.ring;
    auto& L = S.lists;

    const int tz = threadIdx.x, ty = threadIdx.y, t = ty * 32 + tz;
    const int z0 = blockIdx.x * kTileZ, y0 = blockIdx.y * TY, x0 = blockIdx.z * xchunk;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x1 = min(x0 + xchunk, nx);
    const long long N = p.n;
    const long long plane = (long long)ny * nz;
    const int z = z0 + tz, y = y0 + ty;
    const bool inside = (z < nz) && (y < ny);
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    R* __restrict__ vout = static_cast<R*>(a.val_out);

    for (int i = t; i < kTileVolSlots; i += NT) { S.vol_key[i] = -1; S.vol_sum[i] = 0.0; }
    if (t < 3) S.cnt[t] = 0ull;
    unsigned wide = 0, ein = 0, eout = 0;
    uint32_t st = 0;

    load_plane(p, a, ring, 0, x0 == 0 ? nx - 1 : x0 - 1, y0, z0, t, NT);
    load_plane(p, a, ring, 1, x0, y0, z0, t, NT);
    const int rec0 = (ty + 1) * Ring::kCols + (tz + 1);
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;

    for (int x = x0; x < x1; x++)
    {
        const int xi = x - x0;
        const int sl[3] = {xi % 3, (xi + 1) % 3, (xi + 2) % 3};
        if (t <= NF + 1) S.bucket[t] = 0u;
        load_plane(p, a, ring, sl[2], x == nx - 1 ? 0 : x + 1, y0, z0, t, NT);
        __syncthreads();

        // ---- A: flags, bulk copy, list building -----------------------------------------------
        const long long v = (long long)x * plane + (long long)y * nz + z;
        const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
        uint8_t key = 0;
        if (inside)
        {
            const int c = ring.cnt[sl[1]][rec0];
            ein += c;
            int flag = c > 1 ? 2 : 0;
            if (flag == 0)
            {
#pragma unroll
                for (int q = 0; q < 27; q++)
                {
                    const int r = rec0 + ((q / 3) % 3 - 1) * Ring::kCols + (q % 3 - 1);
                    if (ring.cnt[sl[q / 9]][r] > 1) flag = 1;
                }
            }
            if (flag == 0)
            {
                a.cnt_out[v] = (uint8_t)c;
                for (int s = 0; s < c; s++)
                {
                    const int g = s < KT ? ring.g[sl[1]][s < KT ? s : 0][rec0] : a.idx_in[s * N + v];
                    const R phi = s < KT ? ring.phi[sl[1]][s < KT ? s : 0][rec0] : vin[s * N + v];
                    a.idx_out[s * N + v] = (int16_t)g;
                    vout[s * N + v] = phi;
                    tile_vol_insert(S.vol_key, S.vol_sum, a.vol_acc, g, (double)phi);
                }
                eout += c;
            }
            else
            {
                wide++;
                int gl[NF];
                R vl[NF], ll[NF];
#pragma unroll
                for (int k = 0; k < NF; k++) { gl[k] = -1; vl[k] = R(0); ll[k] = R(0); }
                int n = 0;
                bool over = c > NF;
                if (!over)
                {
#pragma unroll
                    for (int k = 0; k < NF; k++)
                    {
                        if (k < c)
                        {
                            gl[k] = k < KT ? ring.g[sl[1]][k < KT ? k : 0][rec0] : a.idx_in[k * N + v];
                            vl[k] = k < KT ? ring.phi[sl[1]][k < KT ? k : 0][rec0] : vin[k * N + v];
                        }
                    }
                    n = c;
                }
                for (int q = 0; q < p.ns && !over; q++)
                {
                    const int dx = p.lap_d[q][0], dy = p.lap_d[q][1], dz = p.lap_d[q][2];
                    const int pl = dx < 0 ? sl[0] : (dx > 0 ? sl[2] : sl[1]);
                    const int r = rec0 + dy * Ring::kCols + dz;
                    const R w = (R)p.lap_w[q];
                    const int cu = ring.cnt[pl][r];
                    for (int s = 0; s < cu; s++)
                    {
                        R phi;
                        int g;
                        if (s < KT)
                        {
                            phi = ring.phi[pl][s][r];
                            g = ring.g[pl][s][r];
                        }
                        else
                        {
                            const long long u = (long long)(dx < 0 ? xm : (dx > 0 ? xp : x)) * plane
                                              + (long long)(dy < 0 ? ym : (dy > 0 ? yp : y)) * nz
                                              + (dz < 0 ? zm : (dz > 0 ? zp : z));
                            phi = vin[s * N + u];
                            g = a.idx_in[s * N + u];
                        }
                        if (phi != R(0)) list_add<R, NF>(gl, vl, ll, n, over, g, w * phi, true);
                    }
                }
                for (int q = 0; q < p.ng && !over; q++)
                {
                    const int dx = p.grad_d[q][0], dy = p.grad_d[q][1], dz = p.grad_d[q][2];
                    const int pl = dx < 0 ? sl[0] : (dx > 0 ? sl[2] : sl[1]);
                    const int r = rec0 + dy * Ring::kCols + dz;
                    const int cu = ring.cnt[pl][r];
                    for (int s = 0; s < cu; s++)
                    {
                        R phi;
                        int g;
                        if (s < KT)
                        {
                            phi = ring.phi[pl][s][r];
                            g = ring.g[pl][s][r];
                        }
                        else
                        {
                            const long long u = (long long)(dx < 0 ? xm : (dx > 0 ? xp : x)) * plane
                                              + (long long)(dy < 0 ? ym : (dy > 0 ? yp : y)) * nz
                                              + (dz < 0 ? zm : (dz > 0 ? zp : z));
                            phi = vin[s * N + u];
                            g = a.idx_in[s * N + u];
                        }
                        if (phi != R(0)) list_add<R, NF>(gl, vl, ll, n, over, g, R(0), false);
                    }
                }
                if (over)
                {
                    key = 255;
                    const unsigned slot = atomicAdd(slow_count, 1u);
                    if (slot < slow_cap) slow_list[slot] = (int)v;
                    else st |= kStOverflowList;
                }
                else
                {
                    key = (uint8_t)n;
#pragma unroll
                    for (int k = 0; k < NF; k++)
                    {
                        if (k < n)
                        {
                            L.g[k][t] = (int16_t)gl[k];
                            L.val[k][t] = vl[k];
                            L.lap[k][t] = ll[k];
                        }
                    }
                    L.flag[t] = (uint8_t)flag;
                    atomicAdd(&S.bucket[n], 1u);
                }
            }
        }
        L.n[t] = key;
        __syncthreads();

        // ---- bucket lists by length -------------------------------------------------------------
        if (t == 0)
        {
            unsigned acc = 0;
            for (int k = NF; k >= 1; k--) { S.base[k] = acc; acc += S.bucket[k]; S.bucket[k] = 0u; }
            S.base[NF + 1] = acc;
        }
        __syncthreads();
        if (key >= 1 && key <= NF)
        {
            const unsigned r = atomicAdd(&S.bucket[key], 1u);
            L.perm[S.base[key] + r] = (uint16_t)t;
        }
        __syncthreads();

        // ---- B: length-specialised processing ---------------------------------------------------
        const unsigned nwork = S.base[NF + 1];
        for (unsigned i = t; i < nwork; i += NT)
        {
            const int u = L.perm[i];
            const int n = L.n[u];
            const int f = L.flag[u];
            int m = 0;
            switch (n)
            {
                case 2: m = process_list<R, 2, NF, NT>(p, a, L, u, f, st); break;
                case 3: if (NF >= 3) m = process_list<R, (NF >= 3 ? 3 : 2), NF, NT>(p, a, L, u, f, st); break;
                case 4: if (NF >= 4) m = process_list<R, (NF >= 4 ? 4 : 2), NF, NT>(p, a, L, u, f, st); break;
                case 5: if (NF >= 5) m = process_list<R, (NF >= 5 ? 5 : 2), NF, NT>(p, a, L, u, f, st); break;
                case 6: if (NF >= 6) m = process_list<R, (NF >= 6 ? 6 : 2), NF, NT>(p, a, L, u, f, st); break;
                default: m = process_list<R, 1, NF, NT>(p, a, L, u, f, st); break;
            }
            L.m[u] = (uint8_t)m;
        }
        __syncthreads();

        // ---- C: write the new records ---------------------------------------------------------
        if (key >= 1 && key <= NF)
        {
            const int m = L.m[t] > KS ? KS : L.m[t];
            if (L.m[t] > KS) st |= kStOverflowK;
            a.cnt_out[v] = (uint8_t)m;
            for (int s = 0; s < m; s++)
            {
                const int g = L.g[s][t];
                const R w = L.val[s][t];
                a.idx_out[s * N + v] = (int16_t)g;
                vout[s * N + v] = w;
                tile_vol_insert(S.vol_key, S.vol_sum, a.vol_acc, g, (double)w);
            }
            eout += m;
        }
    }

    if (st) atomicOr(a.status, st);
    unsigned w = wide, ei = ein, eo = eout;
    for (int o = 16; o > 0; o >>= 1)
    {
        w += __shfl_down_sync(0xffffffffu, w, o);
        ei += __shfl_down_sync(0xffffffffu, ei, o);
        eo += __shfl_down_sync(0xffffffffu, eo, o);
    }
    if (tz == 0)
    {
        if (w) atomicAdd(&S.cnt[0], (unsigned long long)w);
        if (ei) atomicAdd(&S.cnt[1], (unsigned long long)ei);
        if (eo) atomicAdd(&S.cnt[2], (unsigned long long)eo);
    }
    if (st & (kStOverflowK | kStOverflowList)) atomicAdd(&a.counters[kCntOverflowVoxels], 1ull);
    __syncthreads();
    for (int i = t; i < kTileVolSlots; i += NT)
        if (S.vol_key[i] >= 0) atomicAdd(&a.vol_acc[S.vol_key[i]], S.vol_sum[i]);
    if (t < 3 && S.cnt[t])
        atomicAdd(&a.counters[t == 0 ? kCntWide : (t == 1 ? kCntEntriesIn : kCntEntriesOut)], S.cnt[t]);
}

// Voxels whose field + candidate list exceeds the tiled kernel's register capacity, through the
// general per-voxel path (grid-stride over the worklist; the tiled kernel already counted them as
// wide and counted their input entries).
template <class R, int KS, int KL>
__global__ void __launch_bounds__(128) overflow_step_kernel(const __grid_constant__ StepParams p, const StepArrays a,
                                                            const int* __restrict__ slow_list,
                                                            const unsigned* __restrict__ slow_count, unsigned slow_cap)
{
    __shared__ int s_key[kVolSlots];
    __shared__ double s_sum[kVolSlots];
    __shared__ unsigned long long s_out;
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    if (threadIdx.x == 0) s_out = 0ull;
    __syncthreads();
    const unsigned total = min(*slow_count, slow_cap);
    uint32_t st = 0;
    unsigned eo_sum = 0;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
    {
        unsigned wide = 0, ein = 0, eout = 0;
        voxel_step_generic<R, KS, KL>(p, a, slow_list[i], s_key, s_sum, wide, ein, eout, st, false);
        eo_sum += eout;
    }
    if (st) atomicOr(a.status, st);
    if (st & (kStOverflowK | kStOverflowList)) atomicAdd(&a.counters[kCntOverflowVoxels], 1ull);
    if (eo_sum) atomicAdd(&s_out, (unsigned long long)eo_sum);
    __syncthreads();
    for (int i = threadIdx.x; i < kVolSlots; i += blockDim.x)
        if (s_key[i] >= 0) atomicAdd(&a.vol_acc[s_key[i]], s_sum[i]);
    if (threadIdx.x == 0 && s_out) atomicAdd(&a.counters[kCntEntriesOut], s_out);
}

}  // namespace opgpu

namespace opgpu {

constexpr int kTileKT = 4;   // stored slots staged in shared memory
constexpr int kTileNF = 6;   // register list capacity of the tiled kernel
constexpr int kTileTY = 8;   // tile rows (blocks of 32 x 8 threads)

template <class R, int KS, int KL>
int launch_tiled(const StepParams& p, const StepArrays& a, void* stream)
{
    using Smem = TileSmem<R, kTileKT, kTileNF, kTileTY>;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto kern = tile_step_kernel<R, KS, kTileKT, kTileNF, kTileTY>;
    const size_t smem = sizeof(Smem);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    const int tz = (p.nz + kTileZ - 1) / kTileZ, ty = (p.ny + kTileTY - 1) / kTileTY;
    // enough x-chunks for ~8 blocks per SM on small grids, long chunks (halo reuse) on large ones
    int xchunk = (int)((long long)p.nx * tz * ty / (148 * 8));
    xchunk = xchunk < 2 ? 2 : (xchunk > 16 ? 16 : xchunk);
    const int tx = (p.nx + xchunk - 1) / xchunk;
    e = cudaMemsetAsync(a.slow_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    kern<<<dim3(tz, ty, tx), dim3(32, kTileTY), smem, s>>>(p, a, xchunk, a.slow_list, a.slow_count, a.slow_cap);
    e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    overflow_step_kernel<R, KS, KL><<<148 * 2, 128, 0, s>>>(p, a, a.slow_list, a.slow_count, a.slow_cap);
    return (int)cudaGetLastError();
}

template <class R>
int launch_step(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream)
{
    if (variant == kVariantGeneric) return launch_step_generic<R>(p, a, k_slots, stream);
    switch (k_slots)
    {
        case 8:  return launch_tiled<R, 8, 16>(p, a, stream);
        case 12: return launch_tiled<R, 12, 20>(p, a, stream);
        case 16: return launch_tiled<R, 16, 24>(p, a, stream);
        default: return -1;
    }
}

}  // namespace opgpu
