// Tiled form of the fused step (the production path).
//
// A block owns a (y, z) tile of TY x 32 voxels and marches along x over `xchunk` planes.  The 3x3x3
// neighbourhoods come from a ring of three x-planes in shared memory (tile plus a one-voxel halo in
// y and z; periodic wrap by index arithmetic).  The grains present in the three planes of the
// window get block-local slot numbers (at most kSlots, recycled as grains leave the window), and
// every ring plane is held twice:
//   * as per-record slot lists in the record's entry order plus a slot bitmask, and
//   * as dense per-slot value planes dense[slot][plane][record] (zero where the grain is absent).
// Every plane then goes through
//   A  (thread per voxel)  flag from the 27 neighbour counts; bulk voxels are copied straight to
//                          the output; interface voxels discover their candidate fields with
//                          bitmask operations, in the reference's order (own fields, then new
//                          grains in stencil order and neighbour-list order).
//   B  (thread per list)   lists are bucketed by length; each warp runs one length-specialised,
//                          fully unrolled path: Laplacians from the dense planes (27 loads and
//                          multiply-adds per field), pair kinetics, driving force, projection,
//                          merge and finalize, all in registers.
//   C  (thread per voxel)  the new records are written back coalesced; grain volumes accumulate in
//                          a per-block shared-memory table.
// Lists longer than NF and windows with more than kSlots distinct grains go to the overflow
// worklist, which the general per-voxel kernel processes afterwards.
//
// The per-voxel arithmetic and its operation order are those of voxel_step_generic (and of the
// reference: a Laplacian sums w*phi over the stencil in stencil order; adding the zero terms of
// absent neighbours leaves every partial sum unchanged), so the FP64 results agree bit for bit.
#pragma once
#include "step_kernel.cuh"

namespace opgpu {

constexpr int kTileZ = 32;
constexpr int kSlots = 16;           // distinct grains per 3-plane window
constexpr int kTileVolSlots = 512;

template <int TY>
struct TileGeom {
    static constexpr int kRows = TY + 2;
    static constexpr int kCols = kTileZ + 2;
    static constexpr int kRecs = kRows * kCols;
    static constexpr int NT = 32 * TY;
};

template <class R, int KS, int NF, int TY>
struct TileSmem {
    using Geo = TileGeom<TY>;
    R dense[kSlots][3][Geo::kRecs];          // per-slot values of the three ring planes
    R oval[NF][Geo::NT];                     // new record values (phase B -> C)
    double vol_sum[kTileVolSlots];
    uint32_t mask[3][Geo::kRecs];            // slot bitmask per record
    int vol_key[kTileVolSlots];
    int grain_of[kSlots];                    // slot -> grain (-1 = free)
    int lastpos[kSlots];                     // last window position where the slot's grain occurs
    int pending[32];                         // grains of the incoming plane that need a slot
    unsigned bucket[NF + 2];
    unsigned base[NF + 2];
    unsigned long long cnt[3];
    int16_t og[NF][Geo::NT];                 // new record grains (phase B -> C)
    uint16_t perm[Geo::NT];
    uint8_t slot[3][KS][Geo::kRecs];         // slot ids in entry order
    uint8_t cntr[3][Geo::kRecs];             // entries per record
    uint8_t lslot[NF][Geo::NT];              // the list (slot ids) of every interface voxel
    uint8_t key[Geo::NT];                    // 0 bulk/outside, 1..NF list length, 255 overflow
    uint8_t flag[Geo::NT];
    uint8_t m[Geo::NT];
    uint8_t bad[3];                          // ring plane holds a grain without slot
    unsigned npending;
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

// Offsets of the q-th Laplacian stencil element (LaplacianStencil::Set order): 27-point stencils
// enumerate x, y, z in -1..1; the 7-point stencil keeps the centre and the six faces.
template <int NS>
__device__ __forceinline__ constexpr int stencil_dx(int q) { return NS == 27 ? q / 9 - 1 : (q == 0 ? -1 : (q == 6 ? 1 : 0)); }
template <int NS>
__device__ __forceinline__ constexpr int stencil_dy(int q) { return NS == 27 ? (q / 3) % 3 - 1 : (q == 1 ? -1 : (q == 5 ? 1 : 0)); }
template <int NS>
__device__ __forceinline__ constexpr int stencil_dz(int q) { return NS == 27 ? q % 3 - 1 : (q == 2 ? -1 : (q == 4 ? 1 : 0)); }

// Stages 1b-6 for a list of exactly N fields (compile-time), all arrays in registers: Laplacians
// from the dense planes, pair kinetics, driving force, projection, merge, finalize.  The new record
// goes to S.og/S.oval; returns its length.
template <class R, int N, int NS, int KS, int NF, int TY>
__device__ __forceinline__ int process_list(const StepParams& p, const StepArrays& a, TileSmem<R, KS, NF, TY>& S,
                                            int u, int flag, const int (&sl)[3], uint32_t& st)
{
    using Geo = TileGeom<TY>;
    constexpr int NP = N * (N - 1) / 2;
    const int rec0 = (u / 32 + 1) * Geo::kCols + (u % 32 + 1);
    int g[N], s[N];
    R val[N], lap[N];
#pragma unroll
    for (int k = 0; k < N; k++)
    {
        s[k] = S.lslot[k][u];
        g[k] = S.grain_of[s[k]];
        val[k] = S.dense[s[k]][sl[1]][rec0];
        lap[k] = R(0);
    }
    // ---- Laplacians (PhaseField::CalculateDerivativesSR), stencil order ------------------------
#pragma unroll
    for (int q = 0; q < NS; q++)
    {
        const int pl = sl[stencil_dx<NS>(q) + 1];
        const int r = rec0 + stencil_dy<NS>(q) * Geo::kCols + stencil_dz<NS>(q);
        const R w = (R)p.lap_w[q];
#pragma unroll
        for (int k = 0; k < N; k++) lap[k] += w * S.dense[s[k]][pl][r];
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
            const double vra = a.vr[g[i]], vrb = a.vr[g[j]];
            const R scale = (vra == 1.0 && vrb == 1.0) ? R(1) : (R)sqrt(vra * vrb);   // sqrt(1*1) == 1 exactly
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
                // limits (neg/pos reused as the lower / upper limit of each field)
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
            S.og[pos][u] = (int16_t)g[i];
            S.oval[pos][u] = w;
            pos++;
        }
    }
    if (m == 0) st |= kStEmptyVoxel;
    return m;
}

// Slot of a grain in the window table (-1 if absent).
__device__ __forceinline__ int find_slot(const int* grain_of, int g)
{
    int r = -1;
#pragma unroll
    for (int k = 0; k < kSlots; k++) r = (grain_of[k] == g) ? k : r;
    return r;
}

// Bring plane xp (window position wpos) into ring slot `rs`: sparse slot lists, bitmasks and dense
// per-slot values.  Grains not yet in the window get a slot that no grain of the window uses.
template <class R, int KS, int NF, int TY>
__device__ __forceinline__ void load_plane(const StepParams& p, const StepArrays& a, TileSmem<R, KS, NF, TY>& S,
                                           int rs, int xp, int wpos, int y0, int z0, int t)
{
    using Geo = TileGeom<TY>;
    const long long N = p.n;
    const long long base = (long long)xp * p.ny * p.nz;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    // 1. grains of the incoming plane without a slot
    for (int r = t; r < Geo::kRecs; r += Geo::NT)
    {
        const int row = r / Geo::kCols, col = r - row * Geo::kCols;
        int yy = y0 - 1 + row; yy = yy < 0 ? yy + p.ny : (yy >= p.ny ? yy % p.ny : yy);
        int zz = z0 - 1 + col; zz = zz < 0 ? zz + p.nz : (zz >= p.nz ? zz % p.nz : zz);
        const long long v = base + (long long)yy * p.nz + zz;
        const int c = a.cnt_in[v];
        for (int s = 0; s < c; s++)
        {
            const int g = a.idx_in[s * N + v];
            if (find_slot(S.grain_of, g) < 0)
            {
                unsigned h = ((unsigned)g * 2654435761u) & 31u;
                for (int probe = 0; probe < 32; probe++)
                {
                    const int k = atomicCAS(&S.pending[h], -1, g);
                    if (k == -1 || k == g) break;
                    h = (h + 1) & 31u;
                }
            }
        }
    }
    __syncthreads();
    // 2. assign free slots (a slot is free when its grain left the window positions wpos-2.. )
    if (t == 0)
    {
        S.bad[rs] = 0;
        for (int h = 0; h < 32; h++)
        {
            const int g = S.pending[h];
            if (g < 0) continue;
            S.pending[h] = -1;
            int free_slot = -1;
            for (int k = 0; k < kSlots && free_slot < 0; k++)
                if (S.grain_of[k] < 0 || S.lastpos[k] < wpos - 2) free_slot = k;
            if (free_slot < 0) { S.bad[rs] = 1; continue; }
            S.grain_of[free_slot] = g;
            S.lastpos[free_slot] = wpos;
        }
    }
    __syncthreads();
    // 3. slot lists, bitmasks, dense values of the incoming plane
    for (int r = t; r < Geo::kRecs; r += Geo::NT)
    {
        const int row = r / Geo::kCols, col = r - row * Geo::kCols;
        int yy = y0 - 1 + row; yy = yy < 0 ? yy + p.ny : (yy >= p.ny ? yy % p.ny : yy);
        int zz = z0 - 1 + col; zz = zz < 0 ? zz + p.nz : (zz >= p.nz ? zz % p.nz : zz);
        const long long v = base + (long long)yy * p.nz + zz;
        const int c = a.cnt_in[v];
#pragma unroll
        for (int k = 0; k < kSlots; k++) S.dense[k][rs][r] = R(0);
        uint32_t msk = 0;
        for (int s = 0; s < c; s++)
        {
            const int g = a.idx_in[s * N + v];
            const int k = find_slot(S.grain_of, g);
            if (k < 0) { S.bad[rs] = 1; continue; }
            S.dense[k][rs][r] = vin[s * N + v];
            S.slot[rs][s][r] = (uint8_t)k;
            msk |= 1u << k;
            S.lastpos[k] = wpos;
        }
        S.mask[rs][r] = msk;
        S.cntr[rs][r] = (uint8_t)c;
    }
}

template <class R, int KS, int NF, int TY, int NS>
__global__ void __launch_bounds__(32 * TY)
tile_step_kernel(const __grid_constant__ StepParams p, const StepArrays a, int xchunk, int* __restrict__ slow_list,
                 unsigned* __restrict__ slow_count, unsigned slow_cap)
{
    using Geo = TileGeom<TY>;
    using Smem = TileSmem<R, KS, NF, TY>;
    constexpr int NT = Geo::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);

    const int tz = threadIdx.x, ty = threadIdx.y, t = ty * 32 + tz;
    const int z0 = blockIdx.x * kTileZ, y0 = blockIdx.y * TY, x0 = blockIdx.z * xchunk;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x1 = min(x0 + xchunk, nx);
    const long long N = p.n;
    const long long plane = (long long)ny * nz;
    const int z = z0 + tz, y = y0 + ty;
    const bool inside = (z < nz) && (y < ny);
    R* __restrict__ vout = static_cast<R*>(a.val_out);

    for (int i = t; i < kTileVolSlots; i += NT) { S.vol_key[i] = -1; S.vol_sum[i] = 0.0; }
    if (t < kSlots) { S.grain_of[t] = -1; S.lastpos[t] = -1000; }
    if (t < 32) S.pending[t] = -1;
    if (t < 3) S.cnt[t] = 0ull;
    unsigned wide = 0, ein = 0, eout = 0;
    uint32_t st = 0;
    __syncthreads();

    load_plane(p, a, S, 0, x0 == 0 ? nx - 1 : x0 - 1, -1, y0, z0, t);
    __syncthreads();
    load_plane(p, a, S, 1, x0, 0, y0, z0, t);
    const int rec0 = (ty + 1) * Geo::kCols + (tz + 1);

    for (int x = x0; x < x1; x++)
    {
        const int xi = x - x0;
        const int sl[3] = {xi % 3, (xi + 1) % 3, (xi + 2) % 3};
        if (t <= NF + 1) S.bucket[t] = 0u;
        __syncthreads();
        load_plane(p, a, S, sl[2], x == nx - 1 ? 0 : x + 1, xi + 1, y0, z0, t);
        __syncthreads();
        const bool window_bad = S.bad[0] | S.bad[1] | S.bad[2];

        // ---- A: flags, bulk copy, candidate discovery --------------------------------------
        const long long v = (long long)x * plane + (long long)y * nz + z;
        uint8_t key = 0;
        if (inside)
        {
            const int c = S.cntr[sl[1]][rec0];
            ein += c;
            int flag = c > 1 ? 2 : 0;
            if (flag == 0)
            {
#pragma unroll
                for (int q = 0; q < 27; q++)
                {
                    const int r = rec0 + ((q / 3) % 3 - 1) * Geo::kCols + (q % 3 - 1);
                    if (S.cntr[sl[q / 9]][r] > 1) flag = 1;
                }
            }
            if (flag == 0)
            {
                a.cnt_out[v] = (uint8_t)c;
                for (int s = 0; s < c; s++)
                {
                    int g;
                    R phi;
                    if (!window_bad)
                    {
                        const int k = S.slot[sl[1]][s][rec0];
                        g = S.grain_of[k];
                        phi = S.dense[k][sl[1]][rec0];
                    }
                    else
                    {
                        g = a.idx_in[s * N + v];
                        phi = static_cast<const R*>(a.val_in)[s * N + v];
                    }
                    a.idx_out[s * N + v] = (int16_t)g;
                    vout[s * N + v] = phi;
                    tile_vol_insert(S.vol_key, S.vol_sum, a.vol_acc, g, (double)phi);
                }
                eout += c;
            }
            else
            {
                wide++;
                bool over = window_bad || c > NF;
                int n = c;
                if (!over)
                {
                    uint32_t seen = S.mask[sl[1]][rec0];
                    uint8_t ls[NF];
#pragma unroll
                    for (int k = 0; k < NF; k++) ls[k] = k < c ? S.slot[sl[1]][k][rec0] : 0;
                    // Laplacian pass, then (SIMPLE Laplacian only) the gradient pass of
                    // CalculateDerivativesSR: new grains in stencil order, neighbour-list order
                    const int nq = p.ns + p.ng;
                    for (int q = 0; q < nq && !over; q++)
                    {
                        const signed char* d = q < p.ns ? p.lap_d[q] : p.grad_d[q - p.ns];
                        const int pl = d[0] < 0 ? sl[0] : (d[0] > 0 ? sl[2] : sl[1]);
                        const int r = rec0 + d[1] * Geo::kCols + d[2];
                        uint32_t fresh = S.mask[pl][r] & ~seen;
                        if (fresh)
                        {
                            const int cu = S.cntr[pl][r];
                            for (int s = 0; s < cu; s++)
                            {
                                const int k = S.slot[pl][s][r];
                                if ((fresh >> k) & 1u)
                                {
                                    if (n < NF)
                                    {
#pragma unroll
                                        for (int j = 0; j < NF; j++) if (j == n) ls[j] = (uint8_t)k;
                                        n++;
                                    }
                                    else
                                    {
                                        over = true;
                                    }
                                }
                            }
                            seen |= fresh;
                        }
                    }
                    if (!over)
                    {
#pragma unroll
                        for (int k = 0; k < NF; k++) if (k < n) S.lslot[k][t] = ls[k];
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
                    S.flag[t] = (uint8_t)flag;
                    atomicAdd(&S.bucket[n], 1u);
                }
            }
        }
        S.key[t] = key;
        __syncthreads();

        // ---- bucket lists by length ---------------------------------------------------------------
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
            S.perm[S.base[key] + r] = (uint16_t)t;
        }
        __syncthreads();

        // ---- B: length-specialised processing ------------------------------------------------------
        const unsigned nwork = S.base[NF + 1];
        for (unsigned i = t; i < nwork; i += NT)
        {
            const int u = S.perm[i];
            const int n = S.key[u];
            const int f = S.flag[u];
            int m = 0;
            switch (n)
            {
                case 2: m = process_list<R, 2, NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
                case 3: m = process_list<R, (NF >= 3 ? 3 : 2), NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
                case 4: m = process_list<R, (NF >= 4 ? 4 : 2), NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
                case 5: m = process_list<R, (NF >= 5 ? 5 : 2), NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
                case 6: m = process_list<R, (NF >= 6 ? 6 : 2), NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
                default: m = process_list<R, 1, NS, KS, NF, TY>(p, a, S, u, f, sl, st); break;
            }
            S.m[u] = (uint8_t)m;
        }
        __syncthreads();

        // ---- C: write the new records -----------------------------------------------------------
        if (key >= 1 && key <= NF)
        {
            int m = S.m[t];
            if (m > KS) { st |= kStOverflowK; m = KS; }
            a.cnt_out[v] = (uint8_t)m;
            for (int s = 0; s < m; s++)
            {
                const int g = S.og[s][t];
                const R w = S.oval[s][t];
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

// Voxels whose field + candidate list exceeds the tiled kernel's capacity, through the general
// per-voxel path (grid-stride over the worklist; the tiled kernel already counted them as wide and
// counted their input entries).
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

constexpr int kTileNF = 6;   // register list capacity of the tiled kernel
constexpr int kTileTY = 4;   // tile rows (blocks of 32 x 4 threads)

template <class R, int KS, int KL, int NS>
int launch_tiled_ns(const StepParams& p, const StepArrays& a, void* stream)
{
    using Smem = TileSmem<R, KS, kTileNF, kTileTY>;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto kern = tile_step_kernel<R, KS, kTileNF, kTileTY, NS>;
    const size_t smem = sizeof(Smem);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    const int tz = (p.nz + kTileZ - 1) / kTileZ, ty = (p.ny + kTileTY - 1) / kTileTY;
    // enough x-chunks for several blocks per SM on small grids, long chunks (halo reuse) on large ones
    int xchunk = (int)((long long)p.nx * tz * ty / (148 * 8));
    xchunk = xchunk < 2 ? 2 : (xchunk > 32 ? 32 : xchunk);
    const int tx = (p.nx + xchunk - 1) / xchunk;
    e = cudaMemsetAsync(a.slow_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    kern<<<dim3(tz, ty, tx), dim3(32, kTileTY), smem, s>>>(p, a, xchunk, a.slow_list, a.slow_count, a.slow_cap);
    e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    overflow_step_kernel<R, KS, KL><<<148 * 2, 128, 0, s>>>(p, a, a.slow_list, a.slow_count, a.slow_cap);
    return (int)cudaGetLastError();
}

template <class R, int KS, int KL>
int launch_tiled(const StepParams& p, const StepArrays& a, void* stream)
{
    if (p.ns == 27) return launch_tiled_ns<R, KS, KL, 27>(p, a, stream);
    if (p.ns == 7) return launch_tiled_ns<R, KS, KL, 7>(p, a, stream);
    return -1;
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
