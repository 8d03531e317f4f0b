// Tiled production path of the fused step: a classify kernel and one compute kernel per list length.
//
// classify (tile_classify_kernel)
//   A block owns a (y, z) tile of TY x kTileZ voxels and marches along x over `xchunk` planes.  The 3x3x3
//   neighbourhoods come from a ring of three x-planes in shared memory (tile plus a one-voxel halo
//   in y and z; periodic wrap by index arithmetic).  The grains present in the three planes of the
//   window carry block-local slot numbers (at most kSlots, recycled as grains leave the window), and
//   every ring plane is held twice: per record its slots in entry order with a slot bitmask, and as
//   dense per-slot value planes dense[slot][plane][record] (zero where the grain is absent).  For
//   each voxel of the centre plane one thread
//     - derives the flag from the 27 neighbour counts and copies bulk voxels to the output;
//     - discovers the candidate fields with bitmask operations, in the reference's order (own
//       fields, then new grains in stencil order and neighbour-list order);
//     - sums every field's Laplacian from the dense planes (27 loads and multiply-adds in stencil
//       order; the zero terms of absent neighbours leave every partial sum unchanged);
//     - writes the list to the work buffer and appends the voxel to its block's slice of the
//       bucket of its list length.
// compute (list_compute_kernel<N>)
//   One kernel per list length N = 2..kListCap over all the slices' entries of that length (a
//   small scan kernel turns the per-slice counts into offsets), split evenly over the CUDA blocks:
//   fully unrolled, register-only pair kinetics, driving force, projection, merge and finalize
//   (the operation order of list_step), new record written to the output state.
// Lists longer than kListCap and voxels next to a grain without a window slot go to the general-path
// worklist, processed one warp per voxel (warp_step.cuh).
#pragma once
#include "step_kernel.cuh"
#include "warp_step.cuh"

namespace opgpu {

constexpr int kTileZ = kTileCols;
// distinct grains per 3-plane window: 16 for FP32 values, 14 for FP64 (its dense planes would
// otherwise leave room for only two blocks per SM)
template <class R>
struct WindowSlots {
    static constexpr int value = sizeof(R) == 8 ? 14 : 16;
};
constexpr int kSlotHash = 64;        // grain -> slot hash table entries
constexpr int kTileVolSlots = 512;      // grain-volume hash of the compute kernels
constexpr int kKeepEntries = 6;         // entries per record the plane loader keeps in registers
// The FP64 plane loader keeps the slots step 1 found in shared memory for step 3 (measured 5 %
// faster classify); in FP32 the extra addressing costs more than the second hash lookup saves.
template <class R>
struct LoaderSlotCache {
    static constexpr bool value = sizeof(R) == 8;
};
// grain-volume hash of the classify kernel (bulk voxels); smaller where the slot cache needs room
template <class R>
struct ClassifyVolSlots {
    static constexpr int value = LoaderSlotCache<R>::value ? 128 : 256;
};
// Blocks of each per-length compute kernel: one per 4096 voxels of the grid, between 8 and 32 per
// SM (a finer split of each length's entries pays on large grids; on small ones the per-block
// set-up and flush of the grain-volume hash would cost more than it balances).
inline int compute_blocks(long long n)
{
    const long long b = n / 4096;
    return (int)(b < 148 * 8 ? 148 * 8 : (b > 148 * 32 ? 148 * 32 : b));
}
constexpr int kTileTY = kTileRows;   // tile rows (blocks of kTileZ x kTileRows threads)

template <int TY>
struct TileGeom {
    static constexpr int kRows = TY + 2;
    static constexpr int kCols = kTileZ + 2;
    static constexpr int kRecs = kRows * kCols;
    static constexpr int NT = kTileZ * TY;
};

template <class R, int KS, int TY>
struct TileSmem {
    using Geo = TileGeom<TY>;
    static constexpr int kSlots = WindowSlots<R>::value;
    R dense[kSlots][3][Geo::kRecs];          // per-slot values of the three ring planes (zero where absent)
    double vol_sum[ClassifyVolSlots<R>::value];
    uint64_t slotl[3][Geo::kRecs];           // slot ids of the record in entry order, 4 bits each
    uint32_t word[3][Geo::kRecs];            // slot bitmask of the record | (more than one field) << 31
                                             // | (a grain of the record has no slot) << 30
    int vol_key[ClassifyVolSlots<R>::value];
    int grain_of[kSlots];                    // slot -> grain (-1 = free)
    int lastpos[kSlots];                     // last window position where the slot's grain occurs
    int hkey[kSlotHash];                     // grain -> slot hash: key (-1 empty, -2 deleted)
    int pending[32];                         // grains of the incoming plane that need a slot
    unsigned nb[kListCap + 1];               // entries this block appended per list length
    unsigned woff;                           // bytes of work records this block wrote
    unsigned crowded;                        // voxels sent to the general path for a crowded window
    unsigned long long cnt[3];
    uint8_t hslot[kSlotHash];                // grain -> slot hash: slot
    uint8_t cntr[3][Geo::kRecs];             // entries per record
    uint8_t pslot[LoaderSlotCache<R>::value ? Geo::kRecs : 1][kKeepEntries];   // slot step 1 found per kept
                                                                             // entry (0xFF: none)
    uint8_t tomb;                            // deleted hash entries
};

__device__ __forceinline__ unsigned slot_hash(int g) { return ((unsigned)g * 2654435761u) >> 26; }

// One term of the classify kernel's dense-plane Laplacian.  FP64: the reference's separate multiply
// and add (the FP64 unit is compiled without contraction).  FP32: one fused multiply-add, written
// out because the FP32 unit is compiled without contraction too (so that the adjoint can repeat its
// per-voxel arithmetic exactly); these Laplacians reach the forward and the adjoint alike through
// the work records, so their rounding only has to be the same in both, which it is.
__device__ __forceinline__ double lap_acc(double l, double w, double x) { return l + w * x; }
__device__ __forceinline__ float lap_acc(float l, float w, float x) { return __fmaf_rn(w, x, l); }

// Slot of a grain in the window (-1 if the grain has none).
__device__ __forceinline__ int find_slot(const int* hkey, const uint8_t* hslot, int g)
{
    unsigned h = slot_hash(g);
    for (int probe = 0; probe < kSlotHash; probe++)
    {
        const int k = hkey[h];
        if (k == g) return hslot[h];
        if (k == -1) return -1;
        h = (h + 1) & (kSlotHash - 1);
    }
    return -1;
}

__device__ __forceinline__ void hash_insert(int* hkey, uint8_t* hslot, int g, int slot)
{
    unsigned h = slot_hash(g);
    for (int probe = 0; probe < kSlotHash; probe++)
    {
        if (hkey[h] < 0) { hkey[h] = g; hslot[h] = (uint8_t)slot; return; }
        h = (h + 1) & (kSlotHash - 1);
    }
}

__device__ __forceinline__ void hash_erase(int* hkey, int g, uint8_t& tomb)
{
    unsigned h = slot_hash(g);
    for (int probe = 0; probe < kSlotHash; probe++)
    {
        if (hkey[h] == g) { hkey[h] = -2; tomb++; return; }
        if (hkey[h] == -1) return;
        h = (h + 1) & (kSlotHash - 1);
    }
}

// Records of a ring plane each thread handles, and how many entries of each it keeps in registers
// between the two passes of load_plane.
template <int TY>
struct PlaneRegs {
    static constexpr int kPer = (TileGeom<TY>::kRecs + TileGeom<TY>::NT - 1) / TileGeom<TY>::NT;
    static constexpr int kKeep = kKeepEntries;
};

template <int TY>
__device__ __forceinline__ long long plane_voxel(const StepParams& p, long long base, int r, int y0, int z0)
{
    using Geo = TileGeom<TY>;
    const int row = r / Geo::kCols, col = r - row * Geo::kCols;
    int yy = y0 - 1 + row; yy = yy < 0 ? yy + p.ny : (yy >= p.ny ? yy % p.ny : yy);
    int zz = z0 - 1 + col; zz = zz < 0 ? zz + p.nz : (zz >= p.nz ? zz % p.nz : zz);
    return base + (long long)yy * p.nz + zz;
}

// Counts of plane xp for this thread's records (issued one plane ahead of their use).
template <int TY>
__device__ __forceinline__ void prefetch_counts(const StepParams& p, const StepArrays& a, int xp, int y0, int z0,
                                                int t, int (&cr)[PlaneRegs<TY>::kPer])
{
    using Geo = TileGeom<TY>;
    const long long base = (long long)xp * p.ny * p.nz;
#pragma unroll
    for (int i = 0; i < PlaneRegs<TY>::kPer; i++)
    {
        const int r = t + i * Geo::NT;
        cr[i] = r < Geo::kRecs ? (int)a.cnt_in[plane_voxel<TY>(p, base, r, y0, z0)] : 0;
    }
}

// Registers a thread keeps between the passes of the plane loader: the voxel index of each of its
// records and their first kKeep entries.
template <class R, int TY>
struct PlaneLoad {
    long long vv[PlaneRegs<TY>::kPer];
    int gr[PlaneRegs<TY>::kPer][PlaneRegs<TY>::kKeep];
    R vr[PlaneRegs<TY>::kPer][PlaneRegs<TY>::kKeep];
};

// Bringing plane xp (window position wpos) into ring slot `rs` -- slot lists, bitmask words and
// dense per-slot values; grains not yet in the window get a slot that no grain of the window uses --
// takes three passes with a barrier between each:
//   plane_scan    reads the records once (the first kKeep entries stay in registers), marks the
//                 grains already slotted as in use and collects the others in `pending`; it touches
//                 only the hash (read), lastpos, pslot and pending, so it may run while other
//                 threads still read the ring for the previous plane; returns whether this thread
//                 added a pending grain
//   plane_assign  warp 0 hands free slots to the pending grains (only needed when some thread
//                 added one)
//   plane_fill    slot lists, bitmask words and dense values of the incoming plane, clearing what
//                 the ring position held before
// cr holds the plane's counts on entry (prefetched) and the next plane's counts after plane_fill.
// Invariant of the dense planes: dense[k][rs][r] != 0 only if bit k of word[rs][r] is set.
template <class R, int KS, int TY>
__device__ __forceinline__ bool plane_scan(const StepParams& p, const StepArrays& a, TileSmem<R, KS, TY>& S,
                                           int xp, int wpos, int y0, int z0, int t,
                                           const int (&cr)[PlaneRegs<TY>::kPer], PlaneLoad<R, TY>& L)
{
    using Geo = TileGeom<TY>;
    using PR = PlaneRegs<TY>;
    const long long N = p.n;
    const long long base = (long long)xp * p.ny * p.nz;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    bool added = false;
#pragma unroll
    for (int i = 0; i < PR::kPer; i++)
    {
        const int r = t + i * Geo::NT;
        L.vv[i] = r < Geo::kRecs ? plane_voxel<TY>(p, base, r, y0, z0) : 0;
#pragma unroll
        for (int s = 0; s < PR::kKeep; s++)
        {
            if (s < cr[i])
            {
                L.gr[i][s] = a.idx_in[s * N + L.vv[i]];
                L.vr[i][s] = vin[s * N + L.vv[i]];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < PR::kPer; i++)
    {
        for (int s = 0; s < cr[i]; s++)
        {
            int g;
#pragma unroll
            for (int q = 0; q < PR::kKeep; q++)
                if (q == s) g = L.gr[i][q];
            if (s >= PR::kKeep) g = a.idx_in[s * N + L.vv[i]];
            const int k0 = find_slot(S.hkey, S.hslot, g);
            if constexpr (LoaderSlotCache<R>::value)
                if (s < PR::kKeep) S.pslot[t + i * Geo::NT][s] = (uint8_t)(k0 >= 0 ? k0 : 0xFF);
            if (k0 >= 0)
            {
                S.lastpos[k0] = wpos;   // in use by the incoming plane: not free for plane_assign
            }
            else
            {
                added = true;
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
    return added;
}

template <class R, int KS, int TY>
__device__ __forceinline__ void plane_assign(TileSmem<R, KS, TY>& S, int wpos, int t)
{
    // warp 0 hands free slots (grain gone from the window) to the pending grains; lane 0 keeps
    // the grain -> slot hash in step
    if (t < 32)
    {
        const int g = S.pending[t];
        const bool valid = g >= 0;
        constexpr int kSlots = WindowSlots<R>::value;
        const bool is_free = t < kSlots && (S.grain_of[t] < 0 || S.lastpos[t] < wpos - 2);
        const unsigned fm = __ballot_sync(0xffffffffu, is_free);
        const unsigned vm = __ballot_sync(0xffffffffu, valid);
        const int rank = __popc(vm & ((1u << t) - 1u));
        const int k = (valid && rank < __popc(fm)) ? (int)__fns(fm, 0, rank + 1) : -1;
        if (valid) S.pending[t] = -1;
        for (unsigned m = vm; m; m &= m - 1u)
        {
            const int lane = __ffs(m) - 1;
            const int gl = __shfl_sync(0xffffffffu, g, lane);
            const int kl = __shfl_sync(0xffffffffu, k, lane);
            if (t == 0 && kl >= 0)
            {
                const int old = S.grain_of[kl];
                if (old >= 0) hash_erase(S.hkey, old, S.tomb);
                hash_insert(S.hkey, S.hslot, gl, kl);
                S.grain_of[kl] = gl;
                S.lastpos[kl] = wpos;
            }
        }
        // grains left without a slot are marked per record in plane_fill
        if (t == 0 && S.tomb > 24)
        {
            for (int h = 0; h < kSlotHash; h++) S.hkey[h] = -1;
            for (int q = 0; q < kSlots; q++)
                if (S.grain_of[q] >= 0) hash_insert(S.hkey, S.hslot, S.grain_of[q], q);
            S.tomb = 0;
        }
    }
}

template <class R, int KS, int TY>
__device__ __forceinline__ void plane_fill(const StepParams& p, const StepArrays& a, TileSmem<R, KS, TY>& S,
                                           int rs, int xp, int y0, int z0, int t, int (&cr)[PlaneRegs<TY>::kPer],
                                           const PlaneLoad<R, TY>& L)
{
    using Geo = TileGeom<TY>;
    using PR = PlaneRegs<TY>;
    const long long N = p.n;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
#pragma unroll
    for (int i = 0; i < PR::kPer; i++)
    {
        const int r = t + i * Geo::NT;
        if (r >= Geo::kRecs) continue;
        for (uint32_t m = S.word[rs][r] & 0xFFFFu; m; m &= m - 1u) S.dense[__ffs(m) - 1][rs][r] = R(0);
        uint32_t msk = 0;
        uint64_t lst = 0;
        bool unslotted = false;
        const int c = cr[i];
        for (int s = 0; s < c; s++)
        {
            int g;
            R val;
#pragma unroll
            for (int q = 0; q < PR::kKeep; q++)
                if (q == s) { g = L.gr[i][q]; val = L.vr[i][q]; }
            if (s >= PR::kKeep) { g = a.idx_in[s * N + L.vv[i]]; val = vin[s * N + L.vv[i]]; }
            // the slot plane_scan found, else the one plane_assign handed out
            int k = 0xFF;
            if constexpr (LoaderSlotCache<R>::value)
                if (s < PR::kKeep) k = S.pslot[r][s];
            if (k == 0xFF) k = find_slot(S.hkey, S.hslot, g);
            if (k < 0) { unslotted = true; continue; }
            S.dense[k][rs][r] = val;
            lst |= (uint64_t)k << (4 * s);
            msk |= 1u << k;
        }
        S.word[rs][r] = msk | (c > 1 ? 0x80000000u : 0u) | (unslotted ? 0x40000000u : 0u);
        S.slotl[rs][r] = lst;
        S.cntr[rs][r] = (uint8_t)c;
    }
    // counts of the next plane, for the next call
    prefetch_counts<TY>(p, a, xp == p.nx - 1 ? 0 : xp + 1, y0, z0, t, cr);
}

// The three passes with their barriers, for kernels that do not overlap plane_scan with other work.
template <class R, int KS, int TY>
__device__ __forceinline__ void load_plane(const StepParams& p, const StepArrays& a, TileSmem<R, KS, TY>& S,
                                           int rs, int xp, int wpos, int y0, int z0, int t,
                                           int (&cr)[PlaneRegs<TY>::kPer])
{
    PlaneLoad<R, TY> L;
    plane_scan(p, a, S, xp, wpos, y0, z0, t, cr, L);
    __syncthreads();
    plane_assign(S, wpos, t);
    __syncthreads();
    plane_fill(p, a, S, rs, xp, y0, z0, t, cr, L);
}

// Offsets of the q-th Laplacian stencil element (LaplacianStencil::Set order): 27-point stencils
// enumerate x, y, z in -1..1; the 7-point stencil keeps the centre and the six faces.
template <int NS>
__device__ __forceinline__ constexpr int stencil_dx(int q) { return NS == 27 ? q / 9 - 1 : (q == 0 ? -1 : (q == 6 ? 1 : 0)); }
template <int NS>
__device__ __forceinline__ constexpr int stencil_dy(int q) { return NS == 27 ? (q / 3) % 3 - 1 : (q == 1 ? -1 : (q == 5 ? 1 : 0)); }
template <int NS>
__device__ __forceinline__ constexpr int stencil_dz(int q) { return NS == 27 ? q % 3 - 1 : (q == 2 ? -1 : (q == 4 ? 1 : 0)); }

// New grains of neighbour record (pl, r): append them (4-bit slot ids) in the record's entry order.
template <class R, int KS, int TY>
__device__ __forceinline__ void append_fresh(const TileSmem<R, KS, TY>& S, int pl, int r, uint32_t fresh,
                                             uint64_t& ls, int& n, bool& over)
{
    const int cu = S.cntr[pl][r];
    uint64_t lst = S.slotl[pl][r];
    for (int s = 0; s < cu; s++, lst >>= 4)
    {
        const int k = (int)(lst & 15u);
        if ((fresh >> k) & 1u)
        {
            if (n < kListCap) { ls |= (uint64_t)k << (4 * n); n++; }
            else over = true;
        }
    }
}

template <class R, int KS, int TY, int NS>
__global__ void __launch_bounds__(kTileZ * TY)
tile_classify_kernel(const __grid_constant__ StepParams p, const StepArrays a, int xchunk)
{
    using Geo = TileGeom<TY>;
    using Smem = TileSmem<R, KS, TY>;
    constexpr int NT = Geo::NT;
    constexpr int kC = Geo::kCols;
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
    const int blin = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    const long long nblocks = (long long)gridDim.x * gridDim.y * gridDim.z;
    const long long slice0 = (long long)blin * a.slice;
    unsigned char* __restrict__ wbase = a.wl + (long long)blin * a.wl_slice;
    R* __restrict__ vout = static_cast<R*>(a.val_out);

    for (int i = t; i < ClassifyVolSlots<R>::value; i += NT) { S.vol_key[i] = -1; S.vol_sum[i] = 0.0; }
    constexpr int kSlots = WindowSlots<R>::value;
    for (int i = t; i < kSlots * 3 * Geo::kRecs; i += NT) (&S.dense[0][0][0])[i] = R(0);
    for (int i = t; i < 3 * Geo::kRecs; i += NT) (&S.word[0][0])[i] = 0u;
    if (t < kSlots) { S.grain_of[t] = -1; S.lastpos[t] = -1000; }
    if (t < kSlotHash) S.hkey[t] = -1;
    if (t < 32) S.pending[t] = -1;
    if (t <= kListCap) S.nb[t] = 0u;
    if (t < 3) S.cnt[t] = 0ull;
    if (t == 0) { S.woff = 0u; S.crowded = 0u; S.tomb = 0; }
    unsigned wide = 0, ein = 0, eout = 0;
    uint32_t st = 0;
    int acc_g = -1;        // bulk-voxel volume accumulator of this thread
    double acc_v = 0.0;
    int cr[PlaneRegs<TY>::kPer];
    prefetch_counts<TY>(p, a, x0 == 0 ? nx - 1 : x0 - 1, y0, z0, t, cr);
    __syncthreads();

    const int rec0 = (ty + 1) * kC + (tz + 1);

    // plane x0-1+j goes to ring slot j%3 at window position j-1; once three planes are in, the
    // centre plane x = x0+j-2 is processed (one call site of the plane loader keeps the code small)
    const int nj = (x1 - x0) + 2;
    for (int j = 0; j < nj; j++)
    {
        int xp = x0 - 1 + j;
        xp = xp < 0 ? xp + nx : (xp >= nx ? xp - nx : xp);
        // the scan of the incoming plane overlaps the other threads' work on the previous plane;
        // its barrier also ends that work, and the slot hand-out runs only when a grain is new
        {
            PlaneLoad<R, TY> L;
            const bool added = plane_scan(p, a, S, xp, j - 1, y0, z0, t, cr, L);
            if (__syncthreads_or(added))
            {
                plane_assign(S, j - 1, t);
                __syncthreads();
            }
            plane_fill(p, a, S, j % 3, xp, y0, z0, t, cr, L);
        }
        __syncthreads();
        if (j < 2 || !inside) continue;
        const int x = x0 + j - 2;
        const int sl0 = (j - 2) % 3, sl1 = (j - 1) % 3, sl2 = j % 3;
        const long long v = (long long)x * plane + (long long)y * nz + z;

        const int c = S.cntr[sl1][rec0];
        ein += c;
        // ---- flag and (27-point stencils) candidate discovery over the neighbours ----------------
        // One unrolled pass over the 27 bitmask words: the flag bits, and the stencil positions
        // whose record holds a grain not seen at an earlier position (nor in the voxel itself).
        const uint32_t own = S.word[sl1][rec0] & 0xFFFFu;
        uint32_t multi = 0, qfresh = 0;
        {
            uint32_t seen = own;
#pragma unroll
            for (int q = 0; q < 27; q++)
            {
                const int pl = q < 9 ? sl0 : (q < 18 ? sl1 : sl2);
                const int r = rec0 + ((q / 3) % 3 - 1) * kC + (q % 3 - 1);
                const uint32_t w = S.word[pl][r];
                multi |= w;
                if (w & 0xFFFFu & ~seen) qfresh |= 1u << q;
                seen |= w;
            }
        }
        // a neighbour holding a grain the window has no slot for: the general path
        const bool window_bad = (multi >> 30) & 1u;
        uint64_t ls = 0;
        int n = c;
        bool over = window_bad || c > kListCap;
        if (!over) ls = S.slotl[sl1][rec0];   // c <= kListCap entries, unused nibbles are zero
        // candidates in the reference's order: new grains of each neighbour in stencil order and
        // neighbour-list order.  Only the positions marked above bring new grains; the words of the
        // others add nothing to `seen`, so visiting the marked ones in order gives the same list.
        if (NS == 27 && !over && qfresh)
        {
            uint32_t seen = own;
            for (uint32_t m = qfresh; m; m &= m - 1u)
            {
                const int q = __ffs(m) - 1;
                const int pl = q < 9 ? sl0 : (q < 18 ? sl1 : sl2);
                const int r = rec0 + ((q / 3) % 3 - 1) * kC + (q % 3 - 1);
                const uint32_t w = S.word[pl][r] & 0xFFFFu;
                append_fresh(S, pl, r, w & ~seen, ls, n, over);
                if (over) break;
                seen |= w;
            }
        }
        const int flag = c > 1 ? 2 : ((multi >> 31) ? 1 : 0);
        if (flag == 0)
        {
            // bulk voxel: carried over unchanged
            a.cnt_out[v] = (uint8_t)c;
            for (int s = 0; s < c; s++)
            {
                const int g = a.idx_in[s * N + v];
                const R phi = static_cast<const R*>(a.val_in)[s * N + v];
                a.idx_out[s * N + v] = (int16_t)g;
                vout[s * N + v] = phi;
                if (in_volume_window(p, v))
                {
                    // consecutive bulk voxels of a thread mostly belong to one grain: sum them in a
                    // register before the shared-memory add
                    if (g != acc_g)
                    {
                        if (acc_g >= 0) vol_insert_n(S.vol_key, S.vol_sum, ClassifyVolSlots<R>::value, a.vol_acc, acc_g, acc_v);
                        acc_g = g;
                        acc_v = 0.0;
                    }
                    acc_v += (double)phi;
                }
            }
            eout += c;
            continue;
        }
        wide++;
        if (NS != 27 && !over)
        {
            // 7-point Laplacian: its stencil order, then the gradient pass over the 26 neighbours
            uint32_t seen = own;
            const int nq = p.ns + p.ng;
            for (int q = 0; q < nq && !over; q++)
            {
                const signed char* d = q < p.ns ? p.lap_d[q] : p.grad_d[q - p.ns];
                const int pl = d[0] < 0 ? sl0 : (d[0] > 0 ? sl2 : sl1);
                const int r = rec0 + d[1] * kC + d[2];
                const uint32_t fresh = S.word[pl][r] & 0xFFFFu & ~seen;
                if (fresh) append_fresh(S, pl, r, fresh, ls, n, over);
                seen |= fresh;
            }
        }
        if (over || n < 2)
        {
            if (window_bad) atomicAdd(&S.crowded, 1u);
            const unsigned slot = atomicAdd(a.slow_count, 1u);
            if (slot < a.slow_cap) a.slow_list[slot] = (int)v;
            else st |= kStOverflowList;
            continue;
        }
        // ---- values and Laplacians from the dense planes into a work record ----------------------
        const int pad = ((2 * n + 7) / 8) * 8;
        const unsigned off = atomicAdd(&S.woff, (unsigned)(pad + 2 * n * (int)sizeof(R)));
        int16_t* rg = reinterpret_cast<int16_t*>(wbase + off);
        R* rv = reinterpret_cast<R*>(wbase + off + pad);
        for (int k = 0; k < n; k++)
        {
            const int s = (int)((ls >> (4 * k)) & 15u);
            R l = R(0);
#pragma unroll
            for (int q = 0; q < NS; q++)
            {
                const int dx = stencil_dx<NS>(q);
                const int pl = dx < 0 ? sl0 : (dx > 0 ? sl2 : sl1);
                const int r = rec0 + stencil_dy<NS>(q) * kC + stencil_dz<NS>(q);
                l = lap_acc(l, (R)p.lap_w[q], S.dense[s][pl][r]);
            }
            rg[k] = (int16_t)S.grain_of[s];
            rv[k] = S.dense[s][sl1][rec0];
            rv[n + k] = l;
        }
        const unsigned rank = atomicAdd(&S.nb[n], 1u);
        a.bucket[(long long)n * a.bucket_cap + slice0 + rank] =
            make_int2((int)v | (flag == 2 ? (int)0x80000000 : 0), (int)off);
    }
    __syncthreads();
    if (t >= 2 && t <= kListCap) a.bucket_count[t * nblocks + blin] = S.nb[t];
    if (t == 0 && S.crowded) atomicAdd(&a.counters[kCntCrowdedLast], (unsigned long long)S.crowded);
    if (acc_g >= 0) vol_insert_n(S.vol_key, S.vol_sum, ClassifyVolSlots<R>::value, a.vol_acc, acc_g, acc_v);
    flush_block(a, wide, ein, eout, st, S.cnt, S.vol_key, S.vol_sum, ClassifyVolSlots<R>::value, t, NT);
}

// Exclusive prefix of the per-slice bucket counts, one block per list length N = 2..kListCap:
// bucket_off[N][s] = entries of length N in slices before s, bucket_off[N][nslices] = their total.
static __global__ void __launch_bounds__(1024) bucket_scan_kernel(const StepArrays a, int nslices)
{
    __shared__ unsigned s_warp[32];
    const int N = blockIdx.x + 2;
    const unsigned* __restrict__ cnt = a.bucket_count + (long long)N * nslices;
    unsigned* __restrict__ off = a.bucket_off + (long long)N * (nslices + 1);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (nslices + 1023) / 1024;
    const int s0 = min(t * per, nslices), s1 = min(s0 + per, nslices);
    unsigned sum = 0;
    for (int s = s0; s < s1; s++) sum += cnt[s];
    unsigned incl = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        unsigned x = s_warp[lane];
        for (int o = 1; o < 32; o <<= 1)
        {
            const unsigned u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
        }
        s_warp[lane] = x;   // inclusive over warps
    }
    __syncthreads();
    unsigned base = (w > 0 ? s_warp[w - 1] : 0u) + incl - sum;
    for (int s = s0; s < s1; s++) { off[s] = base; base += cnt[s]; }
    if (t == 0) off[nslices] = s_warp[31];
}

constexpr int kChunkTable = 128;   // 32-entry chunks of a compute block whose slices are tabulated
constexpr int kVolCache = 4;       // per-thread grain-volume cache of the compute kernels

// Stages 2-5 for lists of exactly N fields (compile-time), all arrays in registers; the operation
// order is that of list_step.  The entries of length N from all classify slices form one index
// range (bucket_off); each CUDA block takes an equal contiguous part of it, its warps 32
// consecutive entries at a time, so that no warp idles while another drains a long slice.
template <class R, int N, int KS>
__global__ void __launch_bounds__(128) list_compute_kernel(const __grid_constant__ StepParams p, const StepArrays a,
                                                           int nslices)
{
    constexpr int NP = N * (N - 1) / 2;
    __shared__ int s_key[kTileVolSlots];
    __shared__ double s_sum[kTileVolSlots];
    __shared__ unsigned long long s_cnt[3];
    __shared__ int s_chunk[kChunkTable];
    const int t = threadIdx.x;
    const unsigned* __restrict__ off = a.bucket_off + (long long)N * (nslices + 1);
    const unsigned total = off[nslices];
    // whole chunks of 32 entries for every warp of the block: a length with few entries then keeps
    // all warps of fewer blocks busy instead of one warp of many blocks (the others would wait at
    // the final barrier, holding their registers)
    const unsigned per = ((total + gridDim.x * blockDim.x - 1u) / (gridDim.x * blockDim.x)) * blockDim.x;
    const unsigned r0 = blockIdx.x * per;
    if (r0 >= total) return;
    const unsigned r1 = min(total, r0 + per);
    for (int i = t; i < kTileVolSlots; i += blockDim.x) { s_key[i] = -1; s_sum[i] = 0.0; }
    if (t < 3) s_cnt[t] = 0ull;
    // slice of each 32-entry chunk of the block's range
    const unsigned nchunks = (r1 - r0 + 31u) / 32u;
    const bool tabulated = nchunks <= (unsigned)kChunkTable;
    if (tabulated)
        for (unsigned c = t; c < nchunks; c += blockDim.x) s_chunk[c] = slice_of(off, nslices, r0 + 32u * c);
    __syncthreads();
    const long long N_ = p.n;
    const int2* __restrict__ buck = a.bucket + (long long)N * a.bucket_cap;
    // grain-volume contributions of this thread's voxels, most recent grain first (consecutive
    // voxels of a thread lie close together and mostly share their grains)
    int cg[kVolCache];
    double cv[kVolCache];
#pragma unroll
    for (int c = 0; c < kVolCache; c++) { cg[c] = -1; cv[c] = 0.0; }
    constexpr int kPad = ((2 * N + 7) / 8) * 8;
    R* __restrict__ vout = static_cast<R*>(a.val_out);
    uint32_t st = 0;
    unsigned eout = 0;
    const unsigned lane = t & 31u;
    for (unsigned base = r0 + (t - lane); base < r1; base += blockDim.x)   // the same trip count per warp
    {
        const unsigned e = base + lane;
        // slice of the warp's first entry, then of each lane's entry
        int lo = tabulated ? s_chunk[(base - r0) >> 5] : slice_of(off, nslices, base);
        if (e < r1)
        {
        while (off[lo + 1] <= e) lo++;   // off[nslices] = total > e
        const int2 ent = buck[(long long)lo * a.slice + (e - off[lo])];
        const unsigned char* __restrict__ wbase = a.wl + (long long)lo * a.wl_slice;
        const long long v = ent.x & 0x7fffffff;
        const int flag = (ent.x >> 31) ? 2 : 1;
        const int16_t* __restrict__ rg = reinterpret_cast<const int16_t*>(wbase + ent.y);
        const R* __restrict__ rv = reinterpret_cast<const R*>(wbase + ent.y + kPad);
        int g[N];
        R val[N], lap[N];
#pragma unroll
        for (int k = 0; k < N; k++)
        {
            g[k] = rg[k];
            val[k] = rv[k];
            lap[k] = rv[N + k];
        }
        // ---- pair kinetics ---------------------------------------------------------------------
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
        R sg[NP];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i + 1; j < N; j++) sg[pair_pos(i, j, N)] = (R)pair_energy(p, a, g[i], g[j]);
        const R pref = (R)p.pref_do;
        double pv[NP];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i + 1; j < N; j++)
            {
                const int q = pair_pos(i, j, N);
                const double vri = a.vr[g[i]], vrj = a.vr[g[j]];
                const R scale = (vri == 1.0 && vrj == 1.0) ? R(1) : (R)sqrt(vri * vrj);
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
        // ---- driving force (interface voxels only) ----------------------------------------------
        if (p.use_dg && flag == 2)
        {
#pragma unroll
            for (int i = 0; i < N; i++)
#pragma unroll
                for (int j = i + 1; j < N; j++)
                {
                    const double locdG = limited_force(p, a, g[i], g[j]);
                    double norm = sqrt((double)val[i] * (double)val[j]);
                    if (a.gstage[g[i]] == 1 || a.gstage[g[j]] == 1) norm += 1.0e-6;
                    const double dpsi = locdG * (double)(R)pair_mobility(p, a, g[i], g[j]) * norm * p.pref_df;
                    pv[pair_pos(i, j, N)] += dpsi;
                }
        }
        // ---- projection ---------------------------------------------------------------------------
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
        else
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
        // ---- merge (FP64) and finalize --------------------------------------------------------------
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
            if (keep[i] && pos < KS)
            {
                const R w = (m > 1) ? (R)(vd[i] * norm) : R(1);
                if (!isfinite((double)w)) st |= kStNonFinite;
                a.idx_out[pos * N_ + v] = (int16_t)g[i];
                vout[pos * N_ + v] = w;
                if (in_volume_window(p, v))
                {
                    const int gi = g[i];
                    const double wi = (double)w;
                    bool hit = false;
#pragma unroll
                    for (int c = 0; c < kVolCache; c++)
                        if (cg[c] == gi) { cv[c] += wi; hit = true; }
                    if (!hit)
                    {
                        if (cg[kVolCache - 1] >= 0)
                            vol_insert_n(s_key, s_sum, kTileVolSlots, a.vol_acc, cg[kVolCache - 1], cv[kVolCache - 1]);
#pragma unroll
                        for (int c = kVolCache - 1; c > 0; c--) { cg[c] = cg[c - 1]; cv[c] = cv[c - 1]; }
                        cg[0] = gi;
                        cv[0] = wi;
                    }
                }
                pos++;
            }
        }
        if (m == 0) st |= kStEmptyVoxel;
        if (m > KS) st |= kStOverflowK;
        a.cnt_out[v] = (uint8_t)pos;
        eout += pos;
        }
    }
#pragma unroll
    for (int c = 0; c < kVolCache; c++)
        if (cg[c] >= 0) vol_insert_n(s_key, s_sum, kTileVolSlots, a.vol_acc, cg[c], cv[c]);
    flush_block(a, 0u, 0u, eout, st, s_cnt, s_key, s_sum, kTileVolSlots, t, blockDim.x);
}

template <class R, int KS, int KL, int NS>
int launch_tiled_ns(const StepParams& p, const StepArrays& a, void* stream, LaunchInfo* info)
{
    using Smem = TileSmem<R, KS, kTileTY>;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int xchunk = 0, gz = 0, gy = 0, gx = 0;
    tiled_geometry(p.nx, p.ny, p.nz, &xchunk, &gz, &gy, &gx);
    const int nblocks = gz * gy * gx;
    auto kern = tile_classify_kernel<R, KS, kTileTY, NS>;
    const size_t smem = sizeof(Smem);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemsetAsync(a.slow_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    kern<<<dim3(gz, gy, gx), dim3(kTileZ, kTileTY), smem, s>>>(p, a, xchunk);
    if (info && info->after_classify)
    {
        e = cudaEventRecord(static_cast<cudaEvent_t>(info->after_classify), s);
        if (e != cudaSuccess) return (int)e;
    }
    bucket_scan_kernel<<<kListCap - 1, 1024, 0, s>>>(a, nblocks);
    const int cb = compute_blocks(p.n);
    list_compute_kernel<R, 2, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 3, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 4, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 5, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 6, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 7, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    list_compute_kernel<R, 8, KS><<<cb, 128, 0, s>>>(p, a, nblocks);
    // general path: one warp per voxel of the worklist
    {
        auto gk = warp_general_kernel<R, KS, KL>;
        const size_t wsm = 4 * sizeof(WarpScratch<R, KL>);
        e = cudaFuncSetAttribute(gk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
        if (e != cudaSuccess) return (int)e;
        gk<<<148 * 4, 128, wsm, s>>>(p, a);
    }
    if (info) info->kernels += 10;
    return (int)cudaGetLastError();
}

// The classify kernel and the bucket scan (work records, length buckets and their offsets,
// general-path worklist, bulk copies): the adjoint reverses the lists they leave.  Returns the number of classify blocks (the slices of
// the buckets) or a negative error.
template <class R, int KS, int NS>
int launch_classify_ns(const StepParams& p, const StepArrays& a, void* stream)
{
    using Smem = TileSmem<R, KS, kTileTY>;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int xchunk = 0, gz = 0, gy = 0, gx = 0;
    tiled_geometry(p.nx, p.ny, p.nz, &xchunk, &gz, &gy, &gx);
    auto kern = tile_classify_kernel<R, KS, kTileTY, NS>;
    const size_t smem = sizeof(Smem);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return -(int)e;
    e = cudaMemsetAsync(a.slow_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return -(int)e;
    kern<<<dim3(gz, gy, gx), dim3(kTileZ, kTileTY), smem, s>>>(p, a, xchunk);
    bucket_scan_kernel<<<kListCap - 1, 1024, 0, s>>>(a, gz * gy * gx);
    e = cudaGetLastError();
    return e == cudaSuccess ? gz * gy * gx : -(int)e;
}

template <class R>
int launch_classify(const StepParams& p, const StepArrays& a, int k_slots, void* stream)
{
    const bool ns27 = p.ns == 27;
    switch (k_slots)
    {
        case 8:  return ns27 ? launch_classify_ns<R, 8, 27>(p, a, stream) : launch_classify_ns<R, 8, 7>(p, a, stream);
        case 12: return ns27 ? launch_classify_ns<R, 12, 27>(p, a, stream) : launch_classify_ns<R, 12, 7>(p, a, stream);
        case 16: return ns27 ? launch_classify_ns<R, 16, 27>(p, a, stream) : launch_classify_ns<R, 16, 7>(p, a, stream);
        default: return -1;
    }
}

template <class R, int KS, int KL>
int launch_tiled(const StepParams& p, const StepArrays& a, void* stream, LaunchInfo* info)
{
    if (p.ns == 27) return launch_tiled_ns<R, KS, KL, 27>(p, a, stream, info);
    if (p.ns == 7) return launch_tiled_ns<R, KS, KL, 7>(p, a, stream, info);
    return -1;
}

template <class R>
int launch_step(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                LaunchInfo* info)
{
    if (variant == kVariantGeneric || p.aniso || a.df_lim)
    {
        // anisotropic energies need the gradients of every list entry, and the averaged driving
        // force is read per voxel pair: the per-voxel generic kernel only (the tiled kernels stay
        // free of both)
        if (info) info->kernels += 1;
        return launch_step_generic<R>(p, a, k_slots, stream);
    }
    switch (k_slots)
    {
        case 8:  return launch_tiled<R, 8, 16>(p, a, stream, info);
        case 12: return launch_tiled<R, 12, 20>(p, a, stream, info);
        case 16: return launch_tiled<R, 16, 24>(p, a, stream, info);
        default: return -1;
    }
}

}  // namespace opgpu
