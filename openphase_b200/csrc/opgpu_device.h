// Device-side data layout and launch interface of the fused multiphase-field step.
//
// State (one buffer of a ping-pong pair), structure of arrays over N = nx*ny*nz voxels:
//   cnt[N]        uint8   number of stored (positive) fields of the voxel
//   idx[K][N]     int16   grain index of slot s        (slot plane s at idx + s*N)
//   val[K][N]     real    phase-field value of slot s  (real = double or float)
// Slots s >= cnt[v] are never read.  Only positive entries are stored (what NodePF holds after
// NodePF::finalize); the zero-valued candidate entries the reference appends in
// CalculateDerivativesSR are re-derived inside the step kernel from the 3x3x3 neighbourhood.
// A voxel's interface flag is never stored: flag = 2 if cnt > 1, else 1 if any of its 26 periodic
// neighbours has cnt > 1, else 0 (identical to NodePF::finalize + PhaseField::SetFlagsSR).
#pragma once
#include <stdint.h>

namespace opgpu {

constexpr int kMaxPhases = 8;

enum : uint32_t {
    kStOverflowK = 1u << 0,
    kStOverflowList = 1u << 1,
    kStEmptyVoxel = 1u << 2,
    kStNormalizeWarn = 1u << 3,
    kStLimiterCap = 1u << 4,
    kStNonFinite = 1u << 5,
    kStAdjointMismatch = 1u << 6,   // the recomputed step does not reproduce the stored next state
    kStAverageSkipped = 1u << 7,    // driving-force averaging ran out of its pair storage for a voxel
                                    // (its pairs kept the raw force)
};

// Driving-force averaging (average.cu).  Every interface voxel's pairs of stored fields get one
// slot each in compact storage: off[v] is the voxel's first slot (exclusive scan of c(c-1)/2 over
// the voxels with c > 1 stored fields); a voxel whose slots would pass cap is skipped.
struct AvgArrays {
    unsigned* npairs;            // [N] pairs of stored fields of interface voxels, then scanned into off
    unsigned* off;               // [N] first slot of each voxel
    double* tmp;                 // [cap] CollectAverage's tmp per stored pair
    double* lim;                 // [cap] the averaged, limited force per stored pair
    unsigned cap;
    const signed char* off3;     // [noff][3] sphere offsets with Range - |d| > 0, in loop order
    int noff;
    double weight_threshold;     // sqrt(Threshold (1 - Threshold))
    void* scan_tmp;              // device scratch of the scan
    size_t scan_bytes;
};

// counters[] slots: the step kernel adds into the per-step slots 0-2; the grain-update kernel rolls
// them into the running totals and clears them.
enum {
    kCntWide = 0, kCntEntriesIn = 1, kCntEntriesOut = 2, kCntOverflowVoxels = 3,
    kCntWideTotal = 4, kCntEntriesInTotal = 5, kCntEntriesOutTotal = 6, kCntWideLast = 7, kCntSteps = 8,
    kCntGeneralLast = 9,      // voxels the last step sent through the general per-voxel path
    kCntGeneralTotal = 10,
    kCntCrowdedLast = 11,     // of those, voxels whose window held more grains than slots
    kCntCrowdedTotal = 12,
    kNumCounters = 13
};

// Bytes of a work-list record with n fields of type R: grains padded to 8 bytes, values, Laplacians.
__host__ __device__ constexpr int work_record_bytes(int n, int rsz) { return ((2 * n + 7) / 8) * 8 + 2 * n * rsz; }

struct StepParams {
    int nx, ny, nz;
    long long n;
    // Laplacian stencil (LaplacianStencil::Set order) and the neighbour set used to discover
    // candidates after it (GradientStencil::Set order), both with periodic offsets.
    int ns;
    signed char lap_d[27][3];
    double lap_w[27];
    int ng;
    signed char grad_d[27][3];
    double pref_do;          // Pi^2/Eta^2 (DoubleObstacle.cpp:504)
    double pref_df;          // Pi/Eta     (DrivingForce.cpp:507)
    double dt;
    double eps_snap;         // finalize snap/erase threshold (DBL_EPSILON in the FP64 form)
    int nphases;
    double sigma_p[kMaxPhases * kMaxPhases];
    double mu_p[kMaxPhases * kMaxPhases];
    double allowed_p[kMaxPhases * kMaxPhases];   // Limit*Prefactor*MaxEnergy*RegularizationFactor
    int limiting;
    double tj_factor;
    int consider_nucleus_volume;
    int pair_mode;           // OPGPU_PAIRS_*
    unsigned long long hash_seed;
    double hash_lo, hash_span;
    int ngrains;
    int use_dg;
    // anisotropic interface energy (InterfaceProperties::SetSR, src/InterfaceProperties.cpp:617-673):
    // per phase pair the model (0 ISO, 1 CUBIC, 2 DISORIENTATION, 3 HEXBOETTGER, 4 HEXSUN, 5 HEXYANG),
    // its Epsilon1 (eps_p) and Epsilon2..4 (eps_x) and MaxEnergy; per phase solid (1) or
    // liquid (0); the gradient stencil in GradientStencil::Set order with its weights per axis
    int aniso;
    signed char emodel[kMaxPhases * kMaxPhases];
    double eps_p[kMaxPhases * kMaxPhases];
    double eps_x[kMaxPhases * kMaxPhases][3];
    int facet_lo[kMaxPhases * kMaxPhases], facet_hi[kMaxPhases * kMaxPhases];   // FACETED: rows of facets
    signed char mmodel[kMaxPhases * kMaxPhases];   // mobility model per phase pair (codes of emodel)
    int mfacet_lo[kMaxPhases * kMaxPhases], mfacet_hi[kMaxPhases * kMaxPhases];   // FACETED mobility rows
    double meps[kMaxPhases * kMaxPhases][4];       // its Epsilon1..4
    double maxe_p[kMaxPhases * kMaxPhases];
    signed char solid_p[kMaxPhases];
    int ngs;
    signed char gs_d[27][3];
    double gs_w[27][3];
    // x-planes [vol_x0, vol_x1) count in the grain volumes (all planes unless a slab of a larger
    // grid: its halo planes are excluded)
    int vol_x0, vol_x1;
};

// Whether voxel v lies in the planes that count in the grain volumes.
__device__ __forceinline__ bool in_volume_window(const StepParams& p, long long v)
{
    if (p.vol_x0 == 0 && p.vol_x1 == p.nx) return true;
    const int x = (int)(v / ((long long)p.ny * p.nz));
    return x >= p.vol_x0 && x < p.vol_x1;
}

struct StepArrays {
    const uint8_t* cnt_in;
    const int16_t* idx_in;
    const void* val_in;
    uint8_t* cnt_out;
    int16_t* idx_out;
    void* val_out;
    const double* vr;          // [G] VolumeRatio
    const int16_t* gphase;     // [G]
    const int8_t* gstage;      // [G]
    const double* dg;          // [G] or null
    const double* pair_sigma;  // [G*G] or null
    const double* pair_mu;     // [G*G] or null
    const double* dg_pair;     // [G*G] limited driving force per grain pair, or null (evaluated in place)
    const double* df_lim;      // averaged limited force per stored pair (slot df_off[v] + pair), or null
    const unsigned* df_off;    // [N] first pair slot of each voxel (averaging)
    unsigned df_cap;           // pair slots
    const double* grot;        // [G*9] grain rotation matrices (row-major), for anisotropic energies
    double* vol_acc;           // [G] volume accumulator of the output state (zeroed by the caller)
    uint32_t* status;          // soft status bits
    unsigned long long* counters;  // kNumCounters
    // overflow worklist of the tiled kernel (voxels whose lists exceed its register capacity)
    int* slow_list;            // [slow_cap]
    unsigned* slow_count;      // reset by the launcher before every step
    unsigned slow_cap;
    // work buffer between the classify kernel and the per-length compute kernels: every list is a
    // record of n fields (int16 grains padded to 8 bytes, then n values, then n Laplacians) packed
    // in its classify block's byte slice; bucket entries (voxel | flag2 << 31, record offset)
    unsigned char* wl;         // [blocks][wl_slice] bytes
    long long wl_slice;        // bytes per classify block
    int2* bucket;              // [kListCap + 1][bucket_cap] entries per list length, block-private slices
    unsigned* bucket_count;    // [kListCap + 1][max blocks] entries per slice
    unsigned* bucket_off;      // [kListCap + 1][blocks + 1] exclusive prefix of bucket_count per list
                               // length, then the length's total
    const double* facets;      // FACETED: rows of (unit facet normal x, y, z, SigmaF, EpsilonEF)
    long long bucket_cap;
    int slice;                 // entries per classify-block slice
};

constexpr int kListCap = 8;    // list capacity of the split kernels (longer lists: overflow worklist)
constexpr int kTileCols = 16;  // tile of the classify kernel: kTileCols (z) x kTileRows (y) voxels,
constexpr int kTileRows = 8;   // one thread each

// Launch geometry of the classify kernel: tiles of kTileCols (z) x kTileRows (y) voxels marching over
// `xchunk` x-planes; enough x-chunks for several blocks per SM on small grids, long chunks (halo
// reuse) on large ones.  slice = voxels one block can append to a bucket.
inline void tiled_geometry(int nx, int ny, int nz, int* xchunk, int* gz, int* gy, int* gx)
{
    const int tzb = (nz + kTileCols - 1) / kTileCols, tyb = (ny + kTileRows - 1) / kTileRows;
    long long xc = (long long)nx * tzb * tyb / (148 * 8);
    xc = xc < 2 ? 2 : (xc > 32 ? 32 : xc);
    *xchunk = (int)xc;
    *gz = tzb;
    *gy = tyb;
    *gx = (int)((nx + xc - 1) / xc);
}

enum { kVariantTiled = 0, kVariantGeneric = 1 };

// Filled by the launchers: kernels launched, and an event recorded after the classify kernel
// (when `after_classify` is not null) so the caller can time it separately.
struct LaunchInfo {
    void* after_classify = nullptr;   // cudaEvent_t
    int kernels = 0;
};

// Launchers (defined in step_f64.cu / step_f32.cu).  k_slots in {8, 12, 16}; variant selects the
// tiled production kernel or the full-grid generic kernel (same results, used for validation).
int launch_step_f64(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                    LaunchInfo* info);
int launch_step_f32(const StepParams& p, const StepArrays& a, int k_slots, int variant, void* stream,
                    LaunchInfo* info);
// The classify kernel of the tiled step alone; returns the number of classify blocks or < 0.
int launch_classify_f64(const StepParams& p, const StepArrays& a, int k_slots, void* stream);
int launch_classify_f32(const StepParams& p, const StepArrays& a, int k_slots, void* stream);
// Driving-force averaging of a state (average.cu): launch_average_scan counts the pair slots of
// every voxel, scans them into aa.off and writes their total to d_total; launch_average then writes
// aa.tmp and aa.lim.  average_scan_bytes gives the scan's scratch bytes for n voxels.
size_t average_scan_bytes(long long n);
int launch_average_scan(long long n, const AvgArrays& aa, const uint8_t* cnt, unsigned long long* d_total, void* stream);
int launch_average(const StepParams& p, const AvgArrays& aa, const uint8_t* cnt, const int16_t* idx,
                   const void* val, bool fp32, const double* vr, const double* dg, const int16_t* gphase,
                   uint32_t* status, void* stream);
// Add the volumes of the window planes of a state to vol_acc (defined in step_f64.cu).
int launch_volume_recount(const StepParams& p, const uint8_t* cnt, const int16_t* idx, const void* val, int fp32,
                          double* vol_acc, void* stream);

}  // namespace opgpu
