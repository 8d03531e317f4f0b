// opgpu context: device memory, parameter tables, state upload/download, grain records and the
// step loop of the C ABI declared in include/opgpu.h.
#include "opgpu.h"
#include "adjoint.h"
#include "opgpu_device.h"
#include "opgpu_host.h"

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

using namespace opgpu;

struct opgpu_ctx {
    opgpu_grid grid{};
    int device = 0;
    cudaStream_t stream = nullptr;
    void* adj_side = nullptr;            // adjoint: side stream of the worklist kernel, fork / join events
    void* adj_fork = nullptr;
    void* adj_join = nullptr;
    std::string err;
    long long n = 0;
    int K = 8;
    int fp32 = 0;
    size_t rsz = 8;
    // ping-pong state
    uint8_t* cnt[2] = {nullptr, nullptr};
    int16_t* idx[2] = {nullptr, nullptr};
    void* val[2] = {nullptr, nullptr};
    int cur = 0;
    // grain records
    int G = 0;
    double *d_vr = nullptr, *d_volume = nullptr, *d_maxvol = nullptr, *d_refvol = nullptr, *d_vol_acc = nullptr;
    int16_t* d_gphase = nullptr;
    int8_t *d_gstage = nullptr, *d_exist = nullptr;
    double *d_dg = nullptr, *d_pair_sigma = nullptr, *d_pair_mu = nullptr;
    double* d_dg_pair = nullptr;     // limited driving force per grain pair (G <= kMaxPairTableGrains)
    double* d_grot = nullptr;        // [G*9] grain rotation matrices (identity unless oriented)
    double* d_facets = nullptr;      // FACETED: rows of (unit facet normal, SigmaF, EpsilonEF)
    // checkpoints of the state and the grain records (adjoint rollouts)
    struct Slot {
        uint8_t* cnt = nullptr; int16_t* idx = nullptr; void* val = nullptr;
        double *volume = nullptr, *maxvol = nullptr, *vr = nullptr;
        int8_t *exist = nullptr, *stage = nullptr;
    };
    std::vector<Slot> slots;
    // adjoint / tangent-linear buffers (allocated on first use)
    double *d_lam[2] = {nullptr, nullptr};
    double* d_lam_local = nullptr;
    uint8_t* d_lcnt = nullptr;
    int16_t* d_lidx = nullptr;
    double* d_llam = nullptr;
    double *d_gsig = nullptr, *d_gmu = nullptr, *d_gdg = nullptr;
    double *d_tsig = nullptr, *d_tmu = nullptr, *d_tdg = nullptr;
    double* d_dphi[2] = {nullptr, nullptr};
    double* d_tvol = nullptr;
    int lam_cur = 0, dphi_cur = 0;
    bool adjoint_ready = false, tlm_ready = false;
    bool dg_pair_dirty = true;
    // DISORIENTATION energies: per-grain-pair table built on the host from the orientations
    std::vector<int16_t> h_gphase;      // [G] phase of every grain
    std::vector<double> h_quat;         // [G*4] orientations (s, x, y, z) as given; empty: unrotated
    std::vector<double> h_user_sigma;   // [G*G] energies given to opgpu_set_pair_table; empty: none
    std::vector<double> h_dg;           // [G] driving forces given to opgpu_set_driving_force
    std::vector<double> h_dg_pair;      // [G*G] host side of the limited driving-force table
    bool pair_energy_dirty = true;
    uint32_t* d_status = nullptr;
    unsigned long long* d_counters = nullptr;
    int* d_slow_list = nullptr;      // overflow worklist of the tiled kernel (capacity N)
    unsigned* d_slow_count = nullptr;
    // work buffer of the classify / compute split (see tile_kernel.cuh)
    unsigned char* d_wl = nullptr;
    long long wl_slice = 0;
    int2* d_bucket = nullptr;
    unsigned* d_bucket_count = nullptr;
    unsigned* d_bucket_off = nullptr;
    long long bucket_cap = 0;
    int slice = 0;
    int variant = kVariantTiled;
    StepParams sp{};
    bool model_set = false, state_loaded = false, initialized = false;
    uint32_t status = 0;
    double nvf = 1.0;   // NucleusVolumeFactor
    // per-step timing of the step kernels (events: start, after classify, end)
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;          // event triples recorded and not yet read
    long long timed_launches = 0;
    double timed_ms = 0.0;
    double timed_classify_ms = 0.0;
    long long kernel_launches = 0;   // kernels of this library launched on the context's stream
    int8_t* noalloc_scratch = nullptr;   // device address of the allocation-free flag scratch
    bool stream_ordered = false;         // slab calls enqueue only (the caller orders its streams)
    // driving-force averaging ($Average Yes)
    bool averaging = false;
    int avg_range = 0;
    double avg_threshold = 0.0;
    double *d_df_tmp = nullptr, *d_df_lim = nullptr;
    unsigned *d_df_npairs = nullptr, *d_df_off = nullptr;
    unsigned long long* d_df_total = nullptr;
    unsigned df_cap = 0;
    void* d_df_scan = nullptr;
    size_t df_scan_bytes = 0;
    signed char* d_avg_off = nullptr;
    int avg_noff = 0;
};

namespace {

constexpr double kPi = 3.14159265358979323846;   // include/Globals.h:124

uint32_t fail(opgpu_ctx* c, uint32_t code, const std::string& msg)
{
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ctx, OPGPU_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T) + 16);
}

void dfree(void* p)
{
    if (p) cudaFree(p);
}

// ------------------------------------------------------------------------------------ kernels

__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }

// Ragged lists -> K-slot state; voxels with more than one entry go through NodePF::finalize
// (include/Containers/NodePF.h:214-255), which FinalizeSR applies to the flag-2 voxels that
// NodePF::read produced (NodePF.h:751-763).
template <class R>
__global__ void load_kernel(long long N, int K, int G, const int32_t* counts, const long long* offsets,
                            const int32_t* idx, const double* val, uint8_t* cnt_out, int16_t* idx_out,
                            R* val_out, uint32_t* status, double* vol_acc)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int c = counts[v];
    const long long off = offsets[v];
    uint32_t st = 0;
    if (c > 1)
    {
        double total = 0.0;
        int m = 0;
        int gs[64];
        double vs[64];
        for (int i = 0; i < c; i++)
        {
            double w = val[off + i];
            bool erase = false;
            if (w >= 1.0 - DBL_EPSILON) w = 1.0;
            if (w <= 0.0 + DBL_EPSILON) { w = 0.0; erase = true; }
            total += w;
            if (!erase && m < 64) { gs[m] = idx[off + i]; vs[m] = w; m++; }
        }
        if (m > 1)
        {
            const double norm = 1.0 / total;
            for (int i = 0; i < m; i++) vs[i] *= norm;
        }
        else if (m == 1)
        {
            vs[0] = 1.0;
        }
        else
        {
            st |= kStEmptyVoxel;
        }
        if (m > K) { st |= kStOverflowK; m = K; }
        cnt_out[v] = (uint8_t)m;
        for (int i = 0; i < m; i++)
        {
            idx_out[i * N + v] = (int16_t)gs[i];
            val_out[i * N + v] = (R)vs[i];
            atomicAdd(&vol_acc[gs[i]], (double)(R)vs[i]);
        }
    }
    else
    {
        if (c == 0) st |= kStEmptyVoxel;
        cnt_out[v] = (uint8_t)c;
        if (c == 1)
        {
            idx_out[v] = (int16_t)idx[off];
            val_out[v] = (R)val[off];
            atomicAdd(&vol_acc[idx[off]], (double)(R)val[off]);
        }
    }
    if (st) atomicOr(status, st);
}

// PhaseField::CalculateGrainsVolume tail (src/PhaseField.cpp:896-951): MAXVolume, VolumeRatio,
// Exist/Stage bookkeeping; block 0 also rolls the per-step counters into their totals.
__global__ void grains_update_kernel(int G, double* vol_acc, double* volume, double* maxv, const double* refv,
                                     double* vr, int8_t* exist, int8_t* stage, unsigned long long* counters,
                                     int count_step)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0 && count_step)
    {
        counters[kCntWideTotal] += counters[kCntWide];
        counters[kCntEntriesInTotal] += counters[kCntEntriesIn];
        counters[kCntEntriesOutTotal] += counters[kCntEntriesOut];
        counters[kCntWideLast] = counters[kCntWide];
        counters[kCntSteps] += 1;
        counters[kCntGeneralTotal] += counters[kCntGeneralLast];
        counters[kCntGeneralLast] = 0;
        counters[kCntCrowdedTotal] += counters[kCntCrowdedLast];
        counters[kCntCrowdedLast] = 0;
        counters[kCntWide] = 0;
        counters[kCntEntriesIn] = 0;
        counters[kCntEntriesOut] = 0;
    }
    if (g >= G) return;
    double V = vol_acc[g];
    vol_acc[g] = 0.0;
    const double mx = dmax_ref(V, maxv[g]);
    double r = mx / refv[g];
    double m = mx;
    if (exist[g] && V <= 0.0)
    {
        exist[g] = 0;
        stage[g] = OPGPU_STAGE_STABLE;
        V = 0.0;
        m = 0.0;
        r = 1.0;
    }
    else if (V > 0.0)
    {
        exist[g] = 1;
        if (stage[g] == OPGPU_STAGE_SEED) stage[g] = OPGPU_STAGE_NUCLEUS;
        if (r > 1.0)
        {
            stage[g] = OPGPU_STAGE_STABLE;
            r = 1.0;
        }
    }
    volume[g] = V;
    maxv[g] = m;
    vr[g] = r;
}

__global__ void counts_kernel(long long N, const uint8_t* cnt, int32_t* counts, long long* wide)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) { counts[v] = cnt[v]; wide[v] = cnt[v]; }
}

__global__ void widen_kernel(long long N, const int32_t* counts, long long* wide)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) wide[v] = counts[v];
}

template <class R>
__global__ void gather_kernel(long long N, const uint8_t* cnt, const int16_t* idx, const R* val,
                              const long long* offsets, int32_t* idx_out, double* val_out)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int c = cnt[v];
    const long long off = offsets[v];
    for (int s = 0; s < c; s++)
    {
        idx_out[off + s] = idx[s * N + v];
        val_out[off + s] = (double)val[s * N + v];
    }
}

__global__ void flags_kernel(int nx, int ny, int nz, const uint8_t* cnt, int8_t* flags)
{
    const long long N = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int z = (int)(v % nz);
    const int y = (int)((v / nz) % ny);
    const int x = (int)(v / ((long long)ny * nz));
    int f = cnt[v] > 1 ? 2 : 0;
    for (int q = 0; q < 27 && f == 0; q++)
    {
        const int xx = (x + q / 9 - 1 + nx) % nx, yy = (y + (q / 3) % 3 - 1 + ny) % ny, zz = (z + q % 3 - 1 + nz) % nz;
        if (cnt[((long long)xx * ny + yy) * nz + zz] > 1) f = 1;
    }
    flags[v] = (int8_t)f;
}

unsigned grid_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

void free_grains(opgpu_ctx* c)
{
    dfree(c->d_vr); dfree(c->d_volume); dfree(c->d_maxvol); dfree(c->d_refvol); dfree(c->d_vol_acc);
    dfree(c->d_gphase); dfree(c->d_gstage); dfree(c->d_exist); dfree(c->d_dg);
    dfree(c->d_pair_sigma); dfree(c->d_pair_mu); dfree(c->d_dg_pair); dfree(c->d_grot);
    c->d_grot = nullptr;
    c->d_vr = c->d_volume = c->d_maxvol = c->d_refvol = c->d_vol_acc = nullptr;
    c->d_gphase = nullptr; c->d_gstage = c->d_exist = nullptr;
    c->d_dg = c->d_pair_sigma = c->d_pair_mu = c->d_dg_pair = nullptr;
    c->dg_pair_dirty = true;
    c->h_quat.clear();
    c->h_user_sigma.clear();
    c->pair_energy_dirty = true;
}

// Tools::getDisorientationCubic (src/Tools.cpp:626-678): rotation angle 2*acos(max |c|) of
// dQ = A * B.inverted() over the 24 component combinations c of the cubic group (Grimmer 1974),
// with the reference's factors 0.707 and 0.5; quaternion product and inverse as
// include/Containers/Quaternion.h:257-266, 313-339 (component 0 = s).  Host code, so that log and
// acos are the host library's, as in the reference.
double disorientation_cubic(const double* A, const double* B)
{
    const double bs = B[0], bx = B[1], by = B[2], bz = B[3];
    const double n2 = bs * bs + (bx * bx + by * by + bz * bz);
    const double is = bs / n2, ix = (bx * (-1.0)) / n2, iy = (by * (-1.0)) / n2, iz = (bz * (-1.0)) / n2;
    const double as = A[0], ax = A[1], ay = A[2], az = A[3];
    const double d1 = ax * is + ay * iz - az * iy + as * ix;
    const double d2 = -ax * iz + ay * is + az * ix + as * iy;
    const double d3 = ax * iy - ay * ix + az * is + as * iz;
    const double d0 = -ax * ix - ay * iy - az * iz + as * is;
    const double c[24] = {
        d0, d1, d2, d3,
        (d0 + d1) * 0.707, (d0 - d1) * 0.707, (d2 + d3) * 0.707, (d2 - d3) * 0.707,
        (d0 + d2) * 0.707, (d0 - d2) * 0.707, (d1 + d3) * 0.707, (d1 - d3) * 0.707,
        (d0 + d3) * 0.707, (d0 - d3) * 0.707, (d1 + d2) * 0.707, (d1 - d2) * 0.707,
        (d0 + d1 + d2 + d3) * 0.5, (d0 + d1 - d2 - d3) * 0.5, (d0 - d1 + d2 - d3) * 0.5, (d0 - d1 - d2 + d3) * 0.5,
        (d0 + d1 + d2 - d3) * 0.5, (d0 + d1 - d2 + d3) * 0.5, (d0 - d1 + d2 + d3) * 0.5, (d0 - d1 - d2 - d3) * 0.5};
    double m = 0.0;
    for (int k = 0; k < 24; k++)
        if (m < std::fabs(c[k])) m = std::fabs(c[k]);
    return 2 * std::acos(m);
}

// The facet normals a FACETED facet (h, k, l) stands for: itself, or with $NfacetFamilies every
// distinct vector of its family (index permutations with sign changes, the set that
// Tools::findIndexPermutations enumerates, src/Tools.cpp:37-260), each normalised as
// iVector3::normalized (include/Containers/iVector3.h:274-289).  The model takes the facet of
// largest cos^2, so the order within a family does not matter.
void facet_normals(long h, long k, long l, bool family, std::vector<double>& out)
{
    std::vector<std::array<long, 3>> v;
    if (!family)
        v.push_back({h, k, l});
    else
    {
        const long a[3] = {std::labs(h), std::labs(k), std::labs(l)};
        const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        for (const auto& pm : perm)
            for (int sg = 0; sg < 8; sg++)
            {
                std::array<long, 3> w = {a[pm[0]] * ((sg & 1) ? -1 : 1), a[pm[1]] * ((sg & 2) ? -1 : 1),
                                         a[pm[2]] * ((sg & 4) ? -1 : 1)};
                bool dup = false;
                for (const auto& u : v) dup |= u == w;
                if (!dup) v.push_back(w);
            }
    }
    for (const auto& w : v)
    {
        const double norm = std::sqrt((double)(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]));
        if (norm != 0.0)
        {
            const double inv = 1.0 / norm;
            out.push_back(w[0] * inv); out.push_back(w[1] * inv); out.push_back(w[2] * inv);
        }
        else
        {
            out.push_back(0.0); out.push_back(0.0); out.push_back(0.0);
        }
    }
}

// InterfaceEnergyModel::CalculateDisorientation (include/InterfaceProperties/InterfaceEnergyModel.h:
// 308-323): Read-Shockley-type energy of the disorientation angle, constant above 0.349066 rad.
double disorientation_energy(const double* A, const double* B)
{
    const double constant = 0.85;
    const double mis = disorientation_cubic(A, B);
    if (mis <= 0.349066) return mis * constant * (0.8 - std::log(mis));
    return 0.349066 * constant * (0.8 - std::log(0.349066));
}

// Grain counts up to which the limited driving force is tabulated per grain pair (8 * G^2 bytes:
// 3.2 GB of device memory at 20000 grains): every count the int16 grain indices allow.
constexpr int kMaxPairTableGrains = 32767;

// Stencil tables: LaplacianStencil3D_7 / _27a / _LB (include/Containers/LaplacianStencil.h:72-156)
// and the neighbour sets of GradientStencil1D / 3D / 3D_LB (include/Containers/GradientStencil.h),
// enumerated in the x, y, z loop order of LaplacianStencil::Set / GradientStencil::Set.
void set_stencils(StepParams& sp, int lap, int grad, double dx)
{
    sp.ns = 0;
    for (int x = -1; x <= 1; ++x)
    for (int y = -1; y <= 1; ++y)
    for (int z = -1; z <= 1; ++z)
    {
        const int d = (x != 0) + (y != 0) + (z != 0);
        double w;
        if (lap == OPGPU_STENCIL_SIMPLE)
            w = (d == 0) ? -6.0 : (d == 1 ? 1.0 : 0.0);
        else if (lap == OPGPU_STENCIL_ISOTROPIC)
            w = (d == 0) ? -64.0 / 15.0 : (d == 1 ? 7.0 / 15.0 : (d == 2 ? 1.0 / 10.0 : 1.0 / 30.0));
        else
            w = (d == 0) ? -38.0 / 9.0 : (d == 1 ? 4.0 / 9.0 : (d == 2 ? 1.0 / 9.0 : 1.0 / 36.0));
        if (w != 0.0)
        {
            sp.lap_d[sp.ns][0] = (signed char)x;
            sp.lap_d[sp.ns][1] = (signed char)y;
            sp.lap_d[sp.ns][2] = (signed char)z;
            sp.lap_w[sp.ns] = w / (dx * dx);
            sp.ns++;
        }
    }
    // GradientStencil::Set (include/Containers/GradientStencil.h:132-155) over GradientStencil1D
    // (:46-56), GradientStencil3D (:82-92) and GradientStencil3D_LB (:108-118): weight c*table/dx
    sp.ngs = 0;
    for (int x = -1; x <= 1; ++x)
    for (int y = -1; y <= 1; ++y)
    for (int z = -1; z <= 1; ++z)
    {
        const int d = (x != 0) + (y != 0) + (z != 0);
        double t;
        if (grad == OPGPU_STENCIL_SIMPLE)
            t = (d == 1) ? 0.5 : 0.0;
        else if (grad == OPGPU_STENCIL_ISOTROPIC)
            t = (d == 0) ? 0.0 : (d == 1 ? 1.0 / 4.64 : (d == 2 ? 0.245 / 4.64 : 0.085 / 4.64));
        else
            t = (d == 0) ? 0.0 : (d == 1 ? 2.0 / 9.0 : (d == 2 ? 1.0 / 18.0 : 1.0 / 72.0));
        if (t != 0.0)
        {
            sp.gs_d[sp.ngs][0] = (signed char)x;
            sp.gs_d[sp.ngs][1] = (signed char)y;
            sp.gs_d[sp.ngs][2] = (signed char)z;
            sp.gs_w[sp.ngs][0] = x * t / dx;
            sp.gs_w[sp.ngs][1] = y * t / dx;
            sp.gs_w[sp.ngs][2] = z * t / dx;
            sp.ngs++;
        }
    }
    // Candidate discovery by the gradient pass only matters when the Laplacian misses neighbours
    // the gradient stencil visits (SIMPLE Laplacian with a 26-neighbour gradient stencil).
    sp.ng = 0;
    if (sp.ns < 27 && grad != OPGPU_STENCIL_SIMPLE)
    {
        for (int x = -1; x <= 1; ++x)
        for (int y = -1; y <= 1; ++y)
        for (int z = -1; z <= 1; ++z)
        {
            if (!x && !y && !z) continue;
            sp.grad_d[sp.ng][0] = (signed char)x;
            sp.grad_d[sp.ng][1] = (signed char)y;
            sp.grad_d[sp.ng][2] = (signed char)z;
            sp.ng++;
        }
    }
}

uint32_t read_status(opgpu_ctx* ctx)
{
    uint32_t st = 0;
    CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < ctx->ev_used; i++)
    {
        float ms = 0.f, ms_c = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev_pool[3 * i], ctx->ev_pool[3 * i + 2]));
        CK(cudaEventElapsedTime(&ms_c, ctx->ev_pool[3 * i], ctx->ev_pool[3 * i + 1]));
        ctx->timed_ms += ms;
        ctx->timed_classify_ms += ms_c;
        ctx->timed_launches++;
    }
    ctx->ev_used = 0;
    ctx->status |= st;
    return st;
}

uint32_t require(opgpu_ctx* ctx, bool cond, const char* what)
{
    if (!ctx) return OPGPU_E_INVALID;
    if (!cond) return fail(ctx, OPGPU_E_STATE, what);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, OPGPU_E_CUDA, cudaGetErrorString(e));
    return OPGPU_OK;
}

}  // namespace

// ==================================================================================== C ABI

extern "C" int32_t opgpu_abi_version(void) { return OPGPU_ABI_VERSION; }

#ifndef OPGPU_SOURCE_HASH
#define OPGPU_SOURCE_HASH "unstamped"
#endif
extern "C" const char* opgpu_build_info(void)
{
    return "opgpu sm_100a source " OPGPU_SOURCE_HASH;
}

extern "C" int32_t opgpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" const char* opgpu_last_error(const opgpu_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" uint32_t opgpu_create(const opgpu_grid* grid, opgpu_ctx** out)
{
    if (!grid || !out) return OPGPU_E_INVALID;
    *out = nullptr;
    const opgpu_grid& g = *grid;
    if (g.nx < 3 || g.ny < 3 || g.nz < 3 || !(g.dx > 0.0) || !(g.iwidth > 0.0)) return OPGPU_E_INVALID;
    if (g.k_slots != 8 && g.k_slots != 12 && g.k_slots != 16) return OPGPU_E_INVALID;
    if (g.precision != OPGPU_FP64 && g.precision != OPGPU_FP32) return OPGPU_E_INVALID;
    if (g.laplacian_stencil < 0 || g.laplacian_stencil > 2 || g.gradient_stencil < 0 || g.gradient_stencil > 2)
        return OPGPU_E_INVALID;
    if (opgpu_device_count() <= g.device || g.device < 0) return OPGPU_E_NODEVICE;
    opgpu_ctx* ctx = new opgpu_ctx();
    ctx->grid = g;
    ctx->device = g.device;
    ctx->n = (long long)g.nx * g.ny * g.nz;
    ctx->K = g.k_slots;
    ctx->fp32 = g.precision == OPGPU_FP32;
    ctx->rsz = ctx->fp32 ? sizeof(float) : sizeof(double);
    auto bail = [&](uint32_t code) { opgpu_destroy(ctx); return code; };
    if (cudaSetDevice(ctx->device) != cudaSuccess) return bail(OPGPU_E_CUDA);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(OPGPU_E_CUDA);
    for (int b = 0; b < 2; b++)
    {
        if (dalloc(&ctx->cnt[b], (size_t)ctx->n) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (dalloc(&ctx->idx[b], (size_t)ctx->n * ctx->K) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (cudaMalloc(&ctx->val[b], (size_t)ctx->n * ctx->K * ctx->rsz + 16) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (cudaMemset(ctx->cnt[b], 0, (size_t)ctx->n) != cudaSuccess) return bail(OPGPU_E_CUDA);
    }
    if (dalloc(&ctx->d_slow_list, (size_t)ctx->n) != cudaSuccess) return bail(OPGPU_E_CUDA);
    if (dalloc(&ctx->d_slow_count, 1) != cudaSuccess) return bail(OPGPU_E_CUDA);
    {
        int xchunk = 0, gz = 0, gy = 0, gx = 0;
        tiled_geometry(g.nx, g.ny, g.nz, &xchunk, &gz, &gy, &gx);
        const long long nblocks = (long long)gz * gy * gx;
        ctx->slice = kTileCols * kTileRows * xchunk;
        ctx->bucket_cap = nblocks * ctx->slice;
        ctx->wl_slice = (long long)ctx->slice * work_record_bytes(kListCap, (int)ctx->rsz);
        if (dalloc(&ctx->d_wl, (size_t)(nblocks * ctx->wl_slice)) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (dalloc(&ctx->d_bucket, (size_t)(kListCap + 1) * ctx->bucket_cap) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (dalloc(&ctx->d_bucket_count, (size_t)(kListCap + 1) * nblocks) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (cudaMemset(ctx->d_bucket_count, 0, (kListCap + 1) * nblocks * sizeof(unsigned)) != cudaSuccess)
            return bail(OPGPU_E_CUDA);
        if (dalloc(&ctx->d_bucket_off, (size_t)(kListCap + 1) * (nblocks + 1)) != cudaSuccess) return bail(OPGPU_E_CUDA);
        if (cudaMemset(ctx->d_bucket_off, 0, (kListCap + 1) * (nblocks + 1) * sizeof(unsigned)) != cudaSuccess)
            return bail(OPGPU_E_CUDA);
    }
    if (dalloc(&ctx->d_status, 1) != cudaSuccess) return bail(OPGPU_E_CUDA);
    if (dalloc(&ctx->d_counters, kNumCounters) != cudaSuccess) return bail(OPGPU_E_CUDA);
    cudaMemset(ctx->d_status, 0, sizeof(uint32_t));
    cudaMemset(ctx->d_counters, 0, kNumCounters * sizeof(unsigned long long));
    StepParams& sp = ctx->sp;
    sp.nx = g.nx; sp.ny = g.ny; sp.nz = g.nz; sp.n = ctx->n;
    sp.vol_x0 = 0; sp.vol_x1 = g.nx;
    set_stencils(sp, g.laplacian_stencil, g.gradient_stencil, g.dx);
    const double Eta = g.iwidth * g.dx;                 // src/GridParameters.cpp:256
    sp.pref_do = kPi * kPi / (Eta * Eta);               // src/DoubleObstacle.cpp:504
    sp.pref_df = kPi / Eta;                             // src/DrivingForce.cpp:507
    // finalize snaps at DBL_EPSILON in both forms: the FP32 form merges and finalizes in FP64 and
    // rounds only the stored values, so its erase decisions follow the FP64 form's
    sp.eps_snap = DBL_EPSILON;
    sp.consider_nucleus_volume = 1;
    sp.limiting = 1;
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(OPGPU_E_CUDA);
    *out = ctx;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_destroy(opgpu_ctx* ctx)
{
    if (!ctx) return OPGPU_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int b = 0; b < 2; b++) { dfree(ctx->cnt[b]); dfree(ctx->idx[b]); dfree(ctx->val[b]); }
    free_grains(ctx);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    dfree(ctx->d_slow_list);
    dfree(ctx->d_slow_count);
    dfree(ctx->d_wl);
    dfree(ctx->d_bucket); dfree(ctx->d_bucket_count); dfree(ctx->d_bucket_off);
    dfree(ctx->d_facets);
    dfree(ctx->d_df_tmp); dfree(ctx->d_df_lim); dfree(ctx->d_avg_off);
    dfree(ctx->d_df_npairs); dfree(ctx->d_df_off); dfree(ctx->d_df_scan); dfree(ctx->d_df_total);
    dfree(ctx->d_status);
    dfree(ctx->d_counters);
    for (auto& s : ctx->slots)
    {
        dfree(s.cnt); dfree(s.idx); dfree(s.val); dfree(s.volume); dfree(s.maxvol); dfree(s.vr);
        dfree(s.exist); dfree(s.stage);
    }
    for (int b = 0; b < 2; b++) { dfree(ctx->d_lam[b]); dfree(ctx->d_dphi[b]); }
    dfree(ctx->d_lam_local); dfree(ctx->d_lcnt); dfree(ctx->d_lidx); dfree(ctx->d_llam);
    dfree(ctx->d_gsig); dfree(ctx->d_gmu); dfree(ctx->d_gdg);
    dfree(ctx->d_tsig); dfree(ctx->d_tmu); dfree(ctx->d_tdg); dfree(ctx->d_tvol);
    if (ctx->adj_side) cudaStreamDestroy(static_cast<cudaStream_t>(ctx->adj_side));
    if (ctx->adj_fork) cudaEventDestroy(static_cast<cudaEvent_t>(ctx->adj_fork));
    if (ctx->adj_join) cudaEventDestroy(static_cast<cudaEvent_t>(ctx->adj_join));
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return OPGPU_OK;
}

extern "C" void* opgpu_stream(opgpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" uint32_t opgpu_set_model(opgpu_ctx* ctx, const opgpu_model* m)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    if (!m || m->nphases < 1 || m->nphases > kMaxPhases || !m->sigma || !m->mu)
        return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: need 1..8 phases and sigma/mu tables");
    StepParams& sp = ctx->sp;
    const int P = m->nphases;
    sp.nphases = P;
    sp.limiting = m->limiting;
    sp.tj_factor = m->tj_factor;
    sp.consider_nucleus_volume = m->consider_nucleus_volume;
    std::vector<double> facet_rows;
    for (int a = 0; a < P; a++)
    for (int b = 0; b < P; b++)
    {
        const int q = a * P + b;
        sp.sigma_p[q] = m->sigma[q];
        sp.mu_p[q] = m->mu[q];
        const double lim = m->limit ? m->limit[q] : 0.95;   // src/DrivingForce.cpp:161
        const int model = m->energy_model ? m->energy_model[q] : 0;
        if (model < 0 || model > 7)
            return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: energy model 0 (ISO) .. 7 (FACETEDEXP)");
        sp.emodel[q] = (signed char)model;
        const bool normal_model = model == 1 || (model >= 3 && model <= 5);
        sp.eps_p[q] = (normal_model && m->cubic_eps) ? m->cubic_eps[q] : 0.0;
        for (int k = 0; k < 3; k++) sp.eps_x[q][k] = (model >= 4 && m->model_eps) ? m->model_eps[3 * q + k] : 0.0;
        // DISORIENTATION reads no $Sigma: its Energy and MaxEnergy keep the constructor's 0
        // (InterfaceEnergyModel.h:63-70, 303-306), which the triple-junction term and the
        // driving-force limiter use
        if (model == 2) sp.sigma_p[q] = 0.0;
        // MaxEnergy: Energy for ISO and the HEX models (InterfaceEnergyModel.h:82, 105-134),
        // Energy*(1 + Epsilon*1.41) for CUBIC (ReadInputCubic, :87-94), 0 for DISORIENTATION
        sp.maxe_p[q] = model == 1 ? m->sigma[q] * (1.0 + sp.eps_p[q] * 1.41) : (model == 2 ? 0.0 : m->sigma[q]);
        sp.facet_lo[q] = sp.facet_hi[q] = 0;
        if (model == 6)
        {
            // ReadInputFaceted (InterfaceEnergyModel.h:196-246): facet rows, Energy = mean SigmaF
            // (accumulated in facet order), MaxEnergy = max SigmaF
            if (!m->facet_start || !m->facet_data || m->facet_start[q + 1] <= m->facet_start[q])
                return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: a FACETED pair needs facets");
            const int n0 = m->facet_start[q], n1 = m->facet_start[q + 1], nf = n1 - n0;
            const bool family = m->facet_family && m->facet_family[q];
            double energy = 0.0, maxe = 0.0;
            sp.facet_lo[q] = (int)(facet_rows.size() / 5);
            for (int f = n0; f < n1; f++)
            {
                const double* d = m->facet_data + 5 * (size_t)f;
                std::vector<double> nrm;
                facet_normals(std::lround(d[0]), std::lround(d[1]), std::lround(d[2]), family, nrm);
                for (size_t r = 0; r < nrm.size(); r += 3)
                    facet_rows.insert(facet_rows.end(), {nrm[r], nrm[r + 1], nrm[r + 2], d[3], d[4]});
                energy += d[3] / nf;
                if (d[3] > maxe) maxe = d[3];
            }
            sp.facet_hi[q] = (int)(facet_rows.size() / 5);
            sp.sigma_p[q] = energy;
            sp.maxe_p[q] = maxe;
        }
        if (model == 7)
        {
            // ReadInputFacetedEXP (InterfaceEnergyModel.h:248-295): facet rows (unit normal,
            // EpsilonEF, PowerEF); Energy = MaxEnergy = $Sigma
            if (!m->facet_start || !m->facet_data || m->facet_start[q + 1] <= m->facet_start[q])
                return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: a FACETEDEXP pair needs facets");
            const bool family = m->facet_family && m->facet_family[q];
            sp.facet_lo[q] = (int)(facet_rows.size() / 5);
            for (int f = m->facet_start[q]; f < m->facet_start[q + 1]; f++)
            {
                const double* d = m->facet_data + 5 * (size_t)f;
                if (!(d[4] >= 2.0))
                    return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: FACETEDEXP facet power must be >= 2");
                std::vector<double> nrm;
                facet_normals(std::lround(d[0]), std::lround(d[1]), std::lround(d[2]), family, nrm);
                for (size_t r = 0; r < nrm.size(); r += 3)
                    facet_rows.insert(facet_rows.end(), {nrm[r], nrm[r + 1], nrm[r + 2], d[3], d[4]});
            }
            sp.facet_hi[q] = (int)(facet_rows.size() / 5);
        }
        // src/DrivingForce.cpp:548-552: Limit*Prefactor*MaxEnergy, then *= RegularizationFactor
        double allowed = lim * sp.pref_df * sp.maxe_p[q];
        allowed *= m->regularization;
        sp.allowed_p[q] = allowed;
    }
    for (int q = 0; q < P * P; q++)
    {
        const int mm = m->mobility_model ? m->mobility_model[q] : 0;
        if (mm != 0 && mm != 1 && (mm < 3 || mm > 6))
            return fail(ctx, OPGPU_E_INVALID,
                        "opgpu_set_model: mobility model 0 (ISO), 1 (CUBIC), 3..5 (HEX*), 6 (FACETED)");
        sp.mmodel[q] = (signed char)mm;
        for (int k = 0; k < 4; k++) sp.meps[q][k] = (mm != 0 && m->mobility_eps) ? m->mobility_eps[4 * q + k] : 0.0;
        sp.mfacet_lo[q] = sp.mfacet_hi[q] = 0;
        if (mm == 6)
        {
            // InterfaceMobilityModel::ReadInputFaceted (InterfaceMobilityModel.h:165-208): facet
            // rows (unit normal, MuF, EpsilonMF); it reads no $Mu, so its Mobility (the value where
            // no solid grain of the pair counts) keeps the constructor's 0
            const int32_t* fs = m->mobility_facet_start;
            if (!fs || !m->mobility_facet_data || fs[q + 1] <= fs[q])
                return fail(ctx, OPGPU_E_INVALID, "opgpu_set_model: a FACETED mobility pair needs facets");
            const bool family = m->mobility_facet_family && m->mobility_facet_family[q];
            sp.mfacet_lo[q] = (int)(facet_rows.size() / 5);
            for (int f = fs[q]; f < fs[q + 1]; f++)
            {
                const double* d = m->mobility_facet_data + 5 * (size_t)f;
                std::vector<double> nrm;
                facet_normals(std::lround(d[0]), std::lround(d[1]), std::lround(d[2]), family, nrm);
                for (size_t r = 0; r < nrm.size(); r += 3)
                    facet_rows.insert(facet_rows.end(), {nrm[r], nrm[r + 1], nrm[r + 2], d[3], d[4]});
            }
            sp.mfacet_hi[q] = (int)(facet_rows.size() / 5);
            sp.mu_p[q] = 0.0;
        }
    }
    sp.aniso = 0;   // models of the interface normal (the disorientation energy depends on the grain pair only)
    for (int q = 0; q < P * P; q++) sp.aniso |= sp.emodel[q] == 1 || sp.emodel[q] >= 3 || sp.mmodel[q] != 0;
    dfree(ctx->d_facets);
    ctx->d_facets = nullptr;
    if (!facet_rows.empty())
    {
        CK(dalloc(&ctx->d_facets, facet_rows.size()));
        CK(cudaMemcpy(ctx->d_facets, facet_rows.data(), facet_rows.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    for (int a = 0; a < P; a++) sp.solid_p[a] = (signed char)(m->phase_solid ? (m->phase_solid[a] != 0) : 1);
    ctx->nvf = m->nucleus_volume_factor > 0.0 ? m->nucleus_volume_factor : 1.0;
    ctx->model_set = true;
    ctx->dg_pair_dirty = true;
    ctx->pair_energy_dirty = true;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_grains(opgpu_ctx* ctx, int32_t ngrains, const int32_t* phase, const int32_t* stage)
{
    if (uint32_t r = require(ctx, ctx && ctx->model_set, "opgpu_set_grains: call opgpu_set_model first")) return r;
    if (ngrains < 1 || ngrains > 32767) return fail(ctx, OPGPU_E_INVALID, "opgpu_set_grains: 1..32767 grains");
    const int G = ngrains;
    std::vector<int16_t> gp(G);
    std::vector<int8_t> gs(G), ex(G, 1);
    for (int g = 0; g < G; g++)
    {
        const int p = phase ? phase[g] : 0;
        if (p < 0 || p >= ctx->sp.nphases) return fail(ctx, OPGPU_E_INVALID, "opgpu_set_grains: phase out of range");
        gp[g] = (int16_t)p;
        const int s = stage ? stage[g] : OPGPU_STAGE_STABLE;
        if (s < 0 || s > 2) return fail(ctx, OPGPU_E_INVALID, "opgpu_set_grains: bad stage");
        gs[g] = (int8_t)s;
    }
    free_grains(ctx);
    ctx->G = G;
    ctx->sp.ngrains = G;
    CK(dalloc(&ctx->d_vr, G));
    CK(dalloc(&ctx->d_volume, G));
    CK(dalloc(&ctx->d_maxvol, G));
    CK(dalloc(&ctx->d_refvol, G));
    CK(dalloc(&ctx->d_vol_acc, G));
    CK(dalloc(&ctx->d_gphase, G));
    CK(dalloc(&ctx->d_gstage, G));
    CK(dalloc(&ctx->d_exist, G));
    // PhaseField::AddGrainInfo (src/PhaseField.cpp:2970-2979): RefVolume from
    // CalculateReferenceVolume(iWidth) (:367-391, 3-D), VolumeRatio 0, MAXVolume 0, Exist.
    const double r = ctx->grid.iwidth;
    const double ref = (4.0 / 3.0) * kPi * r * r * r * ctx->nvf;
    std::vector<double> refv(G, ref), zeros(G, 0.0);
    CK(cudaMemcpy(ctx->d_refvol, refv.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_vr, zeros.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_volume, zeros.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_maxvol, zeros.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_vol_acc, zeros.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_gphase, gp.data(), G * sizeof(int16_t), cudaMemcpyHostToDevice));
    ctx->h_gphase = gp;
    CK(cudaMemcpy(ctx->d_gstage, gs.data(), G * sizeof(int8_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_exist, ex.data(), G * sizeof(int8_t), cudaMemcpyHostToDevice));
    CK(dalloc(&ctx->d_grot, (size_t)G * 9));
    {
        std::vector<double> rot((size_t)G * 9, 0.0);
        for (int g = 0; g < G; g++) { rot[9 * g] = 1.0; rot[9 * g + 4] = 1.0; rot[9 * g + 8] = 1.0; }
        CK(cudaMemcpy(ctx->d_grot, rot.data(), rot.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    ctx->sp.pair_mode = OPGPU_PAIRS_PHASE;
    ctx->sp.use_dg = 0;
    ctx->initialized = false;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_pair_table(opgpu_ctx* ctx, const double* sigma, const double* mu)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_set_pair_table: call opgpu_set_grains first")) return r;
    const size_t GG = (size_t)ctx->G * ctx->G;
    dfree(ctx->d_pair_sigma); ctx->d_pair_sigma = nullptr;
    dfree(ctx->d_pair_mu); ctx->d_pair_mu = nullptr;
    ctx->h_user_sigma.clear();
    ctx->pair_energy_dirty = true;
    if (sigma)
    {
        CK(dalloc(&ctx->d_pair_sigma, GG));
        CK(cudaMemcpy(ctx->d_pair_sigma, sigma, GG * sizeof(double), cudaMemcpyHostToDevice));
        ctx->h_user_sigma.assign(sigma, sigma + GG);
    }
    if (mu)
    {
        CK(dalloc(&ctx->d_pair_mu, GG));
        CK(cudaMemcpy(ctx->d_pair_mu, mu, GG * sizeof(double), cudaMemcpyHostToDevice));
    }
    ctx->sp.pair_mode = (sigma || mu) ? OPGPU_PAIRS_TABLE : OPGPU_PAIRS_PHASE;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_pair_hash(opgpu_ctx* ctx, uint64_t seed, double lo, double span)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_set_pair_hash: call opgpu_set_grains first")) return r;
    ctx->sp.pair_mode = OPGPU_PAIRS_HASH;
    ctx->pair_energy_dirty = true;
    ctx->sp.hash_seed = seed;
    ctx->sp.hash_lo = lo;
    ctx->sp.hash_span = span;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_driving_force(opgpu_ctx* ctx, const double* dG)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_set_driving_force: call opgpu_set_grains first")) return r;
    if (!dG)
    {
        ctx->sp.use_dg = 0;
        return OPGPU_OK;
    }
    if (!ctx->d_dg) CK(dalloc(&ctx->d_dg, ctx->G));
    CK(cudaMemcpyAsync(ctx->d_dg, dG, ctx->G * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // the pair table is rebuilt only when the forces change (or with the model and the grains)
    const bool same = ctx->sp.use_dg && ctx->h_dg.size() == (size_t)ctx->G &&
                      std::memcmp(ctx->h_dg.data(), dG, ctx->G * sizeof(double)) == 0;
    if (!same)
    {
        ctx->h_dg.assign(dG, dG + ctx->G);
        ctx->dg_pair_dirty = true;
    }
    ctx->sp.use_dg = 1;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_averaging(opgpu_ctx* ctx, int32_t enable, int32_t range, double threshold)
{
    if (uint32_t r = require(ctx, ctx != nullptr, "opgpu_set_averaging: no context")) return r;
    if (!enable)
    {
        ctx->averaging = false;
        return OPGPU_OK;
    }
    // DrivingForce::Initialize / ReadInput (src/DrivingForce.cpp:61-73, 132-133): Range = iWidth,
    // Threshold = iWidth/15 below an interface width of 5 cells, else 1/3
    const double iw = ctx->grid.iwidth;
    const int R = range > 0 ? range : (int)iw;
    const double t = threshold > 0.0 ? threshold : (iw < 5.0 ? iw / 15.0 : 1.0 / 3.0);
    if (R < 1 || !(t < 1.0)) return fail(ctx, OPGPU_E_INVALID, "opgpu_set_averaging: range >= 1 and threshold < 1 required");
    // the sphere of CollectAverage / DistributeAverage in their loop order: offsets with
    // Range - |d| > 0 within +-min(Range, N - 1) per axis
    const int Xr = std::min(R, ctx->grid.nx - 1), Yr = std::min(R, ctx->grid.ny - 1), Zr = std::min(R, ctx->grid.nz - 1);
    std::vector<signed char> off;
    for (int ii = -Xr; ii <= Xr; ii++)
        for (int jj = -Yr; jj <= Yr; jj++)
            for (int kk = -Zr; kk <= Zr; kk++)
            {
                const double wd = R - std::sqrt((double)(ii * ii + jj * jj + kk * kk));
                if (wd > 0.0) off.insert(off.end(), {(signed char)ii, (signed char)jj, (signed char)kk});
            }
    if (R > 127) return fail(ctx, OPGPU_E_INVALID, "opgpu_set_averaging: range above 127");
    dfree(ctx->d_avg_off);
    ctx->d_avg_off = nullptr;
    CK(dalloc(&ctx->d_avg_off, off.size()));
    CK(cudaMemcpy(ctx->d_avg_off, off.data(), off.size(), cudaMemcpyHostToDevice));
    if (!ctx->d_df_npairs)
    {
        // pair slots are sized per step (they grow to the total the scan finds)
        CK(dalloc(&ctx->d_df_total, 1));
        CK(dalloc(&ctx->d_df_npairs, (size_t)ctx->n));
        CK(dalloc(&ctx->d_df_off, (size_t)ctx->n));
        ctx->df_scan_bytes = average_scan_bytes(ctx->n);
        CK(dalloc(reinterpret_cast<unsigned char**>(&ctx->d_df_scan), ctx->df_scan_bytes));
    }
    ctx->avg_noff = (int)(off.size() / 3);
    ctx->avg_range = R;
    ctx->avg_threshold = t;
    ctx->averaging = true;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_orientations(opgpu_ctx* ctx, const double* quat)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_set_orientations: set the grains first")) return r;
    const int G = ctx->G;
    std::vector<double> rot((size_t)G * 9, 0.0);
    for (int g = 0; g < G; g++)
    {
        double* R = rot.data() + 9 * (size_t)g;
        // Quaternion::setRotationMatrix (src/Containers/Quaternion.cpp:78-98) on the quaternion
        // normalised as Quaternion::normalized (include/Containers/Quaternion.h:304-311)
        const double qs = quat ? quat[4 * g] : 1.0, q0 = quat ? quat[4 * g + 1] : 0.0;
        const double q1 = quat ? quat[4 * g + 2] : 0.0, q2 = quat ? quat[4 * g + 3] : 0.0;
        const double len = std::sqrt(qs * qs + q0 * q0 + q1 * q1 + q2 * q2);
        if (len < DBL_EPSILON)
        {
            R[0] = 1.0; R[4] = 1.0; R[8] = 1.0;
            continue;
        }
        const double S = qs / len, V0 = q0 / len, V1 = q1 / len, V2 = q2 / len;
        R[0] = 1.0 - 2.0 * (V1 * V1 + V2 * V2);
        R[1] =       2.0 * (V0 * V1 -  S * V2);
        R[2] =       2.0 * (V0 * V2 +  S * V1);
        R[3] =       2.0 * (V0 * V1 +  S * V2);
        R[4] = 1.0 - 2.0 * (V0 * V0 + V2 * V2);
        R[5] =       2.0 * (V1 * V2 -  S * V0);
        R[6] =       2.0 * (V0 * V2 -  S * V1);
        R[7] =       2.0 * (V1 * V2 +  S * V0);
        R[8] = 1.0 - 2.0 * (V0 * V0 + V1 * V1);
    }
    CK(cudaMemcpy(ctx->d_grot, rot.data(), rot.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (quat) ctx->h_quat.assign(quat, quat + 4 * (size_t)G);
    else ctx->h_quat.clear();
    ctx->pair_energy_dirty = true;
    return OPGPU_OK;
}

// Per-grain-pair energies of the DISORIENTATION model (InterfaceProperties::SetSR,
// src/InterfaceProperties.cpp:629-634): the energy of a pair depends on the two grains'
// orientations only, so it is tabulated once (G*G, with the other phase pairs' values from the
// user table or the phase model) and the step reads it as a per-grain-pair table.
uint32_t refresh_pair_energy(opgpu_ctx* ctx)
{
    const int P = ctx->sp.nphases, G = ctx->G;
    bool any = false;
    for (int q = 0; q < P * P; q++) any |= ctx->sp.emodel[q] == 2;
    if (!any || !ctx->pair_energy_dirty) return OPGPU_OK;
    if (ctx->sp.pair_mode == OPGPU_PAIRS_HASH)
        return fail(ctx, OPGPU_E_INVALID, "DISORIENTATION energies are tabulated per grain pair: not with opgpu_set_pair_hash");
    if (G > kMaxPairTableGrains)
        return fail(ctx, OPGPU_E_INVALID, "DISORIENTATION energies: at most 32767 grains");
    const size_t GG = (size_t)G * G;
    std::vector<double> tab(GG);
    const double unit[4] = {1.0, 0.0, 0.0, 0.0};
#pragma omp parallel for
    for (int a = 0; a < G; a++)
        for (int b = 0; b < G; b++)
        {
            const int q = ctx->h_gphase[a] * P + ctx->h_gphase[b];
            double v;
            if (ctx->sp.emodel[q] == 2)
                v = a == b ? 0.0
                           : disorientation_energy(ctx->h_quat.empty() ? unit : &ctx->h_quat[4 * (size_t)a],
                                                   ctx->h_quat.empty() ? unit : &ctx->h_quat[4 * (size_t)b]);
            else
                v = ctx->h_user_sigma.empty() ? ctx->sp.sigma_p[q] : ctx->h_user_sigma[(size_t)a * G + b];
            tab[(size_t)a * G + b] = v;
        }
    if (!ctx->d_pair_sigma) CK(dalloc(&ctx->d_pair_sigma, GG));
    CK(cudaMemcpy(ctx->d_pair_sigma, tab.data(), GG * sizeof(double), cudaMemcpyHostToDevice));
    ctx->sp.pair_mode = OPGPU_PAIRS_TABLE;
    ctx->pair_energy_dirty = false;
    return OPGPU_OK;
}

// The tanh-limited driving force of every grain pair, allowed*tanh((dG_b - dG_a)/allowed) with
// allowed = Limit*Prefactor*MaxEnergy*RegularizationFactor (src/DrivingForce.cpp:548-583).  It
// depends on the pair only, so it is tabulated (G*G) whenever the forces or the model change, on
// the host with the C library's tanh: the function the reference evaluates per voxel, so that the
// step's values equal the reference's bit for bit (CUDA's tanh differs from it in the last bit for
// some arguments, which can tip a threshold decision of the step).
uint32_t build_dg_pair(opgpu_ctx* ctx)
{
    if (!(ctx->sp.use_dg && ctx->G <= kMaxPairTableGrains && ctx->dg_pair_dirty)) return OPGPU_OK;
    if (ctx->h_dg.size() != (size_t)ctx->G || ctx->h_gphase.size() != (size_t)ctx->G)
        return fail(ctx, OPGPU_E_STATE, "driving-force table: grains and driving forces out of step");
    const int G = ctx->G, P = ctx->sp.nphases;
    const size_t GG = (size_t)G * G;
    if (!ctx->d_dg_pair) CK(dalloc(&ctx->d_dg_pair, GG));
    ctx->h_dg_pair.resize(GG);
    const double* dg = ctx->h_dg.data();
    const int16_t* ph = ctx->h_gphase.data();
    const StepParams& sp = ctx->sp;
    double* out = ctx->h_dg_pair.data();
#pragma omp parallel for schedule(static)
    for (int a = 0; a < G; a++)
        for (int b = 0; b < G; b++)
        {
            double locdG = dg[b] - dg[a];
            if (sp.limiting)
            {
                const double allowed = sp.allowed_p[ph[a] * P + ph[b]];
                locdG = allowed * std::tanh(locdG / allowed);
            }
            out[(size_t)a * G + b] = locdG;
        }
    // pageable source: the call returns once the table is staged, the host copy stays valid
    CK(cudaMemcpyAsync(ctx->d_dg_pair, out, GG * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    ctx->dg_pair_dirty = false;
    return OPGPU_OK;
}

// Device scratch of the list upload / download / entry count, carved from the spare ping-pong
// state buffers (they hold no state between calls: every step rewrites them); a piece that does
// not fit there is allocated for the call and freed with the scratch.
struct IoScratch {
    unsigned char* a;   // spare value planes
    size_t a_left;
    unsigned char* b;   // spare index planes
    size_t b_left;
    std::vector<void*> owned;

    IoScratch(opgpu_ctx* ctx, int spare)
        : a(static_cast<unsigned char*>(ctx->val[spare])), a_left((size_t)ctx->n * ctx->K * ctx->rsz),
          b(reinterpret_cast<unsigned char*>(ctx->idx[spare])), b_left((size_t)ctx->n * ctx->K * sizeof(int16_t))
    {
    }
    ~IoScratch()
    {
        for (void* p : owned) cudaFree(p);
    }
    IoScratch(const IoScratch&) = delete;
    IoScratch& operator=(const IoScratch&) = delete;

    template <class T>
    cudaError_t take(T** p, size_t count, bool prefer_a)
    {
        const size_t bytes = ((count * sizeof(T) + 16 + 255) / 256) * 256;   // bases stay 256-byte aligned
        for (int pass = 0; pass < 2; pass++)
        {
            const bool use_a = (pass == 0) == prefer_a;
            unsigned char*& base = use_a ? a : b;
            size_t& left = use_a ? a_left : b_left;
            if (bytes <= left)
            {
                *p = reinterpret_cast<T*>(base);
                base += bytes;
                left -= bytes;
                return cudaSuccess;
            }
        }
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) return e;
        owned.push_back(q);
        *p = static_cast<T*>(q);
        return cudaSuccess;
    }
};

extern "C" uint32_t opgpu_upload_lists(opgpu_ctx* ctx, const int32_t* counts, const int32_t* idx, const double* val)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_upload_lists: call opgpu_set_grains first")) return r;
    if (!counts || !idx || !val) return fail(ctx, OPGPU_E_INVALID, "opgpu_upload_lists: null array");
    const long long N = ctx->n;
    long long total = 0;
    int bad = 0;
#pragma omp parallel for reduction(+ : total) reduction(| : bad)
    for (long long v = 0; v < N; v++)
    {
        if (counts[v] < 0 || counts[v] > 64) bad |= 1;
        total += counts[v];
    }
    if (bad) return fail(ctx, OPGPU_E_INVALID, "opgpu_upload_lists: a voxel list must hold 0..64 entries");
    const int G = ctx->G;
#pragma omp parallel for reduction(| : bad)
    for (long long q = 0; q < total; q++)
        if (idx[q] < 0 || idx[q] >= G) bad |= 2;
    if (bad) return fail(ctx, OPGPU_E_INVALID, "opgpu_upload_lists: grain index out of range");
    int32_t *d_counts = nullptr, *d_idx = nullptr;
    long long *d_off = nullptr, *d_wide = nullptr;
    double* d_val = nullptr;
    unsigned char* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    uint32_t rc = OPGPU_OK;
    IoScratch scr(ctx, 1);   // the state is loaded into buffer 0
    cudaError_t e = cudaSuccess;
    do {
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_wide, d_off, N, ctx->stream)) != cudaSuccess) break;
        if ((e = scr.take(&d_val, total, true)) != cudaSuccess) break;
        if ((e = scr.take(&d_idx, total, true)) != cudaSuccess) break;
        if ((e = scr.take(&d_off, N, false)) != cudaSuccess) break;
        if ((e = scr.take(&d_wide, N, false)) != cudaSuccess) break;
        if ((e = scr.take(&d_counts, N, false)) != cudaSuccess) break;
        if ((e = scr.take(&d_tmp, tmp_bytes, false)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(d_counts, counts, N * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(d_idx, idx, total * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(d_val, val, total * sizeof(double), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) break;
        widen_kernel<<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, d_counts, d_wide);
        if ((e = cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_wide, d_off, N, ctx->stream)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(ctx->d_vol_acc, 0, ctx->G * sizeof(double), ctx->stream)) != cudaSuccess) break;
        const int cur = 0;
        if (ctx->fp32)
            load_kernel<float><<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->K, ctx->G, d_counts, d_off, d_idx, d_val,
                ctx->cnt[cur], ctx->idx[cur], static_cast<float*>(ctx->val[cur]), ctx->d_status, ctx->d_vol_acc);
        else
            load_kernel<double><<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->K, ctx->G, d_counts, d_off, d_idx, d_val,
                ctx->cnt[cur], ctx->idx[cur], static_cast<double*>(ctx->val[cur]), ctx->d_status, ctx->d_vol_acc);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) break;
        ctx->cur = cur;
        ctx->state_loaded = true;
        ctx->initialized = false;
        return OPGPU_OK;
    } while (0);
    rc = fail(ctx, OPGPU_E_CUDA, std::string("opgpu_upload_lists: ") + cudaGetErrorString(e));
    return rc;
}

extern "C" uint32_t opgpu_read_raw(opgpu_ctx* ctx, const char* path)
{
    if (!ctx || !path) return OPGPU_E_INVALID;
    std::vector<int32_t> counts, idx;
    std::vector<double> val;
    std::string err;
    if (!raw_read(path, ctx->grid.nx, ctx->grid.ny, ctx->grid.nz, counts, idx, val, err))
        return fail(ctx, OPGPU_E_IO, err);
    return opgpu_upload_lists(ctx, counts.data(), idx.data(), val.data());
}

extern "C" uint32_t opgpu_finalize_initialization(opgpu_ctx* ctx)
{
    // The upload already applied NodePF::finalize to every multi-entry voxel and accumulated the
    // grain volumes; what remains of FinalizeSR is the grain-record update.  Flags and candidate
    // derivatives are re-derived by every step.
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded, "opgpu_finalize_initialization: no state uploaded")) return r;
    if (ctx->initialized) return fail(ctx, OPGPU_E_STATE, "opgpu_finalize_initialization: already initialized");
    grains_update_kernel<<<grid_for(ctx->G, 256), 256, 0, ctx->stream>>>(ctx->G, ctx->d_vol_acc, ctx->d_volume,
        ctx->d_maxvol, ctx->d_refvol, ctx->d_vr, ctx->d_exist, ctx->d_gstage, ctx->d_counters, 0);
    CK(cudaGetLastError());
    const uint32_t st = read_status(ctx);
    if (st & OPGPU_E_CUDA) return st;
    ctx->initialized = true;
    return st & OPGPU_SOFT_MASK;
}

static uint32_t enqueue_steps(opgpu_ctx* ctx, double dt, int nsteps, bool partial = false)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_step: call opgpu_finalize_initialization first")) return r;
    if (nsteps < 0 || !(dt > 0.0)) return fail(ctx, OPGPU_E_INVALID, "opgpu_step: dt > 0 and nsteps >= 0 required");
    if (ctx->sp.use_dg && !ctx->d_dg) return fail(ctx, OPGPU_E_STATE, "opgpu_step: driving force enabled without values");
    if (uint32_t r = refresh_pair_energy(ctx)) return r;
    StepParams sp = ctx->sp;
    sp.dt = dt;
    const bool pair_table = sp.use_dg && ctx->G <= kMaxPairTableGrains;
    if (uint32_t r = build_dg_pair(ctx)) return r;
    for (int s = 0; s < nsteps; s++)
    {
        const int in = ctx->cur, out = 1 - ctx->cur;
        StepArrays a{};
        a.cnt_in = ctx->cnt[in]; a.idx_in = ctx->idx[in]; a.val_in = ctx->val[in];
        a.cnt_out = ctx->cnt[out]; a.idx_out = ctx->idx[out]; a.val_out = ctx->val[out];
        a.vr = ctx->d_vr; a.gphase = ctx->d_gphase; a.gstage = ctx->d_gstage;
        a.dg = ctx->d_dg; a.pair_sigma = ctx->d_pair_sigma; a.pair_mu = ctx->d_pair_mu;
        a.dg_pair = pair_table ? ctx->d_dg_pair : nullptr;
        a.grot = ctx->d_grot; a.facets = ctx->d_facets;
        a.vol_acc = ctx->d_vol_acc; a.status = ctx->d_status; a.counters = ctx->d_counters;
        a.df_lim = nullptr;
        if (ctx->averaging && sp.use_dg)
        {
            // DrivingForce::Average on the state the step starts from: slots for every pair of stored
            // fields of the interface voxels (grown to the total this state needs), then the passes
            AvgArrays aa{ctx->d_df_npairs, ctx->d_df_off, ctx->d_df_tmp, ctx->d_df_lim, ctx->df_cap,
                         ctx->d_avg_off, ctx->avg_noff, std::sqrt(ctx->avg_threshold * (1.0 - ctx->avg_threshold)),
                         ctx->d_df_scan, ctx->df_scan_bytes};
            int rc = launch_average_scan(ctx->n, aa, ctx->cnt[in], ctx->d_df_total, ctx->stream);
            if (rc != 0) return fail(ctx, OPGPU_E_CUDA, std::string("averaging scan: ") + cudaGetErrorString((cudaError_t)rc));
            unsigned long long total = 0;
            CK(cudaMemcpyAsync(&total, ctx->d_df_total, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (total > 0xFFFFFFF0ULL) return fail(ctx, OPGPU_E_INVALID, "averaging: more than 2^32 pair slots");
            if (total > ctx->df_cap)
            {
                dfree(ctx->d_df_tmp); dfree(ctx->d_df_lim);
                ctx->d_df_tmp = ctx->d_df_lim = nullptr;
                const unsigned long long cap = std::min<unsigned long long>(total + total / 4 + 1024, 0xFFFFFFF0ULL);
                CK(dalloc(&ctx->d_df_tmp, (size_t)cap));
                CK(dalloc(&ctx->d_df_lim, (size_t)cap));
                ctx->df_cap = (unsigned)cap;
                aa.tmp = ctx->d_df_tmp;
                aa.lim = ctx->d_df_lim;
                aa.cap = ctx->df_cap;
            }
            rc = launch_average(sp, aa, ctx->cnt[in], ctx->idx[in], ctx->val[in], ctx->fp32 != 0,
                                ctx->d_vr, ctx->d_dg, ctx->d_gphase, ctx->d_status, ctx->stream);
            if (rc != 0) return fail(ctx, OPGPU_E_CUDA, std::string("averaging: ") + cudaGetErrorString((cudaError_t)rc));
            ctx->kernel_launches += 5;   // count, scan, total, collect, distribute
            a.df_lim = ctx->d_df_lim;
            a.df_off = ctx->d_df_off;
            a.df_cap = ctx->df_cap;
        }
        a.slow_list = ctx->d_slow_list; a.slow_count = ctx->d_slow_count; a.slow_cap = (unsigned)ctx->n;
        a.wl = ctx->d_wl; a.wl_slice = ctx->wl_slice;
        a.bucket = ctx->d_bucket; a.bucket_count = ctx->d_bucket_count; a.bucket_off = ctx->d_bucket_off;
        a.bucket_cap = ctx->bucket_cap; a.slice = ctx->slice;
        LaunchInfo info;
        if (ctx->timing)
        {
            if (ctx->ev_pool.size() < 3 * (ctx->ev_used + 1))
            {
                for (int k = 0; k < 3; k++)
                {
                    cudaEvent_t e;
                    CK(cudaEventCreate(&e));
                    ctx->ev_pool.push_back(e);
                }
            }
            CK(cudaEventRecord(ctx->ev_pool[3 * ctx->ev_used], ctx->stream));
            // "after classify" is recorded at the start too; the tiled path records it again after
            // its classify kernel (paths without a classify phase leave it at the start)
            CK(cudaEventRecord(ctx->ev_pool[3 * ctx->ev_used + 1], ctx->stream));
            info.after_classify = ctx->ev_pool[3 * ctx->ev_used + 1];
        }
        const int rc = ctx->fp32 ? launch_step_f32(sp, a, ctx->K, ctx->variant, ctx->stream, &info)
                                 : launch_step_f64(sp, a, ctx->K, ctx->variant, ctx->stream, &info);
        if (rc != 0) return fail(ctx, OPGPU_E_CUDA, std::string("step launch: ") + cudaGetErrorString((cudaError_t)rc));
        if (ctx->timing)
        {
            CK(cudaEventRecord(ctx->ev_pool[3 * ctx->ev_used + 2], ctx->stream));
            ctx->ev_used++;
        }
        ctx->kernel_launches += info.kernels;
        if (!partial)
        {
            grains_update_kernel<<<grid_for(ctx->G, 256), 256, 0, ctx->stream>>>(ctx->G, ctx->d_vol_acc, ctx->d_volume,
                ctx->d_maxvol, ctx->d_refvol, ctx->d_vr, ctx->d_exist, ctx->d_gstage, ctx->d_counters, 1);
            CK(cudaGetLastError());
            ctx->kernel_launches++;
        }
        ctx->cur = out;
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_step_async(opgpu_ctx* ctx, double dt, int32_t nsteps)
{
    return enqueue_steps(ctx, dt, nsteps);
}

extern "C" uint32_t opgpu_sync(opgpu_ctx* ctx)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    const uint32_t st = read_status(ctx);
    if (st & OPGPU_E_CUDA) return st;
    return st & OPGPU_SOFT_MASK;
}

extern "C" uint32_t opgpu_step(opgpu_ctx* ctx, double dt, int32_t nsteps)
{
    if (uint32_t r = enqueue_steps(ctx, dt, nsteps)) return r;
    return opgpu_sync(ctx);
}

extern "C" uint32_t opgpu_total_entries(opgpu_ctx* ctx, int64_t* total)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded, "no state")) return r;
    if (!total) return OPGPU_E_INVALID;
    const long long N = ctx->n;
    int32_t* d_counts = nullptr;
    long long *d_sum = nullptr, *d_wide = nullptr;
    unsigned char* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    IoScratch scr(ctx, 1 - ctx->cur);
    CK(cub::DeviceReduce::Sum(nullptr, tmp_bytes, d_wide, d_sum, N, ctx->stream));
    CK(scr.take(&d_counts, N, false));
    CK(scr.take(&d_wide, N, false));
    CK(scr.take(&d_sum, 1, false));
    CK(scr.take(&d_tmp, tmp_bytes, false));
    counts_kernel<<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->cnt[ctx->cur], d_counts, d_wide);
    CK(cub::DeviceReduce::Sum(d_tmp, tmp_bytes, d_wide, d_sum, N, ctx->stream));
    long long t = 0;
    CK(cudaMemcpyAsync(&t, d_sum, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *total = t;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_download_lists(opgpu_ctx* ctx, int32_t* counts, int32_t* idx, double* val)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded, "no state")) return r;
    if (!counts || !idx || !val) return OPGPU_E_INVALID;
    const long long N = ctx->n;
    int64_t total = 0;
    if (uint32_t r = opgpu_total_entries(ctx, &total)) return r;
    int32_t *d_counts = nullptr, *d_idx = nullptr;
    long long *d_off = nullptr, *d_wide = nullptr;
    double* d_val = nullptr;
    unsigned char* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    IoScratch scr(ctx, 1 - ctx->cur);
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_wide, d_off, N, ctx->stream));
    CK(scr.take(&d_val, total, true));
    CK(scr.take(&d_idx, total, true));
    CK(scr.take(&d_off, N, false));
    CK(scr.take(&d_wide, N, false));
    CK(scr.take(&d_counts, N, false));
    CK(scr.take(&d_tmp, tmp_bytes, false));
    counts_kernel<<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->cnt[ctx->cur], d_counts, d_wide);
    CK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_wide, d_off, N, ctx->stream));
    if (ctx->fp32)
        gather_kernel<float><<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->cnt[ctx->cur], ctx->idx[ctx->cur],
            static_cast<const float*>(ctx->val[ctx->cur]), d_off, d_idx, d_val);
    else
        gather_kernel<double><<<grid_for(N, 256), 256, 0, ctx->stream>>>(N, ctx->cnt[ctx->cur], ctx->idx[ctx->cur],
            static_cast<const double*>(ctx->val[ctx->cur]), d_off, d_idx, d_val);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(counts, d_counts, N * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(idx, d_idx, total * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(val, d_val, total * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_download_flags(opgpu_ctx* ctx, int8_t* flags)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded, "no state")) return r;
    if (!flags) return OPGPU_E_INVALID;
    const long long N = ctx->n;
    int8_t* d_flags = nullptr;
    CK(dalloc(&d_flags, N));
    flags_kernel<<<grid_for(N, 256), 256, 0, ctx->stream>>>(ctx->grid.nx, ctx->grid.ny, ctx->grid.nz,
                                                             ctx->cnt[ctx->cur], d_flags);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(flags, d_flags, N, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    dfree(d_flags);
    return OPGPU_OK;
}

// ---- allocation-free flag download ------------------------------------------------------------
// The flags are computed into a file-scope device array instead of a per-call cudaMalloc'd
// buffer.  Its address is looked up by each library context on its first call
// (cudaGetSymbolAddress, with the context's device current) and kept in the context: a context
// lives in one CUDA context (its own device buffers do), so the address cannot go stale even if the
// host program resets a device and creates new contexts afterwards.  Every one of the N bytes is
// written by flags_kernel before the copy, so nothing in the scratch has to start at zero.  The
// scratch is shared by every context on a device: overlapping calls race.  The 16 MiB are reserved
// when the library's device code is loaded on a device (at its first kernel use with lazy
// loading), for every process that loads the library, whether or not this entry point is called.
namespace {
constexpr long long kNoAllocFlagsMax = 16LL << 20;   // bytes = voxels (a 256^3 grid)
__device__ __align__(256) int8_t g_noalloc_flags[kNoAllocFlagsMax];
}  // namespace

extern "C" uint32_t opgpu_download_flags_noalloc(opgpu_ctx* ctx, int8_t* flags)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    if (!flags) return fail(ctx, OPGPU_E_INVALID, "opgpu_download_flags_noalloc: flags is NULL");
    if (ctx->n > kNoAllocFlagsMax)
        return fail(ctx, OPGPU_E_INVALID,
                    "opgpu_download_flags_noalloc: grid of " + std::to_string(ctx->n) +
                    " voxels exceeds its fixed scratch of 16777216 voxels; use opgpu_download_flags");
    if (!ctx->state_loaded) return fail(ctx, OPGPU_E_STATE, "no state");
    if (!ctx->noalloc_scratch)
    {
        // require() made the context's device current
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_flags);
        if (e != cudaSuccess)
            return fail(ctx, OPGPU_E_CUDA, std::string("opgpu_download_flags_noalloc: set-up: ") + cudaGetErrorString(e));
        ctx->noalloc_scratch = static_cast<int8_t*>(p);
    }
    int8_t* scratch = ctx->noalloc_scratch;
    const long long N = ctx->n;
    flags_kernel<<<grid_for(N, 256), 256, 0, ctx->stream>>>(ctx->grid.nx, ctx->grid.ny, ctx->grid.nz,
                                                             ctx->cnt[ctx->cur], scratch);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(flags, scratch, N, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_write_raw(opgpu_ctx* ctx, const char* path)
{
    if (!ctx || !path) return OPGPU_E_INVALID;
    int64_t total = 0;
    if (uint32_t r = opgpu_total_entries(ctx, &total)) return r;
    std::vector<int32_t> counts(ctx->n), idx(total);
    std::vector<double> val(total);
    if (uint32_t r = opgpu_download_lists(ctx, counts.data(), idx.data(), val.data())) return r;
    std::string err;
    if (!raw_write(path, ctx->grid.nx, ctx->grid.ny, ctx->grid.nz, counts.data(), idx.data(), val.data(), err))
        return fail(ctx, OPGPU_E_IO, err);
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_grains(opgpu_ctx* ctx, double* volume, double* volume_ratio, double* max_volume,
                                 int32_t* exist, int32_t* stage)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "no grains")) return r;
    const int G = ctx->G;
    CK(cudaStreamSynchronize(ctx->stream));
    if (volume) CK(cudaMemcpy(volume, ctx->d_volume, G * sizeof(double), cudaMemcpyDeviceToHost));
    if (volume_ratio) CK(cudaMemcpy(volume_ratio, ctx->d_vr, G * sizeof(double), cudaMemcpyDeviceToHost));
    if (max_volume) CK(cudaMemcpy(max_volume, ctx->d_maxvol, G * sizeof(double), cudaMemcpyDeviceToHost));
    if (exist || stage)
    {
        std::vector<int8_t> tmp(G);
        if (exist)
        {
            CK(cudaMemcpy(tmp.data(), ctx->d_exist, G, cudaMemcpyDeviceToHost));
            for (int g = 0; g < G; g++) exist[g] = tmp[g];
        }
        if (stage)
        {
            CK(cudaMemcpy(tmp.data(), ctx->d_gstage, G, cudaMemcpyDeviceToHost));
            for (int g = 0; g < G; g++) stage[g] = tmp[g];
        }
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_get_stats(opgpu_ctx* ctx, opgpu_stats* stats)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    if (!stats) return OPGPU_E_INVALID;
    unsigned long long c[kNumCounters];
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    read_status(ctx);
    stats->steps = (int64_t)c[kCntSteps];
    stats->wide_last = (int64_t)c[kCntWideLast];
    stats->wide_total = (int64_t)c[kCntWideTotal];
    stats->entries_in_total = (int64_t)c[kCntEntriesInTotal];
    stats->entries_out_total = (int64_t)c[kCntEntriesOutTotal];
    stats->status = ctx->status;
    stats->overflow_voxels = (uint32_t)c[kCntOverflowVoxels];
    stats->general_path_total = (int64_t)c[kCntGeneralTotal];
    stats->crowded_window_total = (int64_t)c[kCntCrowdedTotal];
    stats->timed_launches = ctx->timed_launches;
    stats->timed_kernel_ms = ctx->timed_ms;
    stats->timed_classify_ms = ctx->timed_classify_ms;
    stats->kernel_launches = ctx->kernel_launches;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_kernel_variant(opgpu_ctx* ctx, int32_t variant)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    if (variant != kVariantTiled && variant != kVariantGeneric)
        return fail(ctx, OPGPU_E_INVALID, "opgpu_set_kernel_variant: 0 (tiled) or 1 (generic)");
    ctx->variant = variant;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_set_timing(opgpu_ctx* ctx, int32_t enable)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    read_status(ctx);
    ctx->timing = enable != 0;
    if (enable)
    {
        ctx->timed_launches = 0;
        ctx->timed_ms = 0.0;
        ctx->timed_classify_ms = 0.0;
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_clear_status(opgpu_ctx* ctx)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    read_status(ctx);
    ctx->status = 0;
    return OPGPU_OK;
}

// ---- checkpoints, adjoint and tangent-linear model (no reference counterpart) -------------------
namespace {

StepArrays step_arrays(opgpu_ctx* ctx, const uint8_t* cnt_in, const int16_t* idx_in, const void* val_in,
                       const double* vr, int out)
{
    StepArrays a{};
    a.cnt_in = cnt_in; a.idx_in = idx_in; a.val_in = val_in;
    a.cnt_out = ctx->cnt[out]; a.idx_out = ctx->idx[out]; a.val_out = ctx->val[out];
    a.vr = vr; a.gphase = ctx->d_gphase; a.gstage = ctx->d_gstage;
    a.dg = ctx->d_dg; a.pair_sigma = ctx->d_pair_sigma; a.pair_mu = ctx->d_pair_mu;
    a.dg_pair = (ctx->sp.use_dg && ctx->G <= kMaxPairTableGrains && !ctx->dg_pair_dirty) ? ctx->d_dg_pair : nullptr;
    a.grot = ctx->d_grot; a.facets = ctx->d_facets;
    a.vol_acc = ctx->d_vol_acc; a.status = ctx->d_status; a.counters = ctx->d_counters;
    return a;
}

uint32_t copy_state(opgpu_ctx* ctx, uint8_t* dc, int16_t* di, void* dv, const uint8_t* sc, const int16_t* si,
                    const void* sv)
{
    const size_t N = (size_t)ctx->n, K = (size_t)ctx->K;
    CK(cudaMemcpyAsync(dc, sc, N, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(di, si, N * K * sizeof(int16_t), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dv, sv, N * K * ctx->rsz, cudaMemcpyDeviceToDevice, ctx->stream));
    return OPGPU_OK;
}

uint32_t copy_grains(opgpu_ctx* ctx, double* vol, double* mx, double* vr, int8_t* ex, int8_t* stg,
                     const double* svol, const double* smx, const double* svr, const int8_t* sex, const int8_t* sstg)
{
    const size_t G = (size_t)ctx->G;
    CK(cudaMemcpyAsync(vol, svol, G * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(mx, smx, G * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(vr, svr, G * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ex, sex, G, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(stg, sstg, G, cudaMemcpyDeviceToDevice, ctx->stream));
    return OPGPU_OK;
}

// Fill the G*G driving-force table if it is out of date (the forward step does the same).
uint32_t refresh_dg_pair(opgpu_ctx* ctx)
{
    if (uint32_t r = refresh_pair_energy(ctx)) return r;
    return build_dg_pair(ctx);
}

uint32_t ensure_adjoint(opgpu_ctx* ctx)
{
    if (ctx->averaging)
        return fail(ctx, OPGPU_E_INVALID, "the adjoint and tangent-linear steps do not support driving-force averaging");
    if (ctx->adjoint_ready) return OPGPU_OK;
    const size_t N = (size_t)ctx->n, K = (size_t)ctx->K, G = (size_t)ctx->G;
    for (int b = 0; b < 2; b++) CK(dalloc(&ctx->d_lam[b], N * K));
    CK(dalloc(&ctx->d_lam_local, N * K));
    CK(dalloc(&ctx->d_lcnt, N));
    CK(dalloc(&ctx->d_lidx, N * KAdjList));
    CK(dalloc(&ctx->d_llam, N * KAdjList));
    CK(dalloc(&ctx->d_gsig, G * G));
    CK(dalloc(&ctx->d_gmu, G * G));
    CK(dalloc(&ctx->d_gdg, G));
    if (!ctx->adj_side)
    {
        cudaStream_t side;
        cudaEvent_t ef, ej;
        CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        ctx->adj_side = side;
        CK(cudaEventCreateWithFlags(&ef, cudaEventDisableTiming));
        ctx->adj_fork = ef;
        CK(cudaEventCreateWithFlags(&ej, cudaEventDisableTiming));
        ctx->adj_join = ej;
    }
    ctx->adjoint_ready = true;
    return OPGPU_OK;
}

uint32_t ensure_tlm(opgpu_ctx* ctx)
{
    if (ctx->averaging)
        return fail(ctx, OPGPU_E_INVALID, "the adjoint and tangent-linear steps do not support driving-force averaging");
    if (ctx->tlm_ready) return OPGPU_OK;
    const size_t N = (size_t)ctx->n, K = (size_t)ctx->K, G = (size_t)ctx->G;
    for (int b = 0; b < 2; b++) CK(dalloc(&ctx->d_dphi[b], N * K));
    CK(dalloc(&ctx->d_tsig, G * G));
    CK(dalloc(&ctx->d_tmu, G * G));
    CK(dalloc(&ctx->d_tdg, G));
    CK(dalloc(&ctx->d_tvol, G));
    ctx->tlm_ready = true;
    return OPGPU_OK;
}

// upper-triangle (a < b) copy of a symmetric G*G host table into a device table
uint32_t upload_upper(opgpu_ctx* ctx, double* dst, const double* src)
{
    const size_t G = (size_t)ctx->G;
    std::vector<double> h(G * G, 0.0);
    if (src)
        for (size_t a = 0; a < G; a++)
            for (size_t b = a + 1; b < G; b++) h[a * G + b] = src[a * G + b];
    CK(cudaMemcpyAsync(dst, h.data(), G * G * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

}  // namespace

extern "C" uint32_t opgpu_checkpoint_reserve(opgpu_ctx* ctx, int32_t nslots)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_checkpoint_reserve: set the grains first")) return r;
    if (nslots < 0 || nslots > 4096) return fail(ctx, OPGPU_E_INVALID, "opgpu_checkpoint_reserve: 0..4096 slots");
    const size_t N = (size_t)ctx->n, K = (size_t)ctx->K, G = (size_t)ctx->G;
    while ((int)ctx->slots.size() < nslots)
    {
        opgpu_ctx::Slot s;
        CK(dalloc(&s.cnt, N));
        CK(dalloc(&s.idx, N * K));
        CK(cudaMalloc(&s.val, N * K * ctx->rsz + 16));
        CK(dalloc(&s.volume, G)); CK(dalloc(&s.maxvol, G)); CK(dalloc(&s.vr, G));
        CK(dalloc(&s.exist, G)); CK(dalloc(&s.stage, G));
        ctx->slots.push_back(s);
    }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_checkpoint_save(opgpu_ctx* ctx, int32_t slot)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_checkpoint_save: not initialized")) return r;
    if (slot < 0 || slot >= (int)ctx->slots.size()) return fail(ctx, OPGPU_E_INVALID, "opgpu_checkpoint_save: no such slot");
    auto& s = ctx->slots[slot];
    if (uint32_t r = copy_state(ctx, s.cnt, s.idx, s.val, ctx->cnt[ctx->cur], ctx->idx[ctx->cur], ctx->val[ctx->cur])) return r;
    return copy_grains(ctx, s.volume, s.maxvol, s.vr, s.exist, s.stage, ctx->d_volume, ctx->d_maxvol, ctx->d_vr,
                       ctx->d_exist, ctx->d_gstage);
}

extern "C" uint32_t opgpu_step_save_input(opgpu_ctx* ctx, double dt, int32_t slot)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_step_save_input: not initialized")) return r;
    if (slot < 0 || slot >= (int)ctx->slots.size()) return fail(ctx, OPGPU_E_INVALID, "opgpu_step_save_input: no such slot");
    auto& s = ctx->slots[slot];
    // the grain records are updated in place by the step: copy them first (G values)
    if (uint32_t r = copy_grains(ctx, s.volume, s.maxvol, s.vr, s.exist, s.stage, ctx->d_volume, ctx->d_maxvol,
                                 ctx->d_vr, ctx->d_exist, ctx->d_gstage)) return r;
    const int in = ctx->cur;
    if (uint32_t r = enqueue_steps(ctx, dt, 1)) return r;
    // the step read buffer `in` and wrote the other one: the input state moves into the slot, the
    // slot's old buffers become the spare state buffer (every step rewrites it)
    std::swap(ctx->cnt[in], s.cnt);
    std::swap(ctx->idx[in], s.idx);
    std::swap(ctx->val[in], s.val);
    return opgpu_sync(ctx);
}

extern "C" uint32_t opgpu_checkpoint_load(opgpu_ctx* ctx, int32_t slot)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_checkpoint_load: not initialized")) return r;
    if (slot < 0 || slot >= (int)ctx->slots.size()) return fail(ctx, OPGPU_E_INVALID, "opgpu_checkpoint_load: no such slot");
    auto& s = ctx->slots[slot];
    if (uint32_t r = copy_state(ctx, ctx->cnt[ctx->cur], ctx->idx[ctx->cur], ctx->val[ctx->cur], s.cnt, s.idx, s.val)) return r;
    if (uint32_t r = copy_grains(ctx, ctx->d_volume, ctx->d_maxvol, ctx->d_vr, ctx->d_exist, ctx->d_gstage,
                                 s.volume, s.maxvol, s.vr, s.exist, s.stage)) return r;
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_adjoint_begin(opgpu_ctx* ctx, const double* dL_dV)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_adjoint_begin: not initialized")) return r;
    if (!dL_dV) return fail(ctx, OPGPU_E_INVALID, "opgpu_adjoint_begin: dL_dV is NULL");
    if (ctx->sp.aniso) return fail(ctx, OPGPU_E_INVALID, "opgpu_adjoint_begin: anisotropic energy models are not differentiated");
    if (uint32_t r = ensure_adjoint(ctx)) return r;
    const size_t G = (size_t)ctx->G;
    double* d_w = nullptr;
    CK(dalloc(&d_w, G));
    CK(cudaMemcpyAsync(d_w, dL_dV, G * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_lam[ctx->lam_cur], 0, (size_t)ctx->n * ctx->K * sizeof(double), ctx->stream));
    if (launch_lambda_init(ctx->n, ctx->cnt[ctx->cur], ctx->idx[ctx->cur], d_w, ctx->d_lam[ctx->lam_cur], ctx->stream))
        return fail(ctx, OPGPU_E_CUDA, "opgpu_adjoint_begin: launch");
    CK(cudaMemsetAsync(ctx->d_gsig, 0, G * G * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_gmu, 0, G * G * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_gdg, 0, G * sizeof(double), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    dfree(d_w);
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_adjoint_step(opgpu_ctx* ctx, int32_t slot, double dt)
{
    if (uint32_t r = require(ctx, ctx && ctx->adjoint_ready, "opgpu_adjoint_step: call opgpu_adjoint_begin first")) return r;
    if (slot < 0 || slot >= (int)ctx->slots.size()) return fail(ctx, OPGPU_E_INVALID, "opgpu_adjoint_step: no such slot");
    if (!(dt > 0.0)) return fail(ctx, OPGPU_E_INVALID, "opgpu_adjoint_step: dt > 0 required");
    if (uint32_t r = refresh_dg_pair(ctx)) return r;
    auto& s = ctx->slots[slot];
    StepParams sp = ctx->sp;
    sp.dt = dt;
    StepArrays a = step_arrays(ctx, s.cnt, s.idx, s.val, s.vr, 1 - ctx->cur);
    AdjArrays aa{};
    aa.cnt1 = ctx->cnt[ctx->cur]; aa.idx1 = ctx->idx[ctx->cur]; aa.lam1 = ctx->d_lam[ctx->lam_cur];
    aa.lam_local = ctx->d_lam_local; aa.lcnt = ctx->d_lcnt; aa.lidx = ctx->d_lidx; aa.llam = ctx->d_llam;
    aa.gsig = ctx->d_gsig; aa.gmu = ctx->d_gmu; aa.gdg = ctx->d_gdg;
    double* lam0 = ctx->d_lam[1 - ctx->lam_cur];   // every stored entry of the slot's state is written
    // the forward's lists of the slot's state: the classify kernel (its bulk copies go to the spare
    // state buffer, its volume sums and counters are discarded)
    a.slow_list = ctx->d_slow_list; a.slow_count = ctx->d_slow_count; a.slow_cap = (unsigned)ctx->n;
    a.wl = ctx->d_wl; a.wl_slice = ctx->wl_slice;
    a.bucket = ctx->d_bucket; a.bucket_count = ctx->d_bucket_count; a.bucket_off = ctx->d_bucket_off;
    a.bucket_cap = ctx->bucket_cap; a.slice = ctx->slice;
    const int nblocks = ctx->fp32 ? launch_classify_f32(sp, a, ctx->K, ctx->stream)
                                  : launch_classify_f64(sp, a, ctx->K, ctx->stream);
    if (nblocks < 0) return fail(ctx, OPGPU_E_CUDA, "opgpu_adjoint_step: classify launch");
    CK(cudaMemsetAsync(ctx->d_vol_acc, 0, (size_t)ctx->G * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_counters, 0, 3 * sizeof(unsigned long long), ctx->stream));   // wide, entries in/out
    CK(cudaMemsetAsync(ctx->d_counters + kCntCrowdedLast, 0, sizeof(unsigned long long), ctx->stream));
    const AdjStreams fork{ctx->adj_side, ctx->adj_fork, ctx->adj_join};
    if (launch_adjoint_step(sp, a, aa, ctx->K, ctx->fp32 != 0, nblocks, lam0, ctx->stream, fork))
        return fail(ctx, OPGPU_E_CUDA, "opgpu_adjoint_step: launch");
    ctx->kernel_launches += 12;
    ctx->lam_cur = 1 - ctx->lam_cur;
    // the state before the step becomes the current state (the adjoint is aligned with it): the slot
    // and the current state exchange their buffers (same sizes), so no state is copied
    std::swap(ctx->cnt[ctx->cur], s.cnt);
    std::swap(ctx->idx[ctx->cur], s.idx);
    std::swap(ctx->val[ctx->cur], s.val);
    std::swap(ctx->d_volume, s.volume);
    std::swap(ctx->d_maxvol, s.maxvol);
    std::swap(ctx->d_vr, s.vr);
    std::swap(ctx->d_exist, s.exist);
    std::swap(ctx->d_gstage, s.stage);
    const uint32_t st = read_status(ctx);
    if (st & OPGPU_E_CUDA) return st;
    return st & OPGPU_SOFT_MASK;
}

extern "C" uint32_t opgpu_adjoint_gradients(opgpu_ctx* ctx, double* dL_dsigma, double* dL_dmu, double* dL_ddG)
{
    if (uint32_t r = require(ctx, ctx && ctx->adjoint_ready, "opgpu_adjoint_gradients: no adjoint run")) return r;
    const size_t G = (size_t)ctx->G;
    std::vector<double> hs(G * G), hm(G * G);
    CK(cudaMemcpyAsync(hs.data(), ctx->d_gsig, G * G * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hm.data(), ctx->d_gmu, G * G * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (dL_ddG) CK(cudaMemcpyAsync(dL_ddG, ctx->d_gdg, G * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t a = 0; a < G; a++)
        for (size_t b = 0; b < G; b++)
        {
            const size_t k = a < b ? a * G + b : b * G + a;
            if (dL_dsigma) dL_dsigma[a * G + b] = a == b ? 0.0 : hs[k];
            if (dL_dmu) dL_dmu[a * G + b] = a == b ? 0.0 : hm[k];
        }
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_tlm_begin(opgpu_ctx* ctx, const double* dsigma, const double* dmu, const double* ddG)
{
    if (uint32_t r = require(ctx, ctx && ctx->initialized, "opgpu_tlm_begin: not initialized")) return r;
    if (ctx->fp32) return fail(ctx, OPGPU_E_INVALID, "opgpu_tlm_begin: the tangent-linear model runs the FP64 form");
    if (ctx->sp.aniso) return fail(ctx, OPGPU_E_INVALID, "opgpu_tlm_begin: anisotropic energy models are not differentiated");
    if (uint32_t r = ensure_tlm(ctx)) return r;
    const size_t G = (size_t)ctx->G;
    if (uint32_t r = upload_upper(ctx, ctx->d_tsig, dsigma)) return r;
    if (uint32_t r = upload_upper(ctx, ctx->d_tmu, dmu)) return r;
    if (ddG) CK(cudaMemcpyAsync(ctx->d_tdg, ddG, G * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    else CK(cudaMemsetAsync(ctx->d_tdg, 0, G * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_dphi[ctx->dphi_cur], 0, (size_t)ctx->n * ctx->K * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->d_tvol, 0, G * sizeof(double), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_tlm_step(opgpu_ctx* ctx, double dt, int32_t nsteps)
{
    if (uint32_t r = require(ctx, ctx && ctx->tlm_ready, "opgpu_tlm_step: call opgpu_tlm_begin first")) return r;
    if (nsteps < 0 || !(dt > 0.0)) return fail(ctx, OPGPU_E_INVALID, "opgpu_tlm_step: dt > 0 and nsteps >= 0 required");
    if (uint32_t r = refresh_dg_pair(ctx)) return r;
    StepParams sp = ctx->sp;
    sp.dt = dt;
    for (int s = 0; s < nsteps; s++)
    {
        const int in = ctx->cur, out = 1 - ctx->cur;
        StepArrays a = step_arrays(ctx, ctx->cnt[in], ctx->idx[in], ctx->val[in], ctx->d_vr, out);
        AdjArrays aa{};
        aa.tsig = ctx->d_tsig; aa.tmu = ctx->d_tmu; aa.tdg = ctx->d_tdg;
        aa.dphi_in = ctx->d_dphi[ctx->dphi_cur]; aa.dphi_out = ctx->d_dphi[1 - ctx->dphi_cur];
        aa.tvol = ctx->d_tvol;
        CK(cudaMemsetAsync(ctx->d_tvol, 0, (size_t)ctx->G * sizeof(double), ctx->stream));
        CK(cudaMemsetAsync(aa.dphi_out, 0, (size_t)ctx->n * ctx->K * sizeof(double), ctx->stream));
        if (launch_tlm_step(sp, a, aa, ctx->K, ctx->stream)) return fail(ctx, OPGPU_E_CUDA, "opgpu_tlm_step: launch");
        grains_update_kernel<<<grid_for(ctx->G, 256), 256, 0, ctx->stream>>>(ctx->G, ctx->d_vol_acc, ctx->d_volume,
            ctx->d_maxvol, ctx->d_refvol, ctx->d_vr, ctx->d_exist, ctx->d_gstage, ctx->d_counters, 1);
        CK(cudaGetLastError());
        ctx->kernel_launches += 2;
        ctx->cur = out;
        ctx->dphi_cur = 1 - ctx->dphi_cur;
    }
    const uint32_t st = read_status(ctx);
    if (st & OPGPU_E_CUDA) return st;
    return st & OPGPU_SOFT_MASK;
}

extern "C" uint32_t opgpu_tlm_volumes(opgpu_ctx* ctx, double* dV)
{
    if (uint32_t r = require(ctx, ctx && ctx->tlm_ready, "opgpu_tlm_volumes: call opgpu_tlm_begin first")) return r;
    if (!dV) return fail(ctx, OPGPU_E_INVALID, "opgpu_tlm_volumes: dV is NULL");
    CK(cudaMemcpyAsync(dV, ctx->d_tvol, (size_t)ctx->G * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

// ---- slab decomposition support (no reference counterpart: the reference exchanges halo cells with
// MPI, include/BoundaryConditions.h:2747-2854, and all-reduces the grain volumes,
// src/PhaseField.cpp:854-892) -------------------------------------------------------------------
namespace {

__global__ void grains_reset_kernel(int G, double* maxv, int8_t* exist)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) { maxv[g] = 0.0; exist[g] = 1; }
}

}  // namespace

extern "C" uint32_t opgpu_set_volume_window(opgpu_ctx* ctx, int32_t x0, int32_t x1)
{
    if (uint32_t r = require(ctx, true, "")) return r;
    if (x0 < 0 || x1 > ctx->grid.nx || x0 >= x1)
        return fail(ctx, OPGPU_E_INVALID, "opgpu_set_volume_window: need 0 <= x0 < x1 <= nx");
    ctx->sp.vol_x0 = x0;
    ctx->sp.vol_x1 = x1;
    return OPGPU_OK;
}

extern "C" int64_t opgpu_plane_bytes(opgpu_ctx* ctx)
{
    if (!ctx) return 0;
    const long long P = (long long)ctx->grid.ny * ctx->grid.nz;
    return P * (1 + (long long)ctx->K * (2 + (long long)ctx->rsz));
}

static uint32_t plane_copy(opgpu_ctx* ctx, int32_t x, void* buf, bool pack)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded, "plane copy: no state")) return r;
    if (x < 0 || x >= ctx->grid.nx || !buf) return fail(ctx, OPGPU_E_INVALID, "plane copy: x out of range or NULL buffer");
    const size_t P = (size_t)ctx->grid.ny * ctx->grid.nz, N = (size_t)ctx->n, K = (size_t)ctx->K;
    unsigned char* b = static_cast<unsigned char*>(buf);
    uint8_t* c = ctx->cnt[ctx->cur] + (size_t)x * P;
    unsigned char* i = reinterpret_cast<unsigned char*>(ctx->idx[ctx->cur] + (size_t)x * P);
    unsigned char* v = static_cast<unsigned char*>(ctx->val[ctx->cur]) + (size_t)x * P * ctx->rsz;
    unsigned char* bi = b + P;
    unsigned char* bv = bi + P * K * 2;
    const cudaMemcpyKind kind = cudaMemcpyDeviceToDevice;
    if (pack)
    {
        CK(cudaMemcpyAsync(b, c, P, kind, ctx->stream));
        CK(cudaMemcpy2DAsync(bi, P * 2, i, N * 2, P * 2, K, kind, ctx->stream));
        CK(cudaMemcpy2DAsync(bv, P * ctx->rsz, v, N * ctx->rsz, P * ctx->rsz, K, kind, ctx->stream));
    }
    else
    {
        CK(cudaMemcpyAsync(c, b, P, kind, ctx->stream));
        CK(cudaMemcpy2DAsync(i, N * 2, bi, P * 2, P * 2, K, kind, ctx->stream));
        CK(cudaMemcpy2DAsync(v, N * ctx->rsz, bv, P * ctx->rsz, P * ctx->rsz, K, kind, ctx->stream));
    }
    if (!ctx->stream_ordered) CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_pack_plane(opgpu_ctx* ctx, int32_t x, void* dev_buf) { return plane_copy(ctx, x, dev_buf, true); }
extern "C" uint32_t opgpu_unpack_plane(opgpu_ctx* ctx, int32_t x, const void* dev_buf)
{
    return plane_copy(ctx, x, const_cast<void*>(dev_buf), false);
}

extern "C" uint32_t opgpu_volume_recount(opgpu_ctx* ctx)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded && ctx->G > 0, "opgpu_volume_recount: no state")) return r;
    CK(cudaMemsetAsync(ctx->d_vol_acc, 0, (size_t)ctx->G * sizeof(double), ctx->stream));
    if (launch_volume_recount(ctx->sp, ctx->cnt[ctx->cur], ctx->idx[ctx->cur], ctx->val[ctx->cur], ctx->fp32,
                              ctx->d_vol_acc, ctx->stream))
        return fail(ctx, OPGPU_E_CUDA, "opgpu_volume_recount: launch");
    ctx->kernel_launches++;
    if (!ctx->stream_ordered) CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_step_partial(opgpu_ctx* ctx, double dt)
{
    if (ctx && ctx->averaging)
        return fail(ctx, OPGPU_E_INVALID, "opgpu_step_partial: a slab holds one halo plane; averaging needs Range planes");
    if (uint32_t r = enqueue_steps(ctx, dt, 1, true)) return r;
    if (ctx->stream_ordered) return OPGPU_OK;   // the soft status accumulates for opgpu_sync
    return opgpu_sync(ctx);
}

extern "C" uint32_t opgpu_set_stream_ordered(opgpu_ctx* ctx, int32_t enable)
{
    if (uint32_t r = require(ctx, ctx != nullptr, "opgpu_set_stream_ordered: no context")) return r;
    ctx->stream_ordered = enable != 0;
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_volume_accumulator(opgpu_ctx* ctx, double* dev_dst)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_volume_accumulator: no grains")) return r;
    if (!dev_dst) return fail(ctx, OPGPU_E_INVALID, "opgpu_volume_accumulator: NULL buffer");
    CK(cudaMemcpyAsync(dev_dst, ctx->d_vol_acc, (size_t)ctx->G * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if (!ctx->stream_ordered) CK(cudaStreamSynchronize(ctx->stream));
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_step_complete(opgpu_ctx* ctx, const double* dev_src, int32_t initial)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0, "opgpu_step_complete: no grains")) return r;
    if (!dev_src) return fail(ctx, OPGPU_E_INVALID, "opgpu_step_complete: NULL buffer");
    CK(cudaMemcpyAsync(ctx->d_vol_acc, dev_src, (size_t)ctx->G * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if (initial)
    {
        grains_reset_kernel<<<grid_for(ctx->G, 256), 256, 0, ctx->stream>>>(ctx->G, ctx->d_maxvol, ctx->d_exist);
        CK(cudaGetLastError());
    }
    grains_update_kernel<<<grid_for(ctx->G, 256), 256, 0, ctx->stream>>>(ctx->G, ctx->d_vol_acc, ctx->d_volume,
        ctx->d_maxvol, ctx->d_refvol, ctx->d_vr, ctx->d_exist, ctx->d_gstage, ctx->d_counters, initial ? 0 : 1);
    CK(cudaGetLastError());
    ctx->kernel_launches += initial ? 2 : 1;
    if (ctx->stream_ordered) return OPGPU_OK;   // the soft status accumulates for opgpu_sync
    const uint32_t st = read_status(ctx);
    if (st & OPGPU_E_CUDA) return st;
    return st & OPGPU_SOFT_MASK;
}

// ---- restart files and visual output -----------------------------------------------------------

namespace {

// GrainStages of the reference (include/GrainsProperties.h:35-40): Seed 0, Nucleus 1, Stable 2.
int stage_to_reference(int s) { return s == OPGPU_STAGE_SEED ? 0 : (s == OPGPU_STAGE_NUCLEUS ? 1 : 2); }
int stage_from_reference(int s) { return s == 0 ? OPGPU_STAGE_SEED : (s == 1 ? OPGPU_STAGE_NUCLEUS : OPGPU_STAGE_STABLE); }

template <class T>
void put_bytes(std::vector<unsigned char>& b, T x)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&x);
    b.insert(b.end(), p, p + sizeof(T));
}

template <class T>
T get_bytes(const unsigned char*& p)
{
    T x;
    std::memcpy(&x, p, sizeof(T));
    p += sizeof(T);
    return x;
}

// One grain record of GrainsProperties' binary file (Grain::Write, include/GrainsProperties.h:197-231):
// Exist, Mobile (bool); Stage (int); Parent, Phase, Variant (size_t); State (int); Density, RefVolume,
// Volume, MAXVolume; per axis Rcm, Vcm, Acm, aVel, aAcc, Force, Torque and a row of InertiaM; the
// orientation quaternion (s, x, y, z).
constexpr size_t kGrainRecordBytes = 2 * 1 + 4 + 3 * 8 + 4 + 4 * 8 + 3 * 10 * 8 + 4 * 8;

}  // namespace

extern "C" uint32_t opgpu_write_grains(opgpu_ctx* ctx, const char* path)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0 && path, "opgpu_write_grains: no grains or no path")) return r;
    const int G = ctx->G;
    std::vector<double> vol(G), maxv(G), refv(G);
    std::vector<int32_t> ex(G), st(G);
    if (uint32_t r = opgpu_grains(ctx, vol.data(), nullptr, maxv.data(), ex.data(), st.data())) return r;
    CK(cudaMemcpy(refv.data(), ctx->d_refvol, G * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<unsigned char> b;
    b.reserve(8 + (size_t)G * kGrainRecordBytes);
    put_bytes<uint64_t>(b, (uint64_t)G);
    for (int g = 0; g < G; g++)
    {
        const int ph = ctx->h_gphase.empty() ? 0 : ctx->h_gphase[g];
        put_bytes<uint8_t>(b, ex[g] ? 1 : 0);             // Exist
        put_bytes<uint8_t>(b, 1);                         // Mobile (reference default)
        put_bytes<int32_t>(b, stage_to_reference(st[g]));
        put_bytes<uint64_t>(b, 0);                        // Parent
        put_bytes<uint64_t>(b, (uint64_t)ph);             // Phase
        put_bytes<uint64_t>(b, 0);                        // Variant
        put_bytes<int32_t>(b, ctx->sp.solid_p[ph] ? 0 : 1);   // State: AggregateStates Solid 0, Liquid 1
        put_bytes<double>(b, 0.0);                        // Density (no equilibrium density here)
        put_bytes<double>(b, refv[g]);
        put_bytes<double>(b, vol[g]);
        put_bytes<double>(b, maxv[g]);
        for (int i = 0; i < 30; i++) put_bytes<double>(b, 0.0);   // rigid-body motion: not modelled
        for (int i = 0; i < 4; i++)
            put_bytes<double>(b, ctx->h_quat.empty() ? (i == 0 ? 1.0 : 0.0) : ctx->h_quat[4 * (size_t)g + i]);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ctx, OPGPU_E_IO, std::string("cannot open ") + path);
    const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    if (std::fclose(f) != 0 || !ok) return fail(ctx, OPGPU_E_IO, std::string("write failed: ") + path);
    return OPGPU_OK;
}

extern "C" uint32_t opgpu_read_grains(opgpu_ctx* ctx, const char* path)
{
    if (uint32_t r = require(ctx, ctx && ctx->G > 0 && path, "opgpu_read_grains: call opgpu_set_grains first")) return r;
    if (ctx->initialized) return fail(ctx, OPGPU_E_STATE, "opgpu_read_grains: read the grains before the state is finalized");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ctx, OPGPU_E_IO, std::string("cannot open ") + path);
    std::vector<unsigned char> b;
    unsigned char chunk[65536];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) b.insert(b.end(), chunk, chunk + got);
    std::fclose(f);
    const int G = ctx->G;
    if (b.size() < 8) return fail(ctx, OPGPU_E_IO, "opgpu_read_grains: truncated file");
    const unsigned char* p = b.data();
    const uint64_t size = get_bytes<uint64_t>(p);
    if (size != (uint64_t)G) return fail(ctx, OPGPU_E_INVALID, "opgpu_read_grains: the file holds a different number of grains");
    if (b.size() != 8 + (size_t)G * kGrainRecordBytes) return fail(ctx, OPGPU_E_IO, "opgpu_read_grains: file size does not match its grain count");
    std::vector<int16_t> ph(G);
    std::vector<int8_t> ex(G), st(G);
    std::vector<double> refv(G), vol(G), maxv(G), vr(G), quat(4 * (size_t)G);
    bool rotated = false;
    for (int g = 0; g < G; g++)
    {
        ex[g] = get_bytes<uint8_t>(p) ? 1 : 0;
        (void)get_bytes<uint8_t>(p);                      // Mobile
        st[g] = (int8_t)stage_from_reference(get_bytes<int32_t>(p));
        (void)get_bytes<uint64_t>(p);                     // Parent
        const uint64_t phase = get_bytes<uint64_t>(p);
        if (phase >= (uint64_t)ctx->sp.nphases) return fail(ctx, OPGPU_E_INVALID, "opgpu_read_grains: phase out of range");
        ph[g] = (int16_t)phase;
        (void)get_bytes<uint64_t>(p);                     // Variant
        (void)get_bytes<int32_t>(p);                      // State
        (void)get_bytes<double>(p);                       // Density
        refv[g] = get_bytes<double>(p);
        vol[g] = get_bytes<double>(p);
        maxv[g] = get_bytes<double>(p);
        vr[g] = maxv[g] / refv[g];                        // Grain::Read (include/GrainsProperties.h:98)
        p += 30 * sizeof(double);
        for (int i = 0; i < 4; i++) quat[4 * (size_t)g + i] = get_bytes<double>(p);
        rotated |= quat[4 * (size_t)g] != 1.0 || quat[4 * (size_t)g + 1] != 0.0 || quat[4 * (size_t)g + 2] != 0.0 ||
                   quat[4 * (size_t)g + 3] != 0.0;
    }
    CK(cudaMemcpy(ctx->d_gphase, ph.data(), G * sizeof(int16_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_gstage, st.data(), G, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_exist, ex.data(), G, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_refvol, refv.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_volume, vol.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_maxvol, maxv.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_vr, vr.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    ctx->h_gphase = ph;
    ctx->dg_pair_dirty = true;
    ctx->pair_energy_dirty = true;
    return opgpu_set_orientations(ctx, rotated ? quat.data() : nullptr);
}

namespace {

// Append the %.16g / integer text of one VTK point-data array in x-fastest order, formatted by
// OpenMP threads over z-planes (the reference streams the same text, VTK::ForEach,
// include/VTK.h:70-81).
template <class F>
void vtk_array(std::string& out, int nx, int ny, int nz, bool integral, F value)
{
    std::vector<std::string> part(nz);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nz; k++)
    {
        std::string& s = part[k];
        s.reserve((size_t)nx * ny * 18);
        char buf[40];
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
            {
                const long long v = ((long long)i * ny + j) * nz + k;
                const double x = value(v);
                const int len = integral ? std::snprintf(buf, sizeof(buf), "%lld\n", (long long)x)
                                         : std::snprintf(buf, sizeof(buf), "%.16g\n", x);
                s.append(buf, len);
            }
    }
    for (auto& s : part) out += s;
    out += "</DataArray>\n";
}

void vtk_header(std::string& out, const char* type, const std::string& name)
{
    out += std::string("<DataArray type = \"") + type + "\" Name = \"" + name +
           "\" NumberOfComponents=\"1\" format=\"ascii\">\n";
}

}  // namespace

extern "C" uint32_t opgpu_write_vtk_host(int32_t nx, int32_t ny, int32_t nz, const int32_t* counts, const int32_t* idx,
                                         const double* val, int32_t ngrains, const int32_t* grain_phase,
                                         int32_t nphases, int32_t laplacian_stencil, int32_t gradient_stencil,
                                         const char* path)
{
    if (nx < 1 || ny < 1 || nz < 1 || !counts || !path || ngrains < 1 || nphases < 1 || nphases > kMaxPhases)
        return OPGPU_E_INVALID;
    if (laplacian_stencil < 0 || laplacian_stencil > 2 || gradient_stencil < 0 || gradient_stencil > 2)
        return OPGPU_E_INVALID;
    const long long N = (long long)nx * ny * nz;
    std::vector<long long> off(N + 1, 0);
    for (long long v = 0; v < N; v++) off[v + 1] = off[v] + counts[v];
    for (long long e = 0; e < off[N]; e++)
        if (idx[e] < 0 || idx[e] >= ngrains) return OPGPU_E_INVALID;
    auto phase_of = [&](int g) { return grain_phase ? grain_phase[g] : 0; };
    for (int g = 0; g < ngrains; g++)
        if (phase_of(g) < 0 || phase_of(g) >= nphases) return OPGPU_E_INVALID;
    StepParams sp{};
    set_stencils(sp, laplacian_stencil, gradient_stencil, 1.0);
    auto wrap = [](int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); };
    // NodePF flag (PhaseField::SetFlagsSR, src/PhaseField.cpp:953-969) and the list length after
    // CalculateDerivativesSR (src/PhaseField.cpp:566-615): stored fields plus the zero-valued
    // candidates every stencil neighbour brings to a flag != 0 voxel
    std::vector<int8_t> flag(N);
    std::vector<int32_t> junctions(N);
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < N; v++)
    {
        const int x = (int)(v / ((long long)ny * nz)), y = (int)((v / nz) % ny), z = (int)(v % nz);
        int f = counts[v] > 1 ? 2 : 0;
        for (int dx = -1; dx <= 1 && f == 0; dx++)
            for (int dy = -1; dy <= 1 && f == 0; dy++)
                for (int dz = -1; dz <= 1 && f == 0; dz++)
                {
                    const long long u = ((long long)wrap(x + dx, nx) * ny + wrap(y + dy, ny)) * nz + wrap(z + dz, nz);
                    if (counts[u] > 1) f = 1;
                }
        flag[v] = (int8_t)f;
        int n = counts[v];
        if (f != 0)
        {
            std::vector<int32_t> seen(idx + off[v], idx + off[v + 1]);
            for (int q = 0; q < sp.ns + sp.ng; q++)
            {
                const signed char* d = q < sp.ns ? sp.lap_d[q] : sp.grad_d[q - sp.ns];
                const long long u = ((long long)wrap(x + d[0], nx) * ny + wrap(y + d[1], ny)) * nz + wrap(z + d[2], nz);
                for (long long e = off[u]; e < off[u + 1]; e++)
                    if (val[e] != 0.0 && std::find(seen.begin(), seen.end(), idx[e]) == seen.end()) seen.push_back(idx[e]);
            }
            n = (int)seen.size();
        }
        junctions[v] = n;
    }
    std::string out;
    char line[160];
    out += "<?xml version= \"1.0\" encoding=\"UTF-8\" standalone=\"yes\"?>\n";
    out += "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    std::snprintf(line, sizeof(line), "<StructuredGrid WholeExtent=\"0 %d 0 %d 0 %d\">\n", nx - 1, ny - 1, nz - 1);
    out += line;
    out += "<PointData Scalars= \"ScalarData\">\n";
    // PhaseField::Interfaces (src/PhaseField.cpp:3765-3777)
    vtk_header(out, "Float64", "Interfaces");
    vtk_array(out, nx, ny, nz, false, [&](long long v) {
        double sum = 0.5;
        if (flag[v] == 2)
            for (long long a = off[v]; a < off[v + 1]; a++)
                for (long long b = a + 1; b < off[v + 1]; b++) sum -= val[a] * val[b];
        return 1.0 / (sum * 2.0);
    });
    vtk_header(out, "Int32", "Flags");
    vtk_array(out, nx, ny, nz, true, [&](long long v) { return (double)flag[v]; });
    // NodePF::majority_index (include/Containers/NodePF.h:194-211)
    vtk_header(out, "Int32", "PhaseFields");
    vtk_array(out, nx, ny, nz, true, [&](long long v) {
        if (junctions[v] == 1) return (double)idx[off[v]];
        double mv = 0.0;
        int mi = 0;
        for (long long a = off[v]; a < off[v + 1]; a++)
            if (val[a] > mv) { mv = val[a]; mi = idx[a]; }
        return (double)mi;
    });
    // PhaseField::CalculateFractions (src/PhaseField.cpp:411-423)
    for (int ph = 0; ph < nphases; ph++)
    {
        vtk_header(out, "Float64", "PhaseFraction_" + std::to_string(ph));
        vtk_array(out, nx, ny, nz, false, [&](long long v) {
            double s = 0.0;
            for (long long a = off[v]; a < off[v + 1]; a++)
                if (phase_of(idx[a]) == ph) s += val[a];
            return s;
        });
    }
    vtk_header(out, "UInt64", "Junctions");
    vtk_array(out, nx, ny, nz, true, [&](long long v) { return (double)junctions[v]; });
    // Variant and Parent of the majority grain: 0 for every grain here (PhaseField::Variants,
    // ::ParentGrain, src/PhaseField.cpp:3793-3839)
    vtk_header(out, "Float64", "Variants");
    vtk_array(out, nx, ny, nz, false, [&](long long) { return 0.0; });
    vtk_header(out, "Float64", "ParentGrain");
    vtk_array(out, nx, ny, nz, false, [&](long long) { return 0.0; });
    out += "</PointData>\n";
    // VTK::WriteCoordinates (include/VTK.h:420-471), single resolution
    out += "<Points>\n";
    out += "<DataArray type = \"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    {
        std::vector<std::string> part(nz);
#pragma omp parallel for schedule(dynamic)
        for (int k = 0; k < nz; k++)
        {
            char buf[80];
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++)
                    part[k].append(buf, std::snprintf(buf, sizeof(buf), "%d %d %d\n", i, j, k));
        }
        for (auto& s : part) out += s;
    }
    out += "</DataArray>\n";
    out += "</Points>\n";
    out += "</StructuredGrid>\n";
    out += "</VTKFile>\n";
    FILE* f = std::fopen(path, "wb");
    if (!f) return OPGPU_E_IO;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return (std::fclose(f) == 0 && ok) ? OPGPU_OK : OPGPU_E_IO;
}

extern "C" uint32_t opgpu_write_vtk(opgpu_ctx* ctx, const char* path)
{
    if (uint32_t r = require(ctx, ctx && ctx->state_loaded && path, "opgpu_write_vtk: no state")) return r;
    int64_t total = 0;
    if (uint32_t r = opgpu_total_entries(ctx, &total)) return r;
    std::vector<int32_t> counts(ctx->n), idx(total), gp(ctx->G);
    std::vector<double> val(total);
    if (uint32_t r = opgpu_download_lists(ctx, counts.data(), idx.data(), val.data())) return r;
    for (int g = 0; g < ctx->G; g++) gp[g] = ctx->h_gphase.empty() ? 0 : ctx->h_gphase[g];
    const uint32_t r = opgpu_write_vtk_host(ctx->grid.nx, ctx->grid.ny, ctx->grid.nz, counts.data(), idx.data(),
                                            val.data(), ctx->G, gp.data(), ctx->sp.nphases,
                                            ctx->grid.laplacian_stencil, ctx->grid.gradient_stencil, path);
    if (r) return fail(ctx, r, std::string("opgpu_write_vtk: cannot write ") + path);
    return OPGPU_OK;
}
