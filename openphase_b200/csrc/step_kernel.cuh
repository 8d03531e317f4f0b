// Per-voxel arithmetic of the fused multiphase-field time step, and the full-grid generic kernel.
//
// For one voxel, what the reference spreads over five grid passes:
//   1. derivatives + candidates   PhaseField::CalculateDerivativesSR  (src/PhaseField.cpp:566-615)
//   2. pairwise kinetics          DoubleObstacle::CalculatePhaseFieldIncrementsSR
//                                 (src/DoubleObstacle.cpp:502-571)
//   3. driving-force merge        DrivingForce::MergePhaseFieldIncrementsSR (src/DrivingForce.cpp:497-602)
//   4. simplex projection         PhaseField::NormalizeIncrementsSR (src/PhaseField.cpp:1351-1561)
//   5. merge + finalize           PhaseField::MergeIncrementsSR (:1268-1299), NodePF::finalize
//                                 (include/Containers/NodePF.h:214-255)
// Stage 1 differs between the kernels (global-memory scan here, shared-memory dense planes in the
// tiled kernel); stages 2-5 are `list_step`, shared by both.  The flags of PhaseField::SetFlagsSR
// are derived from neighbour counts, the periodic boundary copies become index wrap-around, and
// the grain volumes of the new state (PhaseField::CalculateGrainsVolume, src/PhaseField.cpp:812-951)
// accumulate through per-block shared-memory tables.
//
// Exactness: in the FP64 form (compiled with --fmad=false) every floating-point expression is
// evaluated in the reference's order, so results are bit-identical to the reference except for
// tanh (CUDA vs. libm, a few ulp) and the grain-volume summation order.
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

// The driving force of a grain pair after the tanh limiter (src/DrivingForce.cpp:548-583):
// allowed*tanh((dG_b - dG_a)/allowed).  It depends on the pair only, so the step reads it from a
// G*G table filled once per parameter change (same arithmetic), else evaluates it in place.
__device__ __forceinline__ double limited_force(const StepParams& p, const StepArrays& a, int ga, int gb)
{
    if (a.dg_pair) return a.dg_pair[(long long)ga * p.ngrains + gb];
    double locdG = a.dg[gb] - a.dg[ga];
    if (p.limiting)
    {
        const double allowed = p.allowed_p[a.gphase[ga] * p.nphases + a.gphase[gb]];
        locdG = allowed * tanh(locdG / allowed);
    }
    return locdG;
}

// The limited driving force of list entries i < j of an interface voxel v with c stored fields (the
// leading entries of its list): with driving-force averaging, the averaged force of a pair of
// stored fields; else, and for the zero-valued candidates (weight 0: their force is multiplied by
// 0 unless a Seed takes part, which the reference gives the raw force), the pair's own force.
__device__ __forceinline__ double pair_force(const StepParams& p, const StepArrays& a, long long v, int c, int i,
                                             int j, int gi, int gj)
{
    if (a.df_lim && j < c)
    {
        const unsigned o = a.df_off[v];
        if ((unsigned long long)o + (unsigned)(c * (c - 1) / 2) <= a.df_cap) return a.df_lim[o + pair_pos(i, j, c)];
    }
    return limited_force(p, a, gi, gj);
}

// Slice of entry e of one list length in the concatenated length buckets: the s with
// off[s] <= e < off[s + 1] (off[nslices] > e).
__device__ __forceinline__ int slice_of(const unsigned* __restrict__ off, int nslices, unsigned e)
{
    int lo = 0, hi = nslices;
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-block grain-volume table in shared memory.
constexpr int kVolSlots = 1024;

__device__ __forceinline__ void vol_insert_n(int* keys, double* sums, int nslots, double* global_acc, int g, double v)
{
    unsigned h = ((unsigned)g * 2654435761u) & (unsigned)(nslots - 1);
    for (int probe = 0; probe < nslots; probe++)
    {
        const int k = atomicCAS(&keys[h], -1, g);
        if (k == -1 || k == g)
        {
            atomicAdd(&sums[h], v);
            return;
        }
        h = (h + 1) & (unsigned)(nslots - 1);
    }
    atomicAdd(&global_acc[g], v);
}

// Working arrays of one voxel: element k of an array at base[k*stride] (stride 1 for per-thread
// local arrays, the block size for a column of shared memory).
template <class R>
struct ListScratch {
    int16_t* g;      // [KL] grain indices (in: list, out: new record)
    R* val;          // [KL] values        (in: list, out: new record)
    R* lap;          // [KL] Laplacians
    R* sg;           // [KL*(KL-1)/2] pair energies
    double* pv;      // [KL*(KL-1)/2] pair increments
    double* pos;     // [KL] positive increments / upper limits
    double* neg;     // [KL] negative increments / lower limits
    int stride;
    const R* grad;   // [KL*3] gradients, entry k at grad[3k..3k+2] (anisotropic energies), or null
};

// InterfaceOrientation (src/InterfaceProperties.cpp:39-45): -grad normalised (dVector3::normalize,
// include/Containers/dVector3.h:301-316), rotated back with the transposed RotationMatrix
// (include/Containers/MatrixVectorOperators.h:43-52).
__device__ __forceinline__ void interface_orientation(const double* g3, const double* R, double* out)
{
    double n0 = g3[0] * (-1.0), n1 = g3[1] * (-1.0), n2 = g3[2] * (-1.0);
    const double norm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (norm > DBL_EPSILON)
    {
        const double inv = 1.0 / norm;
        n0 *= inv; n1 *= inv; n2 *= inv;
    }
    else
    {
        n0 = 0.0; n1 = 0.0; n2 = 0.0;
    }
    for (int i = 0; i < 3; i++)
    {
        double t = 0.0;
        t += R[i] * n0;
        t += R[3 + i] * n1;
        t += R[6 + i] * n2;
        out[i] = t;
    }
}

// InterfaceEnergyModel::Calculate (include/InterfaceProperties/InterfaceEnergyModel.h:325-399) for
// the models of the interface normal n: CUBIC, HEXBOETTGER (Boettger et al. 2006), HEXSUN (Sun et
// al. 2006), HEXYANG (Yang et al. 2015), FACETED (facet rows: unit normal, SigmaF, EpsilonEF) and
// FACETEDEXP (rows: unit normal, EpsilonEF, PowerEF), in the reference's operation order.
__device__ __forceinline__ double model_energy(const StepParams& p, int q, const double* n, const double* facets)
{
    const double E = p.sigma_p[q], e1 = p.eps_p[q];
    const double x = n[0], y = n[1], z = n[2];
    switch (p.emodel[q])
    {
        case 3:
            return E * (1.0 - e1 * (pow(x, 6.0) - pow(y, 6.0) - 15.0 * pow(x, 4.0) * y * y + 15.0 * pow(y, 4.0) * x * x
                                    + (5.0 * pow(z, 4.0) - 5.0 * pow(z, 2.0) + pow(z, 6.0))));
        case 4:
        {
            const double pi = 3.14159265358979323846;
            const double e2 = p.eps_x[q][0], e3 = p.eps_x[q][1], e4 = p.eps_x[q][2];
            return E * (1.0 + e1 * sqrt(5.0 / 16.0 / pi) * (3.0 * z * z - 1.0)
                        + e2 * 3.0 / 16.0 / sqrt(pi) * (35.0 * pow(z, 4.0) - 30.0 * z * z + 3.0)
                        + e3 * sqrt(13.0 / pi) / 32.0 * (231.0 * pow(z, 6.0) - 315.0 * pow(z, 4.0) + 105.0 * z * z - 5.0)
                        + e4 * sqrt(6006.0 / pi) / 64.0
                              * (pow(x, 6.0) - 15.0 * pow(x, 4.0) * y * y + 15.0 * x * x * pow(y, 4.0) - pow(y, 6.0)));
        }
        case 5:
        {
            const double e2 = p.eps_x[q][0], e3 = p.eps_x[q][1];
            return E * (1.0 + e1 * pow((3.0 * z * z - 1.0), 2.0)
                        + e2 * pow((x * x * x - 3.0 * x * y * y), 2.0) * pow((9.0 * z * z - 1.0 + e3), 2.0));
        }
        case 6:
        {
            // FACETED (Salama et al. 2020): the facet of largest cos^2 of its inclination sets the
            // energy EnergyA*EpsilonA^2*(sin^2 + EpsilonA^2 cos^2)^(-3/2)
            double cos2 = 0.0, ea = 0.0, epa = 0.0;
            for (int f = p.facet_lo[q]; f < p.facet_hi[q]; f++)
            {
                const double* r = facets + 5 * f;
                const double c = x * r[0] + y * r[1] + z * r[2];
                const double c2 = c * c;
                if (c2 > cos2) { cos2 = c2; ea = r[3]; epa = r[4]; }
            }
            const double sin2 = 1.0 - cos2;
            return ea * epa * epa * pow(sqrt(sin2 + epa * epa * cos2), -3.0);
        }
        case 7:
        {
            // FACETEDEXP (InterfaceEnergyModel.h:389-413): every facet facing the normal lowers the
            // energy by E*eps*cos^p and adds its second-order term E*eps*p*cos^p (rows: unit
            // normal, EpsilonEF, PowerEF)
            double loc = E;
            for (int f = p.facet_lo[q]; f < p.facet_hi[q]; f++)
            {
                const double* r = facets + 5 * f;
                const double c = x * r[0] + y * r[1] + z * r[2];
                if (c > 0.0)
                {
                    loc -= E * r[3] * pow(c, r[4]);
                    loc += E * r[3] * r[4] * pow(c, r[4]);
                }
            }
            return loc;
        }
        default:
            return E * (1.0 + e1 * (1.5 - 2.5 * (pow(x, 4.0) + pow(y, 4.0) + pow(z, 4.0))));
    }
}

// InterfaceMobilityModel::Calculate (include/InterfaceProperties/InterfaceMobilityModel.h:210-265):
// CUBIC, HEXBOETTGER, HEXSUN, HEXYANG and FACETED of the interface normal n, in the reference's operation order
// (the signs of the anisotropy terms differ from the energy models').
__device__ __forceinline__ double mobility_model(const StepParams& p, int q, const double* n, const double* facets)
{
    const double M = p.mu_p[q], e1 = p.meps[q][0], e2 = p.meps[q][1], e3 = p.meps[q][2], e4 = p.meps[q][3];
    const double x = n[0], y = n[1], z = n[2];
    switch (p.mmodel[q])
    {
        case 6:
        {
            // FACETED (InterfaceMobilityModel.h:266-288): the facet of smallest inclination
            // acos(n.f) (the last one on ties) sets MuF*(EpsMF + (1 - EpsMF)|tan i| tanh(1/|tan i|))
            double incl = 3.14159265358979323846, ma = 0.0, ea = 0.0;
            for (int f = p.mfacet_lo[q]; f < p.mfacet_hi[q]; f++)
            {
                const double* r = facets + 5 * f;
                const double d = acos(x * r[0] + y * r[1] + z * r[2]);
                if (fabs(d) <= fabs(incl)) { incl = d; ma = r[3]; ea = r[4]; }
            }
            return ma * (ea + (1.0 - ea) * fabs(tan(incl)) * tanh(pow(fabs(tan(incl)), -1.0)));
        }
        case 3:
            return M * (1.0 + e1 * (pow(x, 6.0) - pow(y, 6.0) - 15.0 * pow(x, 4.0) * y * y + 15.0 * pow(y, 4.0) * x * x
                                    + (5.0 * pow(z, 4.0) - 5.0 * pow(z, 2.0) + pow(z, 6.0))));
        case 4:
        {
            const double pi = 3.14159265358979323846;
            return M * (1.0 - e1 * sqrt(5.0 / 16.0 / pi) * (3.0 * z * z - 1.0)
                        - e2 * 3.0 / 16.0 / sqrt(pi) * (35.0 * pow(z, 4.0) - 30.0 * z * z + 3.0)
                        - e3 * sqrt(13.0 / pi) / 32.0 * (231.0 * pow(z, 6.0) - 315.0 * pow(z, 4.0) + 105.0 * z * z - 5.0)
                        - e4 * sqrt(6006.0 / pi) / 64.0
                              * (pow(x, 6.0) - 15.0 * pow(x, 4.0) * y * y + 15.0 * x * x * pow(y, 4.0) - pow(y, 6.0)));
        }
        case 5:
            return M * (1.0 - e1 * pow((3.0 * z * z - 1.0), 2.0)
                        - e2 * pow((x * x * x - 3.0 * x * y * y), 2.0) * pow((9.0 * z * z - 1.0 + e3), 2.0));
        default:
            return M * (1.0 - e1 * (1.5 - 2.5 * (pow(x, 4.0) + pow(y, 4.0) + pow(z, 4.0))));
    }
}

// The interface mobility of the pair (i, j) of a voxel's list as InterfaceProperties::SetSR stores
// it (src/InterfaceProperties.cpp:680-707): ISO (or the per-grain-pair table), or the anisotropic
// model summed over the solid grains whose value is neither 0 nor 1 (Mobility when there is none).
template <class R>
__device__ __forceinline__ double voxel_mobility(const StepParams& p, const StepArrays& a, const ListScratch<R>& sc,
                                                 int i, int j)
{
    const int S = sc.stride;
    const int gi = sc.g[i * S], gj = sc.g[j * S];
    const int pA = a.gphase[gi], pB = a.gphase[gj];
    const int q = pA * p.nphases + pB;
    if (p.mmodel[q] == 0) return pair_mobility(p, a, gi, gj);
    double loc = 0.0;
    int solids = 0;
    for (int side = 0; side < 2; side++)
    {
        const int e = side == 0 ? i : j;
        const int g = side == 0 ? gi : gj;
        if (!p.solid_p[side == 0 ? pA : pB]) continue;
        const double v = (double)sc.val[e * S];
        if (v == 0.0 || v == 1.0) continue;
        const double g3[3] = {(double)sc.grad[(3 * e) * S], (double)sc.grad[(3 * e + 1) * S], (double)sc.grad[(3 * e + 2) * S]};
        double n[3];
        interface_orientation(g3, a.grot + 9 * (long long)g, n);
        loc += mobility_model(p, q, n, a.facets);
        solids++;
    }
    if (solids == 0) loc = p.mu_p[q];
    return loc;
}

// The interface energy of the pair (i, j) of a voxel's list as InterfaceProperties::SetSR stores it
// (src/InterfaceProperties.cpp:617-673): the ISO value, or the anisotropic model averaged over the
// solid grains' interface orientations with weights |phi(1 - phi)| (MaxEnergy when no weight counts).
template <class R>
__device__ __forceinline__ double voxel_energy(const StepParams& p, const StepArrays& a, const ListScratch<R>& sc,
                                               int i, int j)
{
    const int S = sc.stride;
    const int gi = sc.g[i * S], gj = sc.g[j * S];
    const int pA = a.gphase[gi], pB = a.gphase[gj];
    const int q = pA * p.nphases + pB;
    if (p.emodel[q] == 0 || p.emodel[q] == 2) return pair_energy(p, a, gi, gj);   // ISO, per-pair table
    double loc = 0.0, wA = 0.0, wB = 0.0;
    if (p.solid_p[pA])
    {
        const double v = (double)sc.val[i * S];
        wA = fabs(v * (1.0 - v));
        if (wA > DBL_EPSILON)
        {
            const double g3[3] = {(double)sc.grad[(3 * i) * S], (double)sc.grad[(3 * i + 1) * S], (double)sc.grad[(3 * i + 2) * S]};
            double n[3];
            interface_orientation(g3, a.grot + 9 * (long long)gi, n);
            loc += model_energy(p, q, n, a.facets) * wA;
        }
        else wA = 0.0;
    }
    if (p.solid_p[pB])
    {
        const double v = (double)sc.val[j * S];
        wB = fabs(v * (1.0 - v));
        if (wB > DBL_EPSILON)
        {
            const double g3[3] = {(double)sc.grad[(3 * j) * S], (double)sc.grad[(3 * j + 1) * S], (double)sc.grad[(3 * j + 2) * S]};
            double n[3];
            interface_orientation(g3, a.grot + 9 * (long long)gj, n);
            loc += model_energy(p, q, n, a.facets) * wB;
        }
        else wB = 0.0;
    }
    if (wA + wB > DBL_EPSILON) loc /= wA + wB;
    else loc = p.maxe_p[q];
    return loc;
}

// Stages 2-5 for a list of n fields (own fields first, then candidates, as CalculateDerivativesSR
// leaves them) with their Laplacians, of voxel v with c stored fields.  Leaves the new record (the
// fields that survive finalize, in list order) in sc.g / sc.val and returns its length.
template <class R>
__device__ __forceinline__ int list_step(const StepParams& p, const StepArrays& a, const ListScratch<R>& sc, int n,
                                         int flag, uint32_t& st, long long v, int c)
{
    const int S = sc.stride;
#define G_(k) sc.g[(k) * S]
#define V_(k) sc.val[(k) * S]
#define L_(k) sc.lap[(k) * S]
#define SG_(q) sc.sg[(q) * S]
#define PV_(q) sc.pv[(q) * S]
#define POS_(k) sc.pos[(k) * S]
#define NEG_(k) sc.neg[(k) * S]
    // ---- 2. pair kinetics -----------------------------------------------------------------------
    double localN;
    if (p.consider_nucleus_volume)
    {
        localN = 0.0;
        for (int k = 0; k < n; k++) localN += a.vr[G_(k)];
    }
    else
    {
        localN = (double)n;
    }
    const R norm_1 = (R)(1.0 / localN);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            SG_(pair_pos(i, j, n)) = (R)(p.aniso ? voxel_energy<R>(p, a, sc, i, j) : pair_energy(p, a, G_(i), G_(j)));
    const R pref = (R)p.pref_do;
    for (int i = 0; i < n; i++)
    {
        const int gi = G_(i);
        const double vri = a.vr[gi];
        const R vali = V_(i), lapi = L_(i);
        for (int j = i + 1; j < n; j++)
        {
            const int gj = G_(j);
            const int q = pair_pos(i, j, n);
            const double vrj = a.vr[gj];
            const R scale = (vri == 1.0 && vrj == 1.0) ? R(1) : (R)sqrt(vri * vrj);   // sqrt(1*1) == 1
            const R h = R(0.5) * (R(1) + scale) * pref;
            const R valj = V_(j);
            R dphi = SG_(q) * ((lapi + h * vali) - (L_(j) + h * valj));
            if (n > 2)
            {
                for (int k = 0; k < n; k++)
                {
                    if (k == i || k == j) continue;
                    const R sbk = SG_(j < k ? pair_pos(j, k, n) : pair_pos(k, j, n));
                    const R sak = SG_(i < k ? pair_pos(i, k, n) : pair_pos(k, i, n));
                    const R valk = V_(k);
                    dphi += (sbk - sak) * (L_(k) + h * valk);
                    if (p.tj_factor != 0.0 || scale < R(1))
                    {
                        const int pA = a.gphase[gi], pB = a.gphase[gj], pG = a.gphase[G_(k)];
                        const int P = p.nphases;
                        const R tj = (R)dmax_ref(p.tj_factor, (double)(R(1) - scale));
                        dphi += tj * pref
                              * (((R)p.sigma_p[pA * P + pB] + (R)p.sigma_p[pB * P + pG]) + (R)p.sigma_p[pA * P + pG])
                              * (vali * valk - valj * valk);
                    }
                }
            }
            dphi *= (R)(p.aniso ? voxel_mobility<R>(p, a, sc, i, j) : pair_mobility(p, a, gi, gj)) * norm_1 * scale;
            PV_(q) = (double)dphi;
        }
    }
    // ---- 3. driving force (interface voxels only) ----------------------------------------------
    if (p.use_dg && flag == 2)
    {
        for (int i = 0; i < n; i++)
        {
            const int gi = G_(i);
            const double vi = (double)V_(i);
            for (int j = i + 1; j < n; j++)
            {
                const int gj = G_(j);
                const double locdG = pair_force(p, a, v, c, i, j, gi, gj);
                double norm = sqrt(vi * (double)V_(j));
                if (a.gstage[gi] == 1 || a.gstage[gj] == 1) norm += 1.0e-6;
                const double mob = p.aniso ? voxel_mobility<R>(p, a, sc, i, j) : pair_mobility(p, a, gi, gj);
                const double dpsi = locdG * (double)(R)mob * norm * p.pref_df;
                PV_(pair_pos(i, j, n)) += dpsi;
            }
        }
    }
    // ---- 4. projection (NormalizeIncrementsSR) ---------------------------------------------------
    const double dt = p.dt;
    const int np = n * (n - 1) / 2;
    if (np == 1)
    {
        const double valueA = (PV_(0) + 0.0) * dt;
        const double old_value = (double)V_(0);
        if ((old_value == 0.0 && valueA < 0.0) || (old_value == 1.0 && valueA > 0.0))
        {
            PV_(0) = 0.0;
        }
        else
        {
            const double new_value = old_value + valueA;
            double norm = 1.0;
            if (new_value < 0.0) norm *= -old_value / valueA;
            else if (new_value > 1.0) norm *= (1.0 - old_value) / valueA;
            if (norm > DBL_EPSILON) PV_(0) *= norm;
            else PV_(0) = 0.0;
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
                dpsi += (i < j) ? PV_(pair_pos(i, j, n)) : PV_(pair_pos(j, i, n)) * (-1.0);
            }
            const double vi = (double)V_(i);
            if ((vi == 0.0 && dpsi < 0.0) || (vi == 1.0 && dpsi > 0.0))
            {
                for (int j = 0; j < n; j++)
                {
                    if (j == i) continue;
                    PV_(i < j ? pair_pos(i, j, n) : pair_pos(j, i, n)) = 0.0;
                }
            }
        }
        bool any = false;
        for (int q = 0; q < np; q++) any |= (PV_(q) != 0.0);
        if (any)
        {
            for (int it = 1; it <= 25; it++)
            {
                for (int i = 0; i < n; i++) { POS_(i) = 0.0; NEG_(i) = 0.0; }
                for (int i = 0; i < n; i++)
                    for (int j = i + 1; j < n; j++)
                    {
                        const double w = PV_(pair_pos(i, j, n));
                        if (w < 0.0) { NEG_(i) += w; POS_(j) += -w; }
                        if (w > 0.0) { POS_(i) += w; NEG_(j) += -w; }
                    }
                // limits: NEG_ becomes the lower limit, POS_ the upper limit of each field
                for (int i = 0; i < n; i++)
                {
                    const double vi = (double)V_(i);
                    const double pi = POS_(i), ni = NEG_(i);
                    const double newPF = vi + (pi + ni) * dt;
                    double limN = 1.0, limP = 1.0;
                    if (newPF < 0.0) limN = dmin_ref(1.0, -(vi + pi * dt) / (ni * dt));
                    if (newPF > 1.0) limP = dmin_ref(1.0, (1.0 - (vi + ni * dt)) / (pi * dt));
                    NEG_(i) = limN;
                    POS_(i) = limP;
                }
                bool needed = false;
                for (int i = 0; i < n; i++)
                    for (int j = i + 1; j < n; j++)
                    {
                        const int q = pair_pos(i, j, n);
                        double w = PV_(q);
                        if (w < 0.0)
                        {
                            const double lim = dmin_ref(NEG_(i), POS_(j));
                            w *= lim;
                            if (lim < 1.0) needed = true;
                        }
                        if (w > 0.0)
                        {
                            const double lim = dmin_ref(POS_(i), NEG_(j));
                            w *= lim;
                            if (lim < 1.0) needed = true;
                        }
                        PV_(q) = w;
                    }
                if (!needed) break;
                if (it == 25) st |= kStLimiterCap;
            }
            for (int q = 0; q < np; q++)
                if (fabs(PV_(q) * dt) < DBL_EPSILON) PV_(q) = 0.0;
            // plausibility check (a warning in the reference); POS_ holds the trial values
            for (int i = 0; i < n; i++) POS_(i) = (double)V_(i);
            for (int i = 0; i < n; i++)
                for (int j = i + 1; j < n; j++)
                {
                    const double w = PV_(pair_pos(i, j, n));
                    if (w != 0.0) { POS_(i) += w * dt; POS_(j) += -w * dt; }
                }
            for (int i = 0; i < n; i++)
            {
                const double c = POS_(i);
                if (c < -(double)FLT_EPSILON || c > 1.0 + (double)FLT_EPSILON) st |= kStNormalizeWarn;
            }
        }
    }
    // ---- 5. merge (accumulated in FP64, NEG_ holds the new values) and finalize -----------------
    for (int i = 0; i < n; i++) NEG_(i) = (double)V_(i);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
        {
            const double value = 1.0 * (PV_(pair_pos(i, j, n)) + 0.0) * dt;
            if (fabs(value) >= DBL_EPSILON)
            {
                NEG_(i) += value;
                NEG_(j) += -value;
            }
        }
    const double hi_snap = 1.0 - p.eps_snap;
    const double lo_snap = 0.0 + p.eps_snap;
    double total = 0.0;
    int m = 0;
    for (int i = 0; i < n; i++)
    {
        double w = NEG_(i);
        bool erase = false;
        if (w >= hi_snap) w = 1.0;
        if (w <= lo_snap) { w = 0.0; erase = true; }
        total += w;
        if (!erase)
        {
            G_(m) = G_(i);
            NEG_(m) = w;
            m++;
        }
    }
    if (m > 1)
    {
        const double norm = 1.0 / total;
        for (int i = 0; i < m; i++) V_(i) = (R)(NEG_(i) * norm);
    }
    else if (m == 1)
    {
        V_(0) = R(1);
    }
    else
    {
        st |= kStEmptyVoxel;
    }
    for (int i = 0; i < m; i++)
        if (!isfinite((double)V_(i))) st |= kStNonFinite;
#undef G_
#undef V_
#undef L_
#undef SG_
#undef PV_
#undef POS_
#undef NEG_
    return m;
}

// Periodic neighbour offsets of voxel v: X[i] + Y[j] + Z[k] is the voxel at (x+i-1, y+j-1, z+k-1).
struct Neighbourhood {
    long long X[3], Y[3], Z[3];
    __device__ __forceinline__ Neighbourhood(const StepParams& p, long long v)
    {
        const int nx = p.nx, ny = p.ny, nz = p.nz;
        const int z = (int)(v % nz);
        const long long t = v / nz;
        const int y = (int)(t % ny);
        const int x = (int)(t / ny);
        const long long plane = (long long)ny * nz;
        X[0] = (long long)(x == 0 ? nx - 1 : x - 1) * plane; X[1] = (long long)x * plane;
        X[2] = (long long)(x == nx - 1 ? 0 : x + 1) * plane;
        Y[0] = (long long)(y == 0 ? ny - 1 : y - 1) * nz; Y[1] = (long long)y * nz;
        Y[2] = (long long)(y == ny - 1 ? 0 : y + 1) * nz;
        Z[0] = (z == 0 ? nz - 1 : z - 1); Z[1] = z; Z[2] = (z == nz - 1 ? 0 : z + 1);
    }
    __device__ __forceinline__ long long at(int dx, int dy, int dz) const { return X[dx + 1] + Y[dy + 1] + Z[dz + 1]; }
};

// Flag of voxel v from the neighbour counts (PhaseField::SetFlagsSR, src/PhaseField.cpp:953-969).
__device__ __forceinline__ int voxel_flag(const uint8_t* cnt, const Neighbourhood& nb, long long v)
{
    const int c = cnt[v];
    if (c > 1) return 2;
    for (int q = 0; q < 27; q++)
        if (cnt[nb.X[q / 9] + nb.Y[(q / 3) % 3] + nb.Z[q % 3]] > 1) return 1;
    return 0;
}

// Stage 1 for one voxel from global memory: own fields (stored order), then the candidates in
// the order CalculateDerivativesSR appends them (Laplacian stencil order and neighbour-list order,
// then the gradient pass), each with its Laplacian summed in stencil order.  Returns the list
// length (capacity KL; a longer list raises kStOverflowList).
template <class R, int KL>
__device__ __forceinline__ int gather_list(const StepParams& p, const uint8_t* __restrict__ cnt,
                                           const int16_t* __restrict__ gin, const R* __restrict__ vin,
                                           const Neighbourhood& nb, long long v, int16_t* gL, R* val, R* lap,
                                           R* grad, uint32_t& st)
{
    const long long N = p.n;
    const int c = cnt[v];
    if (c > KL)
    {
        // more stored fields than the list holds: nothing is written; the caller defers or reports
        st |= kStOverflowList;
        return 0;
    }
    int n = 0;
    for (int s = 0; s < c; s++)
    {
        gL[n] = gin[s * N + v];
        val[n] = vin[s * N + v];
        lap[n] = R(0);
        n++;
    }
    for (int q = 0; q < p.ns; q++)
    {
        const long long u = nb.at(p.lap_d[q][0], p.lap_d[q][1], p.lap_d[q][2]);
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
                else if (n < KL) { gL[n] = (int16_t)g; val[n] = R(0); lap[n] = l; n++; }
                else st |= kStOverflowList;
            }
        }
    }
    // the gradient pass of CalculateDerivativesSR appends indices it meets first
    for (int q = 0; q < p.ng; q++)
    {
        const long long u = nb.at(p.grad_d[q][0], p.grad_d[q][1], p.grad_d[q][2]);
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
                    if (n < KL) { gL[n] = (int16_t)g; val[n] = R(0); lap[n] = R(0); n++; }
                    else st |= kStOverflowList;
                }
            }
        }
    }
    // gradients of every list entry (anisotropic energies only), summed in gradient-stencil order
    if (p.aniso && grad)
    {
        for (int k = 0; k < 3 * n; k++) grad[k] = R(0);
        for (int q = 0; q < p.ngs; q++)
        {
            const long long u = nb.at(p.gs_d[q][0], p.gs_d[q][1], p.gs_d[q][2]);
            const int cu = cnt[u];
            for (int s = 0; s < cu; s++)
            {
                const R phi = vin[s * N + u];
                if (phi != R(0))
                {
                    const int g = gin[s * N + u];
                    int f = 0;
                    while (f < n && gL[f] != g) f++;
                    if (f < n)
                    {
                        const R gx = (R)p.gs_w[q][0] * phi;
                        const R gy = (R)p.gs_w[q][1] * phi;
                        const R gz = (R)p.gs_w[q][2] * phi;
                        grad[3 * f] += gx;
                        grad[3 * f + 1] += gy;
                        grad[3 * f + 2] += gz;
                    }
                }
            }
        }
    }
    return n;
}

// One voxel of the step, reading its 3x3x3 neighbourhood straight from global memory, with its
// working arrays in local memory (capacity KL fields).  This is the general path: the full-grid
// kernel below and the overflow kernel of the tiled step (lists longer than the tiled kernel's
// capacity) both run it.
// ANISO: gradients for anisotropic energies.
template <class R, int KS, int KL, bool ANISO>
__device__ __forceinline__ void voxel_step_generic(const StepParams& p, const StepArrays& a, long long v,
                                                   int* s_key, double* s_sum, int nslots, unsigned& wide,
                                                   unsigned& ein, unsigned& eout, uint32_t& st, bool count_in)
{
    const long long N = p.n;
    const uint8_t* __restrict__ cnt = a.cnt_in;
    const int16_t* __restrict__ gin = a.idx_in;
    const R* __restrict__ vin = static_cast<const R*>(a.val_in);
    R* __restrict__ vout = static_cast<R*>(a.val_out);
    const Neighbourhood nb(p, v);

    const int c = cnt[v];
    if (count_in) ein = c;
    const int flag = voxel_flag(cnt, nb, v);

    if (flag == 0)
    {
        // bulk voxel: the state is carried over unchanged (no stage touches it)
        a.cnt_out[v] = (uint8_t)c;
        for (int s = 0; s < c; s++)
        {
            const int g = gin[s * N + v];
            const R phi = vin[s * N + v];
            a.idx_out[s * N + v] = (int16_t)g;
            vout[s * N + v] = phi;
            if (in_volume_window(p, v)) vol_insert_n(s_key, s_sum, nslots, a.vol_acc, g, (double)phi);
        }
        eout = c;
        return;
    }
    wide = 1;
    // ---- 1. own fields, then candidates, with Laplacians (stencil order) ------------------------
    constexpr int KP = KL * (KL - 1) / 2;
    int16_t gL[KL];
    R val[KL], lap[KL], sg[KP];
    double pv[KP], pos[KL], neg[KL];
    R grad[ANISO ? 3 * KL : 1];
    const int n = gather_list<R, KL>(p, cnt, gin, vin, nb, v, gL, val, lap, ANISO ? grad : nullptr, st);
    const ListScratch<R> sc{gL, val, lap, sg, pv, pos, neg, 1, ANISO ? grad : nullptr};
    int m = list_step<R>(p, a, sc, n, flag, st, v, (int)cnt[v]);
    if (m > KS) { st |= kStOverflowK; m = KS; }
    a.cnt_out[v] = (uint8_t)m;
    for (int i = 0; i < m; i++)
    {
        a.idx_out[i * N + v] = gL[i];
        vout[i * N + v] = val[i];
        if (in_volume_window(p, v)) vol_insert_n(s_key, s_sum, nslots, a.vol_acc, gL[i], (double)val[i]);
    }
    eout = m;
}

// Per-block totals of the counters and the grain-volume table, flushed to global memory.
__device__ __forceinline__ void flush_block(const StepArrays& a, unsigned wide, unsigned ein, unsigned eout,
                                            uint32_t st, unsigned long long* s_cnt, const int* keys,
                                            const double* sums, int nslots, int t, int nt)
{
    if (st) atomicOr(a.status, st);
    unsigned w = wide, ei = ein, eo = eout;
    for (int o = 16; o > 0; o >>= 1)
    {
        w += __shfl_down_sync(0xffffffffu, w, o);
        ei += __shfl_down_sync(0xffffffffu, ei, o);
        eo += __shfl_down_sync(0xffffffffu, eo, o);
    }
    if ((t & 31) == 0)
    {
        if (w) atomicAdd(&s_cnt[0], (unsigned long long)w);
        if (ei) atomicAdd(&s_cnt[1], (unsigned long long)ei);
        if (eo) atomicAdd(&s_cnt[2], (unsigned long long)eo);
    }
    if (st & (kStOverflowK | kStOverflowList)) atomicAdd(&a.counters[kCntOverflowVoxels], 1ull);
    __syncthreads();
    for (int i = t; i < nslots; i += nt)
        if (keys[i] >= 0) atomicAdd(&a.vol_acc[keys[i]], sums[i]);
    if (t < 3 && s_cnt[t])
        atomicAdd(&a.counters[t == 0 ? kCntWide : (t == 1 ? kCntEntriesIn : kCntEntriesOut)], s_cnt[t]);
}

template <class R, int KS, int KL, bool ANISO>
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
    if (v < p.n) voxel_step_generic<R, KS, KL, ANISO>(p, a, v, s_key, s_sum, kVolSlots, wide, ein, eout, st, true);
    flush_block(a, wide, ein, eout, st, s_cnt, s_key, s_sum, kVolSlots, threadIdx.x, blockDim.x);
}

template <class R>
int launch_step_generic(const StepParams& p, const StepArrays& a, int k_slots, void* stream)
{
    const int threads = 256;
    const long long blocks = (p.n + threads - 1) / threads;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (k_slots * 2 + (p.aniso ? 1 : 0))
    {
        case 16: step_kernel<R, 8, 16, false><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 17: step_kernel<R, 8, 16, true><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 24: step_kernel<R, 12, 20, false><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 25: step_kernel<R, 12, 20, true><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 32: step_kernel<R, 16, 24, false><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        case 33: step_kernel<R, 16, 24, true><<<(unsigned)blocks, threads, 0, s>>>(p, a); break;
        default: return -1;
    }
    return (int)cudaGetLastError();
}

}  // namespace opgpu
