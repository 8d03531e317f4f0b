/* TEST INFRASTRUCTURE ONLY — the oracle (see pf_oracle.h).
 *
 * A plain-C restatement of the OpenPhase single-resolution multiphase-field step.  Every function
 * below names the reference function it restates (paths relative to the OpenPhase source tree).
 * The operation order of every floating-point expression follows the reference statement by
 * statement, so that in IEEE double arithmetic without FMA contraction (built with
 * -ffp-contract=off) the results are bit-identical to the reference's own release build.
 *
 * Storage: one fixed-capacity list per voxel of (index, value, laplacian) entries, the analogue of
 * NodePF (include/Containers/NodePF.h:40-180).  The per-voxel increment store FieldsDot
 * (NodeAB<double,double>, include/Containers/NodeAB.h:38-180) lives in per-thread scratch,
 * because every stage between CalculatePhaseFieldIncrements and NodePF::finalize only reads and
 * writes the voxel's own lists; the grid-wide passes (flags, derivatives, volumes) run after the
 * per-voxel stages exactly as in PhaseField::FinalizeSR (src/PhaseField.cpp:1008-1033).
 */
#include "pf_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* include/Globals.h:124 */
static const double OP_PI = 3.14159265358979323846;

typedef struct { int32_t idx; double val; double lap; double grad[3]; } entry;
typedef struct { int a, b; double v1; int alive; } pair;

struct op_sim {
    op_params p;
    int* grain_phase;
    int* phase_solid;
    double *sigma_phase, *mu_phase, *limit_phase, *pair_sigma, *pair_mu, *dg;
    int* energy_model;            /* [P*P] OP_ENERGY_*                                           */
    double* cubic_eps;            /* [P*P] Epsilon1                                              */
    double* model_eps;            /* [P*P*3] Epsilon2..4                                         */
    double* facets;               /* FACETED rows: unit facet normal (3), SigmaF, EpsilonEF      */
    int* facet_lo; int* facet_hi; /* [P*P] rows of each pair                                     */
    int* mfacet_lo; int* mfacet_hi;   /* [P*P] FACETED mobility rows (unit normal, MuF, EpsilonMF) */
    double* phase_e; double* phase_maxe;   /* [P*P] FACETED Energy (mean SigmaF), MaxEnergy      */
    int* mobility_model;          /* [P*P]                                                       */
    double* mobility_eps;         /* [P*P*4]                                                     */
    double* rot;                  /* [G*9] grain RotationMatrix, row-major                       */
    double* quat;                 /* [G*4] grain Orientation (s, x, y, z) as given               */
    int aniso;                    /* some phase pair uses an anisotropic energy model            */
    long n;
    int cap;
    int32_t* cnt;   entry* e;     /* Fields                                */
    int32_t* cnt2;  entry* e2;    /* tmpFields of CalculateDerivativesSR   */
    int8_t* flag;
    double *volume, *max_volume, *ref_volume, *vr;
    int32_t *exist, *stage;
    int ns; int sdi[27], sdj[27], sdk[27]; double sw[27];
    int ng; int gdi[27], gdj[27], gdk[27]; double gw[27][3];
    uint32_t status;
    /* driving-force averaging: per interface voxel, per pair of its positive entries (a < b in
     * list order) the intermediate (tmp) and averaged driving force; npos[v] positive entries */
    double *df_tmp, *df_avg;
    int32_t* npos;
    int maxpp;
};

static double dmax(double a, double b) { return (a < b) ? b : a; }   /* std::max */

/* The facet vectors a FACETED facet (h, k, l) stands for: itself, or with facet families every
 * distinct vector of its family (index permutations with sign changes, the set
 * Tools::findIndexPermutations enumerates, src/Tools.cpp:37-260).  Returns their number (<= 48). */
static int facet_family_vectors(long h, long k, long l, int family, long w[48][3])
{
    if (!family) { w[0][0] = h; w[0][1] = k; w[0][2] = l; return 1; }
    const long a[3] = {labs(h), labs(k), labs(l)};
    static const int perm[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};
    int n = 0;
    for (int pm = 0; pm < 6; pm++)
    for (int sg = 0; sg < 8; sg++)
    {
        const long v0 = a[perm[pm][0]]*((sg & 1) ? -1 : 1);
        const long v1 = a[perm[pm][1]]*((sg & 2) ? -1 : 1);
        const long v2 = a[perm[pm][2]]*((sg & 4) ? -1 : 1);
        int dup = 0;
        for (int i = 0; i < n; i++) dup |= (w[i][0] == v0 && w[i][1] == v1 && w[i][2] == v2);
        if (!dup) { w[n][0] = v0; w[n][1] = v1; w[n][2] = v2; n++; }
    }
    return n;
}
static double dmin(double a, double b) { return (b < a) ? b : a; }   /* std::min */

/* Append the normalised facet vectors of facet row d (h, k, l, c1, c2) to the row table, each with
 * the row's two values; iVector3::normalized (include/Containers/iVector3.h:274-289). */
static void append_facet(double** rows_p, int* rows, int* cap_rows, const double* d, int family)
{
    long w[48][3];
    const int nw = facet_family_vectors(lround(d[0]), lround(d[1]), lround(d[2]), family, w);
    if (*rows + nw > *cap_rows)
    {
        *cap_rows = 2*(*rows + nw);
        *rows_p = (double*)realloc(*rows_p, (size_t)(*cap_rows)*5*sizeof(double));
    }
    for (int k = 0; k < nw; k++)
    {
        double* r = *rows_p + 5*(size_t)(*rows)++;
        const double norm = sqrt((double)(w[k][0]*w[k][0] + w[k][1]*w[k][1] + w[k][2]*w[k][2]));
        if (norm != 0.0)
        {
            const double inv = 1.0/norm;
            r[0] = w[k][0]*inv; r[1] = w[k][1]*inv; r[2] = w[k][2]*inv;
        }
        else { r[0] = 0.0; r[1] = 0.0; r[2] = 0.0; }
        r[3] = d[3]; r[4] = d[4];
    }
}

static double* dup_d(const double* src, size_t n)
{
    if (!src) return NULL;
    double* d = (double*)malloc(n * sizeof(double));
    memcpy(d, src, n * sizeof(double));
    return d;
}

/* LaplacianStencil::Set (include/Containers/LaplacianStencil.h:197-219) over the 3-D tables
 * LaplacianStencil3D_7 (:72-82), LaplacianStencil3D_27a (:109-119), LaplacianStencil3D_LB
 * (:146-156): elements in x, y, z loop order, zero weights skipped, weight = table/(dx*dx). */
static void set_stencil(op_sim* s)
{
    double t[3][3][3];
    const int st = s->p.stencil;
    for (int x = 0; x < 3; x++)
    for (int y = 0; y < 3; y++)
    for (int z = 0; z < 3; z++)
    {
        const int d = (x != 1) + (y != 1) + (z != 1);
        double w = 0.0;
        if (st == OP_STENCIL_SIMPLE)
            w = (d == 0) ? -6.0 : (d == 1 ? 1.0 : 0.0);
        else if (st == OP_STENCIL_ISOTROPIC)
            w = (d == 0) ? -64.0/15.0 : (d == 1 ? 7.0/15.0 : (d == 2 ? 1.0/10.0 : 1.0/30.0));
        else
            w = (d == 0) ? -38.0/9.0 : (d == 1 ? 4.0/9.0 : (d == 2 ? 1.0/9.0 : 1.0/36.0));
        t[x][y][z] = w;
    }
    s->ns = 0;
    for (int x = -1; x <= 1; ++x)
    for (int y = -1; y <= 1; ++y)
    for (int z = -1; z <= 1; ++z)
    if (t[x+1][y+1][z+1] != 0.0)
    {
        s->sdi[s->ns] = x; s->sdj[s->ns] = y; s->sdk[s->ns] = z;
        s->sw[s->ns] = t[x+1][y+1][z+1]/(s->p.dx*s->p.dx);
        s->ns++;
    }
    /* GradientStencil::Set (include/Containers/GradientStencil.h:132-155) over GradientStencil1D
     * (:46-56), GradientStencil3D (:82-92) and GradientStencil3D_LB (:108-118):
     * weight_c = c*table/dx. */
    const int gs = s->p.gradient_stencil;
    for (int x = 0; x < 3; x++)
    for (int y = 0; y < 3; y++)
    for (int z = 0; z < 3; z++)
    {
        const int d = (x != 1) + (y != 1) + (z != 1);
        double w = 0.0;
        if (gs == OP_STENCIL_SIMPLE)
            w = (d == 1) ? 0.5 : 0.0;
        else if (gs == OP_STENCIL_ISOTROPIC)
            w = (d == 0) ? 0.0 : (d == 1 ? 1.0/4.64 : (d == 2 ? 0.245/4.64 : 0.085/4.64));
        else
            w = (d == 0) ? 0.0 : (d == 1 ? 2.0/9.0 : (d == 2 ? 1.0/18.0 : 1.0/72.0));
        t[x][y][z] = w;
    }
    s->ng = 0;
    for (int x = -1; x <= 1; ++x)
    for (int y = -1; y <= 1; ++y)
    for (int z = -1; z <= 1; ++z)
    if (t[x+1][y+1][z+1] != 0.0)
    {
        s->gdi[s->ng] = x; s->gdj[s->ng] = y; s->gdk[s->ng] = z;
        s->gw[s->ng][0] = x*t[x+1][y+1][z+1]/s->p.dx;
        s->gw[s->ng][1] = y*t[x+1][y+1][z+1]/s->p.dx;
        s->gw[s->ng][2] = z*t[x+1][y+1][z+1]/s->p.dx;
        s->ng++;
    }
}

op_sim* op_create(const op_params* p, int cap)
{
    if (cap < 2 || cap > 64) return NULL;
    op_sim* s = (op_sim*)calloc(1, sizeof(op_sim));
    s->p = *p;
    const int G = p->ngrains, P = p->nphases;
    s->grain_phase = (int*)malloc(G * sizeof(int));
    for (int g = 0; g < G; g++) s->grain_phase[g] = p->grain_phase ? p->grain_phase[g] : 0;
    s->phase_solid = (int*)malloc(P * sizeof(int));
    for (int q = 0; q < P; q++) s->phase_solid[q] = p->phase_solid ? p->phase_solid[q] : 1;
    s->sigma_phase = dup_d(p->sigma_phase, (size_t)P*P);
    s->mu_phase    = dup_d(p->mu_phase, (size_t)P*P);
    s->limit_phase = dup_d(p->limit_phase, (size_t)P*P);
    s->pair_sigma  = dup_d(p->pair_sigma, (size_t)G*G);
    s->pair_mu     = dup_d(p->pair_mu, (size_t)G*G);
    s->dg          = dup_d(p->dg, (size_t)G);
    s->p.grain_phase = s->grain_phase; s->p.phase_solid = s->phase_solid;
    s->p.sigma_phase = s->sigma_phase; s->p.mu_phase = s->mu_phase; s->p.limit_phase = s->limit_phase;
    s->p.pair_sigma = s->pair_sigma; s->p.pair_mu = s->pair_mu; s->p.dg = s->dg;
    s->energy_model = (int*)calloc((size_t)P*P, sizeof(int));
    s->cubic_eps = (double*)calloc((size_t)P*P, sizeof(double));
    s->model_eps = (double*)calloc((size_t)P*P*3, sizeof(double));
    s->mobility_model = (int*)calloc((size_t)P*P, sizeof(int));
    s->mobility_eps = (double*)calloc((size_t)P*P*4, sizeof(double));
    for (int q = 0; q < P*P; q++)
    {
        if (p->mobility_model) s->mobility_model[q] = p->mobility_model[q];
        if (p->mobility_eps) for (int k = 0; k < 4; k++) s->mobility_eps[4*q + k] = p->mobility_eps[4*q + k];
        if (s->mobility_model[q] != OP_ENERGY_ISO) s->aniso = 1;
    }
    if (p->model_eps) memcpy(s->model_eps, p->model_eps, (size_t)P*P*3*sizeof(double));
    /* ReadInputFaceted (InterfaceEnergyModel.h:196-246): facet normals (families expanded), Energy
     * = mean SigmaF accumulated in facet order, MaxEnergy = max SigmaF.  ReadInputFacetedEXP
     * (:248-295): the same rows with EpsilonEF and PowerEF; Energy = MaxEnergy = $Sigma.  The
     * FACETED mobility (InterfaceMobilityModel.h:165-208): rows with MuF and EpsilonMF. */
    s->facet_lo = (int*)calloc((size_t)P*P, sizeof(int));
    s->facet_hi = (int*)calloc((size_t)P*P, sizeof(int));
    s->mfacet_lo = (int*)calloc((size_t)P*P, sizeof(int));
    s->mfacet_hi = (int*)calloc((size_t)P*P, sizeof(int));
    s->phase_e = (double*)calloc((size_t)P*P, sizeof(double));
    s->phase_maxe = (double*)calloc((size_t)P*P, sizeof(double));
    s->facets = NULL;
    {
        int rows = 0, cap_rows = 0;
        for (int q = 0; q < P*P; q++)
        {
            const int em = p->energy_model ? p->energy_model[q] : 0;
            if ((em != OP_ENERGY_FACETED && em != OP_ENERGY_FACETEDEXP) || !p->facet_start) continue;
            const int n0 = p->facet_start[q], n1 = p->facet_start[q + 1], nf = n1 - n0;
            const int family = p->facet_family ? p->facet_family[q] : 0;
            double energy = 0.0, maxe = 0.0;
            s->facet_lo[q] = rows;
            for (int f = n0; f < n1; f++)
            {
                const double* d = p->facet_data + 5*(size_t)f;
                append_facet(&s->facets, &rows, &cap_rows, d, family);
                energy += d[3]/nf;
                if (d[3] > maxe) maxe = d[3];
            }
            s->facet_hi[q] = rows;
            if (em == OP_ENERGY_FACETED) { s->phase_e[q] = energy; s->phase_maxe[q] = maxe; }
        }
        for (int q = 0; q < P*P; q++)
        {
            const int mm = p->mobility_model ? p->mobility_model[q] : 0;
            if (mm != OP_MOBILITY_FACETED || !p->mobility_facet_start) continue;
            const int family = p->mobility_facet_family ? p->mobility_facet_family[q] : 0;
            s->mfacet_lo[q] = rows;
            for (int f = p->mobility_facet_start[q]; f < p->mobility_facet_start[q + 1]; f++)
                append_facet(&s->facets, &rows, &cap_rows, p->mobility_facet_data + 5*(size_t)f, family);
            s->mfacet_hi[q] = rows;
        }
    }
    s->aniso = 0;
    for (int q = 0; q < P*P; q++)
    {
        if (p->energy_model) s->energy_model[q] = p->energy_model[q];
        if (p->cubic_eps) s->cubic_eps[q] = p->cubic_eps[q];
        if (s->energy_model[q] != OP_ENERGY_ISO) s->aniso = 1;
    }
    /* Quaternion::setRotationMatrix (src/Containers/Quaternion.cpp:78-98) of each grain's
     * orientation, normalised as Quaternion::normalized (include/Containers/Quaternion.h:304-311);
     * unit rotation without orientations. */
    s->rot = (double*)calloc((size_t)G*9, sizeof(double));
    s->quat = (double*)malloc((size_t)G*4*sizeof(double));
    for (int g = 0; g < G; g++)
    {
        s->quat[4*g]     = p->quat ? p->quat[4*g]     : 1.0;
        s->quat[4*g + 1] = p->quat ? p->quat[4*g + 1] : 0.0;
        s->quat[4*g + 2] = p->quat ? p->quat[4*g + 2] : 0.0;
        s->quat[4*g + 3] = p->quat ? p->quat[4*g + 3] : 0.0;
    }
    for (int g = 0; g < G; g++)
    {
        double* R = s->rot + 9*g;
        const double qs = p->quat ? p->quat[4*g] : 1.0;
        const double q0 = p->quat ? p->quat[4*g + 1] : 0.0;
        const double q1 = p->quat ? p->quat[4*g + 2] : 0.0;
        const double q2 = p->quat ? p->quat[4*g + 3] : 0.0;
        const double len = sqrt(qs*qs + q0*q0 + q1*q1 + q2*q2);
        if (len < DBL_EPSILON)
        {
            R[0] = 1.0; R[4] = 1.0; R[8] = 1.0;
            continue;
        }
        const double S = qs/len, V0 = q0/len, V1 = q1/len, V2 = q2/len;
        R[0] = 1.0 - 2.0*(V1*V1 + V2*V2);
        R[1] =       2.0*(V0*V1 -  S*V2);
        R[2] =       2.0*(V0*V2 +  S*V1);
        R[3] =       2.0*(V0*V1 +  S*V2);
        R[4] = 1.0 - 2.0*(V0*V0 + V2*V2);
        R[5] =       2.0*(V1*V2 -  S*V0);
        R[6] =       2.0*(V0*V2 -  S*V1);
        R[7] =       2.0*(V1*V2 +  S*V0);
        R[8] = 1.0 - 2.0*(V0*V0 + V1*V1);
    }
    s->p.energy_model = s->energy_model; s->p.cubic_eps = s->cubic_eps; s->p.model_eps = s->model_eps;
    s->p.quat = NULL;
    if (s->p.nucleus_volume_factor == 0.0) s->p.nucleus_volume_factor = 1.0;
    s->n = (long)p->nx * p->ny * p->nz;
    s->cap = cap;
    s->cnt  = (int32_t*)calloc(s->n, sizeof(int32_t));
    s->cnt2 = (int32_t*)calloc(s->n, sizeof(int32_t));
    s->e  = (entry*)calloc((size_t)s->n * cap, sizeof(entry));
    s->e2 = (entry*)calloc((size_t)s->n * cap, sizeof(entry));
    s->flag = (int8_t*)calloc(s->n, 1);
    s->volume = (double*)calloc(G, sizeof(double));
    s->max_volume = (double*)calloc(G, sizeof(double));
    s->ref_volume = (double*)calloc(G, sizeof(double));
    s->vr = (double*)calloc(G, sizeof(double));
    s->npos = (int32_t*)calloc((size_t)s->n, sizeof(int32_t));
    s->exist = (int32_t*)calloc(G, sizeof(int32_t));
    s->stage = (int32_t*)calloc(G, sizeof(int32_t));
    /* PhaseField::AddGrainInfo (src/PhaseField.cpp:2970-2979) on a fresh Grain
     * (include/GrainsProperties.h:312-336, add_grain :708-730), and
     * PhaseField::CalculateReferenceVolume (src/PhaseField.cpp:367-391) in 3-D. */
    const double r = p->iwidth;
    const double ref = (4.0/3.0)*OP_PI*r*r*r*s->p.nucleus_volume_factor;
    for (int g = 0; g < G; g++)
    {
        s->exist[g] = 1; s->stage[g] = OP_STAGE_STABLE;
        s->ref_volume[g] = ref; s->vr[g] = 0.0;
    }
    set_stencil(s);
    if (p->threads > 0) omp_set_num_threads(p->threads);
    return s;
}

void op_destroy(op_sim* s)
{
    if (!s) return;
    free(s->grain_phase); free(s->phase_solid);
    free(s->sigma_phase); free(s->mu_phase); free(s->limit_phase);
    free(s->pair_sigma); free(s->pair_mu); free(s->dg);
    free(s->energy_model); free(s->cubic_eps); free(s->model_eps); free(s->rot); free(s->quat);
    free(s->facets); free(s->facet_lo); free(s->facet_hi); free(s->phase_e); free(s->phase_maxe);
    free(s->mfacet_lo); free(s->mfacet_hi);
    free(s->mobility_model); free(s->mobility_eps);
    free(s->cnt); free(s->cnt2); free(s->e); free(s->e2); free(s->flag);
    free(s->volume); free(s->max_volume); free(s->ref_volume); free(s->vr);
    free(s->npos); free(s->df_tmp); free(s->df_avg);
    free(s->exist); free(s->stage);
    free(s);
}

static long vox(const op_sim* s, int i, int j, int k)
{
    /* periodic wrap; storage order of Storage3D (include/Containers/Storage3D.h:2054-2064):
     * x slowest, z fastest */
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    i = (i + nx) % nx; j = (j + ny) % ny; k = (k + nz) % nz;
    return ((long)i * ny + j) * nz + k;
}

/* NodePF::read (include/Containers/NodePF.h:751-763): flag 2 when more than one entry. */
int op_load(op_sim* s, const int32_t* counts, const int32_t* idx, const double* val)
{
    long off = 0;
    for (long v = 0; v < s->n; v++)
    {
        const int c = counts[v];
        if (c > s->cap) return -1;
        s->cnt[v] = c;
        s->flag[v] = (c > 1) ? 2 : 0;
        for (int q = 0; q < c; q++)
        {
            s->e[v*s->cap + q].idx = idx[off + q];
            s->e[v*s->cap + q].val = val[off + q];
            s->e[v*s->cap + q].lap = 0.0;
            s->e[v*s->cap + q].grad[0] = 0.0;
            s->e[v*s->cap + q].grad[1] = 0.0;
            s->e[v*s->cap + q].grad[2] = 0.0;
        }
        off += c;
    }
    return 0;
}

/* ---------------- interface properties (InterfaceProperties::SetSR, src/InterfaceProperties.cpp:603-762)
 * ISO energy model (:617-620) and ISO mobility (:677-680, MaxMobility = Mobility); a per-grain-pair
 * table replaces the per-voxel values the way the oracle driver writes them into IP.Properties. */
static double ip_energy(const op_sim* s, int ga, int gb)
{
    if (s->pair_sigma) return s->pair_sigma[(size_t)ga*s->p.ngrains + gb];
    const int P = s->p.nphases;
    return s->sigma_phase[s->grain_phase[ga]*P + s->grain_phase[gb]];
}
static double ip_mobility(const op_sim* s, int ga, int gb)
{
    if (s->pair_mu) return s->pair_mu[(size_t)ga*s->p.ngrains + gb];
    const int P = s->p.nphases;
    return s->mu_phase[s->grain_phase[ga]*P + s->grain_phase[gb]];
}
/* InterfaceEnergyModel::Energy of a phase pair; the DISORIENTATION model reads no $Sigma and keeps
 * the constructor's 0 (include/InterfaceProperties/InterfaceEnergyModel.h:63-70, 303-306). */
static double phase_energy(const op_sim* s, int pa, int pb)
{
    const int q = pa*s->p.nphases + pb;
    if (s->energy_model[q] == OP_ENERGY_DISORIENTATION) return 0.0;
    if (s->energy_model[q] == OP_ENERGY_FACETED) return s->phase_e[q];
    return s->sigma_phase[q];
}

/* InterfaceEnergyModel::MaxEnergy of a phase pair: Energy for ISO (ReadInputIso), Energy*(1 +
 * Epsilon1*1.41) for CUBIC (ReadInputCubic, include/InterfaceProperties/InterfaceEnergyModel.h:78-94). */
static double phase_max_energy(const op_sim* s, int pa, int pb)
{
    const int q = pa*s->p.nphases + pb;
    if (s->energy_model[q] == OP_ENERGY_CUBIC) return s->sigma_phase[q]*(1.0 + s->cubic_eps[q]*1.41);
    if (s->energy_model[q] == OP_ENERGY_DISORIENTATION) return 0.0;   /* MaxEnergy keeps its 0 */
    if (s->energy_model[q] == OP_ENERGY_FACETED) return s->phase_maxe[q];
    return s->sigma_phase[q];
}

/* Tools::getDisorientationCubic (src/Tools.cpp:626-678): the rotation angle 2*acos(max |c|) of
 * dQ = A * B.inverted() over the 24 combinations c of its components (Grimmer 1974), with the
 * reference's factors 0.707 and 0.5.  Quaternion product and inverse as
 * include/Containers/Quaternion.h:257-266, 313-339 (component 0 = s). */
static double disorientation_cubic(const double* A, const double* B)
{
    const double bs = B[0], bx = B[1], by = B[2], bz = B[3];
    const double n2 = bs*bs + (bx*bx + by*by + bz*bz);
    const double is = bs/n2, ix = (bx*(-1.0))/n2, iy = (by*(-1.0))/n2, iz = (bz*(-1.0))/n2;
    const double as = A[0], ax = A[1], ay = A[2], az = A[3];
    double d[4];
    d[1] =  ax*is + ay*iz - az*iy + as*ix;
    d[2] = -ax*iz + ay*is + az*ix + as*iy;
    d[3] =  ax*iy - ay*ix + az*is + as*iz;
    d[0] = -ax*ix - ay*iy - az*iz + as*is;
    double c[24];
    c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
    c[4]  = (d[0] + d[1])*0.707; c[5]  = (d[0] - d[1])*0.707;
    c[6]  = (d[2] + d[3])*0.707; c[7]  = (d[2] - d[3])*0.707;
    c[8]  = (d[0] + d[2])*0.707; c[9]  = (d[0] - d[2])*0.707;
    c[10] = (d[1] + d[3])*0.707; c[11] = (d[1] - d[3])*0.707;
    c[12] = (d[0] + d[3])*0.707; c[13] = (d[0] - d[3])*0.707;
    c[14] = (d[1] + d[2])*0.707; c[15] = (d[1] - d[2])*0.707;
    c[16] = (d[0] + d[1] + d[2] + d[3])*0.5;
    c[17] = (d[0] + d[1] - d[2] - d[3])*0.5;
    c[18] = (d[0] - d[1] + d[2] - d[3])*0.5;
    c[19] = (d[0] - d[1] - d[2] + d[3])*0.5;
    c[20] = (d[0] + d[1] + d[2] - d[3])*0.5;
    c[21] = (d[0] + d[1] - d[2] + d[3])*0.5;
    c[22] = (d[0] - d[1] + d[2] + d[3])*0.5;
    c[23] = (d[0] - d[1] - d[2] - d[3])*0.5;
    double m = 0.0;
    for (int k = 0; k < 24; k++)
        if (m < fabs(c[k])) m = fabs(c[k]);
    return 2*acos(m);
}

/* InterfaceEnergyModel::CalculateDisorientation (InterfaceEnergyModel.h:308-323): a
 * Read-Shockley-type energy of the disorientation angle, constant above 0.349066 rad. */
static double disorientation_energy(const double* A, const double* B)
{
    const double constant = 0.85;
    const double mis = disorientation_cubic(A, B);
    if (mis <= 0.349066) return mis*constant*(0.8 - log(mis));
    return 0.349066*constant*(0.8 - log(0.349066));
}

/* InterfaceOrientation (src/InterfaceProperties.cpp:39-45): the normal -grad(phi) normalised
 * (dVector3::normalize, include/Containers/dVector3.h:301-316) and rotated back to the grain's
 * reference frame with the transposed RotationMatrix (MatrixVectorOperators.h:43-52). */
static void interface_orientation(const op_sim* s, const entry* e, double out[3])
{
    double n[3] = {e->grad[0]*(-1.0), e->grad[1]*(-1.0), e->grad[2]*(-1.0)};
    const double norm = sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
    if (norm > DBL_EPSILON)
    {
        const double inv = 1.0/norm;
        n[0] *= inv; n[1] *= inv; n[2] *= inv;
    }
    else
    {
        n[0] = 0.0; n[1] = 0.0; n[2] = 0.0;
    }
    const double* R = s->rot + 9*e->idx;
    for (int i = 0; i < 3; i++)
    {
        double t = 0.0;
        for (int j = 0; j < 3; j++) t += R[3*j + i]*n[j];
        out[i] = t;
    }
}

/* InterfaceEnergyModel::Calculate (InterfaceEnergyModel.h:325-399) of the normal n for the phase
 * pair q: CUBIC, HEXBOETTGER, HEXSUN, HEXYANG, each expression in the reference's operation order. */
static double model_energy(const op_sim* s, int q, const double n[3])
{
    const double E = s->sigma_phase[q], e1 = s->cubic_eps[q];
    const double* ex = s->model_eps + 3*q;
    const double x = n[0], y = n[1], z = n[2];
    switch (s->energy_model[q])
    {
        case OP_ENERGY_HEXBOETTGER:
            return E*(1.0 - e1*(pow(x, 6) - pow(y, 6) - 15.0*pow(x, 4)*y*y + 15.0*pow(y, 4)*x*x
                                + (5.0*pow(z, 4) - 5.0*pow(z, 2) + pow(z, 6))));
        case OP_ENERGY_HEXSUN:
            return E*(1.0 + e1*sqrt(5.0/16.0/OP_PI)*(3.0*z*z - 1.0)
                      + ex[0]*3.0/16.0/sqrt(OP_PI)*(35.0*pow(z, 4) - 30.0*z*z + 3.0)
                      + ex[1]*sqrt(13.0/OP_PI)/32.0*(231.0*pow(z, 6) - 315.0*pow(z, 4) + 105.0*z*z - 5.0)
                      + ex[2]*sqrt(6006.0/OP_PI)/64.0*(pow(x, 6) - 15.0*pow(x, 4)*y*y + 15.0*x*x*pow(y, 4) - pow(y, 6)));
        case OP_ENERGY_FACETED:
        {
            /* InterfaceEnergyModel::Calculate, Faceted (:417-438): the facet of largest cos^2 */
            double cos2 = 0.0, ea = 0.0, epa = 0.0;
            for (int f = s->facet_lo[q]; f < s->facet_hi[q]; f++)
            {
                const double* r = s->facets + 5*f;
                const double c = x*r[0] + y*r[1] + z*r[2];
                const double c2 = c*c;
                if (c2 > cos2) { cos2 = c2; ea = r[3]; epa = r[4]; }
            }
            const double sin2 = 1.0 - cos2;
            return ea*epa*epa*pow(sqrt(sin2 + epa*epa*cos2), -3.0);
        }
        case OP_ENERGY_FACETEDEXP:
        {
            /* InterfaceEnergyModel::Calculate, FacetedEXP (:389-413): every facet with cos > 0
             * subtracts E*eps*cos^p and adds E*eps*p*cos^p */
            double loc = E;
            for (int f = s->facet_lo[q]; f < s->facet_hi[q]; f++)
            {
                const double* r = s->facets + 5*f;
                const double c = x*r[0] + y*r[1] + z*r[2];
                if (c > 0.0)
                {
                    loc -= E*r[3]*pow(c, r[4]);
                    loc += E*r[3]*r[4]*pow(c, r[4]);
                }
            }
            return loc;
        }
        case OP_ENERGY_HEXYANG:
            return E*(1.0 + e1*pow((3.0*z*z - 1.0), 2) + ex[0]*pow((x*x*x - 3.0*x*y*y), 2)*pow((9.0*z*z - 1.0 + ex[1]), 2));
        default:   /* CUBIC */
            return E*(1.0 + e1*(1.5 - 2.5*(pow(x, 4) + pow(y, 4) + pow(z, 4))));
    }
}

/* The energy InterfaceProperties::SetSR (src/InterfaceProperties.cpp:617-673) stores for the pair of
 * list entries a, b of one voxel: ISO (or the per-grain-pair table) as ip_energy; an anisotropic
 * model averages the model energy of each solid grain's interface orientation, weighted by
 * |phi(1 - phi)|, falling back to MaxEnergy when neither weight exceeds DBL_EPSILON. */
static double voxel_energy(const op_sim* s, const entry* L, int a, int b)
{
    const int ga = L[a].idx, gb = L[b].idx;
    const int pA = s->grain_phase[ga], pB = s->grain_phase[gb];
    const int q = pA*s->p.nphases + pB;
    if (s->energy_model[q] == OP_ENERGY_ISO) return ip_energy(s, ga, gb);
    if (s->energy_model[q] == OP_ENERGY_DISORIENTATION)   /* InterfaceProperties.cpp:629-634 */
        return disorientation_energy(s->quat + 4*ga, s->quat + 4*gb);
    double loc = 0.0, wA = 0.0, wB = 0.0;
    if (s->phase_solid[pA])
    {
        wA = fabs(L[a].val*(1.0 - L[a].val));
        if (wA > DBL_EPSILON)
        {
            double n[3];
            interface_orientation(s, &L[a], n);
            loc += model_energy(s, q, n)*wA;
        }
        else wA = 0.0;
    }
    if (s->phase_solid[pB])
    {
        wB = fabs(L[b].val*(1.0 - L[b].val));
        if (wB > DBL_EPSILON)
        {
            double n[3];
            interface_orientation(s, &L[b], n);
            loc += model_energy(s, q, n)*wB;
        }
        else wB = 0.0;
    }
    if (wA + wB > DBL_EPSILON) loc /= wA + wB;
    else loc = phase_max_energy(s, pA, pB);
    return loc;
}

/* InterfaceMobilityModel::Calculate (include/InterfaceProperties/InterfaceMobilityModel.h:210-265)
 * for CUBIC, HEXBOETTGER, HEXSUN, HEXYANG, in the reference's operation order. */
static double mobility_model(const op_sim* s, int q, const double n[3])
{
    const double M = s->mu_phase[q];
    const double* e = s->mobility_eps + 4*q;
    const double x = n[0], y = n[1], z = n[2];
    switch (s->mobility_model[q])
    {
        case OP_MOBILITY_FACETED:
        {
            /* InterfaceMobilityModel::Calculate, Faceted (:266-288): the facet of smallest
             * inclination acos(n.f), the last one on ties */
            double incl = OP_PI, ma = 0.0, ea = 0.0;
            for (int f = s->mfacet_lo[q]; f < s->mfacet_hi[q]; f++)
            {
                const double* r = s->facets + 5*f;
                const double d = acos(x*r[0] + y*r[1] + z*r[2]);
                if (fabs(d) <= fabs(incl)) { incl = d; ma = r[3]; ea = r[4]; }
            }
            return ma*(ea + (1.0 - ea)*fabs(tan(incl))*tanh(pow(fabs(tan(incl)), -1.0)));
        }
        case OP_ENERGY_HEXBOETTGER:
            return M*(1.0 + e[0]*(pow(x, 6) - pow(y, 6) - 15.0*pow(x, 4)*y*y + 15.0*pow(y, 4)*x*x
                                  + (5.0*pow(z, 4) - 5.0*pow(z, 2) + pow(z, 6))));
        case OP_ENERGY_HEXSUN:
            return M*(1.0 - e[0]*sqrt(5.0/16.0/OP_PI)*(3.0*z*z - 1.0)
                      - e[1]*3.0/16.0/sqrt(OP_PI)*(35.0*pow(z, 4) - 30.0*z*z + 3.0)
                      - e[2]*sqrt(13.0/OP_PI)/32.0*(231.0*pow(z, 6) - 315.0*pow(z, 4) + 105.0*z*z - 5.0)
                      - e[3]*sqrt(6006.0/OP_PI)/64.0*(pow(x, 6) - 15.0*pow(x, 4)*y*y + 15.0*x*x*pow(y, 4) - pow(y, 6)));
        case OP_ENERGY_HEXYANG:
            return M*(1.0 - e[0]*pow((3.0*z*z - 1.0), 2) - e[1]*pow((x*x*x - 3.0*x*y*y), 2)*pow((9.0*z*z - 1.0 + e[2]), 2));
        default:   /* CUBIC */
            return M*(1.0 - e[0]*(1.5 - 2.5*(pow(x, 4) + pow(y, 4) + pow(z, 4))));
    }
}

/* The mobility InterfaceProperties::SetSR (src/InterfaceProperties.cpp:680-707) stores for the pair
 * of list entries a < b: ISO (or the per-grain-pair table) as ip_mobility; an anisotropic model is
 * summed over the solid grains whose value is neither 0 nor 1, Mobility when there is none. */
static double voxel_mobility(const op_sim* s, const entry* L, int a, int b)
{
    const int ga = L[a].idx, gb = L[b].idx;
    const int pA = s->grain_phase[ga], pB = s->grain_phase[gb];
    const int q = pA*s->p.nphases + pB;
    if (s->mobility_model[q] == OP_ENERGY_ISO) return ip_mobility(s, ga, gb);
    double loc = 0.0;
    int solids = 0;
    if (s->phase_solid[pA] && L[a].val != 0.0 && L[a].val != 1.0)
    {
        double n[3];
        interface_orientation(s, &L[a], n);
        loc += mobility_model(s, q, n);
        solids++;
    }
    if (s->phase_solid[pB] && L[b].val != 0.0 && L[b].val != 1.0)
    {
        double n[3];
        interface_orientation(s, &L[b], n);
        loc += mobility_model(s, q, n);
        solids++;
    }
    /* Mobility: $Mu, except the FACETED model, which reads none and keeps the constructor's 0
     * (InterfaceMobilityModel.h:51-56, 165-208) */
    if (solids == 0) loc = s->mobility_model[q] == OP_MOBILITY_FACETED ? 0.0 : s->mu_phase[q];
    return loc;
}

/* PhaseField::LocalN (include/PhaseField.h:84-95) */
static double local_n(const op_sim* s, const entry* L, int n)
{
    if (!s->p.consider_nucleus_volume) return (double)n;
    double norm = 0.0;
    for (int a = 0; a < n; a++) norm += s->vr[L[a].idx];
    return norm;
}

/* pair position for a < b in a list of n entries (DO creates the pairs in this order) */
static int pair_pos(int a, int b, int n)
{
    return a*(2*n - a - 1)/2 + (b - a - 1);
}

/* NodeAB::get_asym1 (include/Containers/NodeAB.h:517-531) for the list positions a != b. */
static double get_asym1(const pair* P, int a, int b, int n)
{
    if (a < b) { const pair* q = &P[pair_pos(a, b, n)]; return q->alive ? q->v1 : 0.0; }
    const pair* q = &P[pair_pos(b, a, n)];
    return q->alive ? q->v1*(-1.0) : 0.0;
}

/* DoubleObstacle::CalculatePhaseFieldIncrementsSR (src/DoubleObstacle.cpp:502-571), one voxel. */
static int do_increments(const op_sim* s, const entry* L, int n, pair* P)
{
    const double Eta = s->p.iwidth*s->p.dx;             /* src/GridParameters.cpp:256 */
    const double Prefactor = OP_PI*OP_PI/(Eta*Eta);
    const double norm_1 = 1.0/local_n(s, L, n);
    int np = 0;
    for (int a = 0; a < n; a++)
    for (int b = a + 1; b < n; b++)
    {
        const int ga = L[a].idx, gb = L[b].idx;
        const double scale = sqrt(s->vr[ga]*s->vr[gb]);
        double dPhi_dt = (s->aniso ? voxel_energy(s, L, a, b) : ip_energy(s, ga, gb))
                         *((L[a].lap + 0.5*(1.0 + scale)*Prefactor*L[a].val) -
                           (L[b].lap + 0.5*(1.0 + scale)*Prefactor*L[b].val));
        if (n > 2)
        for (int c = 0; c < n; c++)
        if (c != a && c != b)
        {
            const int gc = L[c].idx;
            /* IP.Properties holds one energy per grain pair, evaluated by SetSR with the pair's
             * earlier list entry first (InterfaceProperties.cpp:609-614): an order-dependent model
             * is evaluated here in that order too */
            dPhi_dt += (s->aniso ? voxel_energy(s, L, b < c ? b : c, b < c ? c : b)
                                   - voxel_energy(s, L, a < c ? a : c, a < c ? c : a)
                                 : ip_energy(s, gb, gc) - ip_energy(s, ga, gc))
                      *(L[c].lap + 0.5*(1.0 + scale)*Prefactor*L[c].val);
            /* TripleJunctionModels::Model (:536-552) */
            if (s->p.tj_factor != 0.0 || scale < 1.0)
            {
                const int pA = s->grain_phase[ga], pB = s->grain_phase[gb], pG = s->grain_phase[gc];
                dPhi_dt += dmax(s->p.tj_factor, (1.0 - scale))*Prefactor
                               *(phase_energy(s, pA, pB) + phase_energy(s, pB, pG) + phase_energy(s, pA, pG))
                               *(L[a].val*L[c].val - L[b].val*L[c].val);
            }
        }
        dPhi_dt *= (s->aniso ? voxel_mobility(s, L, a, b) : ip_mobility(s, ga, gb))*norm_1*scale;
        /* NodeAB::add_asym1 on an empty FieldsDot creates the entry (NodeAB.h:467-490) */
        P[np].a = a; P[np].b = b; P[np].v1 = dPhi_dt; P[np].alive = 1;
        np++;
    }
    return np;
}

/* Driving-force averaging, DrivingForce::Average with $Average Yes (src/DrivingForce.cpp:242-256):
 * SetWeights (:276-291), CollectAverage (:293-383) and DistributeAverage (:384-478) in the default
 * PHASEFIELDS weights mode (:59, :137), with Range = iWidth and Threshold = iWidth/15 below an
 * interface width of 5 cells, else 1/3 (:64-73), for the per-grain driving force raw(A,B) =
 * dG_B - dG_A that the oracle driver adds on every pair of an interface voxel.  Only the pairs of
 * positive entries have a weight; the entries of the zero-valued candidates keep weight 0, tmp 0
 * and average 0 (raw for a Seed). */
static int df_range(const op_sim* s) { return (int)s->p.iwidth; }   /* int Range = double iWidth */

static double df_threshold(const op_sim* s)
{
    return s->p.iwidth < 5.0 ? s->p.iwidth/15.0 : 1.0/3.0;
}

/* Force(u).get_weight(A, B): sqrt(phi_A*phi_B) of an interface voxel u holding both (SetWeights),
 * 0 elsewhere; *sa, *sb get the list positions of A and B. */
static double df_weight(const op_sim* s, long u, int A, int B, int* sa, int* sb)
{
    *sa = -1; *sb = -1;
    if (s->flag[u] != 2) return 0.0;
    const entry* L = s->e + u*s->cap;
    for (int k = 0; k < s->cnt[u]; k++)
    {
        if (L[k].idx == A) *sa = k;
        if (L[k].idx == B) *sb = k;
    }
    if (*sa < 0 || *sb < 0) return 0.0;
    return sqrt(L[*sa].val*L[*sb].val);
}

static void df_average(op_sim* s)
{
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const int R = df_range(s);
    const int Xr = R < nx - 1 ? R : nx - 1, Yr = R < ny - 1 ? R : ny - 1, Zr = R < nz - 1 ? R : nz - 1;
    const double thr = df_threshold(s);
    const double weight_threshold = sqrt(thr*(1.0 - thr));
    int maxpos = 2;
    for (long v = 0; v < s->n; v++)
    {
        const entry* L = s->e + v*s->cap;
        int c = 0;
        while (c < s->cnt[v] && L[c].val > 0.0) c++;
        s->npos[v] = c;
        if (s->flag[v] == 2 && c > maxpos) maxpos = c;
    }
    const int maxpp = maxpos*(maxpos - 1)/2;
    if (maxpp > s->maxpp)
    {
        free(s->df_tmp); free(s->df_avg);
        s->df_tmp = (double*)malloc((size_t)s->n*maxpp*sizeof(double));
        s->df_avg = (double*)malloc((size_t)s->n*maxpp*sizeof(double));
        s->maxpp = maxpp;
    }
    const int MP = s->maxpp;
    /* CollectAverage */
    #pragma omp parallel for schedule(dynamic, 64)
    for (long v = 0; v < s->n; v++)
    {
        if (s->flag[v] != 2) continue;
        const int i = (int)(v/((long)ny*nz)), j = (int)((v/nz) % ny), k = (int)(v % nz);
        const entry* L = s->e + v*s->cap;
        const int c = s->npos[v];
        for (int a = 0; a < c; a++)
        for (int b = a + 1; b < c; b++)
        {
            const int A = L[a].idx, B = L[b].idx;
            const double raw = s->dg[B] - s->dg[A];
            const double weight = sqrt(L[a].val*L[b].val);
            const double scale = s->vr[A]*s->vr[B];
            double tmp = 0.0;
            if (weight > weight_threshold*scale)
            {
                double value = 0.0, sum_weights = 0.0;
                for (int ii = -Xr; ii <= Xr; ii++)
                for (int jj = -Yr; jj <= Yr; jj++)
                for (int kk = -Zr; kk <= Zr; kk++)
                {
                    const double weight_dist = R - sqrt((double)(ii*ii + jj*jj + kk*kk));
                    int sa, sb;
                    const double weight_phi = df_weight(s, vox(s, i + ii, j + jj, k + kk), A, B, &sa, &sb);
                    if (weight_dist > 0.0 && weight_phi > 0.0)
                    {
                        sum_weights += weight_phi;
                        value += weight_phi*raw;   /* get_raw(A, B) at the neighbour: raw of (A, B) */
                    }
                }
                tmp = sum_weights > 0.0 ? value/sum_weights : raw;
            }
            s->df_tmp[v*MP + pair_pos(a, b, c)] = tmp;
        }
    }
    /* DistributeAverage */
    #pragma omp parallel for schedule(dynamic, 64)
    for (long v = 0; v < s->n; v++)
    {
        if (s->flag[v] != 2) continue;
        const int i = (int)(v/((long)ny*nz)), j = (int)((v/nz) % ny), k = (int)(v % nz);
        const entry* L = s->e + v*s->cap;
        const int c = s->npos[v];
        for (int a = 0; a < c; a++)
        for (int b = a + 1; b < c; b++)
        {
            const int A = L[a].idx, B = L[b].idx;
            const double scale = s->vr[A]*s->vr[B];
            double value = 0.0, sum_weights = 0.0;
            for (int ii = -Xr; ii <= Xr; ii++)
            for (int jj = -Yr; jj <= Yr; jj++)
            for (int kk = -Zr; kk <= Zr; kk++)
            {
                const double weight_dist = R - sqrt((double)(ii*ii + jj*jj + kk*kk));
                const long u = vox(s, i + ii, j + jj, k + kk);
                int sa, sb;
                const double weight_phi = df_weight(s, u, A, B, &sa, &sb);
                if (weight_dist > 0.0 && weight_phi > weight_threshold*scale)
                {
                    sum_weights += weight_phi;
                    /* get_tmp(A, B): the neighbour's tmp, negated when it lists B before A */
                    const double t = s->df_tmp[u*MP + (sa < sb ? pair_pos(sa, sb, s->npos[u]) : pair_pos(sb, sa, s->npos[u]))];
                    value += weight_phi*(sa < sb ? t : -t);
                }
            }
            s->df_avg[v*MP + pair_pos(a, b, c)] =
                sum_weights > 0.0 ? value/sum_weights : s->df_tmp[v*MP + pair_pos(a, b, c)];
        }
    }
}

/* DrivingForce::MergePhaseFieldIncrementsSR (src/DrivingForce.cpp:497-602) for the per-grain
 * driving force raw(a,b) = dG_b - dG_a that the oracle driver adds with NodeDF::add_raw for each
 * pair (a before b) of an interface voxel: locdG = raw (SkipAverage, $Average No, :258-274) or the
 * average above ($Average Yes). */
static void df_merge(const op_sim* s, long v, const entry* L, int n, pair* P)
{
    const double Eta = s->p.iwidth*s->p.dx;
    const double Prefactor = OP_PI/Eta;
    const int NP = s->p.nphases;
    for (int a = 0; a < n; a++)
    for (int b = a + 1; b < n; b++)
    {
        const int ga = L[a].idx, gb = L[b].idx;
        const int seed = s->stage[ga] == OP_STAGE_SEED || s->stage[gb] == OP_STAGE_SEED;
        double locdG = s->dg[gb] - s->dg[ga];
        if (s->p.average)
        {
            const int c = s->npos[v];
            if (b < c) locdG = s->df_avg[v*s->maxpp + pair_pos(a, b, c)];
            else if (!seed) locdG = 0.0;   /* weight 0, no Seed: the average stays 0 (:464-468) */
        }
        double norm = sqrt(L[a].val*L[b].val);
        if (seed) norm += 1.0e-6;
        if (s->p.limiting)
        {
            const int pA = s->grain_phase[ga], pB = s->grain_phase[gb];
            const double lim = s->limit_phase ? s->limit_phase[pA*NP + pB] : 0.95;
            double allowedDG = lim*Prefactor*phase_max_energy(s, pA, pB);
            allowedDG *= s->p.regularization;
            locdG = allowedDG*tanh(locdG/allowedDG);
        }
        const double dPsi_dt = locdG*(s->aniso ? voxel_mobility(s, L, a, b) : ip_mobility(s, ga, gb))*norm*Prefactor;
        P[pair_pos(a, b, n)].v1 += dPsi_dt;
    }
}

/* PhaseField::NormalizeIncrementsSR (src/PhaseField.cpp:1351-1561), one voxel. */
static uint32_t normalize(const entry* L, int n, pair* P, int np, double dt)
{
    uint32_t st = 0;
    const double precision = FLT_EPSILON;
    if (np == 0) return 0;
    if (np == 1)
    {
        /* :1368-1404 — the single pair's first index is list entry 0 */
        const double valueA = (P[0].v1 + 0.0)*dt;
        const double old_value = L[P[0].a].val;
        if ((old_value == 0.0 && valueA < 0.0) || (old_value == 1.0 && valueA > 0.0))
        {
            P[0].alive = 0;
        }
        else
        {
            const double new_value = old_value + valueA;
            double norm = 1.0;
            if (new_value < 0.0)      norm *= -old_value/valueA;
            else if (new_value > 1.0) norm *= (1.0 - old_value)/valueA;
            if (norm > DBL_EPSILON) P[0].v1 *= norm;
            else P[0].alive = 0;
        }
        return 0;
    }
    /* :1407-1431 zero all pairs of a field that would leave [0,1] */
    for (int a = 0; a < n; a++)
    {
        double dPsiAlpha = 0.0;
        for (int b = 0; b < n; b++)
        if (a != b)
        {
            dPsiAlpha += get_asym1(P, a, b, n);
        }
        if ((L[a].val == 0.0 && dPsiAlpha < 0.0) || (L[a].val == 1.0 && dPsiAlpha > 0.0))
        {
            for (int b = 0; b < n; b++)
            if (a != b)
            {
                pair* q = (a < b) ? &P[pair_pos(a, b, n)] : &P[pair_pos(b, a, n)];
                q->v1 = 0.0;   /* set_sym_pair(.., 0, 0); an erased pair would be re-added as zero */
            }
        }
    }
    /* :1433-1445 erase zero pairs */
    int nalive = 0;
    for (int q = 0; q < np; q++)
    {
        if (P[q].alive && P[q].v1 == 0.0) P[q].alive = 0;
        nalive += P[q].alive;
    }
    if (!nalive) return 0;
    /* :1447-1519 iterative limiting */
    double pos[64], neg[64], limP[64], limN[64];
    int iterations = 0;
    int limiting_needed = 1;
    while (limiting_needed)
    {
        iterations++;
        limiting_needed = 0;
        for (int a = 0; a < n; a++) { pos[a] = 0.0; neg[a] = 0.0; }
        for (int q = 0; q < np; q++)
        if (P[q].alive)
        {
            const double v = P[q].v1;
            if (v < 0.0) { neg[P[q].a] += v; pos[P[q].b] += -v; }
            if (v > 0.0) { pos[P[q].a] += v; neg[P[q].b] += -v; }
        }
        for (int a = 0; a < n; a++)
        {
            const double newPFvalue = L[a].val + (pos[a] + neg[a])*dt;
            limN[a] = 1.0;
            limP[a] = 1.0;
            if (newPFvalue < 0.0)
                limN[a] = dmin(1.0, -(L[a].val + pos[a]*dt)/(neg[a]*dt));
            if (newPFvalue > 1.0)
                limP[a] = dmin(1.0, (1.0 - (L[a].val + neg[a]*dt))/(pos[a]*dt));
        }
        for (int q = 0; q < np; q++)
        if (P[q].alive)
        {
            if (P[q].v1 < 0.0)
            {
                const double lim = dmin(limN[P[q].a], limP[P[q].b]);
                P[q].v1 *= lim;
                if (lim < 1.0) limiting_needed = 1;
            }
            if (P[q].v1 > 0.0)
            {
                const double lim = dmin(limP[P[q].a], limN[P[q].b]);
                P[q].v1 *= lim;
                if (lim < 1.0) limiting_needed = 1;
            }
        }
        if (iterations > 24)
        {
            if (limiting_needed) st |= OP_S_LIMITER_CAP;
            limiting_needed = 0;
        }
    }
    /* :1521-1533 erase increments below DBL_EPSILON */
    for (int q = 0; q < np; q++)
    if (P[q].alive && fabs(P[q].v1*dt) < DBL_EPSILON) P[q].alive = 0;
    /* :1535-1561 plausibility check (warning only) */
    double tmp[64];
    for (int a = 0; a < n; a++) tmp[a] = L[a].val;
    for (int q = 0; q < np; q++)
    if (P[q].alive && P[q].v1 != 0.0)
    {
        tmp[P[q].a] += P[q].v1*dt;
        tmp[P[q].b] += -P[q].v1*dt;
    }
    for (int a = 0; a < n; a++)
    if (tmp[a] < -precision || tmp[a] > 1.0 + precision) st |= OP_S_NORMALIZE_WARN;
    return st;
}

/* PhaseField::MergeIncrementsSR (src/PhaseField.cpp:1268-1299), one voxel; growth-constraint
 * factor 1 (GrowthConstraintsViolations::None for every grain). */
static void merge(entry* L, const pair* P, int np, double dt)
{
    for (int q = 0; q < np; q++)
    if (P[q].alive)
    {
        const double factor = 1.0;
        const double value = factor*(P[q].v1 + 0.0)*dt;
        if (fabs(value) >= DBL_EPSILON)
        {
            L[P[q].a].val += value;
            L[P[q].b].val += -value;
        }
    }
}

/* NodePF::finalize (include/Containers/NodePF.h:214-255); returns the new flag. */
static int node_finalize(entry* L, int32_t* cnt, uint32_t* st)
{
    double total = 0.0;
    int n = *cnt, m = 0;
    for (int a = 0; a < n; a++)
    {
        int erase = 0;
        if (L[a].val >= 1.0 - DBL_EPSILON) L[a].val = 1.0;
        if (L[a].val <= 0.0 + DBL_EPSILON) { L[a].val = 0.0; erase = 1; }
        total += L[a].val;
        if (!erase) L[m++] = L[a];
    }
    *cnt = m;
    if (m > 1)
    {
        const double norm = 1.0/total;
        for (int a = 0; a < m; a++)
        {
            L[a].val *= norm; L[a].lap = 0.0;
            L[a].grad[0] = 0.0; L[a].grad[1] = 0.0; L[a].grad[2] = 0.0;
        }
        return 2;
    }
    if (m == 0) { *st |= OP_S_EMPTY_VOXEL; return 0; }
    L[0].val = 1.0;
    L[0].lap = 0.0;
    L[0].grad[0] = 0.0; L[0].grad[1] = 0.0; L[0].grad[2] = 0.0;
    return 0;
}

/* PhaseField::SetFlagsSR (src/PhaseField.cpp:953-969) with periodic halos. */
static void set_flags(op_sim* s)
{
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
    for (int k = 0; k < nz; k++)
    {
        const long v = ((long)i*ny + j)*nz + k;
        if (s->flag[v] != 0) continue;
        int f = 0;
        for (int di = -1; di <= 1 && !f; di++)
        for (int dj = -1; dj <= 1 && !f; dj++)
        for (int dk = -1; dk <= 1 && !f; dk++)
        if (s->flag[vox(s, i+di, j+dj, k+dk)] == 2) f = 1;
        if (f) s->flag[v] = -1;   /* mark, resolved below so that marks do not propagate */
    }
    #pragma omp parallel for schedule(static)
    for (long v = 0; v < s->n; v++) if (s->flag[v] == -1) s->flag[v] = 1;
}

/* PhaseField::CalculateDerivativesSR (src/PhaseField.cpp:566-615): Laplacian pass, then gradient
 * pass, both appending zero-valued candidate entries for indices met in the neighbourhood;
 * NodePF::set_temporary / add_laplacian_tmp / add_gradient_tmp / copy_from_temporary
 * (NodePF.h:183-192, 351-366, 411-427). */
static void calculate_derivatives(op_sim* s)
{
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, cap = s->cap;
    uint32_t st = 0;
    #pragma omp parallel for collapse(2) schedule(static) reduction(|:st)
    for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
    for (int k = 0; k < nz; k++)
    {
        const long v = ((long)i*ny + j)*nz + k;
        if (s->flag[v] == 0) continue;
        entry* T = s->e2 + v*cap;
        int n = s->cnt[v];
        memcpy(T, s->e + v*cap, n*sizeof(entry));
        for (int q = 0; q < s->ns; q++)
        {
            const long u = vox(s, i + s->sdi[q], j + s->sdj[q], k + s->sdk[q]);
            const entry* U = s->e + u*cap;
            for (int r = 0; r < s->cnt[u]; r++)
            if (U[r].val != 0.0)
            {
                const double laplacian = s->sw[q]*U[r].val;
                int f = 0;
                for (; f < n; f++) if (T[f].idx == U[r].idx) break;
                if (f < n) T[f].lap += laplacian;
                else if (n < cap)
                {
                    T[n].idx = U[r].idx; T[n].val = 0.0; T[n].lap = laplacian;
                    T[n].grad[0] = 0.0; T[n].grad[1] = 0.0; T[n].grad[2] = 0.0;
                    n++;
                }
                else st |= OP_S_LIST_OVERFLOW;
            }
        }
        for (int q = 0; q < s->ng; q++)
        {
            const long u = vox(s, i + s->gdi[q], j + s->gdj[q], k + s->gdk[q]);
            const entry* U = s->e + u*cap;
            for (int r = 0; r < s->cnt[u]; r++)
            if (U[r].val != 0.0)
            {
                const double gx = s->gw[q][0]*U[r].val;
                const double gy = s->gw[q][1]*U[r].val;
                const double gz = s->gw[q][2]*U[r].val;
                int f = 0;
                for (; f < n; f++) if (T[f].idx == U[r].idx) break;
                if (f < n) { T[f].grad[0] += gx; T[f].grad[1] += gy; T[f].grad[2] += gz; }
                else if (n < cap)
                {
                    T[n].idx = U[r].idx; T[n].val = 0.0; T[n].lap = 0.0;
                    T[n].grad[0] = gx; T[n].grad[1] = gy; T[n].grad[2] = gz;
                    n++;
                }
                else st |= OP_S_LIST_OVERFLOW;
            }
        }
        s->cnt2[v] = n;
    }
    s->status |= st;
    #pragma omp parallel for schedule(static)
    for (long v = 0; v < s->n; v++)
    if (s->flag[v] != 0)
    {
        s->cnt[v] = s->cnt2[v];
        memcpy(s->e + v*cap, s->e2 + v*cap, s->cnt2[v]*sizeof(entry));
    }
}

/* PhaseField::CalculateGrainsVolume (src/PhaseField.cpp:812-951), single process.  The volume sum
 * runs over static per-thread chunks added in thread order (the reference adds per-thread partial
 * arrays of a dynamic schedule; the two orders differ only in the last bits). */
static void calculate_grains_volume(op_sim* s)
{
    const int G = s->p.ngrains;
    const int T = omp_get_max_threads();
    double* part = (double*)calloc((size_t)T*G, sizeof(double));
    #pragma omp parallel
    {
        double* mine = part + (size_t)omp_get_thread_num()*G;
        #pragma omp for schedule(static)
        for (long v = 0; v < s->n; v++)
        {
            const entry* L = s->e + v*s->cap;
            for (int a = 0; a < s->cnt[v]; a++) mine[L[a].idx] += L[a].val;
        }
    }
    for (int g = 0; g < G; g++)
    {
        s->volume[g] = 0.0;
        for (int t = 0; t < T; t++) s->volume[g] += part[(size_t)t*G + g];
    }
    free(part);
    for (int g = 0; g < G; g++)
    {
        s->max_volume[g] = dmax(s->volume[g], s->max_volume[g]);
        s->vr[g] = s->max_volume[g]/s->ref_volume[g];
    }
    for (int g = 0; g < G; g++)
    {
        if (s->exist[g] && s->volume[g] <= 0.0)
        {
            s->exist[g] = 0; s->stage[g] = OP_STAGE_STABLE;
            s->volume[g] = 0.0; s->max_volume[g] = 0.0; s->vr[g] = 1.0;
        }
        else if (s->volume[g] > 0.0)
        {
            s->exist[g] = 1;
            if (s->stage[g] == OP_STAGE_SEED) s->stage[g] = OP_STAGE_NUCLEUS;
            if (s->vr[g] > 1.0) { s->stage[g] = OP_STAGE_STABLE; s->vr[g] = 1.0; }
        }
    }
}

/* PhaseField::FinalizeSR (src/PhaseField.cpp:1008-1033): node finalize on wide-interface voxels,
 * then flags, derivatives and grain volumes (the periodic BoundaryConditions calls are implicit in
 * the periodic neighbour indexing). */
static void finalize_sr(op_sim* s)
{
    uint32_t st = 0;
    #pragma omp parallel for schedule(static) reduction(|:st)
    for (long v = 0; v < s->n; v++)
    if (s->flag[v] != 0)
    {
        s->flag[v] = (int8_t)node_finalize(s->e + v*s->cap, &s->cnt[v], &st);
    }
    s->status |= st;
    set_flags(s);
    calculate_derivatives(s);
    calculate_grains_volume(s);
}

void op_finalize_initialization(op_sim* s)
{
    finalize_sr(s);
}

uint32_t op_step(op_sim* s, double dt, int nsteps)
{
    const int cap = s->cap;
    const int maxpairs = cap*(cap - 1)/2;
    for (int t = 0; t < nsteps; t++)
    {
        uint32_t st = 0;
        if (s->dg && s->p.average) df_average(s);
        #pragma omp parallel reduction(|:st)
        {
            pair* P = (pair*)malloc(maxpairs*sizeof(pair));
            #pragma omp for schedule(static)
            for (long v = 0; v < s->n; v++)
            {
                if (s->flag[v] == 0) continue;
                entry* L = s->e + v*cap;
                const int n = s->cnt[v];
                const int np = do_increments(s, L, n, P);
                if (s->dg && s->flag[v] == 2) df_merge(s, v, L, n, P);
                st |= normalize(L, n, P, np, dt);
                merge(L, P, np, dt);
            }
            free(P);
        }
        s->status |= st;
        finalize_sr(s);
    }
    const uint32_t r = s->status;
    s->status = 0;
    return r;
}

long op_total_entries(const op_sim* s)
{
    long t = 0;
    for (long v = 0; v < s->n; v++) t += s->cnt[v];
    return t;
}

void op_get_state(const op_sim* s, int32_t* counts, int32_t* idx, double* val)
{
    long off = 0;
    for (long v = 0; v < s->n; v++)
    {
        counts[v] = s->cnt[v];
        for (int a = 0; a < s->cnt[v]; a++)
        {
            idx[off] = s->e[v*s->cap + a].idx;
            val[off] = s->e[v*s->cap + a].val;
            off++;
        }
    }
}

void op_get_flags(const op_sim* s, int8_t* flags)
{
    memcpy(flags, s->flag, s->n);
}

long op_wide_count(const op_sim* s)
{
    long w = 0;
    for (long v = 0; v < s->n; v++) w += (s->flag[v] != 0);
    return w;
}

void op_get_grains(const op_sim* s, double* volume, double* volume_ratio, double* max_volume,
                   int32_t* exist, int32_t* stage)
{
    const int G = s->p.ngrains;
    if (volume) memcpy(volume, s->volume, G*sizeof(double));
    if (volume_ratio) memcpy(volume_ratio, s->vr, G*sizeof(double));
    if (max_volume) memcpy(max_volume, s->max_volume, G*sizeof(double));
    if (exist) memcpy(exist, s->exist, G*sizeof(int32_t));
    if (stage) memcpy(stage, s->stage, G*sizeof(int32_t));
}

void op_set_grains(op_sim* s, const double* volume_ratio, const double* max_volume,
                   const int32_t* exist, const int32_t* stage, const double* ref_volume)
{
    const int G = s->p.ngrains;
    if (volume_ratio) memcpy(s->vr, volume_ratio, G*sizeof(double));
    if (max_volume) memcpy(s->max_volume, max_volume, G*sizeof(double));
    if (exist) memcpy(s->exist, exist, G*sizeof(int32_t));
    if (stage) memcpy(s->stage, stage, G*sizeof(int32_t));
    if (ref_volume) memcpy(s->ref_volume, ref_volume, G*sizeof(double));
}

/* Per-voxel entry counts of a raw PhaseField file (the format of PhaseField::Write,
 * src/PhaseField.cpp:2340-2388: after the 3 x int32 header, per voxel a size_t count and that many
 * (size_t index, double value) pairs).  `words` are the 8-byte words after the header.  Returns the
 * number of words the n voxels take, or -1 if they run past nwords. */
long op_raw_counts(const uint64_t* words, long nwords, long n, int32_t* counts)
{
    long pos = 0;
    for (long v = 0; v < n; v++)
    {
        if (pos >= nwords) return -1;
        const uint64_t c = words[pos];
        if (c > (uint64_t)(nwords - pos - 1) / 2) return -1;
        counts[v] = (int32_t)c;
        pos += 1 + 2 * (long)c;
    }
    return pos;
}
