/* TEST INFRASTRUCTURE ONLY — the oracle.  A CPU restatement, in plain C, of the OpenPhase
 * multiphase-field time step (double-obstacle pairwise kinetics, per-grain driving force,
 * increment normalisation, merge, finalize, flags, derivatives, grain volumes).  It exists to
 * check the CUDA path; only the tests, the smoke check and the bench's CPU-baseline leg load it.
 * It is never part of the product and the product never falls back to it.
 *
 * Parity pinning: the restatement is checked against the unmodified reference (compiled from its
 * own sources into oracle/_ref by oracle/Makefile) through golden fixtures under tests/golden/
 * and direct runs; see the header of pf_oracle.c for the per-function reference citations.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OP_STENCIL_SIMPLE = 0, OP_STENCIL_ISOTROPIC = 1, OP_STENCIL_LB = 2 };
enum { OP_STAGE_STABLE = 0, OP_STAGE_SEED = 1, OP_STAGE_NUCLEUS = 2 };
enum { OP_ENERGY_ISO = 0, OP_ENERGY_CUBIC = 1, OP_ENERGY_DISORIENTATION = 2, OP_ENERGY_HEXBOETTGER = 3,
       OP_ENERGY_HEXSUN = 4, OP_ENERGY_HEXYANG = 5, OP_ENERGY_FACETED = 6, OP_ENERGY_FACETEDEXP = 7 };
enum { OP_MOBILITY_FACETED = 6 };   /* mobility models use the energy codes 0, 1, 3..5, and this */

/* Status bits reported by op_step (OR-ed over all voxels and steps since the last call). */
enum {
    OP_S_LIST_OVERFLOW  = 1u << 0,  /* a voxel list needed more than `cap` entries            */
    OP_S_EMPTY_VOXEL    = 1u << 1,  /* finalize left a voxel without entries (reference: UB)   */
    OP_S_NORMALIZE_WARN = 1u << 2,  /* NormalizeIncrements plausibility warning was raised     */
    OP_S_LIMITER_CAP    = 1u << 3,  /* the increment limiter stopped after 25 iterations       */
};

typedef struct op_params {
    int nx, ny, nz;
    double dx;
    double iwidth;                    /* interface width in grid cells; Eta = iwidth*dx       */
    int stencil;                      /* Laplacian stencil, OP_STENCIL_*                        */
    int gradient_stencil;             /* gradient stencil, OP_STENCIL_* (reference default ISOTROPIC) */
    int nphases;
    int ngrains;
    const int* grain_phase;           /* [G] thermodynamic phase of each grain                  */
    const int* phase_solid;           /* [P] 1 = solid, 0 = liquid (NULL: all solid)            */
    const double* sigma_phase;        /* [P*P] ISO interface energy per phase pair              */
    const double* mu_phase;           /* [P*P] ISO interface mobility per phase pair            */
    const int* energy_model;          /* [P*P] OP_ENERGY_* (NULL: all ISO)                      */
    const double* cubic_eps;          /* [P*P] Epsilon1 of the CUBIC / HEX models (NULL: 0)     */
    const double* model_eps;          /* [P*P*3] Epsilon2..4 of the HEX models (NULL: 0)        */
    const int* facet_start;           /* [P*P+1] FACETED: facets of pair q in facet_data rows    */
    const double* facet_data;         /* rows of h, k, l, SigmaF, EpsilonEF (FACETEDEXP: h, k, l,
                                         EpsilonEF, PowerEF)                                       */
    const int* facet_family;          /* [P*P] 1: facets stand for their families                */
    const int* mobility_model;        /* [P*P] 0 ISO, 1 CUBIC, 3..5 HEX* (NULL: all ISO)         */
    const double* mobility_eps;       /* [P*P*4] its Epsilon1..4                                  */
    const int* mobility_facet_start;  /* [P*P+1] FACETED mobility: facets of pair q               */
    const double* mobility_facet_data;/* rows of h, k, l, MuF, EpsilonMF                          */
    const int* mobility_facet_family; /* [P*P] 1: facets stand for their families                */
    const double* quat;               /* [G*4] grain orientation quaternions (w,x,y,z) or NULL  */
    const double* pair_sigma;         /* [G*G] per-grain-pair sigma overriding the phase value, or NULL */
    const double* pair_mu;            /* [G*G] per-grain-pair mobility, or NULL                 */
    const double* dg;                 /* [G] per-grain stored-energy driving force, or NULL     */
    int limiting;                     /* tanh driving-force limiting (reference default: on)    */
    const double* limit_phase;        /* [P*P] limit factor (reference default 0.95), or NULL   */
    double regularization;            /* InterfaceProperties RegularizationFactor (default 1)   */
    double tj_factor;                 /* TripleJunctionFactor (default 0)                       */
    int consider_nucleus_volume;      /* PhaseField ConsiderNucleusVolume (default 1)           */
    double nucleus_volume_factor;     /* PhaseField NucleusVolumeFactor (default 1)             */
    int threads;                      /* OpenMP threads (0 = runtime default)                   */
    int average;                      /* DrivingForce $Average (reference default Yes; the
                                         benchmark set-ups use No)                               */
} op_params;

typedef struct op_sim op_sim;

op_sim* op_create(const op_params* p, int cap);
void    op_destroy(op_sim* s);

/* Load a state: counts[N] entries per voxel (voxel order x slowest, z fastest), then the entries
 * (index, value) of all voxels concatenated in that order.  Equivalent of PhaseField::Read. */
int     op_load(op_sim* s, const int32_t* counts, const int32_t* idx, const double* val);
/* PhaseField::FinalizeInitialization for a single-resolution grid. */
void    op_finalize_initialization(op_sim* s);
/* Run nsteps time steps of size dt; returns the OR of OP_S_* bits. */
uint32_t op_step(op_sim* s, double dt, int nsteps);

/* Total number of stored entries (sum of per-voxel list sizes). */
long    op_total_entries(const op_sim* s);
/* Copy the state out in the op_load layout (idx/val sized op_total_entries). */
void    op_get_state(const op_sim* s, int32_t* counts, int32_t* idx, double* val);
/* Per-voxel interface flag (0 bulk, 1 halo, 2 interface) as kept by the reference. */
void    op_get_flags(const op_sim* s, int8_t* flags);
long    op_wide_count(const op_sim* s);
/* Per-grain records after the last volume update. */
void    op_get_grains(const op_sim* s, double* volume, double* volume_ratio, double* max_volume,
                      int32_t* exist, int32_t* stage);
void    op_set_grains(op_sim* s, const double* volume_ratio, const double* max_volume,
                      const int32_t* exist, const int32_t* stage, const double* ref_volume);

/* Per-voxel counts of the n voxel lists of a raw PhaseField file (words after the 12-byte header);
 * returns the words they take or -1 if nwords is too short. */
long    op_raw_counts(const uint64_t* words, long nwords, long n, int32_t* counts);

#ifdef __cplusplus
}
#endif
#endif
