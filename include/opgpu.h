/*
 * opgpu — B200-native multiphase-field time step of OpenPhase, C ABI.
 *
 * This is the drop-in boundary for the OpenPhase single-resolution phase-field step.  Every entry
 * point names the reference interface it replaces (paths relative to the OpenPhase source tree).
 * Plain C types only: pointers to host memory, sizes and status codes.  No exception ever crosses
 * this boundary; every call returns OPGPU_OK (0) or a bitmask of OPGPU_E_* codes.
 *
 * Threading: one context is driven by one host thread at a time; distinct contexts are
 * independent.  Each context owns one CUDA stream on its device; calls that return data to the
 * host are synchronous, opgpu_step returns after the requested steps completed on the device.
 *
 * Voxel order everywhere: x slowest, z fastest (v = (x*ny + y)*nz + z), the order of the
 * reference's Storage3D (include/Containers/Storage3D.h:2054-2064) and of its raw files.
 */
#ifndef OPGPU_H
#define OPGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OPGPU_ABI_VERSION 2

/* ---- codes --------------------------------------------------------------------------------- */
#define OPGPU_OK                0u
/* soft conditions raised by the step (the reference would warn or misbehave silently) */
#define OPGPU_E_OVERFLOW_K      (1u << 0)  /* a voxel ended a step with more than K positive fields */
#define OPGPU_E_OVERFLOW_LIST   (1u << 1)  /* a voxel's field+candidate list exceeded its capacity   */
#define OPGPU_E_EMPTY_VOXEL     (1u << 2)  /* finalize left a voxel with no field (reference: UB)     */
#define OPGPU_E_NORMALIZE_WARN  (1u << 3)  /* NormalizeIncrements plausibility warning                */
#define OPGPU_E_LIMITER_CAP     (1u << 4)  /* increment limiter stopped after its 25 iterations       */
#define OPGPU_E_NONFINITE       (1u << 5)  /* a non-finite phase-field value was produced             */
#define OPGPU_E_ADJOINT_MISMATCH (1u << 6) /* adjoint step: recomputed step differs from the stored one */
#define OPGPU_E_AVERAGE_SKIPPED (1u << 7)  /* driving-force averaging could not store a voxel's pairs;
                                              that voxel's pairs kept the raw force                      */
/* hard errors */
#define OPGPU_E_INVALID         (1u << 8)  /* invalid argument                                         */
#define OPGPU_E_CUDA            (1u << 9)  /* CUDA runtime error (message: opgpu_last_error)           */
#define OPGPU_E_IO              (1u << 10) /* file could not be read or written                         */
#define OPGPU_E_STATE           (1u << 11) /* call order violated (e.g. step before initialization)     */
#define OPGPU_E_NODEVICE        (1u << 12) /* no CUDA device / the library was built without one        */
#define OPGPU_SOFT_MASK         0xFFu

enum opgpu_precision { OPGPU_FP64 = 0, OPGPU_FP32 = 1 };
enum opgpu_stencil   { OPGPU_STENCIL_SIMPLE = 0, OPGPU_STENCIL_ISOTROPIC = 1, OPGPU_STENCIL_LB = 2 };
enum opgpu_stage     { OPGPU_STAGE_STABLE = 0, OPGPU_STAGE_SEED = 1, OPGPU_STAGE_NUCLEUS = 2 };
enum opgpu_pair_mode { OPGPU_PAIRS_PHASE = 0, OPGPU_PAIRS_TABLE = 1, OPGPU_PAIRS_HASH = 2 };

typedef struct opgpu_ctx opgpu_ctx;

/* Grid and storage.  Replaces GridParameters (@GridParameters $Nx,$Ny,$Nz,$dx,$IWidth,
 * src/GridParameters.cpp:233-265) and the @PhaseField stencil keys (src/PhaseField.cpp:108-178). */
typedef struct opgpu_grid {
    int32_t nx, ny, nz;        /* periodic grid                                                   */
    double  dx;                /* grid spacing                                                    */
    double  iwidth;            /* interface width in grid cells; Eta = iwidth*dx                  */
    int32_t laplacian_stencil; /* OPGPU_STENCIL_* ($PhaseFieldLaplacianStencil, default ISOTROPIC) */
    int32_t gradient_stencil;  /* OPGPU_STENCIL_* ($PhaseFieldGradientStencil, default ISOTROPIC)  */
    int32_t precision;         /* OPGPU_FP64 (parity drop-in) or OPGPU_FP32                        */
    int32_t k_slots;           /* stored fields per voxel: 8, 12 or 16                            */
    int32_t device;            /* CUDA device ordinal                                             */
} opgpu_grid;

/* Phase-pair model.  Replaces the ISO energy/mobility models of InterfaceProperties
 * (src/InterfaceProperties.cpp:150-300; InterfaceEnergyModel.h:78-84) and the DrivingForce
 * limiter settings (src/DrivingForce.cpp:127-168), PhaseField ConsiderNucleusVolume /
 * NucleusVolumeFactor (src/PhaseField.cpp:112-113). */
typedef struct opgpu_model {
    int32_t nphases;               /* <= 8                                                        */
    const double* sigma;           /* [P*P] interface energy per phase pair ($Sigma_a_b)          */
    const double* mu;              /* [P*P] interface mobility per phase pair ($Mu_a_b)           */
    const double* limit;           /* [P*P] driving-force limit ($Limit_a_b) or NULL for 0.95     */
    int32_t limiting;              /* $Limiting (reference default 1)                             */
    double  regularization;        /* $RegularizationFactor (default 1.0)                         */
    double  tj_factor;             /* $TripleJunctionFactor (default 0.0)                         */
    int32_t consider_nucleus_volume; /* default 1                                                 */
    double  nucleus_volume_factor;   /* default 1.0                                               */
    /* Anisotropic interface energy (InterfaceEnergyModel.h:78-94, 325-345; InterfaceProperties.cpp:
     * 617-673); any may be NULL (all ISO, all phases solid). */
    const int32_t* energy_model;   /* [P*P] 0 = ISO, 1 = CUBIC, 2 = DISORIENTATION, 3 = HEXBOETTGER,
                                      4 = HEXSUN, 5 = HEXYANG, 6 = FACETED, 7 = FACETEDEXP
                                      ($EnergyModel_a_b;
                                      DISORIENTATION: InterfaceEnergyModel.h:303-323, the energy of
                                      a grain pair from the cubic disorientation of the two grains'
                                      orientations (opgpu_set_orientations), tabulated per grain pair;
                                      its Energy and MaxEnergy are 0 as in the reference, so with
                                      $Limiting on the driving force of such pairs is limited to 0) */
    const double* cubic_eps;       /* [P*P] Epsilon1 of the CUBIC and HEX* models ($EpsilonE_a_b;
                                      HEXSUN $EpsilonE20_a_b, HEXYANG $EpsilonE1_a_b)              */
    const int32_t* phase_solid;    /* [P] 1 = Solid, 0 = Liquid ($State_p); anisotropy weights
                                      only count solid grains                                     */
    const double* model_eps;       /* [P*P*3] Epsilon2..4 of the HEX models (HEXSUN: $EpsilonE40,
                                      $EpsilonE60, $EpsilonE66; HEXYANG: $EpsilonE2, $EpsilonE3, -;
                                      InterfaceEnergyModel.h:105-134, 365-399); NULL: zeros       */
    /* FACETED (InterfaceEnergyModel.h:196-246, 417-438): the facets of phase pair q are entries
     * facet_start[q] .. facet_start[q+1]-1 of facet_data, 5 doubles each: h, k, l ($Facet_a_b_n),
     * SigmaF ($SigmaF_a_b_n), EpsilonEF ($EpsilonEF_a_b_n); facet_family[q] = 1 makes every facet
     * stand for its family of index permutations ($NfacetFamilies_a_b), 0 for itself ($Nfacets_a_b).
     * Energy = mean SigmaF, MaxEnergy = max SigmaF.  All three may be NULL without FACETED pairs.
     * FACETEDEXP (InterfaceEnergyModel.h:248-295, 389-413) reads the same table with the last two
     * columns EpsilonEF ($EpsilonEF_a_b_n) and PowerEF ($PowerEF_a_b_n, >= 2); its Energy and
     * MaxEnergy are $Sigma_a_b (sigma[q]). */
    const int32_t* facet_start;    /* [P*P+1]                                                      */
    const double* facet_data;      /* [facet_start[P*P]*5]                                         */
    const int32_t* facet_family;   /* [P*P]                                                        */
    /* Anisotropic interface mobility (InterfaceMobilityModel.h:71-113, 210-265; InterfaceProperties.cpp:
     * 680-707): per phase pair 0 = ISO, 1 = CUBIC, 3 = HEXBOETTGER, 4 = HEXSUN, 5 = HEXYANG,
     * 6 = FACETED ($MobilityModel_a_b) and Epsilon1..4 ($EpsilonM_a_b; HEXSUN $EpsilonM20/40/60/66_a_b; HEXYANG
     * $EpsilonM1/2/3_a_b).  Per voxel and pair the model is summed over the solid grains whose value
     * is neither 0 nor 1 (not averaged, as in the reference), else Mobility.  NULL: all ISO.      */
    const int32_t* mobility_model; /* [P*P]                                                        */
    const double* mobility_eps;    /* [P*P*4]                                                      */
    /* FACETED mobility (mobility model 6; InterfaceMobilityModel.h:165-208, 266-287): the facets of
     * phase pair q are rows mobility_facet_start[q] .. [q+1]-1 of mobility_facet_data, 5 doubles
     * each: h, k, l ($Facet_a_b_n), MuF ($MuF_a_b_n), EpsilonMF ($EpsilonMF_a_b_n);
     * mobility_facet_family as facet_family.  The model reads no $Mu: its Mobility, used where no
     * solid grain of the pair counts, is 0 as in the reference.  NULL without such pairs.        */
    const int32_t* mobility_facet_start;   /* [P*P+1]                                              */
    const double* mobility_facet_data;     /* [mobility_facet_start[P*P]*5]                        */
    const int32_t* mobility_facet_family;  /* [P*P]                                                */
} opgpu_model;

typedef struct opgpu_stats {
    int64_t steps;                 /* steps run since creation                                    */
    int64_t wide_last;             /* wide-interface voxels (flag != 0) processed by the last step */
    int64_t wide_total;            /* sum of wide-interface voxels over all steps                 */
    int64_t entries_in_total;      /* sum over steps of stored entries read                       */
    int64_t entries_out_total;     /* sum over steps of stored entries written                    */
    uint32_t status;               /* OR of soft OPGPU_E_* bits since the last opgpu_clear_status  */
    uint32_t overflow_voxels;      /* voxels that raised OPGPU_E_OVERFLOW_K / _LIST               */
    int64_t timed_launches;        /* steps timed since opgpu_set_timing(ctx, 1)                   */
    double  timed_kernel_ms;       /* their summed device duration: CUDA events on the context's
                                      stream around each step's kernel sequence                    */
    int64_t general_path_total;    /* voxels processed by the general per-voxel path (long lists,
                                      windows with too many grains) summed over all steps          */
    int64_t crowded_window_total;  /* of those, voxels whose 3-plane window held too many grains  */
    double  timed_classify_ms;     /* of timed_kernel_ms, the part spent in the classify kernel     */
    int64_t kernel_launches;       /* kernels this library launched for steps since creation       */
} opgpu_stats;

/* ---- lifecycle ------------------------------------------------------------------------------ */
/* Replaces PhaseField::Initialize + AllocateStorages (src/PhaseField.cpp:44-73, 341-365). */
uint32_t opgpu_create(const opgpu_grid* grid, opgpu_ctx** out);
uint32_t opgpu_destroy(opgpu_ctx* ctx);
const char* opgpu_last_error(const opgpu_ctx* ctx);
int32_t  opgpu_abi_version(void);
/* Build stamp: "opgpu sm_100a source <hash>", the hash of the sources and compile flags the library
 * was built from (openphase_b200/build_ext.py: source_hash).  No reference counterpart. */
const char* opgpu_build_info(void);
/* Number of CUDA devices visible (0 without a GPU). */
int32_t  opgpu_device_count(void);

/* ---- parameters ----------------------------------------------------------------------------- */
uint32_t opgpu_set_model(opgpu_ctx* ctx, const opgpu_model* model);
/* Grain records: replaces PhaseField::AddGrainInfo (src/PhaseField.cpp:2970-2979) for G grains of
 * the given phases; stage NULL = all Stable (GrainsProperties.h:319). */
uint32_t opgpu_set_grains(opgpu_ctx* ctx, int32_t ngrains, const int32_t* phase, const int32_t* stage);
/* Per-grain-pair interface energy/mobility written into every voxel's interface properties
 * (what InterfaceProperties::Properties(i,j,k).set_energy_and_mobility would hold after IP.Set,
 * InterfaceProperties.h:97, NodeIP.h:413-431).  sigma/mu are symmetric [G*G]; either may be NULL
 * to keep the phase-pair value. */
uint32_t opgpu_set_pair_table(opgpu_ctx* ctx, const double* sigma, const double* mu);
/* Per-grain-pair energy generated on the device: sigma(a,b) = lo + span*u(seed, min(a,b), max(a,b))
 * with the counter-based generator of opgpu_uniform(); for grain counts where a G*G table is
 * impractical.  Mobility stays the phase-pair value. */
uint32_t opgpu_set_pair_hash(opgpu_ctx* ctx, uint64_t seed, double lo, double span);
/* Per-grain driving force dG[G]: on every interface voxel each pair (a before b in the voxel's
 * list) receives raw = dG[b] - dG[a] (replaces DrivingForce::Clear + NodeDF::add_raw on Force,
 * src/DrivingForce.cpp:176-183, NodeDF.h:412-435, then Average->SkipAverage :242-274).
 * NULL disables the driving-force merge. */
uint32_t opgpu_set_driving_force(opgpu_ctx* ctx, const double* dG);
/* Driving-force averaging, $Average Yes of @DrivingForce (the reference default; the benchmark
 * set-ups use No): DrivingForce::Average -> SetWeights, CollectAverage, DistributeAverage
 * (src/DrivingForce.cpp:242-256, 276-478) in the default PHASEFIELDS weights mode, run on the state
 * each step starts from.  range ($Range) <= 0: iWidth; threshold ($Threshold) <= 0: iWidth/15 below
 * an interface width of 5 cells, else 1/3.  The averaged force of a pair replaces its raw force in
 * the merge (a pair whose weight exceeds the threshold nowhere within range gets none, as in the
 * reference).  Costs two passes over a sphere of radius range per interface pair, 8 bytes of device
 * memory per voxel and 16 per pair of stored fields of the interface voxels, and one host
 * synchronisation per step; not with the adjoint, the tangent-linear model or slab steps. */
uint32_t opgpu_set_averaging(opgpu_ctx* ctx, int32_t enable, int32_t range, double threshold);
/* Grain orientations as quaternions (s, x, y, z) per grain, quat[4*G] (GrainsProperties::Orientation,
 * include/GrainsProperties.h:76); NULL = unrotated.  Used by anisotropic energy models. */
uint32_t opgpu_set_orientations(opgpu_ctx* ctx, const double* quat);

/* ---- state ---------------------------------------------------------------------------------- */
/* Upload ragged per-voxel lists: counts[N], then (idx, val) of all entries concatenated in voxel
 * order.  Equivalent of PhaseField::Read (src/PhaseField.cpp:2477-2539, NodePF::read
 * NodePF.h:751-763).  Lists longer than K are accepted if finalize brings them to <= K. */
uint32_t opgpu_upload_lists(opgpu_ctx* ctx, const int32_t* counts, const int32_t* idx, const double* val);
/* Read / write a raw PhaseField file (3 x int32 header, per voxel size_t n and n x (size_t index,
 * double value)); replaces PhaseField::Read(FileName) / Write(FileName)
 * (src/PhaseField.cpp:2340-2388, 2477-2539). */
uint32_t opgpu_read_raw(opgpu_ctx* ctx, const char* path);
uint32_t opgpu_write_raw(opgpu_ctx* ctx, const char* path);
/* PhaseField::FinalizeInitialization (src/PhaseField.cpp:1068-1077). */
uint32_t opgpu_finalize_initialization(opgpu_ctx* ctx);
/* Total stored entries, then download in the opgpu_upload_lists layout. */
uint32_t opgpu_total_entries(opgpu_ctx* ctx, int64_t* total);
uint32_t opgpu_download_lists(opgpu_ctx* ctx, int32_t* counts, int32_t* idx, double* val);
/* Per-voxel flags (0 bulk, 1 interface halo, 2 interface) of the current state
 * (PhaseField::SetFlagsSR, src/PhaseField.cpp:953-969). */
uint32_t opgpu_download_flags(opgpu_ctx* ctx, int8_t* flags);
/* Same result as opgpu_download_flags, but the call allocates no device memory (no cudaMalloc /
 * cudaFree, no allocating library routine): the flags are computed into a fixed 16 MiB scratch
 * array in the library's device memory and copied from there.  No reference counterpart.
 * For callers that cannot allocate: a host whose device memory is fully handed out to its own
 * pool, and callers that must not stall other streams (cudaFree waits for all work on the
 * device), e.g. a monitor that reads the flags while steps run on other contexts.
 * Limit: grids of at most 16,777,216 voxels (256^3); larger grids get OPGPU_E_INVALID with a
 * message.  The first call on each context does a one-time set-up (it looks up the scratch
 * address on the context's device) and should come before any stream capture.  The 16 MiB are
 * taken from device memory when the library's device code is loaded on a device, in every process
 * that loads the library, not at the call.  The scratch is shared by all contexts on a device:
 * overlapping calls (from several threads) race, so serialise them. */
uint32_t opgpu_download_flags_noalloc(opgpu_ctx* ctx, int8_t* flags);

/* Grain records in the reference's restart format: the binary file of GrainsProperties::Write /
 * Read (include/GrainsProperties.h:762-825, one Grain::Write record per grain, :197-231): size_t G,
 * then per grain Exist, Mobile, Stage, Parent, Phase, Variant, State, Density, RefVolume, Volume,
 * MAXVolume, the rigid-body vectors and the orientation quaternion.  Fields this library does not
 * model are written with the reference's defaults (Mobile true, Parent/Variant 0, Density 0, motion
 * zero) and ignored when read.  A restart, like PhaseField::Read(Settings, BC, tStep)
 * (src/PhaseField.cpp:2541-2554: raw state, FieldsProperties.Read, Finalize), is
 *   opgpu_read_raw -> opgpu_read_grains -> opgpu_finalize_initialization,
 * the last of which then keeps the MAXVolume read from the file.  opgpu_read_grains needs
 * opgpu_set_grains with the same grain count first and replaces phases, stages, reference volumes,
 * volumes, MAXVolume (VolumeRatio = MAXVolume/RefVolume as Grain::Read) and orientations. */
uint32_t opgpu_write_grains(opgpu_ctx* ctx, const char* path);
uint32_t opgpu_read_grains(opgpu_ctx* ctx, const char* path);
/* VTK output of the current state, byte for byte what PhaseField::WriteVTK writes for a single-
 * resolution grid without curvature output (src/PhaseField.cpp:2128-2150, VTK::Write
 * src/VTK.cpp:75-95): an ASCII StructuredGrid (.vts) with the point data Interfaces, Flags,
 * PhaseFields (majority grain), PhaseFraction_<p>, Junctions (list length including the zero-valued
 * candidates), Variants, ParentGrain, then the point coordinates. */
uint32_t opgpu_write_vtk(opgpu_ctx* ctx, const char* path);
/* The same file from ragged host lists (no device needed): counts[N], idx/val of all entries in
 * voxel order, grain_phase[ngrains] (NULL: all phase 0), the grid's OPGPU_STENCIL_* choices (they
 * decide which neighbours bring candidates). */
uint32_t opgpu_write_vtk_host(int32_t nx, int32_t ny, int32_t nz, const int32_t* counts, const int32_t* idx,
                              const double* val, int32_t ngrains, const int32_t* grain_phase, int32_t nphases,
                              int32_t laplacian_stencil, int32_t gradient_stencil, const char* path);

/* ---- the time step -------------------------------------------------------------------------- */
/* nsteps repetitions of the reference step sequence
 *   IP.Set -> [dG fill + Average] -> DoubleObstacle::CalculatePhaseFieldIncrements
 *   (src/DoubleObstacle.cpp:461-571) -> [DrivingForce::MergePhaseFieldIncrements
 *   (src/DrivingForce.cpp:480-602)] -> PhaseField::NormalizeIncrements (src/PhaseField.cpp:1334-1561)
 *   -> PhaseField::MergeIncrements + Finalize (src/PhaseField.cpp:1248-1299, 989-1033),
 * fused into one device pass per step plus a per-grain update.  Returns the soft status bits
 * raised by these steps (also accumulated in opgpu_stats.status). */
uint32_t opgpu_step(opgpu_ctx* ctx, double dt, int32_t nsteps);
/* Same, but does not synchronise: returns once the steps are enqueued on the context's stream.
 * opgpu_sync waits and returns the accumulated soft status. */
uint32_t opgpu_step_async(opgpu_ctx* ctx, double dt, int32_t nsteps);
uint32_t opgpu_sync(opgpu_ctx* ctx);
/* Grain records after the last step (PhaseField::CalculateGrainsVolume, src/PhaseField.cpp:812-951):
 * any pointer may be NULL. */
uint32_t opgpu_grains(opgpu_ctx* ctx, double* volume, double* volume_ratio, double* max_volume,
                      int32_t* exist, int32_t* stage);
uint32_t opgpu_get_stats(opgpu_ctx* ctx, opgpu_stats* stats);
/* Kernel variant of opgpu_step: 0 = tiled production kernel (default), 1 = full-grid generic
 * kernel with identical arithmetic (kept for validation).  No reference counterpart. */
uint32_t opgpu_set_kernel_variant(opgpu_ctx* ctx, int32_t variant);
/* Time every fused step-kernel launch with a pair of CUDA events on the context's stream
 * (enable = 1 resets the accumulated figures; 0 stops timing).  No reference counterpart: the
 * reference's TimeInfo stamps (include/Tools/TimeInfo.h:36-86) are host wall-clock only. */
uint32_t opgpu_set_timing(opgpu_ctx* ctx, int32_t enable);
uint32_t opgpu_clear_status(opgpu_ctx* ctx);
/* CUDA stream of the context (a cudaStream_t), for callers that order their own work after it. */
void*    opgpu_stream(opgpu_ctx* ctx);

/* ---- checkpoints, adjoint and tangent-linear model ------------------------------------------ */
/* None of these has a reference counterpart: OpenPhase has no adjoint.  Parameters are the
 * per-grain-pair interface energy sigma(a,b) and mobility mu(a,b) the step uses (symmetric G*G
 * tables, diagonal unused) and the per-grain driving force dG(g); the loss is any function of the
 * grain volumes V(g) of the current state.  The discrete decisions of each step (list members,
 * zeroed and limited increments, snapped and erased fields) are those of the forward run and held
 * fixed; VolumeRatio is held fixed.  Both precisions record states; the adjoint arithmetic and the
 * gradient accumulation are FP64.  The tangent-linear model runs the FP64 form. */
/* Reserve nslots device checkpoints (state plus grain records). */
uint32_t opgpu_checkpoint_reserve(opgpu_ctx* ctx, int32_t nslots);
/* Copy the current state and grain records into / out of a checkpoint slot. */
uint32_t opgpu_checkpoint_save(opgpu_ctx* ctx, int32_t slot);
uint32_t opgpu_checkpoint_load(opgpu_ctx* ctx, int32_t slot);
/* One step (opgpu_step with nsteps = 1) that leaves the state it started from, with its grain
 * records, in checkpoint `slot`: opgpu_checkpoint_save(slot) + opgpu_step without copying the state
 * (the slot takes the input buffers; its old buffers become the step's scratch). */
uint32_t opgpu_step_save_input(opgpu_ctx* ctx, double dt, int32_t slot);
/* Start a reverse sweep at the current state: the adjoint of every stored value is dL_dV[grain]
 * (dL_dV[G]); the gradient accumulators are zeroed. */
uint32_t opgpu_adjoint_begin(opgpu_ctx* ctx, const double* dL_dV);
/* One step backwards.  `slot` holds the state from which one forward step of length dt produced the
 * current state.  Accumulates the parameter gradients of that step, turns the adjoint into that of
 * the slot's state and makes the slot's state current: the slot and the current state exchange
 * their buffers, so that afterwards the slot holds the state that was current.  OPGPU_E_* bit 6 is
 * raised when the recomputed step does not reproduce the current state's lists. */
uint32_t opgpu_adjoint_step(opgpu_ctx* ctx, int32_t slot, double dt);
/* Accumulated gradients: dL_dsigma[G*G], dL_dmu[G*G] (symmetric, zero diagonal), dL_ddG[G]; any may
 * be NULL. */
uint32_t opgpu_adjoint_gradients(opgpu_ctx* ctx, double* dL_dsigma, double* dL_dmu, double* dL_ddG);
/* Tangent-linear model: parameter tangents (symmetric G*G tables, G values; NULL = zero); the
 * tangent of the current state starts at zero. */
uint32_t opgpu_tlm_begin(opgpu_ctx* ctx, const double* dsigma, const double* dmu, const double* ddG);
/* nsteps forward steps carrying the tangent (FP64 form; the state advances exactly as opgpu_step's). */
uint32_t opgpu_tlm_step(opgpu_ctx* ctx, double dt, int32_t nsteps);
/* Tangent of the grain volumes of the current state, dV[G]. */
uint32_t opgpu_tlm_volumes(opgpu_ctx* ctx, double* dV);

/* ---- slab decomposition --------------------------------------------------------------------- */
/* A rank holds an x-slab of the global grid plus one halo plane on each side (local nx = slab + 2);
 * before each step the halo planes are refreshed from the neighbouring ranks, and the grain
 * volumes are summed over the slab only and all-reduced across ranks.  The reference does the
 * same with MPI (halo cells, include/BoundaryConditions.h:2747-2854; volume all-reduce,
 * src/PhaseField.cpp:854-892); these entry points have no direct counterpart. */
/* Only planes x0 <= x < x1 count in the grain volumes (call before uploading the state). */
uint32_t opgpu_set_volume_window(opgpu_ctx* ctx, int32_t x0, int32_t x1);
/* Bytes of one packed x-plane: ny*nz count bytes, then K index planes (int16), then K value planes. */
int64_t  opgpu_plane_bytes(opgpu_ctx* ctx);
/* Copy x-plane x of the current state to / from a device buffer of opgpu_plane_bytes bytes. */
uint32_t opgpu_pack_plane(opgpu_ctx* ctx, int32_t x, void* dev_buf);
uint32_t opgpu_unpack_plane(opgpu_ctx* ctx, int32_t x, const void* dev_buf);
/* Stream-ordered slab calls (enable != 0): opgpu_pack_plane, opgpu_unpack_plane,
 * opgpu_volume_recount, opgpu_volume_accumulator, opgpu_step_partial and opgpu_step_complete only
 * enqueue their work on the context's stream (opgpu_stream) and return; the caller orders its own
 * streams against it (e.g. events) before it reads or writes the device buffers involved, and
 * reads the accumulated soft status with opgpu_sync.  Default (0): each call returns with its work
 * done.  No reference counterpart. */
uint32_t opgpu_set_stream_ordered(opgpu_ctx* ctx, int32_t enable);
/* Recompute the grain-volume accumulator from the window planes of the current state. */
uint32_t opgpu_volume_recount(opgpu_ctx* ctx);
/* One step whose grain update is deferred: the window's volume sums stay in the accumulator. */
uint32_t opgpu_step_partial(opgpu_ctx* ctx, double dt);
/* Copy the accumulator (G doubles) to a device buffer (for the all-reduce). */
uint32_t opgpu_volume_accumulator(opgpu_ctx* ctx, double* dev_dst);
/* Set the accumulator from a device buffer (the all-reduced sums) and run the grain update; with
 * initial != 0 it is the update of FinalizeInitialization (MAXVolume and Exist restart). */
uint32_t opgpu_step_complete(opgpu_ctx* ctx, const double* dev_src, int32_t initial);

/* ---- host-side initial states (no GPU needed) ---------------------------------------------- */
/* Counter-based generator shared by host and device: SplitMix64 (Steele, Lea, Flood 2014) over
 * the key (seed, stream, a, b); uniform in [0,1) with 53 bits. */
double   opgpu_uniform(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b);
/* Voronoi tessellation: G seeds at integer positions floor(u*n) per axis (stream 1, b = axis);
 * owner[v] = nearest seed under the periodic minimum-image distance, ties to the lowest index.
 * The reference counterpart is Initializations::VoronoiTessellation (src/Initializations.cpp:
 * 2014-2194), whose seeds are fixed, so the seeded variant here is what both engines load. */
uint32_t opgpu_voronoi_owner_host(int32_t nx, int32_t ny, int32_t nz, int32_t ngrains, uint64_t seed,
                                  int32_t threads, int32_t* owner);
/* Grain-boundary spreading of an owner map (periodic, order independent): every voxel lists its
 * own grain first, then each distinct grain among its 26 neighbours in x,y,z-lexicographic offset
 * order, all with value 1.0 (finalize normalises).  Call with idx == NULL to get counts and the
 * total; then with idx sized total. */
uint32_t opgpu_spread_boundaries_host(int32_t nx, int32_t ny, int32_t nz, const int32_t* owner,
                                      int32_t threads, int32_t* counts, int32_t* idx, int64_t* total);

/* Symmetric per-grain-pair table out[a*G+b] = lo + span*u(seed, stream, min(a,b), max(a,b)) with
 * out[a*G+a] = lo; the table opgpu_set_pair_table takes (stream 2 for interface energies). */
uint32_t opgpu_pair_table_host(int32_t ngrains, uint64_t seed, uint64_t stream, double lo, double span,
                               double* out);
/* Per-grain values out[g] = scale*u(seed, stream, g, 0) (stream 3 for driving forces). */
uint32_t opgpu_grain_values_host(int32_t ngrains, uint64_t seed, uint64_t stream, double scale, double* out);

#ifdef __cplusplus
}
#endif
#endif /* OPGPU_H */
