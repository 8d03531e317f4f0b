/*
 * opgpu.hpp — C++ mirror of the OpenPhase classes on the phase-field step, over the opgpu C ABI.
 *
 * A caller written against the reference (examples/NormalGG/NormalGG.cpp:74-83) keeps its call
 * sequence and swaps the types:
 *
 *     IP.Set(Phi, BC);
 *     dG.Clear();                                   // then dG.SetGrainForces(...)
 *     dG.Average(Phi, BC);
 *     DO.CalculatePhaseFieldIncrements(Phi, IP, dG);
 *     dG.MergePhaseFieldIncrements(Phi, IP);
 *     Phi.NormalizeIncrements(BC, dt);
 *     Phi.MergeIncrements(BC, dt);                  // the fused device step runs here
 *
 * Each call checks that it comes in the reference's order and records what the fused step needs;
 * PhaseField::MergeIncrements launches the step.  Error behaviour follows the reference: a hard
 * error prints a message and exits (ConsoleOutput::WriteExit + OP_Exit, include/Globals.h:98-110);
 * soft conditions print a warning (ConsoleOutput::WriteWarning, src/PhaseField.cpp:1560) and are
 * also returned by LastStatus().  Periodic boundaries only.  Header-only; link -lopgpu.
 */
#ifndef OPGPU_HPP
#define OPGPU_HPP

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "opgpu.h"

namespace opgpu_cxx {

inline void write_exit(const std::string& where, const std::string& msg)
{
    std::fprintf(stderr, "ERROR: %s: %s\n", where.c_str(), msg.c_str());
    std::exit(EXIT_FAILURE);
}

inline void write_warning(const std::string& where, const std::string& msg)
{
    std::fprintf(stderr, "WARNING: %s: %s\n", where.c_str(), msg.c_str());
}

/* GridParameters (src/GridParameters.cpp:233-265): periodic Nx x Ny x Nz, dx, iWidth. */
struct GridParameters {
    int Nx = 0, Ny = 0, Nz = 0;
    double dx = 1.0;
    double iWidth = 5.0;
    int LaplacianStencil = OPGPU_STENCIL_ISOTROPIC;   /* $PhaseFieldLaplacianStencil */
    int GradientStencil = OPGPU_STENCIL_ISOTROPIC;    /* $PhaseFieldGradientStencil  */
    int Precision = OPGPU_FP64;
    int KSlots = 16;
    int Device = 0;
};

/* BoundaryConditions: this step supports periodic boundaries in all directions only. */
struct BoundaryConditions {};

class InterfaceProperties;
class DrivingForce;

/* PhaseField (include/PhaseField.h:60-260): owns the device state. */
class PhaseField {
public:
    explicit PhaseField(const GridParameters& g) : grid_(g)
    {
        opgpu_grid d{};
        d.nx = g.Nx; d.ny = g.Ny; d.nz = g.Nz; d.dx = g.dx; d.iwidth = g.iWidth;
        d.laplacian_stencil = g.LaplacianStencil; d.gradient_stencil = g.GradientStencil;
        d.precision = g.Precision; d.k_slots = g.KSlots; d.device = g.Device;
        check(opgpu_create(&d, &ctx_), "PhaseField::Initialize");
    }
    ~PhaseField() { if (ctx_) opgpu_destroy(ctx_); }
    PhaseField(const PhaseField&) = delete;
    PhaseField& operator=(const PhaseField&) = delete;

    /* PhaseField::AddGrainInfo (src/PhaseField.cpp:2970-2979) for all grains at once. */
    void AddGrains(const std::vector<int32_t>& phase, const std::vector<int32_t>& stage = {})
    {
        check(opgpu_set_grains(ctx_, (int32_t)phase.size(), phase.data(), stage.empty() ? nullptr : stage.data()),
              "PhaseField::AddGrainInfo");
        ngrains_ = (int)phase.size();
    }
    /* PhaseField::Read / Write (src/PhaseField.cpp:2477-2539, 2340-2388): false on an IO error. */
    bool Read(const std::string& FileName)
    {
        const uint32_t st = opgpu_read_raw(ctx_, FileName.c_str());
        if (st & OPGPU_E_IO) return false;
        check(st, "PhaseField::Read");
        return true;
    }
    bool Write(const std::string& FileName)
    {
        const uint32_t st = opgpu_write_raw(ctx_, FileName.c_str());
        if (st & OPGPU_E_IO) return false;
        check(st, "PhaseField::Write");
        return true;
    }
    /* PhaseField::FinalizeInitialization (src/PhaseField.cpp:1068-1077). */
    void FinalizeInitialization(const BoundaryConditions&)
    {
        check(opgpu_finalize_initialization(ctx_), "PhaseField::FinalizeInitialization");
        stage_ = Stage::Idle;
    }
    /* Restart pair of PhaseField::Write(Settings, tStep) / Read(Settings, BC, tStep)
     * (src/PhaseField.cpp:2390-2402, 2541-2554): the raw state and the grain records
     * (GrainsProperties::Write / Read, include/GrainsProperties.h:762-825); Read finalizes. */
    bool WriteRestart(const std::string& RawFileName, const std::string& GrainsFileName)
    {
        if (!Write(RawFileName)) return false;
        const uint32_t st = opgpu_write_grains(ctx_, GrainsFileName.c_str());
        if (st & OPGPU_E_IO) return false;
        check(st, "PhaseField::Write");
        return true;
    }
    bool ReadRestart(const BoundaryConditions& BC, const std::string& RawFileName, const std::string& GrainsFileName)
    {
        if (!Read(RawFileName)) return false;
        const uint32_t st = opgpu_read_grains(ctx_, GrainsFileName.c_str());
        if (st & OPGPU_E_IO) return false;
        check(st, "PhaseField::Read");
        FinalizeInitialization(BC);
        return true;
    }
    /* PhaseField::WriteVTK (src/PhaseField.cpp:2128-2150), single resolution, no curvature output. */
    void WriteVTK(const std::string& FileName)
    {
        check(opgpu_write_vtk(ctx_, FileName.c_str()), "PhaseField::WriteVTK");
    }
    /* PhaseField::NormalizeIncrements (src/PhaseField.cpp:1334-1349). */
    void NormalizeIncrements(const BoundaryConditions&, double dt)
    {
        if (stage_ != Stage::IncrementsMerged && stage_ != Stage::Increments)
            write_exit("PhaseField::NormalizeIncrements", "called before DoubleObstacle::CalculatePhaseFieldIncrements");
        dt_ = dt;
        stage_ = Stage::Normalized;
    }
    /* PhaseField::MergeIncrements (src/PhaseField.cpp:1248-1299) with Finalize: runs the fused step. */
    void MergeIncrements(const BoundaryConditions&, double dt, bool finalize = true, bool clear = true)
    {
        if (stage_ != Stage::Normalized)
            write_exit("PhaseField::MergeIncrements", "called before PhaseField::NormalizeIncrements");
        if (!finalize || !clear)
            write_exit("PhaseField::MergeIncrements", "only finalize = clear = true is supported by the fused step");
        if (dt != dt_)
            write_exit("PhaseField::MergeIncrements", "dt differs from the one given to NormalizeIncrements");
        status_ = opgpu_step(ctx_, dt, 1);
        check(status_, "PhaseField::MergeIncrements");
        stage_ = Stage::Idle;
    }
    /* FieldsProperties[g].Volume after the last step (src/PhaseField.cpp:812-951). */
    std::vector<double> GrainVolumes()
    {
        std::vector<double> v(ngrains_);
        check(opgpu_grains(ctx_, v.data(), nullptr, nullptr, nullptr, nullptr), "PhaseField::CalculateGrainsVolume");
        return v;
    }
    /* Ragged host copy of Fields: counts[N], then (index, value) in voxel order. */
    void Download(std::vector<int32_t>& counts, std::vector<int32_t>& idx, std::vector<double>& val)
    {
        int64_t total = 0;
        check(opgpu_total_entries(ctx_, &total), "PhaseField::Fields");
        counts.resize((size_t)grid_.Nx * grid_.Ny * grid_.Nz);
        idx.resize((size_t)total);
        val.resize((size_t)total);
        check(opgpu_download_lists(ctx_, counts.data(), idx.data(), val.data()), "PhaseField::Fields");
    }
    uint32_t LastStatus() const { return status_; }
    opgpu_ctx* Handle() { return ctx_; }

private:
    friend class InterfaceProperties;
    friend class DrivingForce;
    friend class DoubleObstacle;
    enum class Stage { Idle, PropertiesSet, Increments, IncrementsMerged, Normalized };

    void check(uint32_t st, const char* where)
    {
        if (st & ~OPGPU_SOFT_MASK)
        {
            const char* m = opgpu_last_error(ctx_);
            write_exit(where, m && *m ? m : "opgpu error");
        }
        if (st & OPGPU_E_OVERFLOW_K) write_warning(where, "a voxel holds more phase fields than the K slots");
        if (st & OPGPU_E_OVERFLOW_LIST) write_warning(where, "a voxel's field and candidate list overflowed");
        if (st & OPGPU_E_NORMALIZE_WARN) write_warning(where, "NormalizeIncrements: phase field out of bounds");
        if (st & OPGPU_E_NONFINITE) write_warning(where, "non-finite phase-field value");
        if (st & OPGPU_E_EMPTY_VOXEL) write_warning(where, "a voxel lost all its phase fields");
    }

    GridParameters grid_;
    opgpu_ctx* ctx_ = nullptr;
    int ngrains_ = 0;
    double dt_ = 0.0;
    uint32_t status_ = 0;
    Stage stage_ = Stage::Idle;
};

/* InterfaceProperties (src/InterfaceProperties.cpp): the phase-pair model plus optional per-grain-
 * pair tables.  Set() only marks the step: the properties are evaluated inside the fused step. */
class InterfaceProperties {
public:
    /* ISO energy / mobility per phase pair ($Sigma_a_b, $Mu_a_b), limiter settings of DrivingForce. */
    void SetModel(PhaseField& Phi, const opgpu_model& m)
    {
        Phi.check(opgpu_set_model(Phi.ctx_, &m), "InterfaceProperties::ReadInput");
    }
    /* Per-grain-pair energies / mobilities (symmetric G*G; either may be null). */
    void SetPairTable(PhaseField& Phi, const double* sigma, const double* mu)
    {
        Phi.check(opgpu_set_pair_table(Phi.ctx_, sigma, mu), "InterfaceProperties::Properties");
    }
    void Set(PhaseField& Phi, const BoundaryConditions&)
    {
        Phi.stage_ = PhaseField::Stage::PropertiesSet;
    }
};

/* DrivingForce (src/DrivingForce.cpp) with per-grain forces: raw(a, b) = dG[b] - dG[a]. */
class DrivingForce {
public:
    void Clear() { cleared_ = true; }
    void SetGrainForces(PhaseField& Phi, const std::vector<double>& dG)
    {
        Phi.check(opgpu_set_driving_force(Phi.ctx_, dG.data()), "DrivingForce::Force");
    }
    /* $Average / $Range / $Threshold of @DrivingForce (src/DrivingForce.cpp:129-133; Range <= 0 and
     * Threshold <= 0 take the reference's defaults).  The reference's default is Yes. */
    void SetAveraging(PhaseField& Phi, bool Averaging, int Range = 0, double Threshold = 0.0)
    {
        Phi.check(opgpu_set_averaging(Phi.ctx_, Averaging ? 1 : 0, Range, Threshold), "DrivingForce::ReadInput");
    }
    /* DrivingForce::Average (src/DrivingForce.cpp:242-256): with averaging on, SetWeights,
     * CollectAverage and DistributeAverage run inside the fused step on the state it starts from;
     * else SkipAverage (:258-274). */
    void Average(PhaseField&, const BoundaryConditions&) {}
    void MergePhaseFieldIncrements(PhaseField& Phi, InterfaceProperties&)
    {
        if (Phi.stage_ != PhaseField::Stage::Increments)
            write_exit("DrivingForce::MergePhaseFieldIncrements", "called before DoubleObstacle::CalculatePhaseFieldIncrements");
        Phi.stage_ = PhaseField::Stage::IncrementsMerged;
    }

private:
    bool cleared_ = false;
};

/* DoubleObstacle (src/DoubleObstacle.cpp:461-500): stateless. */
class DoubleObstacle {
public:
    void CalculatePhaseFieldIncrements(PhaseField& Phi, InterfaceProperties&)
    {
        if (Phi.stage_ != PhaseField::Stage::PropertiesSet)
            write_exit("DoubleObstacle::CalculatePhaseFieldIncrements", "called before InterfaceProperties::Set");
        Phi.stage_ = PhaseField::Stage::Increments;
    }
    void CalculatePhaseFieldIncrements(PhaseField& Phi, InterfaceProperties& IP, DrivingForce&)
    {
        CalculatePhaseFieldIncrements(Phi, IP);
    }
};

}  // namespace opgpu_cxx

#endif  // OPGPU_HPP
