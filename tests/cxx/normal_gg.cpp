// A caller written in the shape of examples/NormalGG/NormalGG.cpp:74-83, on the opgpu C++ mirror.
//
//     normal_gg <in.raw> <out.raw> <nx> <ny> <nz> <ngrains> <iwidth> <dt> <nsteps> [dg_file]
//
// Reads a raw PhaseField state, runs nsteps of the reference step sequence (LB stencil, sigma = mu
// = 1 for all pairs, optional per-grain driving forces from a text file), writes the final state
// and prints the grain volumes, one per line.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "opgpu.hpp"

int main(int argc, char** argv)
{
    using namespace opgpu_cxx;
    if (argc < 10)
    {
        std::fprintf(stderr, "usage: %s in.raw out.raw nx ny nz ngrains iwidth dt nsteps [dg_file]\n", argv[0]);
        return 2;
    }
    GridParameters G;
    G.Nx = std::atoi(argv[3]); G.Ny = std::atoi(argv[4]); G.Nz = std::atoi(argv[5]);
    G.iWidth = std::atof(argv[7]);
    G.LaplacianStencil = OPGPU_STENCIL_LB;
    G.Precision = OPGPU_FP64;
    G.KSlots = 16;
    const int ngrains = std::atoi(argv[6]);
    const double dt = std::atof(argv[8]);
    const int nsteps = std::atoi(argv[9]);

    BoundaryConditions BC;
    PhaseField Phi(G);
    InterfaceProperties IP;
    DrivingForce dG;
    DoubleObstacle DO;

    double sigma = 1.0, mu = 1.0;
    opgpu_model m{};
    m.nphases = 1; m.sigma = &sigma; m.mu = &mu; m.limit = nullptr; m.limiting = 1;
    m.regularization = 1.0; m.tj_factor = 0.0; m.consider_nucleus_volume = 1; m.nucleus_volume_factor = 1.0;
    IP.SetModel(Phi, m);
    Phi.AddGrains(std::vector<int32_t>(ngrains, 0));
    bool with_dg = false;
    if (argc > 10)
    {
        std::vector<double> f(ngrains);
        std::ifstream in(argv[10]);
        for (int g = 0; g < ngrains; ++g) in >> f[g];
        dG.SetGrainForces(Phi, f);
        with_dg = true;
    }
    if (!Phi.Read(argv[1])) { std::fprintf(stderr, "cannot read %s\n", argv[1]); return 1; }
    Phi.FinalizeInitialization(BC);

    for (int tStep = 1; tStep <= nsteps; ++tStep)
    {
        IP.Set(Phi, BC);
        if (with_dg)
        {
            dG.Clear();
            dG.Average(Phi, BC);
            DO.CalculatePhaseFieldIncrements(Phi, IP, dG);
            dG.MergePhaseFieldIncrements(Phi, IP);
        }
        else
        {
            DO.CalculatePhaseFieldIncrements(Phi, IP);
        }
        Phi.NormalizeIncrements(BC, dt);
        Phi.MergeIncrements(BC, dt);
    }
    if (!Phi.Write(argv[2])) { std::fprintf(stderr, "cannot write %s\n", argv[2]); return 1; }
    for (double v : Phi.GrainVolumes()) std::printf("%.17g\n", v);
    return 0;
}
