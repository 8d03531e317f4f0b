// Test infrastructure (checker only): drives the UNMODIFIED OpenPhase reference through its own
// public C++ API for the multiphase-field time step, so that the oracle restatement and the CUDA
// path can be pinned against the reference's own output.  Built by oracle/Makefile into
// oracle/_ref/ref_driver; never linked into the product.
//
// Call order per time step (reference: examples/SolidificationFe/SolidificationFe.cpp:64-98,
// examples/NormalGG/NormalGG.cpp:74-83):
//     dG.Clear()                                  src/DrivingForce.cpp:176-183
//     IP.Set(Phi, BC)                             src/InterfaceProperties.cpp:557-576
//     <per-grain-pair sigma/mu written into IP.Properties on wide-interface voxels>
//     <per-grain driving force written with NodeDF::add_raw on interface voxels>
//     dG.Average(Phi, BC)                         src/DrivingForce.cpp:242-256 ($Average No: SkipAverage;
//                                                 "average 1": SetWeights, CollectAverage, DistributeAverage)
//     DO.CalculatePhaseFieldIncrements(Phi,IP,dG) src/DoubleObstacle.cpp:479-500
//     dG.MergePhaseFieldIncrements(Phi, IP)       src/DrivingForce.cpp:480-602
//     Phi.NormalizeIncrements(BC, dt)             src/PhaseField.cpp:1334-1349
//     Phi.MergeIncrements(BC, dt)                 src/PhaseField.cpp:1248-1299 (-> Finalize)
//
// The initial state is loaded with PhaseField::Read(FileName) (src/PhaseField.cpp:2477-2539)
// followed by PhaseField::FinalizeInitialization (src/PhaseField.cpp:1068-1077); grains are
// registered with PhaseField::AddGrainInfo (src/PhaseField.cpp:2970-2979).
//
// Usage: ref_driver <case.txt> <initial_raw.dat> <out_dir>
// case.txt holds "key value..." lines (see parse_case below).  Outputs in <out_dir>:
//     PF_<step>.dat    PhaseField::Write raw state at every requested dump step
//     V_<step>.bin     per-grain Volume (double[G]) at the same steps
//     VR_<step>.bin    per-grain VolumeRatio (double[G])
//     FP_<step>.dat    grain records in the restart format (GrainsProperties::Write)
//     PhaseField_<step>.vts  PhaseField::WriteVTK output at the vtk_steps
// With "restart_grains_file" the run starts from the raw state and those grain records followed
// by PhaseField::Finalize, the reference's restart (src/PhaseField.cpp:2541-2554).
//     stats.txt        wide-interface voxel count per step, step-loop wall time, threads

#include "Settings.h"
#include "DoubleObstacle.h"
#include "PhaseField.h"
#include "DrivingForce.h"
#include "BoundaryConditions.h"
#include "InterfaceProperties.h"

#include <omp.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

using namespace openphase;

struct Case
{
    int nx = 0, ny = 0, nz = 0;
    double dx = 1.0;
    double iwidth = 5.0;
    std::string stencil = "LB";
    double dt = 0.1;
    int nsteps = 0;
    int nphases = 1;
    std::vector<std::string> phase_state;
    std::vector<double> quat;      // [G*4] grain orientations (s, x, y, z), empty: none
    std::map<std::pair<int,int>, double> sigma, mu, limit, cubic_eps;
    std::map<std::pair<int,int>, std::vector<double>> model_eps;   // Epsilon2..4 of the HEX models
    std::map<std::pair<int,int>, std::vector<std::vector<double>>> facets;   // FACETED: h k l SigmaF EpsilonEF
    std::map<std::pair<int,int>, int> facet_family;
    std::map<std::pair<int,int>, std::vector<std::vector<double>>> mobility_facets;   // FACETED mobility: h k l MuF EpsilonMF
    std::map<std::pair<int,int>, int> mobility_facet_family;
    std::map<std::pair<int,int>, std::string> mobility_model;
    std::map<std::pair<int,int>, std::vector<double>> mobility_eps;
    std::map<std::pair<int,int>, std::string> energy_model;
    int ngrains = 0;
    std::vector<int> grain_phase;
    std::vector<double> pair_sigma, pair_mu, dg;
    bool limiting = true;
    bool average = false;          // DrivingForce $Average
    double regularization = 1.0;
    double tj_factor = 0.0;
    bool consider_nucleus_volume = true;
    std::set<int> dump_steps;
    std::set<int> vtk_steps;       // PhaseField::WriteVTK at these steps
    std::string restart_grains;    // FieldsProperties file to restart from (with the raw state)
    int threads = 0;
};

static std::vector<double> read_doubles(const std::string& path, size_t count)
{
    std::vector<double> v(count);
    std::ifstream f(path, std::ios::binary);
    if (!f) { fprintf(stderr, "ref_driver: cannot open %s\n", path.c_str()); exit(2); }
    f.read(reinterpret_cast<char*>(v.data()), count*sizeof(double));
    if (size_t(f.gcount()) != count*sizeof(double))
    {
        fprintf(stderr, "ref_driver: short read %s\n", path.c_str()); exit(2);
    }
    return v;
}

static std::vector<int> read_ints(const std::string& path, size_t count)
{
    std::vector<int> v(count);
    std::ifstream f(path, std::ios::binary);
    if (!f) { fprintf(stderr, "ref_driver: cannot open %s\n", path.c_str()); exit(2); }
    f.read(reinterpret_cast<char*>(v.data()), count*sizeof(int));
    return v;
}

static Case parse_case(const std::string& path)
{
    Case c;
    std::ifstream f(path);
    if (!f) { fprintf(stderr, "ref_driver: cannot open %s\n", path.c_str()); exit(2); }
    std::string line;
    std::string grain_phase_file, pair_sigma_file, pair_mu_file, dg_file, orientation_file;
    while (std::getline(f, line))
    {
        std::istringstream is(line);
        std::string key;
        if (!(is >> key) or key[0] == '#') continue;
        if      (key == "nx") is >> c.nx;
        else if (key == "ny") is >> c.ny;
        else if (key == "nz") is >> c.nz;
        else if (key == "dx") is >> c.dx;
        else if (key == "iwidth") is >> c.iwidth;
        else if (key == "stencil") is >> c.stencil;
        else if (key == "dt") is >> c.dt;
        else if (key == "nsteps") is >> c.nsteps;
        else if (key == "nphases") { is >> c.nphases; c.phase_state.assign(c.nphases, "SOLID"); }
        else if (key == "phase_state") { int p; std::string s; is >> p >> s; c.phase_state.at(p) = s; }
        else if (key == "sigma") { int a, b; double v; is >> a >> b >> v; c.sigma[{a,b}] = v; }
        else if (key == "mu") { int a, b; double v; is >> a >> b >> v; c.mu[{a,b}] = v; }
        else if (key == "limit") { int a, b; double v; is >> a >> b >> v; c.limit[{a,b}] = v; }
        else if (key == "energy_model") { int a, b; std::string m; is >> a >> b >> m; c.energy_model[{a,b}] = m; }
        else if (key == "cubic_eps") { int a, b; double v; is >> a >> b >> v; c.cubic_eps[{a,b}] = v; }
        else if (key == "mobility_model") { int a, b; std::string m; is >> a >> b >> m; c.mobility_model[{a,b}] = m; }
        else if (key == "mobility_eps") { int a, b; std::vector<double> e(4); is >> a >> b >> e[0] >> e[1] >> e[2] >> e[3]; c.mobility_eps[{a,b}] = e; }
        else if (key == "facet_family") { int a, b, f; is >> a >> b >> f; c.facet_family[{a,b}] = f; }
        else if (key == "facet") { int a, b; std::vector<double> f(5); is >> a >> b >> f[0] >> f[1] >> f[2] >> f[3] >> f[4]; c.facets[{a,b}].push_back(f); }
        else if (key == "mobility_facet_family") { int a, b, f; is >> a >> b >> f; c.mobility_facet_family[{a,b}] = f; }
        else if (key == "mobility_facet") { int a, b; std::vector<double> f(5); is >> a >> b >> f[0] >> f[1] >> f[2] >> f[3] >> f[4]; c.mobility_facets[{a,b}].push_back(f); }
        else if (key == "model_eps") { int a, b; double e2, e3, e4; is >> a >> b >> e2 >> e3 >> e4; c.model_eps[{a,b}] = {e2, e3, e4}; }
        else if (key == "ngrains") is >> c.ngrains;
        else if (key == "grain_phase_file") is >> grain_phase_file;
        else if (key == "pair_sigma_file") is >> pair_sigma_file;
        else if (key == "pair_mu_file") is >> pair_mu_file;
        else if (key == "dg_file") is >> dg_file;
        else if (key == "orientation_file") is >> orientation_file;
        else if (key == "limiting") { int v; is >> v; c.limiting = v != 0; }
        else if (key == "average") { int v; is >> v; c.average = v != 0; }
        else if (key == "regularization") is >> c.regularization;
        else if (key == "tj_factor") is >> c.tj_factor;
        else if (key == "consider_nucleus_volume") { int v; is >> v; c.consider_nucleus_volume = v != 0; }
        else if (key == "dump_steps") { int s; while (is >> s) c.dump_steps.insert(s); }
        else if (key == "vtk_steps") { int s; while (is >> s) c.vtk_steps.insert(s); }
        else if (key == "restart_grains_file") is >> c.restart_grains;
        else if (key == "threads") is >> c.threads;
        else { fprintf(stderr, "ref_driver: unknown key %s\n", key.c_str()); exit(2); }
    }
    if (c.phase_state.empty()) c.phase_state.assign(c.nphases, "SOLID");
    const size_t G = c.ngrains;
    c.grain_phase = grain_phase_file.empty() ? std::vector<int>(G, 0) : read_ints(grain_phase_file, G);
    if (!orientation_file.empty()) c.quat = read_doubles(orientation_file, 4*G);
    if (!pair_sigma_file.empty()) c.pair_sigma = read_doubles(pair_sigma_file, G*G);
    if (!pair_mu_file.empty())    c.pair_mu    = read_doubles(pair_mu_file, G*G);
    if (!dg_file.empty())         c.dg         = read_doubles(dg_file, G);
    return c;
}

static void write_opi(const Case& c, const std::string& path)
{
    std::ofstream o(path);
    o.precision(17);
    o << "OpenPhase input written by ref_driver\n\n";
    o << "@Settings\n";
    for (int p = 0; p < c.nphases; p++)
    {
        o << "$Phase_" << p << " : Phase" << p << "\n";
        o << "$State_" << p << " : " << c.phase_state[p] << "\n";
    }
    o << "\n@GridParameters\n";
    o << "$Nx : " << c.nx << "\n$Ny : " << c.ny << "\n$Nz : " << c.nz << "\n";
    o << "$dx : " << c.dx << "\n$IWidth : " << c.iwidth << "\n";
    o << "\n@PhaseField\n";
    o << "$PhaseFieldLaplacianStencil : " << c.stencil << "\n";
    o << "$PhaseFieldGradientStencil : ISOTROPIC\n";
    o << "$ConsiderNucleusVolume : " << (c.consider_nucleus_volume ? "Yes" : "No") << "\n";
    o << "\n@InterfaceProperties\n";
    for (int a = 0; a < c.nphases; a++)
    for (int b = a; b < c.nphases; b++)
    {
        std::string model = "ISO";
        auto it = c.energy_model.find({a,b});
        if (it != c.energy_model.end()) model = it->second;
        double s = c.sigma.count({a,b}) ? c.sigma.at({a,b}) : 1.0;
        double m = c.mu.count({a,b}) ? c.mu.at({a,b}) : 1.0;
        o << "$EnergyModel_" << a << "_" << b << " : " << model << "\n";
        o << "$Sigma_" << a << "_" << b << " : " << s << "\n";
        const double e1 = c.cubic_eps.count({a,b}) ? c.cubic_eps.at({a,b}) : 0.0;
        const std::vector<double> ex = c.model_eps.count({a,b}) ? c.model_eps.at({a,b}) : std::vector<double>(3, 0.0);
        const std::string ab = std::to_string(a) + "_" + std::to_string(b);
        if (model == "CUBIC" or model == "HEXBOETTGER") o << "$EpsilonE_" << ab << " : " << e1 << "\n";
        if (model == "HEXSUN")
            o << "$EpsilonE20_" << ab << " : " << e1 << "\n" << "$EpsilonE40_" << ab << " : " << ex[0] << "\n"
              << "$EpsilonE60_" << ab << " : " << ex[1] << "\n" << "$EpsilonE66_" << ab << " : " << ex[2] << "\n";
        if (model == "FACETED" or model == "FACETEDEXP")
        {
            const auto& fs = c.facets.at({a,b});
            const bool fam = c.facet_family.count({a,b}) and c.facet_family.at({a,b});
            o << (fam ? "$NfacetFamilies_" : "$Nfacets_") << ab << " : " << fs.size() << "\n";
            for (size_t n = 0; n < fs.size(); n++)
            {
                o << "$Facet_" << ab << "_" << n << " : " << (long)fs[n][0] << " " << (long)fs[n][1] << " " << (long)fs[n][2] << "\n";
                if (model == "FACETED")
                    o << "$SigmaF_" << ab << "_" << n << " : " << fs[n][3] << "\n"
                      << "$EpsilonEF_" << ab << "_" << n << " : " << fs[n][4] << "\n";
                else
                    o << "$EpsilonEF_" << ab << "_" << n << " : " << fs[n][3] << "\n"
                      << "$PowerEF_" << ab << "_" << n << " : " << fs[n][4] << "\n";
            }
        }
        if (model == "HEXYANG")
            o << "$EpsilonE1_" << ab << " : " << e1 << "\n" << "$EpsilonE2_" << ab << " : " << ex[0] << "\n"
              << "$EpsilonE3_" << ab << " : " << ex[1] << "\n";
        const std::string mmodel = c.mobility_model.count({a,b}) ? c.mobility_model.at({a,b}) : "ISO";
        const std::vector<double> me = c.mobility_eps.count({a,b}) ? c.mobility_eps.at({a,b}) : std::vector<double>(4, 0.0);
        o << "$MobilityModel_" << a << "_" << b << " : " << mmodel << "\n";
        if (mmodel == "CUBIC" or mmodel == "HEXBOETTGER") o << "$EpsilonM_" << ab << " : " << me[0] << "\n";
        if (mmodel == "HEXSUN")
            o << "$EpsilonM20_" << ab << " : " << me[0] << "\n" << "$EpsilonM40_" << ab << " : " << me[1] << "\n"
              << "$EpsilonM60_" << ab << " : " << me[2] << "\n" << "$EpsilonM66_" << ab << " : " << me[3] << "\n";
        if (mmodel == "HEXYANG")
            o << "$EpsilonM1_" << ab << " : " << me[0] << "\n" << "$EpsilonM2_" << ab << " : " << me[1] << "\n"
              << "$EpsilonM3_" << ab << " : " << me[2] << "\n";
        if (mmodel == "FACETED")
        {
            // the energy and mobility models read the same $NfacetFamilies / $Facet keys: a pair
            // with both FACETED shares its facet vectors (not used here)
            const auto& fs = c.mobility_facets.at({a,b});
            const bool fam = c.mobility_facet_family.count({a,b}) and c.mobility_facet_family.at({a,b});
            o << (fam ? "$NfacetFamilies_" : "$Nfacets_") << ab << " : " << fs.size() << "\n";
            for (size_t n = 0; n < fs.size(); n++)
                o << "$Facet_" << ab << "_" << n << " : " << (long)fs[n][0] << " " << (long)fs[n][1] << " " << (long)fs[n][2] << "\n"
                  << "$MuF_" << ab << "_" << n << " : " << fs[n][3] << "\n"
                  << "$EpsilonMF_" << ab << "_" << n << " : " << fs[n][4] << "\n";
        }
        o << "$Mu_" << a << "_" << b << " : " << m << "\n";
    }
    o << "$TripleJunctionModel : MODEL\n";
    o << "$TripleJunctionFactor : " << c.tj_factor << "\n";
    o << "$RegularizationFactor : " << c.regularization << "\n";
    o << "\n@DrivingForce\n";
    o << "$Average : " << (c.average ? "Yes" : "No") << "\n";
    o << "$Limiting : " << (c.limiting ? "Yes" : "No") << "\n";
    for (int a = 0; a < c.nphases; a++)
    for (int b = a; b < c.nphases; b++)
    {
        double l = c.limit.count({a,b}) ? c.limit.at({a,b}) : 0.95;
        o << "$Limit_" << a << "_" << b << " : " << l << "\n";
    }
    o << "\n@BoundaryConditions\n";
    o << "$BC0X : Periodic\n$BCNX : Periodic\n$BC0Y : Periodic\n$BCNY : Periodic\n";
    o << "$BC0Z : Periodic\n$BCNZ : Periodic\n";
    o << "\n@DoubleObstacle\n\n";
}

static void write_doubles(const std::string& path, const std::vector<double>& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), v.size()*sizeof(double));
}

static void dump(const Case& c, PhaseField& Phi, const std::string& out, int step)
{
    const std::string tag = std::to_string(step);
    Phi.Write(out + "/PF_" + tag + ".dat");
    std::vector<double> V(c.ngrains), VR(c.ngrains);
    for (int g = 0; g < c.ngrains; g++)
    {
        V[g]  = Phi.FieldsProperties[g].Volume;
        VR[g] = Phi.FieldsProperties[g].VolumeRatio;
    }
    write_doubles(out + "/V_" + tag + ".bin", V);
    write_doubles(out + "/VR_" + tag + ".bin", VR);
    // grain records in the restart format (GrainsProperties::Write, include/GrainsProperties.h:762-792)
    Phi.FieldsProperties.Write(out + "/FP_" + tag + ".dat");
}

int main(int argc, char* argv[])
{
    if (argc < 4)
    {
        fprintf(stderr, "usage: ref_driver <case.txt> <initial_raw.dat> <out_dir>\n");
        return 2;
    }
    const Case c = parse_case(argv[1]);
    const std::string raw_in = argv[2];
    const std::string out = argv[3];
    const std::string opi = out + "/ProjectInput.opi";
    write_opi(c, opi);
    if (c.threads > 0) omp_set_num_threads(c.threads);

    Settings S;
    S.ReadInput(opi);
    PhaseField          Phi(S, opi);
    DoubleObstacle      DO(S, opi);
    InterfaceProperties IP(S, opi);
    DrivingForce        dG(S, opi);
    BoundaryConditions  BC(S, opi);

    for (int g = 0; g < c.ngrains; g++) Phi.AddGrainInfo(c.grain_phase[g]);
    if (!c.quat.empty())
    {
        // grain orientations (s, x, y, z) per grain: GrainsProperties::Orientation
        // (include/GrainsProperties.h:76) with its rotation matrix
        const std::vector<double>& q = c.quat;
        for (int g = 0; g < c.ngrains; g++)
            Phi.FieldsProperties[g].Orientation = Quaternion({q[4*g], q[4*g + 1], q[4*g + 2], q[4*g + 3]});
    }
    if (!Phi.Read(raw_in)) { fprintf(stderr, "ref_driver: Read failed\n"); return 3; }
    if (c.restart_grains.empty())
    {
        Phi.FinalizeInitialization(BC);
    }
    else
    {
        // restart: the raw state plus the grain records, then Finalize
        // (PhaseField::Read(Settings, BC, tStep), src/PhaseField.cpp:2541-2554)
        if (!Phi.FieldsProperties.Read(c.restart_grains)) { fprintf(stderr, "ref_driver: grains Read failed\n"); return 3; }
        Phi.Finalize(BC);
    }
    S.VTKDir = out + "/";
    if (c.dump_steps.count(0)) dump(c, Phi, out, 0);
    if (c.vtk_steps.count(0)) Phi.WriteVTK(S, 0);

    const bool use_pair = !c.pair_sigma.empty();
    const bool use_dg   = !c.dg.empty();
    const size_t G = c.ngrains;

    std::vector<long> wide(c.nsteps + 1, 0);
    std::vector<double> step_seconds(c.nsteps + 1, 0.0);
    double t_loop = 0.0;
    for (int step = 1; step <= c.nsteps; step++)
    {
        const double t0 = omp_get_wtime();
        if (use_dg) dG.Clear();
        IP.Set(Phi, BC);
        if (use_pair)
        {
            // Per-grain-pair sigma/mu: written into the public per-voxel interface property
            // storage for every pair of every wide-interface voxel (InterfaceProperties.h:97,
            // NodeIP::set_energy_and_mobility NodeIP.h:413-431).
            OMP_PARALLEL_STORAGE_LOOP_BEGIN(i,j,k,Phi.Fields,0,)
            {
                if (Phi.Fields(i,j,k).wide_interface())
                for (auto a = Phi.Fields(i,j,k).cbegin(); a != Phi.Fields(i,j,k).cend(); ++a)
                for (auto b = a + 1; b != Phi.Fields(i,j,k).cend(); ++b)
                {
                    const size_t ga = a->index, gb = b->index;
                    const double s = c.pair_sigma[ga*G + gb];
                    const double m = c.pair_mu.empty() ? IP.Properties(i,j,k).get_mobility(ga, gb)
                                                       : c.pair_mu[ga*G + gb];
                    IP.Properties(i,j,k).set_energy_and_mobility(ga, gb, s, m);
                }
            }
            OMP_PARALLEL_STORAGE_LOOP_END
        }
        if (use_dg)
        {
            // Per-grain stored-energy driving force: raw(a,b) = dG_b - dG_a for every pair
            // (a before b in the voxel's list) of every interface voxel; positive raw grows a.
            // Idiom of src/UserDrivingForce.cpp:152-175.
            OMP_PARALLEL_STORAGE_LOOP_BEGIN(i,j,k,Phi.Fields,0,)
            {
                if (Phi.Fields(i,j,k).interface())
                for (auto a = Phi.Fields(i,j,k).cbegin(); a != Phi.Fields(i,j,k).cend(); ++a)
                for (auto b = a + 1; b != Phi.Fields(i,j,k).cend(); ++b)
                {
                    dG.Force(i,j,k).add_raw(a->index, b->index, c.dg[b->index] - c.dg[a->index]);
                }
            }
            OMP_PARALLEL_STORAGE_LOOP_END
            dG.Average(Phi, BC);
            DO.CalculatePhaseFieldIncrements(Phi, IP, dG);
            dG.MergePhaseFieldIncrements(Phi, IP);
        }
        else
        {
            DO.CalculatePhaseFieldIncrements(Phi, IP);
        }
        Phi.NormalizeIncrements(BC, c.dt);
        Phi.MergeIncrements(BC, c.dt);
        step_seconds[step] = omp_get_wtime() - t0;
        t_loop += step_seconds[step];

        long w = 0;
        #pragma omp parallel for collapse(3) reduction(+:w)
        for (int i = 0; i < c.nx; i++)
        for (int j = 0; j < c.ny; j++)
        for (int k = 0; k < c.nz; k++)
        {
            if (Phi.Fields(i,j,k).wide_interface()) w++;
        }
        wide[step] = w;
        if (c.dump_steps.count(step)) dump(c, Phi, out, step);
        if (c.vtk_steps.count(step)) Phi.WriteVTK(S, step);
    }

    std::ofstream st(out + "/stats.txt");
    st.precision(17);
    st << "threads " << omp_get_max_threads() << "\n";
    st << "step_loop_seconds " << t_loop << "\n";
    st << "nsteps " << c.nsteps << "\n";
    st << "wide";
    for (int s = 1; s <= c.nsteps; s++) st << " " << wide[s];
    st << "\n";
    st << "step_seconds";
    for (int s = 1; s <= c.nsteps; s++) st << " " << step_seconds[s];
    st << "\n";
    return 0;
}
