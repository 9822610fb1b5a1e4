// driver.cpp — headless driver of the reference CPU solver SPH::TimeStepDFSPH (test infrastructure:
// the timed CPU baseline and a physics pin of the oracle). It replaces the GUI application's
// DemoBase::buildModel (Demos/Common/DemoBase.cpp:400-513) for one scene: fluid points, one static
// wall body given as sample points, the XSPH viscosity, the given kernel (0 = analytic cubic,
// 3 = the reference default 10000-sample table), then runs TimeStepDFSPH::step().
//
// usage: dfsph_ref <input.bin> <output.bin>
// input:  "DFRF" int32 version=1; doubles r, rho0, viscosity, gx, gy, gz, dt, max_error, max_error_v,
//         mass; int32 max_iter, max_iter_v, enable_div, kernel, n_fluid, n_boundary, warmup, steps;
//         double time_budget_s; float32 fluid xyz[3 n_fluid], boundary xyz[3 n_boundary]
// output: int32 steps_done; double ms_per_step; int32 iterations[steps_done], iterations_v[steps_done];
//         then, in original particle order: double x[3n], v[3n], density[n], factor[n], psi[nb]
//
// The reference step appends to fluid_simulation_timmings_cpu.csv in the working directory and
// exits once the simulation time passes 5 s (SPlisHSPlasH/DFSPH/TimeStepDFSPH.cpp:98-125): run it in
// a scratch directory; the driver resets the simulation time before every step.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "SPlisHSPlasH/Common.h"
#include "SPlisHSPlasH/DFSPH/TimeStepDFSPH.h"
#include "SPlisHSPlasH/DFSPH/SimulationDataDFSPH.h"
#include "SPlisHSPlasH/FluidModel.h"
#include "SPlisHSPlasH/StaticRigidBody.h"
#include "SPlisHSPlasH/TimeManager.h"
#include "SPlisHSPlasH/Viscosity/ViscosityBase.h"

using namespace SPH;

namespace {
template <class T> T rd(std::ifstream& f) {
    T v;
    f.read(reinterpret_cast<char*>(&v), sizeof(T));
    return v;
}
}  // namespace

// Exposes the per-particle arrays of the solver's simulation data for the final dump.
class DumpableDFSPH : public TimeStepDFSPH {
public:
    using TimeStepDFSPH::TimeStepDFSPH;
    SimulationDataDFSPH& data() { return m_simulationData; }
};

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: dfsph_ref <input.bin> <output.bin>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    char magic[4];
    in.read(magic, 4);
    if (std::memcmp(magic, "DFRF", 4) != 0 || rd<int32_t>(in) != 1) {
        std::cerr << "bad input\n";
        return 2;
    }
    const double r = rd<double>(in), rho0 = rd<double>(in), visc = rd<double>(in);
    const double gx = rd<double>(in), gy = rd<double>(in), gz = rd<double>(in);
    const double dt = rd<double>(in), max_err = rd<double>(in), max_err_v = rd<double>(in), mass = rd<double>(in);
    const int max_it = rd<int32_t>(in), max_it_v = rd<int32_t>(in), enable_div = rd<int32_t>(in);
    const int kernel = rd<int32_t>(in), n = rd<int32_t>(in), nb = rd<int32_t>(in);
    const int warmup = rd<int32_t>(in), steps = rd<int32_t>(in);
    const double budget = rd<double>(in);
    std::vector<float> fx(3 * (size_t)n), bx(3 * (size_t)nb);
    in.read(reinterpret_cast<char*>(fx.data()), fx.size() * sizeof(float));
    in.read(reinterpret_cast<char*>(bx.data()), bx.size() * sizeof(float));
    if (!in) {
        std::cerr << "truncated input\n";
        return 2;
    }

    TimeManager::getCurrent()->setTimeStepSize(dt);
    FluidModel model;
    model.setParticleRadius(r);
    std::vector<Vector3r> bpts(nb), fpts(n), fvel(n, Vector3r::Zero());
    for (int i = 0; i < nb; ++i) bpts[i] = Vector3r(bx[3 * i], bx[3 * i + 1], bx[3 * i + 2]);
    for (int i = 0; i < n; ++i) fpts[i] = Vector3r(fx[3 * i], fx[3 * i + 1], fx[3 * i + 2]);
    StaticRigidBody* rb = new StaticRigidBody();
    model.addRigidBodyObject(rb, (unsigned int)nb, bpts.data());
    model.initModel((unsigned int)n, fpts.data(), fvel.data(), 0);
    model.setKernel(kernel);
    model.setGradKernel(kernel);
    DumpableDFSPH* sim = new DumpableDFSPH(&model);
    sim->setMaxIterations(max_it);
    sim->setMaxError(max_err);
    sim->setMaxIterationsV(max_it_v);
    sim->setMaxErrorV(max_err_v);
    if (sim->getViscosityBase()) sim->getViscosityBase()->setViscosity(visc);
    model.setDensity0(rho0);  // FluidModel::initMasses (0.8 rho0 (2r)^3) + boundary psi
    if (mass > 0.0)
        for (int i = 0; i < n; ++i) model.setMass(i, mass);
    model.setGravitation(Vector3r(gx, gy, gz));
    sim->setEnableDivergenceSolver(enable_div != 0);

    std::vector<int32_t> its, itsv;
    for (int s = 0; s < warmup; ++s) {
        TimeManager::getCurrent()->setTime(0.0);
        sim->step();
    }
    const auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    for (int s = 0; s < steps; ++s) {
        TimeManager::getCurrent()->setTime(0.0);
        sim->step();
        its.push_back((int32_t)sim->getIterationCount());
        itsv.push_back((int32_t)sim->getIterationCountV());
        ++done;
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (budget > 0.0 && el > budget && done >= 1) break;
    }
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    std::ofstream out(argv[2], std::ios::binary);
    const int32_t d32 = done;
    const double ms = done ? total * 1e3 / done : 0.0;
    out.write(reinterpret_cast<const char*>(&d32), 4);
    out.write(reinterpret_cast<const char*>(&ms), 8);
    out.write(reinterpret_cast<const char*>(its.data()), 4 * its.size());
    out.write(reinterpret_cast<const char*>(itsv.data()), 4 * itsv.size());
    // dump in original particle order (the solver z-sorts particles every 500 steps)
    const auto& orig = model.getNeighborhoodSearch()->point_set(0).original_index();
    std::vector<double> X(3 * (size_t)n), V(3 * (size_t)n), D(n), F(n), P(nb);
    for (int i = 0; i < n; ++i) {
        const unsigned int o = orig.empty() ? (unsigned int)i : orig[i];
        for (int a = 0; a < 3; ++a) {
            X[3 * (size_t)o + a] = model.getPosition(0, i)[a];
            V[3 * (size_t)o + a] = model.getVelocity(0, i)[a];
        }
        D[o] = model.getDensity(i);
        F[o] = sim->data().getFactor(i);
    }
    for (int i = 0; i < nb; ++i) P[i] = model.getRigidBodyParticleObject(0)->m_boundaryPsi[i];
    out.write(reinterpret_cast<const char*>(X.data()), 8 * X.size());
    out.write(reinterpret_cast<const char*>(V.data()), 8 * V.size());
    out.write(reinterpret_cast<const char*>(D.data()), 8 * D.size());
    out.write(reinterpret_cast<const char*>(F.data()), 8 * F.size());
    out.write(reinterpret_cast<const char*>(P.data()), 8 * P.size());
    return out ? 0 : 1;
}
