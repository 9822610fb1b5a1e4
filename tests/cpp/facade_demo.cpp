// facade_demo.cpp — drives the library through the C++ facade (include/dfsph.hpp) the way the
// reference's callers drive SPH::DFSPHCUDA: construct from a scene, step(), read the state back.
// Test program: tests/test_cpp_facade.py writes the scene, runs this and compares with the Python
// facade.
//
//   facade_demo <scene.bin> <steps> <out.bin>
//
// scene.bin: int32 n_fluid, int32 n_boundary, float64 config[10] = {r, rho0, viscosity, dt,
// max_error, max_error_v, cfl_method, precision, cfl_factor, cfl_max_time_step}, float32 fluid[3 n],
// float32 boundary[3 nb].
// out.bin: for the fused step() run then for the piecewise cuda_* run: int32 n, float32 pos[3 n],
// float32 vel[3 n], then int32 iterations_sum and iterations_v_sum of the fused run.
// Exit codes: 0 ok, 2 usage / input error, 3 dfsph::Error (message on stderr).
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "dfsph.hpp"

namespace {
template <class T> bool rd(std::ifstream& f, T* p, size_t n) {
    return (bool)f.read(reinterpret_cast<char*>(p), (std::streamsize)(n * sizeof(T)));
}
template <class T> void wr(std::ofstream& f, const T* p, size_t n) {
    f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
}
void dump(std::ofstream& f, dfsph::DFSPHCData& d) {
    std::vector<float> x, v;
    d.readDynamicData(x, v);
    const int32_t n = (int32_t)(x.size() / 3);
    wr(f, &n, 1);
    wr(f, x.data(), x.size());
    wr(f, v.data(), v.size());
}
}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        std::cerr << "usage: facade_demo <scene.bin> <steps> <out.bin>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t n = 0, nb = 0;
    double cfg[10];
    if (!rd(in, &n, 1) || !rd(in, &nb, 1) || !rd(in, cfg, 10) || n < 0 || nb < 0) {
        std::cerr << "bad scene file\n";
        return 2;
    }
    std::vector<float> fluid(3 * (size_t)n), boundary(3 * (size_t)nb);
    if (!rd(in, fluid.data(), fluid.size()) || !rd(in, boundary.data(), boundary.size())) {
        std::cerr << "truncated scene file\n";
        return 2;
    }
    const int steps = std::atoi(argv[2]);
    try {
        dfsph_scene s;
        dfsph::check(nullptr, dfsph_scene_defaults(&s));
        s.particle_radius = cfg[0];
        s.density0 = cfg[1];
        s.viscosity = cfg[2];
        s.time_step = cfg[3];
        s.max_error = cfg[4];
        s.max_error_v = cfg[5];
        s.cfl_method = (int32_t)cfg[6];
        s.precision = (int32_t)cfg[7];
        s.cfl_factor = cfg[8];
        s.cfl_max_time_step = cfg[9];
        dfsph::DFSPHCUDA fused(s, fluid, boundary);
        dfsph::DFSPHCUDA piecewise(s, fluid, boundary);
        if (fused.getMaxError() != cfg[4] || fused.getCflMethod() != (unsigned)cfg[6]) {
            std::cerr << "parameters not applied\n";
            return 2;
        }
        int32_t its = 0, itv = 0;
        for (int k = 0; k < steps; ++k) {
            fused.step();
            its += (int32_t)fused.getIterationCount();
            itv += (int32_t)fused.getIterationCountV();
            // the sequence of DFSPHCUDA::step through the host functions of DFSPH_core_cuda.h
            dfsph::DFSPHCData& d = piecewise.m_data;
            dfsph::cuda_neighborsSearch(d, true);
            dfsph::cuda_divergenceSolve(d, piecewise.getMaxIterationsV(), piecewise.getMaxErrorV());
            dfsph::cuda_externalForces(d);
            if (piecewise.getCflMethod() != 0)
                dfsph::cuda_CFL(d, 0.0001, piecewise.getCflFactor(), piecewise.getCflMaxTimeStepSize());
            else
                d.updateTimeStep(cfg[3]);
            dfsph::cuda_update_vel(d);
            dfsph::cuda_pressureSolve(d, piecewise.getMaxIterations(), piecewise.getMaxError());
            dfsph::cuda_update_pos(d);
            d.onSimulationStepEnd();
        }
        std::ofstream out(argv[3], std::ios::binary);
        dump(out, fused.m_data);
        dump(out, piecewise.m_data);
        wr(out, &its, 1);
        wr(out, &itv, 1);
        std::cout << "steps " << steps << " fluid " << fused.m_data.getFluidParticlesCount() << " iterations "
                  << its << " " << itv << " h " << fused.m_data.h() << "\n";
    } catch (const dfsph::Error& e) {
        std::cerr << e.what() << "\n";
        return 3;
    }
    return 0;
}
