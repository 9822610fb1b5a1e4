// host_ops_demo.cpp — the host-side operations of the reference's SPH::DFSPHCUDA through the C++
// facade (include/dfsph.hpp): handleSimulationSave / handleSimulationLoad, zeroFluidVelocities,
// updateTimeStepDuration, updateRigidBodies, handleDynamicBodiesPause, updateRigidBodiesStateToFile /
// updateRigidBodiesStatefromFile, getFluidImpactOnDynamicBodies, getFluidBoyancyOnDynamicBodies,
// getFluidLevel and handleFLuidLevelControl. Test program:
// tests/test_cpp_facade.py writes the scene, runs this and reads its exit code; the checks are made
// here.
//
//   host_ops_demo <scene.bin> <folder/>
//
// scene.bin as for facade_demo. Exit codes: 0 ok, 1 a check failed (message on stderr), 2 usage /
// input error, 3 dfsph::Error.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <iostream>
#include <vector>

#include "dfsph.hpp"

namespace {
template <class T> bool rd(std::ifstream& f, T* p, size_t n) {
    return (bool)f.read(reinterpret_cast<char*>(p), (std::streamsize)(n * sizeof(T)));
}
int fail(const char* what) {
    std::cerr << "check failed: " << what << "\n";
    return 1;
}
bool close(double a, double b, double tol) { return std::fabs(a - b) <= tol * std::max(1.0, std::fabs(b)); }
}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: host_ops_demo <scene.bin> <folder/>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t n = 0, nb = 0;
    double cfg[10];
    if (!rd(in, &n, 1) || !rd(in, &nb, 1) || !rd(in, cfg, 10) || n <= 0 || nb <= 0) {
        std::cerr << "bad scene file\n";
        return 2;
    }
    std::vector<float> fluid(3 * (size_t)n), boundary(3 * (size_t)nb);
    if (!rd(in, fluid.data(), fluid.size()) || !rd(in, boundary.data(), boundary.size())) {
        std::cerr << "truncated scene file\n";
        return 2;
    }
    try {
        dfsph_scene s;
        dfsph::check(nullptr, dfsph_scene_defaults(&s));
        s.particle_radius = cfg[0];
        s.time_step = cfg[3];
        dfsph::DFSPHCUDA sim(s, fluid, boundary);
        sim.set("boundary_forces", 1);
        for (int k = 0; k < 8; ++k) sim.step();

        // getFluidImpactOnDynamicBodies: the whole boundary as one body, against dfsph_body_wrench
        const double c[3] = {0.5, 0.25, 0.5};
        sim.addDynamicBody(0u, (uint32_t)nb, {c[0], c[1], c[2]});
        std::vector<std::array<double, 3>> F, M;
        sim.getFluidImpactOnDynamicBodies(F, M, {{1.0, 1.0, 1.0}});
        const uint32_t first = 0, count = (uint32_t)nb;
        double ft[6];
        dfsph::check(sim.handle(), dfsph_body_wrench(sim.handle(), 1, &first, &count, c, ft));
        for (int a = 0; a < 3; ++a)
            if (!close(F[0][a], ft[a], 1e-9) || !close(M[0][a], ft[3 + a], 1e-9)) return fail("wrench");
        if (!(F[0][1] < 0.0)) return fail("the fluid pushes the walls down");
        std::vector<std::array<double, 3>> F2, M2;
        sim.getFluidImpactOnDynamicBodies(F2, M2, {{0.5, 1.0, 2.0}});
        if (!close(F2[0][0], 0.5 * F[0][0], 1e-12) || !close(F2[0][1], F[0][1], 1e-12) ||
            !close(F2[0][2], 2.0 * F[0][2], 1e-12))
            return fail("reduction factor");

        // getFluidBoyancyOnDynamicBodies: the vertical force, applied inside the box of the samples
        std::vector<std::array<double, 3>> B, P;
        sim.getFluidBoyancyOnDynamicBodies(B, P);
        if (B[0][0] != 0.0 || B[0][2] != 0.0 || !close(B[0][1], F[0][1], 1e-9)) return fail("buoyancy force");
        for (int a = 0; a < 3; ++a) {
            float lo = boundary[a], hi = boundary[a];
            for (size_t k = a; k < boundary.size(); k += 3) {
                lo = std::min(lo, boundary[k]);
                hi = std::max(hi, boundary[k]);
            }
            if (!(P[0][a] >= lo && P[0][a] <= hi)) return fail("buoyancy point");
        }

        // handleSimulationSave / zeroFluidVelocities / handleSimulationLoad
        std::vector<float> x0, v0, x1, v1, x2, v2;
        sim.m_data.readDynamicData(x0, v0);
        sim.fluid_files_folder = argv[2];
        sim.handleSimulationSave(true, false, true);
        sim.zeroFluidVelocities();
        sim.m_data.readDynamicData(x1, v1);
        if (x1 != x0) return fail("zeroFluidVelocities keeps the positions");
        for (float q : v1)
            if (q != 0.0f) return fail("zeroFluidVelocities");
        sim.handleSimulationLoad(true, true, false, false, false);
        sim.m_data.readDynamicData(x2, v2);
        if (x2.size() != x0.size()) return fail("loaded count");
        for (size_t k = 0; k < x0.size(); ++k)
            if (!close(x2[k], x0[k], 1e-6) || !close(v2[k], v0[k], 1e-6)) return fail("load round trip");

        // updateRigidBodies: the whole boundary translated by 1 mm, no rotation, at rest
        std::vector<double> b0(3 * (size_t)nb), b1(3 * (size_t)nb);
        dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64, b0.data(),
                                                  b0.size(), DFSPH_ORDER_ID));
        sim.updateRigidBodies({{{c[0] + 0.001, c[1], c[2]}, {0.1, 0.0, 0.0}, {0.0, 0.0, 0.0}, {1.0, 0.0, 0.0, 0.0}}});
        dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64, b1.data(),
                                                  b1.size(), DFSPH_ORDER_ID));
        for (size_t k = 0; k < b0.size(); ++k)
            if (!close(b1[k], b0[k] + (k % 3 == 0 ? 0.001 : 0.0), 1e-6)) return fail("updateRigidBodies");
        if (sim.dynamic_bodies[0].position[0] != c[0] + 0.001) return fail("body position");
        std::vector<double> bv(3 * (size_t)nb), b2(3 * (size_t)nb);
        dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_VELOCITY, DFSPH_DTYPE_F64, bv.data(),
                                                  bv.size(), DFSPH_ORDER_ID));
        for (size_t k = 0; k < bv.size(); ++k)
            if (!close(bv[k], k % 3 == 0 ? 0.1 : 0.0, 1e-6)) return fail("rigid velocity");

        // handleDynamicBodiesPause: velocities zero, pose kept
        sim.handleDynamicBodiesPause(true);
        if (!sim.is_dynamic_bodies_paused) return fail("pause flag");
        dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_VELOCITY, DFSPH_DTYPE_F64, bv.data(),
                                                  bv.size(), DFSPH_ORDER_ID));
        dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64, b2.data(),
                                                  b2.size(), DFSPH_ORDER_ID));
        for (size_t k = 0; k < bv.size(); ++k)
            if (bv[k] != 0.0 || !close(b2[k], b1[k], 1e-7)) return fail("handleDynamicBodiesPause");

        // updateRigidBodiesStateToFile: the body-frame positions and the fluid's forces, per particle
        sim.solids_files_folder = argv[2];
        sim.step();
        sim.updateRigidBodiesStateToFile();
        {
            std::vector<double> f(3 * (size_t)nb), x(3 * (size_t)nb);
            dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_FORCE, DFSPH_DTYPE_F64, f.data(),
                                                      f.size(), DFSPH_ORDER_ID));
            dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64,
                                                      x.data(), x.size(), DFSPH_ORDER_ID));
            std::ifstream sf(std::string(argv[2]) + "solids_file.txt");
            int bodies = 0;
            if (!(sf >> bodies) || bodies != 1) return fail("solids_file.txt");
            std::ifstream ff(std::string(argv[2]) + "solid_forces_file_0.txt");
            uint32_t count = 0;
            if (!(ff >> count) || count != (uint32_t)nb) return fail("solid_forces_file_0.txt count");
            double fmax = 0;
            for (double q : f) fmax = std::max(fmax, std::fabs(q));
            for (uint32_t i = 0; i < count; ++i) {
                double v[6];
                for (double& q : v)
                    if (!(ff >> q)) return fail("solid_forces_file_0.txt line");
                for (int a = 0; a < 3; ++a) {
                    const double x0 = x[3 * (size_t)i + a] - sim.dynamic_bodies[0].position[a];
                    if (std::fabs(v[a] - x0) > 1e-5 * std::max(1.0, std::fabs(x0))) return fail("body-frame position");
                    if (std::fabs(v[3 + a] - f[3 * (size_t)i + a]) > 1e-5 * std::fabs(f[3 * (size_t)i + a]) + 1e-9 * fmax)
                        return fail("particle force");
                }
            }
        }

        // updateRigidBodiesStatefromFile: position x y z, velocity, q as x y z w, angular velocity
        {
            const std::string path = std::string(argv[2]) + "update_solids.txt";
            std::ofstream uf(path);
            uf.precision(17);
            uf << c[0] + 0.002 << " " << c[1] << " " << c[2] << " 0 0 0  0 0 0 1  0 0 0\n";
            uf.close();
            sim.updateRigidBodiesStatefromFile(5.0);
            if (std::ifstream(path).good()) return fail("update_solids.txt not removed");
            dfsph::check(sim.handle(), dfsph_download(sim.handle(), DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64,
                                                      b2.data(), b2.size(), DFSPH_ORDER_ID));
            for (size_t k = 0; k < b0.size(); ++k)
                if (!close(b2[k], b0[k] + (k % 3 == 0 ? 0.002 : 0.0), 1e-6)) return fail("updateRigidBodiesStatefromFile");
        }

        // getFluidLevel / handleFLuidLevelControl: a target within 5 cm of the level changes nothing,
        // one 6 cm below it removes every particle above it
        const double level = sim.getFluidLevel();
        if (!(level > 0.0)) return fail("getFluidLevel");
        const uint32_t n_before = sim.m_data.getFluidParticlesCount();
        sim.handleFLuidLevelControl(level + 0.04);
        if (sim.m_data.getFluidParticlesCount() != n_before) return fail("level control near the level");
        sim.handleFLuidLevelControl(level - 0.06);
        std::vector<float> x3, v3;
        sim.m_data.readDynamicData(x3, v3);
        if (!(sim.m_data.getFluidParticlesCount() < n_before)) return fail("level control removal");
        for (size_t k = 1; k < x3.size(); k += 3)
            if (x3[k] > (float)(level - 0.06)) return fail("a particle above the target remains");

        // updateTimeStepDuration
        sim.updateTimeStepDuration(0.00125);
        if (sim.get("time_step") != 0.00125) return fail("updateTimeStepDuration");
        sim.step();
        std::cout << "ok: force " << F[0][0] << " " << F[0][1] << " " << F[0][2] << "\n";
    } catch (const dfsph::Error& e) {
        std::cerr << e.what() << "\n";
        return 3;
    }
    return 0;
}
