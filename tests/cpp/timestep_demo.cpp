// timestep_demo.cpp — a C++ caller written against the reference's SPH::TimeStepDFSPH interface,
// constructed from a reference JSON scene read by the library (no Python): load, step, read back.
// Test program for tests/test_cpp_facade.py.
//
//   timestep_demo <scene.json> <steps> <out.bin>     out.bin: int32 n, float32 pos[3 n], vel[3 n],
//                                                     int32 iterations_sum, iterations_v_sum
//   timestep_demo --load <scene.json>                prints "fluid <n> boundary <nb> radius <r>"
// Exit codes: 0 ok, 2 usage, 3 dfsph::Error (message on stderr).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "dfsph.hpp"

int main(int argc, char** argv) {
    try {
        if (argc == 3 && std::strcmp(argv[1], "--load") == 0) {
            const dfsph::SceneData d = dfsph::SceneData::load(argv[2]);
            std::cout << "fluid " << d.fluid.size() / 3 << " boundary " << d.boundary.size() / 3 << " radius "
                      << d.scene.particle_radius << "\n";
            return 0;
        }
        if (argc != 4) {
            std::cerr << "usage: timestep_demo <scene.json> <steps> <out.bin> | --load <scene.json>\n";
            return 2;
        }
        dfsph::TimeStepDFSPH ts{std::string(argv[1])};
        const int steps = std::atoi(argv[2]);
        int32_t its = 0, itv = 0;
        for (int k = 0; k < steps; ++k) {
            ts.step();
            its += (int32_t)ts.getIterationCount();
            itv += (int32_t)ts.getIterationCountV();
        }
        std::vector<float> x, v;
        ts.m_data.readDynamicData(x, v);
        const int32_t n = (int32_t)(x.size() / 3);
        std::ofstream out(argv[3], std::ios::binary);
        out.write(reinterpret_cast<const char*>(&n), 4);
        out.write(reinterpret_cast<const char*>(x.data()), (std::streamsize)(x.size() * 4));
        out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 4));
        out.write(reinterpret_cast<const char*>(&its), 4);
        out.write(reinterpret_cast<const char*>(&itv), 4);
    } catch (const dfsph::Error& e) {
        std::cerr << e.what() << "\n";
        return 3;
    }
    return 0;
}
