// C entry points over the reference's own PartioReaderWriter (Utilities/PartioReaderWriter.cpp:8-66,
// 189-231) and the vendored partio library it calls (extern/partio/src/lib/io/BGEO.cpp), compiled from
// the reference's sources by the Makefile beside this file. Test infrastructure only: the parity
// tests of the .bgeo reader and writer use it to read what the product writes and to write files for
// the product to read.
#include <cstring>
#include <vector>
#include <cstdio>
#include "Utilities/PartioReaderWriter.h"
#include "Utilities/FileSystem.h"

// Utilities/FileSystem.cpp pulls in platform directory code and md5; the one function the reader
// calls (FileSystem.cpp:157-166, "can the file be opened for reading") is restated here.
bool SPH::FileSystem::fileExists(const std::string& fileName) {
    if (FILE* f = std::fopen(fileName.c_str(), "r")) {
        std::fclose(f);
        return true;
    }
    return false;
}

using SPH::Vector3r;
using SPH::Matrix3r;

extern "C" {

// Positions and velocities of a partio file (velocity zero when the file has none), untransformed.
// Returns the particle count, -1 if the file cannot be read, -2 if cap is too small.
long pin_partio_read(const char* path, float* xyz, float* vxyz, long cap) {
    std::vector<Vector3r> pos, vel;
    if (!SPH::PartioReaderWriter::readParticles(path, Vector3r::Zero(), Matrix3r::Identity(), Real(1), pos, vel))
        return -1;
    const long n = (long)pos.size();
    if (n > cap) return -2;
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            xyz[3 * i + c] = (float)pos[i][c];
            vxyz[3 * i + c] = (float)vel[i][c];
        }
    return n;
}

// The reference's export of a fluid (StaticBoundaryDemo/main.cpp:485-496): position, velocity (when
// vxyz is not null), pscale (when radius != 0) and id, gzip-compressed .bgeo.
void pin_partio_write(const char* path, long n, const float* xyz, const float* vxyz, float radius) {
    std::vector<Vector3r> pos(n), vel(n + 1);  // +1: a non-null velocity pointer also when n == 0
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            pos[i][c] = xyz[3 * i + c];
            if (vxyz) vel[i][c] = vxyz[3 * i + c];
        }
    SPH::PartioReaderWriter::writeParticles(path, (unsigned)n, pos.data(), vxyz ? vel.data() : nullptr, radius);
}
}
