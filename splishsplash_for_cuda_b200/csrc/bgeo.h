// bgeo.h — particle files in Houdini's binary geometry format (BGEO v5, as partio writes it).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dfsph {

// Writes n particles: position, velocity (when vxyz is not null), pscale = radius (when radius != 0)
// and id = index, gzip-compressed. False with a message in err on failure.
bool bgeo_write(const std::string& path, uint64_t n, const float* xyz, const float* vxyz, float radius,
                std::string& err);

// Reads positions and, when the file has a "velocity" attribute, velocities (zeros otherwise).
bool bgeo_read(const std::string& path, std::vector<float>& xyz, std::vector<float>& vxyz, bool& has_velocity,
               std::string& err);

}  // namespace dfsph
