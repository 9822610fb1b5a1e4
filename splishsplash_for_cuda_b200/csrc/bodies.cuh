// bodies.cuh — per-body force and torque of the fluid on boundary bodies (bodies.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dfsph {

// out[6 b + 0..2] = sum of force[u], out[6 b + 3..5] = sum of (pos[u] - centers[b]) x force[u] over
// u in [first[b], first[b] + count[b]) (upload order, 3 doubles per particle). One block per body.
void launch_body_wrench(const double* pos, const double* force, const uint32_t* first, const uint32_t* count,
                        const double* centers, uint32_t n_bodies, double* out, cudaStream_t s);

}  // namespace dfsph
