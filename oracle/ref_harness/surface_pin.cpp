// surface_pin.cpp — runs the reference's own BufferFluidSurface (SPlisHSPlasH/DFSPH/BufferFluidSurface.cu,
// the shapes of the simple open boundary) on the host: its __host__ __device__ members compile as host
// code. Test infrastructure only: the open-boundary pins compare the oracle's restatement of
// isinside / getNormal with it. The mesh shape is not used (it needs managed memory).
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>

#include <cuda_runtime.h>

#include "SPH_kernels.h"
#include "DFSPH_macro_cuda.h"
using namespace SPH;
#include "BufferFluidSurface.cu"

// Layout of the C ABI's dfsph_surface.
struct PinSurface {
    int32_t type, reversed;
    float origin[3], normal[3], center[3], half_lengths[3];
    float radius, radius_internal;
    uint32_t points;
    float direction[3];
};

extern "C" {

// inside[i] = S.isinside(p_i), normal[3 i..] = S.getNormal(p_i). Returns -1 for an unsupported type.
int pin_surface_eval(const PinSurface* s, const float* p, uint32_t n, uint8_t* inside, float* normal) {
    BufferFluidSurface S;
    const Vector3d c(s->center[0], s->center[1], s->center[2]);
    switch (s->type) {
        case 0: S.setPlane(Vector3d(s->origin[0], s->origin[1], s->origin[2]),
                           Vector3d(s->normal[0], s->normal[1], s->normal[2])); break;
        case 1: S.setCuboid(c, Vector3d(s->half_lengths[0], s->half_lengths[1], s->half_lengths[2])); break;
        case 2: S.setCylinder(c, s->half_lengths[1], s->radius); break;
        case 4: S.setSphere(c, s->radius); break;
        case 5: S.setStar(c, s->half_lengths[1], s->radius, s->radius_internal, s->points,
                          Vector3d(s->direction[0], s->direction[1], s->direction[2])); break;
        default: return -1;
    }
    S.setReversedSurface(s->reversed != 0);
    for (uint32_t i = 0; i < n; ++i) {
        const Vector3d x(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
        inside[i] = S.isinside(x) ? 1 : 0;
        const Vector3d nr = S.getNormal(x);
        normal[3 * i] = nr.x;
        normal[3 * i + 1] = nr.y;
        normal[3 * i + 2] = nr.z;
    }
    return 0;
}
}
