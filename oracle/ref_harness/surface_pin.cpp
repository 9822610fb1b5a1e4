// surface_pin.cpp — runs the reference's own BufferFluidSurface (SPlisHSPlasH/DFSPH/BufferFluidSurface.cu,
// the shapes of the simple open boundary) on the host: its __host__ __device__ members compile as host
// code. Test infrastructure only: the open-boundary pins compare the oracle's restatement of
// isinside / getNormal with it. The mesh shape's class needs managed memory, so pin_mesh_inside runs
// the steps of MeshPerso::isInside (BufferFluidSurface.cu:224-270: the box of the vertices and the
// origin, the fixed ray, the reference's own RayIntersectsTriangle) on host arrays.
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

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

// The triangles MeshPerso::loadFromFile reads (OBJ_Loader, its first mesh): 9 floats per triangle,
// the three vertex positions in index order. out null: only the count.
int pin_obj_triangles(const char* path, float* out, uint32_t cap, uint32_t* count) {
    objl::Loader L;
    if (!L.LoadFile(path) || L.LoadedMeshes.empty()) return -1;
    const objl::Mesh& m = L.LoadedMeshes[0];
    const uint32_t nt = (uint32_t)(m.Indices.size() / 3);
    *count = nt;
    if (!out) return 0;
    if (cap < nt) return -2;
    for (uint32_t t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k) {
            const objl::Vector3& q = m.Vertices[m.Indices[3 * t + k]].Position;
            out[9 * t + 3 * k] = q.X;
            out[9 * t + 3 * k + 1] = q.Y;
            out[9 * t + 3 * k + 2] = q.Z;
        }
    return 0;
}

// MeshPerso::isInside for the mesh (vertices v[3 nv], triangles t[3 nt]) moved by offset[3].
int pin_mesh_inside(const float* v, uint32_t nv, const uint32_t* t, uint32_t nt, const float* offset,
                    const float* p, uint32_t n, uint8_t* inside) {
    Vector3d bmin(0, 0, 0), bmax(0, 0, 0);
    std::vector<Vector3d> V(nv);
    for (uint32_t i = 0; i < nv; ++i) {
        V[i] = Vector3d(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        bmin.toMin(V[i]);
        bmax.toMax(V[i]);
    }
    const Vector3d off(offset[0], offset[1], offset[2]);
    Vector3d u(2.575, 6.19763, 5.986);
    u.toUnit();
    for (uint32_t k = 0; k < n; ++k) {
        const Vector3d x(p[3 * k], p[3 * k + 1], p[3 * k + 2]);
        if ((x < bmin + off) || x > bmax + off) {
            inside[k] = 0;
            continue;
        }
        int count = 0;
        for (uint32_t f = 0; f < nt; ++f) {
            Vector3d ip(0);
            RealCuda dist = 0;
            if (RayIntersectsTriangle<true, false>(x, u, V[t[3 * f]] + off, V[t[3 * f + 1]] + off, V[t[3 * f + 2]] + off,
                                                   ip, dist)) {
                if (dist > 0) count++;
            }
        }
        inside[k] = (count & 1) ? 1 : 0;
    }
    return 0;
}
}
