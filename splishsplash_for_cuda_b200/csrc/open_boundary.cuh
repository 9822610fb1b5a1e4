// open_boundary.cuh — the simple open boundary (inflow from a layer of sample positions, outflow
// through the boundary layer above the fluid surface), stable compaction of the fluid, and the
// exclusive scan both use.
#pragma once
#include "dfsph_state.cuh"

namespace dfsph {

// A surface as the kernels see it: the C ABI's description and, for DFSPH_SURFACE_MESH, the mesh
// registered under its id (`points`) in device memory. The mesh is translated by the surface's
// `center` (the reference's MeshPerso offset).
struct SurfaceMesh {
    const float4* tri = nullptr;  // 3 per triangle: vertices 0, 1, 2 (w unused), untranslated
    uint32_t nt = 0;
    float bmin[3] = {0.f, 0.f, 0.f}, bmax[3] = {0.f, 0.f, 0.f};  // box of the vertices and the origin
    float dir[3] = {0.f, 0.f, 0.f};                              // the ray's direction (unit)
};
struct DevSurface {
    dfsph_surface s;
    SurfaceMesh m;
};
inline DevSurface plain_surface(const dfsph_surface& s) {
    DevSurface d;
    d.s = s;
    return d;
}
// The ray direction of the mesh inside test, normalise((2.575, 6.19763, 5.986)) in FP32 with each
// operation rounded (BufferFluidSurface.cu:242-243).
void mesh_ray_direction(float dir[3]);

// Scratch words of exclusive_scan_u32 for n inputs.
inline size_t scan_scratch_words(uint32_t n) { return (size_t)(n / 4096u) + 2u; }

// out[i] = sum of in[0..i) and *total = sum of in[0..n), for n <= 2^32 - 1 with a sum below 2^32.
// scratch: scan_scratch_words(n) words. Deterministic; three launches.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, uint32_t* total,
                        cudaStream_t s);

// keep[i] = 1 for samples outside `interior` and inside `fluid_surface` whose cell lies in the grid
// (OpenBoundariesSimple::init, OpenBoundariesSimple.cu:283-318).
template <class Real>
void launch_open_boundary_select(const float4* samples, uint32_t ns, DevSurface interior, DevSurface fluid_surface,
                                 const StepParams<Real>& p, uint32_t* keep, cudaStream_t s);

// Compacts samples[i] with keep[i] to out[rank[i]].
void launch_compact_samples(const float4* samples, const uint32_t* keep, const uint32_t* rank, uint32_t ns,
                            float4* out, cudaStream_t s);

// Shifts every sample by d (the dynamic-window displacement, OpenBoundariesSimple.cu:527-553).
void launch_shift_samples(float4* samples, uint32_t ns, float dx, float dy, float dz, cudaStream_t s);

// Inflow decision per sample (inflow_with_predefined_positions_kernel, OpenBoundariesSimple.cu:352-470)
// over the binned fluid (fluid_table) and boundary (boundary_table): flag[i] = 1 and vel[i] = the
// kernel-weighted fluid velocity when no fluid particle of the 27 cells is within allowed_distance, the
// density estimate is at most allowed_density and the velocity does not point out of `boundary`.
template <class Real>
void launch_inflow(const DevState<Real>* d, const float4* samples, uint32_t ns, float allowed_distance,
                   float allowed_density, Real mass, DevSurface boundary, const uint2* fluid_table,
                   const uint2* boundary_table, uint32_t* flag, float4* vel, cudaStream_t s);

// Appends the flagged samples at n + rank (ranks past capacity are dropped): position, velocity,
// mass, kappa = kappa_v = 0, id = n + rank; kappaT / kappaVT = 0 when not null.
template <class Real>
void launch_append_inflow(const float4* samples, const float4* svel, const uint32_t* flag, const uint32_t* rank,
                          uint32_t ns, uint32_t n, uint32_t capacity, Real mass, Vec4<Real>* pos, Vec4<Real>* vel,
                          Real* kappa, Real* kappaV, uint32_t* id, Real* kappaT, Real* kappaVT, cudaStream_t s);

// alive[i] = 0 for particles outside `interior` and outside `fluid_surface` (outflow_basic_kernel,
// OpenBoundariesSimple.cu:475-492), 1 otherwise.
template <class Real>
void launch_outflow_tag(const Vec4<Real>* pos, uint32_t n, DevSurface interior, DevSurface fluid_surface,
                        uint32_t* alive, cudaStream_t s);

// Stable compaction of the fluid state (cur -> nxt) keeping the particles with alive[i], and the
// renumbering of ids that keeps them dense and in their previous relative order:
// alive_by_id[id] = alive, new_id = exclusive scan of alive_by_id.
template <class Real>
void launch_compact_fluid(const uint32_t* alive, const uint32_t* dst, uint32_t n, const Vec4<Real>* pos_in,
                          const Vec4<Real>* vel_in, const Real* kappa_in, const Real* kappaV_in, const uint32_t* id_in,
                          const Real* kT_in, const Real* kVT_in, Vec4<Real>* pos_out, Vec4<Real>* vel_out,
                          Real* kappa_out, Real* kappaV_out, uint32_t* id_out, Real* kT_out, Real* kVT_out,
                          cudaStream_t s);
// alive[i] = 0 (and *count += 1) for particles with a coordinate outside [lo, hi]
// (checkParticlesPositions(2), SPH_other_systems_cuda.cu:1242-1281), 1 otherwise.
template <class Real>
void launch_box_tag(const Vec4<Real>* pos, uint32_t n, const float lo[3], const float hi[3], uint32_t* alive,
                    uint32_t* count, cudaStream_t s);
void launch_alive_by_id(const uint32_t* id, const uint32_t* alive, uint32_t n, uint32_t* alive_by_id, cudaStream_t s);
void launch_renumber_ids(uint32_t* id, uint32_t n, const uint32_t* new_id, cudaStream_t s);

}  // namespace dfsph
