// dfsph_state.cuh — the device-resident state block every kernel of the time step reads.
//
// The reference passes DFSPHCData by value to every kernel (DFSPH_core_cuda.cu, e.g. :221) and
// swaps nothing: it sorts into scratch buffers and copies back (cuda_sortData, :2057-2120). Here the
// fluid arrays are double-buffered (the reorder writes the other half, no copy back) and all
// pointers and per-step parameters live in one struct in device memory, refreshed by a small copy
// when they change. Kernels take only a pointer to it, so the divergence and pressure loops can be
// captured once as CUDA graphs and replayed every step.
#pragma once

#include "dfsph_common.cuh"

namespace dfsph {

template <class Real> struct DevState {
    StepParams<Real> p;
    // fluid, current (cell-sorted) order
    Vec4<Real>* pos;       // x, y, z, mass
    Vec4<Real>* vel;       // vx, vy, vz, (unused)
    Real* kappa;           // pressure warm-start accumulator
    Real* kappaV;          // divergence warm-start accumulator
    uint32_t* id;          // stable particle id
    Real* density;         // density deviation rho - rho0 (stored instead of rho: see density_alpha_kernel)
    Real* factor;          // DFSPH alpha
    Real* densityAdv;      // clamped residual (divergence or density)
    Real* kcoef;           // densityAdv * factor, the Jacobi coefficient read by neighbours
    Vec4<Real>* acc;       // non-pressure acceleration
    uint32_t* counts;      // fluid count | boundary count << 16
    uint32_t* nbr;         // interleaved neighbour table nbr[k * nbr_stride + i]
    // boundary, cell-sorted order
    const Vec4<Real>* bpos;  // x, y, z, psi
    const Vec4<Real>* bvel;  // vx, vy, vz, (unused)
    // reductions and control
    double* partials;      // one FP64 partial per block
    LoopCtl* ctl;          // [0] divergence loop, [1] pressure loop, [2] CFL / misc
    uint32_t* status;      // DFSPH_ST_* bits
    float* cfl_partials;   // per-block max |v + a h|^2
    // learned warm start (null when off)
    float* features;       // 4 per particle, written by the density+alpha pass
    float* predicted;      // 2 per particle: kappa, kappa_v predictions
};

// ---- launch wrappers (neighbors.cu) ----------------------------------------------------------------
template <class Real>
void launch_cell_keys(const Vec4<Real>* pos, uint32_t n, const StepParams<Real>& p, uint32_t* keys, uint32_t* status,
                      cudaStream_t s);
template <class Real>
void launch_reorder_fluid(const uint32_t* perm, uint32_t n, const Vec4<Real>* pos_in, const Vec4<Real>* vel_in,
                          const Real* kappa_in, const Real* kappaV_in, const uint32_t* id_in, Vec4<Real>* pos_out,
                          Vec4<Real>* vel_out, Real* kappa_out, Real* kappaV_out, uint32_t* id_out, cudaStream_t s);
void launch_cell_bounds(const uint32_t* sorted_keys, uint32_t n, int dim_x, int dim_y, int dim_z, uint2* table,
                        cudaStream_t s);
template <class Real>
void launch_build_neighbors(const DevState<Real>* d, uint32_t n, const uint2* fluid_table, const uint2* boundary_table,
                            cudaStream_t s);
template <class Real>
void launch_boundary_psi(const Vec4<Real>* bpos_in, Vec4<Real>* bpos_out, uint32_t nb, const StepParams<Real>& p,
                         const uint2* boundary_table, uint32_t* status, cudaStream_t s);
template <class Real>
void launch_scatter_by_id(const uint32_t* id, uint32_t n, const Real* src, int comps, int src_stride, Real* dst,
                          cudaStream_t s);

// ---- launch wrappers (solver.cu) ------------------------------------------------------------------
template <class Real> void launch_density_alpha(const DevState<Real>* d, uint32_t n, bool warm_v, cudaStream_t s);
template <class Real> void launch_divergence_warm_jacobi(const DevState<Real>* d, uint32_t n, cudaStream_t s);
template <class Real>
void launch_divergence_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                                cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s);
template <class Real>
void launch_divergence_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                              cudaStream_t s);
template <class Real> void launch_viscosity(const DevState<Real>* d, uint32_t n, bool cfl, cudaStream_t s);
template <class Real> void launch_update_vel(const DevState<Real>* d, uint32_t n, cudaStream_t s);
template <class Real> void launch_pressure_warm_jacobi(const DevState<Real>* d, uint32_t n, bool fused_vel, cudaStream_t s);
template <class Real>
void launch_pressure_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                              cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s);
template <class Real>
void launch_pressure_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                            cudaStream_t s);
template <class Real> void launch_update_pos(const DevState<Real>* d, uint32_t n, cudaStream_t s);
template <class Real> void launch_cfl_reduce(const DevState<Real>* d, uint32_t n_blocks, cudaStream_t s);

inline unsigned grid_for(uint32_t n) { return (n + kBlock - 1) / kBlock; }

}  // namespace dfsph
