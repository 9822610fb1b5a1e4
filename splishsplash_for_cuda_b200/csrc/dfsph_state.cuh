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
    // Force of the fluid on each boundary particle, x, y, z, accumulated as 64-bit fixed point
    // (kForceScale units per newton): integer additions commute, so the sums do not depend on the
    // order in which the atomics land (null: not accumulated).
    unsigned long long* bforce;
    // reductions and control
    double* partials;      // one FP64 partial per block
    LoopCtl* ctl;          // [0] divergence loop, [1] pressure loop, [2] CFL / misc, [3] candidate probe
    double* dtd;           // dt history in FP64 (see DtSlot); the kernels read their Real copies in p
    uint32_t* status;      // [0] DFSPH_ST_* bits, [1] scratch, [2] learned warm start kept (bit 0 div, 1 pressure)
    float* cfl_partials;   // per-block max |v + a h|^2
    // learned warm start (see mlp.cuh)
    float* features;       // kMlpIn per particle, written by the density+alpha pass
    float* pred;           // 2 per particle: network outputs (normalised corrections)
    Real* kappaT;          // previous step's total applied kappa (warm start + corrections)
    Real* kappaVT;         // previous step's total applied kappa_v
    Real* kappaW;          // warm-start value used by this step's pressure solve
    Real* kappaVW;         // warm-start value used by this step's divergence solve
    Real* kappaP;          // plain (reference) pressure warm-start candidate
    Real* kappaVP;         // plain (reference) divergence warm-start candidate
    Vec4<Real>* velP;      // velocities after the plain candidate's warm-start pass (probe)
    Real* resid;           // unclamped density residual of the last pressure pass (null: not kept)
    Real* residV;          // unclamped divergence residual of the last divergence pass (null: not kept)
    Real* dadvP;           // plain candidate's clamped init residual (both candidates in one pass)
    Real* kcP;             // plain candidate's Jacobi coefficient
    Real* rawP;            // plain candidate's unclamped init residual
    const float* out_scale;  // 2 floats: scales of the network outputs
};

// ---- launch wrappers (neighbors.cu) ----------------------------------------------------------------
template <class Real>
// clear0 / clear1 (words0 / words1 32-bit words each, may be null / 0): buffers the same launch sets
// to zero (the fluid cell table and the sort's workspace before a fluid binning).
void launch_cell_keys(const Vec4<Real>* pos, uint32_t n, const StepParams<Real>& p, uint32_t* keys, uint32_t* status,
                      cudaStream_t s, uint32_t* clear0 = nullptr, size_t words0 = 0, uint32_t* clear1 = nullptr,
                      size_t words1 = 0);
template <class Real>
void launch_reorder_fluid(const uint32_t* perm, uint32_t n, const Vec4<Real>* pos_in, const Vec4<Real>* vel_in,
                          const Real* kappa_in, const Real* kappaV_in, const uint32_t* id_in, Vec4<Real>* pos_out,
                          Vec4<Real>* vel_out, Real* kappa_out, Real* kappaV_out, uint32_t* id_out, cudaStream_t s);
// Reorders two more per-particle arrays by the same permutation (learned warm-start totals).
template <class Real>
void launch_reorder_pair(const uint32_t* perm, uint32_t n, const Real* a_in, const Real* b_in, Real* a_out,
                         Real* b_out, cudaStream_t s);
void launch_cell_bounds(const uint32_t* sorted_keys, uint32_t n, int dim_x, int dim_y, int dim_z, uint2* table,
                        cudaStream_t s);
template <class Real>
void launch_build_neighbors(const DevState<Real>* d, uint32_t n, const uint2* fluid_table, const uint2* boundary_table,
                            cudaStream_t s, bool boundary_shifted = false);
// Checked builds only (no-ops otherwise): particle 0's first list entry := value; the range check of
// every list entry and count (DFSPH_ST_INDEX, the offending particle's list emptied).
void launch_corrupt_first_neighbor(uint32_t* nbr, const uint32_t* counts, uint32_t value, cudaStream_t s);
void launch_validate_neighbors(uint32_t* counts, const uint32_t* nbr, uint32_t n, uint32_t n_boundary, uint32_t stride,
                               uint32_t cap, uint32_t* status, cudaStream_t s);
constexpr bool kCheckedBuild =
#ifdef DFSPH_CHECKED
    true;
#else
    false;
#endif
template <class Real>
void launch_boundary_psi(const Vec4<Real>* bpos_in, Vec4<Real>* bpos_out, uint32_t nb, const StepParams<Real>& p,
                         const uint2* boundary_table, uint32_t* status, cudaStream_t s);
template <class Real>
void launch_scatter_by_id(const uint32_t* id, uint32_t n, const Real* src, int comps, int src_stride, Real* dst,
                          cudaStream_t s);

// ---- launch wrappers (solver.cu) ------------------------------------------------------------------
// warm_v: scale kappa_v into the reference warm start; features: write the MLP inputs instead.
template <class Real>
void launch_density_alpha(const DevState<Real>* d, uint32_t n, bool warm_v, bool features, cudaStream_t s);
// kw: warm-start coefficients (null = kappa_v); vout: output velocities (null = in place).
template <class Real>
void launch_divergence_warm_jacobi(const DevState<Real>* d, uint32_t n, const Real* kw, Vec4<Real>* vout,
                                   cudaStream_t s, bool forces = false);
// Sum of the divergence (which = 0) or density (which = 1) residual of velocities `vel`, into ctl[3]
// (no other write): the initial residual of a warm-start candidate.
template <class Real>
void launch_probe_residual(const DevState<Real>* d, uint32_t n, int which, const Vec4<Real>* vel, cudaStream_t s);
// Warm-start candidates: which = 0 divergence (kappa_v), 1 pressure (kappa). Writes the plain
// (reference) candidate to kappaVP / kappaP and, when learned, the learned one to kappa_v + kappaVW /
// kappaW (otherwise the plain one there too).
template <class Real>
void launch_warm_values(const DevState<Real>* d, uint32_t n, int which, bool learned, bool use_pred, double damping,
                        cudaStream_t s);
// kappaT / kappaVT = the pressure / divergence coefficients this step's solves needed: applied
// totals (warm start + corrections) less the excess the unclamped final residuals show.
template <class Real> void launch_restore_totals(const DevState<Real>* d, uint32_t n, cudaStream_t s);
template <class Real> void launch_totals(const DevState<Real>* d, uint32_t n, bool div_ran, cudaStream_t s);
// Training pairs of `batch` particles spread over [0, n): x = features, t = targets
// [(needed kappa)/r2 - kappaT_prev, (needed kappa_v)/hr - kappaVT_prev] / out_scale.
template <class Real>
void launch_gather_training(const DevState<Real>* d, uint32_t n, uint32_t batch, uint32_t offset, bool div_ran, float* x,
                            float* t, cudaStream_t s);
// keep: also store the unclamped residual in residV (learned warm start).
template <class Real>
void launch_divergence_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                                cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s, bool keep = false);
template <class Real>
void launch_divergence_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                              cudaStream_t s, bool forces = false);
template <class Real> void launch_viscosity(const DevState<Real>* d, uint32_t n, bool cfl, cudaStream_t s);
template <class Real> void launch_update_vel(const DevState<Real>* d, uint32_t n, cudaStream_t s);
// kw null: kappa scaled by (h/h_f)^2 and clamped (reference warm start); otherwise the given final
// warm-start coefficients. vout: output velocities (null = in place).
template <class Real>
void launch_pressure_warm_jacobi(const DevState<Real>* d, uint32_t n, bool fused_vel, const Real* kw,
                                 Vec4<Real>* vout, cudaStream_t s, bool forces = false);
// keep: also store the unclamped residual in resid (learned warm start).
template <class Real>
void launch_pressure_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                              cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s, bool keep = false);
// Both warm-start candidates in one pass (which = 0 divergence, 1 pressure): the plain candidate
// (kappaVP / kappaP) into velP, the learned one (kappaVW / kappaW) into vel; then their init residuals
// in one pass (learned into the solver's arrays and ctl[0 or 1], plain into dadvP / kcP / rawP and
// ctl[3]); then the selection, which installs the plain candidate if the learned one's sum |r| is
// larger. Replaces the probe + warm-start + init + fallback sequence with three launches.
template <class Real>
void launch_warm_dual(const DevState<Real>* d, uint32_t n, int which, bool fused_vel, cudaStream_t s, bool forces);
template <class Real>
void launch_residual_dual(const DevState<Real>* d, uint32_t n, int which, double eta, int min_it, int max_it,
                          cudaStream_t s);
template <class Real> void launch_select_candidate(const DevState<Real>* d, uint32_t n, int which, cudaStream_t s);
// Fallback init pass of the learned warm start (which = 0 divergence, 1 pressure): if the plain
// candidate's probed residual (ctl[3]) is below the learned candidate's init residual, installs the
// plain candidate and redoes the init pass; otherwise records the learned one as kept (status[2]).
template <class Real>
void launch_fallback_residual(const DevState<Real>* d, uint32_t n, int which, double eta, int min_it, int max_it,
                              cudaStream_t s);
template <class Real>
void launch_pressure_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                            cudaStream_t s, bool forces = false);
template <class Real> void launch_update_pos(const DevState<Real>* d, uint32_t n, cudaStream_t s);
template <class Real> void launch_cfl_reduce(const DevState<Real>* d, uint32_t n_blocks, cudaStream_t s);

inline unsigned grid_for(uint32_t n) { return (n + kBlock - 1) / kBlock; }

}  // namespace dfsph
