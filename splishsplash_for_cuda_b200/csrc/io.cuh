// io.cuh — launch wrappers of io.cu.
#pragma once
#include "dfsph_state.cuh"

namespace dfsph {

// Publishes the host's DevState block. The dt fields of p are kept from the device: the dt history
// lives on the device (DtSlot) and only launch_dt changes it.
template <class Real> void launch_set_state(DevState<Real>* dst, const DevState<Real>& v, cudaStream_t s);

// Slots of the FP64 dt block (DevState::dtd).
enum DtSlot { kDtH = 0, kDtHFuture, kDtHPast, kDtInvH, kDtInvHFuture, kDtRatio, kDtRatio2, kDtFixed, kDtRatioUsedV,
              kDtRatio2UsedP, kDtSlots };
struct DtArgs {
    double v[kDtSlots];
};
// op 0: set every slot from a; op 1: h_future = a.v[0] (or the fixed step kDtFixed if a.v[0] <= 0);
// op 2: CFL (cuda_CFL, DFSPH_core_cuda.cu:3321-3394): h_future = factor 0.4 diameter / sqrt(max |v + a h|^2)
// from ctl[2].sum, clamped to [min, max] (a.v = factor, min, max, diameter); op 3: onSimulationStepEnd.
// Ops 1 and 2 then set 1/h_future and the ratios (DFSPHCData::updateTimeStep,
// DFSPH_c_arrays_structure.cpp:1100-1112), all in FP64, and refresh the Real copies in p.
template <class Real> void launch_dt(DevState<Real>* d, int op, const DtArgs& a, cudaStream_t s);

// Writes n particles (positions, optional velocities and masses; kappa and kappa_v zero) at pos..,
// with ids id0, id0 + 1, ...
template <class Real>
void launch_unpack_fluid(const float* xyz, const float* vxyz, const float* mass, float default_mass, uint32_t n,
                         Vec4<Real>* pos, Vec4<Real>* vel, Real* kappa, Real* kappaV, uint32_t* id, cudaStream_t s,
                         uint32_t id0 = 0);
// Overwrites positions (xyz not null) and, with set_vel, velocities (zero for a null vxyz) of the
// particles, both given in id order.
template <class Real>
void launch_update_fluid(const float* xyz, const float* vxyz, uint32_t n, const uint32_t* id, Vec4<Real>* pos,
                         Vec4<Real>* vel, cudaStream_t s, bool set_vel = true);
template <class Real>
void launch_unpack_boundary(const float* xyz, const float* psi, uint32_t n, Vec4<Real>* bpos, Vec4<Real>* bvel,
                            cudaStream_t s);
template <class Real>
void launch_reorder_boundary(const uint32_t* perm, uint32_t n, const Vec4<Real>* bpos_in, const Vec4<Real>* bvel_in,
                             Vec4<Real>* bpos_out, Vec4<Real>* bvel_out, uint32_t* bid_out, cudaStream_t s);
template <class Real>
void launch_move_boundary(const float* xyz, const float* vxyz, uint32_t n, const uint32_t* bid, Vec4<Real>* bpos,
                          Vec4<Real>* bvel, cudaStream_t s);
// Rotation (row-major), translation, linear and angular velocity of one rigid range of boundary
// particles (upload indices [first, first + count)).
struct RigidMotion {
    double R[9], p[3], v[3], w[3];
    uint32_t first, count;
};
template <class Real>
void launch_rigid_boundary(const float* rest, uint32_t n, const uint32_t* bid, const RigidMotion& m, Vec4<Real>* bpos,
                           Vec4<Real>* bvel, cudaStream_t s);
// Boundary forces from their fixed-point sums (x, y, z, 0 per particle).
template <class Real>
void launch_force_from_fx(const unsigned long long* fx, uint32_t n, Real* out, cudaStream_t s);
// The dynamic window's stabilisation: particles with id >= first (the ones the last shift added) are
// the tagged ones. save: spos[id] = pos, svel[id] = vel for the untagged; restore: the untagged get
// their saved position and velocity back; damp: the tagged velocities are multiplied by f.
template <class Real>
void launch_save_untagged(const Vec4<Real>* pos, const Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first,
                          Vec4<Real>* spos, Vec4<Real>* svel, cudaStream_t s);
template <class Real>
void launch_restore_untagged(Vec4<Real>* pos, Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first,
                             const Vec4<Real>* spos, const Vec4<Real>* svel, cudaStream_t s);
template <class Real>
void launch_damp_tagged(Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first, Real f, cudaStream_t s);
template <class Real, class Out>
void launch_pack_field(const Real* src, int src_stride, int comps, const uint32_t* id, uint32_t n, Out* dst,
                       cudaStream_t s);
void launch_pack_u32(const uint32_t* src, int comps, const uint32_t* id, uint32_t n, uint32_t* dst, cudaStream_t s);
void launch_unpack_counts(const uint32_t* counts, const uint32_t* id, uint32_t n, uint32_t* dst, cudaStream_t s);

}  // namespace dfsph
