// io.cu — device-side packing between the caller's packed xyz arrays and the solver's SoA layout.
//
// Replaces load_UnifiedParticleSet_cuda / read_UnifiedParticleSet_cuda
// (DFSPH_memory_management_cuda.cu:613-656), which copy AoS Vector3d arrays through managed memory.
#include "io.cuh"

namespace dfsph {

namespace {

template <class Real>
__global__ void __launch_bounds__(kBlock) unpack_fluid_kernel(const float* __restrict__ xyz,
                                                              const float* __restrict__ vxyz,
                                                              const float* __restrict__ mass, float default_mass,
                                                              uint32_t n, Vec4<Real>* __restrict__ pos,
                                                              Vec4<Real>* __restrict__ vel, Real* __restrict__ kappa,
                                                              Real* __restrict__ kappaV, uint32_t* __restrict__ id,
                                                              uint32_t id0) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Vec4<Real> x, v;
    x.x = (Real)xyz[3 * i + 0];
    x.y = (Real)xyz[3 * i + 1];
    x.z = (Real)xyz[3 * i + 2];
    x.w = (Real)(mass ? mass[i] : default_mass);
    v.x = vxyz ? (Real)vxyz[3 * i + 0] : Real(0);
    v.y = vxyz ? (Real)vxyz[3 * i + 1] : Real(0);
    v.z = vxyz ? (Real)vxyz[3 * i + 2] : Real(0);
    v.w = Real(0);
    pos[i] = x;
    vel[i] = v;
    kappa[i] = Real(0);
    kappaV[i] = Real(0);
    id[i] = id0 + i;
}

// Overwrites positions/velocities of each slot from the caller's arrays indexed by particle id.
template <class Real>
__global__ void __launch_bounds__(kBlock) update_fluid_kernel(const float* __restrict__ xyz,
                                                              const float* __restrict__ vxyz, uint32_t n,
                                                              const uint32_t* __restrict__ id,
                                                              Vec4<Real>* __restrict__ pos,
                                                              Vec4<Real>* __restrict__ vel, bool set_vel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id[i];
    if (xyz) {
        Vec4<Real> x = pos[i];
        x.x = (Real)xyz[3 * t + 0];
        x.y = (Real)xyz[3 * t + 1];
        x.z = (Real)xyz[3 * t + 2];
        pos[i] = x;
    }
    if (!set_vel) return;
    Vec4<Real> v;
    v.x = vxyz ? (Real)vxyz[3 * t + 0] : Real(0);
    v.y = vxyz ? (Real)vxyz[3 * t + 1] : Real(0);
    v.z = vxyz ? (Real)vxyz[3 * t + 2] : Real(0);
    v.w = Real(0);
    vel[i] = v;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) unpack_boundary_kernel(const float* __restrict__ xyz,
                                                                 const float* __restrict__ psi, uint32_t n,
                                                                 Vec4<Real>* __restrict__ bpos,
                                                                 Vec4<Real>* __restrict__ bvel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Vec4<Real> x;
    x.x = (Real)xyz[3 * i + 0];
    x.y = (Real)xyz[3 * i + 1];
    x.z = (Real)xyz[3 * i + 2];
    x.w = psi ? (Real)psi[i] : Real(0);
    bpos[i] = x;
    Vec4<Real> v;
    v.x = v.y = v.z = v.w = Real(0);
    bvel[i] = v;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) reorder_boundary_kernel(const uint32_t* __restrict__ perm, uint32_t n,
                                                                  const Vec4<Real>* __restrict__ bpos_in,
                                                                  const Vec4<Real>* __restrict__ bvel_in,
                                                                  Vec4<Real>* __restrict__ bpos_out,
                                                                  Vec4<Real>* __restrict__ bvel_out,
                                                                  uint32_t* __restrict__ bid_out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t j = perm[i];
    if (j >= n) j = i;  // only after a failed sort (flagged in the status word); stay in range
    bpos_out[i] = bpos_in[j];
    bvel_out[i] = bvel_in[j];
    bid_out[i] = j;
}

// Moves boundary particles given in original order (bid maps sorted slot -> original index).
template <class Real>
__global__ void __launch_bounds__(kBlock) move_boundary_kernel(const float* __restrict__ xyz,
                                                               const float* __restrict__ vxyz, uint32_t n,
                                                               const uint32_t* __restrict__ bid,
                                                               Vec4<Real>* __restrict__ bpos,
                                                               Vec4<Real>* __restrict__ bvel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = bid[i];
    Vec4<Real> x = bpos[i];
    x.x = (Real)xyz[3 * t + 0];
    x.y = (Real)xyz[3 * t + 1];
    x.z = (Real)xyz[3 * t + 2];
    bpos[i] = x;
    Vec4<Real> v;
    v.x = vxyz ? (Real)vxyz[3 * t + 0] : Real(0);
    v.y = vxyz ? (Real)vxyz[3 * t + 1] : Real(0);
    v.z = vxyz ? (Real)vxyz[3 * t + 2] : Real(0);
    v.w = Real(0);
    bvel[i] = v;
}

// Rigid motion of the boundary particles whose upload index lies in [first, first + count), the
// reference's update of a dynamic object's particles (DFSPH_updateDynamicObjectParticles_kernel,
// DFSPH_core_cuda.cu:3412-3423): x = R x0 + p, v = w x (x - p) + v_lin, with x0 the particle's
// position given at dfsph_set_boundary (upload order); psi is kept. i runs over the sorted slots.
template <class Real>
__global__ void __launch_bounds__(kBlock) rigid_boundary_kernel(const float* __restrict__ rest, uint32_t n,
                                                                const uint32_t* __restrict__ bid, RigidMotion m,
                                                                Vec4<Real>* __restrict__ bpos,
                                                                Vec4<Real>* __restrict__ bvel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = bid[i];
    if (t - m.first >= m.count) return;  // unsigned: also t < first
    const Real x0 = (Real)rest[3 * (size_t)t], y0 = (Real)rest[3 * (size_t)t + 1], z0 = (Real)rest[3 * (size_t)t + 2];
    const Real R[9] = {(Real)m.R[0], (Real)m.R[1], (Real)m.R[2], (Real)m.R[3], (Real)m.R[4],
                       (Real)m.R[5], (Real)m.R[6], (Real)m.R[7], (Real)m.R[8]};
    const Real px = (Real)m.p[0], py = (Real)m.p[1], pz = (Real)m.p[2];
    Vec4<Real> x = bpos[i];
    x.x = R[0] * x0 + R[1] * y0 + R[2] * z0 + px;
    x.y = R[3] * x0 + R[4] * y0 + R[5] * z0 + py;
    x.z = R[6] * x0 + R[7] * y0 + R[8] * z0 + pz;
    bpos[i] = x;
    const Real rx = x.x - px, ry = x.y - py, rz = x.z - pz;
    const Real wx = (Real)m.w[0], wy = (Real)m.w[1], wz = (Real)m.w[2];
    Vec4<Real> v;
    v.x = wy * rz - wz * ry + (Real)m.v[0];
    v.y = wz * rx - wx * rz + (Real)m.v[1];
    v.z = wx * ry - wy * rx + (Real)m.v[2];
    v.w = Real(0);
    bvel[i] = v;
}

// Boundary forces: 64-bit fixed-point sums (kForceScale units per newton) -> Real x, y, z, 0.
template <class Real>
__global__ void __launch_bounds__(kBlock) force_from_fx_kernel(const unsigned long long* __restrict__ fx, uint32_t n,
                                                               Real* __restrict__ out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[4 * (size_t)i + c] = (Real)((double)(long long)fx[3 * (size_t)i + c] / kForceScale);
    out[4 * (size_t)i + 3] = Real(0);
}

// Field download: element c of slot i of src (stride src_stride Real elements) goes to
// dst[(id ? id[i] : i) * comps + c], converted to Out.
template <class Real, class Out>
__global__ void __launch_bounds__(kBlock) pack_field_kernel(const Real* __restrict__ src, int src_stride, int comps,
                                                            const uint32_t* __restrict__ id, uint32_t n,
                                                            Out* __restrict__ dst) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id ? id[i] : i;
    for (int c = 0; c < comps; ++c) dst[(size_t)t * comps + c] = (Out)src[(size_t)i * src_stride + c];
}

__global__ void __launch_bounds__(kBlock) pack_u32_kernel(const uint32_t* __restrict__ src, int comps,
                                                          const uint32_t* __restrict__ id, uint32_t n,
                                                          uint32_t* __restrict__ dst) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id ? id[i] : i;
    for (int c = 0; c < comps; ++c) dst[(size_t)t * comps + c] = src[(size_t)i * comps + c];
}

__global__ void __launch_bounds__(kBlock) unpack_counts_kernel(const uint32_t* __restrict__ counts,
                                                               const uint32_t* __restrict__ id, uint32_t n,
                                                               uint32_t* __restrict__ dst) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id ? id[i] : i;
    dst[2 * (size_t)t + 0] = counts[i] & 0xFFFFu;
    dst[2 * (size_t)t + 1] = counts[i] >> 16;
}

// Publishes a new device state block. The block travels as a kernel parameter, so the update is
// ordered with the surrounding work on the stream and never reads host memory asynchronously.
template <class Real> __global__ void set_state_kernel(DevState<Real>* __restrict__ dst, DevState<Real> v) {
    DFSPH_PDL_ENTER;
    const StepParams<Real>& o = dst->p;  // dt fields stay as the device has them
    v.p.h = o.h;
    v.p.h_future = o.h_future;
    v.p.inv_h = o.inv_h;
    v.p.inv_h_future = o.inv_h_future;
    v.p.h_ratio_to_past = o.h_ratio_to_past;
    v.p.h_ratio_to_past2 = o.h_ratio_to_past2;
    *dst = v;
    // The solver loops' last-block tickets start from zero (each reduction leaves them at zero too);
    // resetting them here, with the state, saves a memset before every solve.
    if (v.ctl)
        for (int k = 0; k < 4; ++k) v.ctl[k].ticket = 0;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) save_untagged_kernel(const Vec4<Real>* __restrict__ pos,
                                                               const Vec4<Real>* __restrict__ vel,
                                                               const uint32_t* __restrict__ id, uint32_t n,
                                                               uint32_t first, Vec4<Real>* __restrict__ spos,
                                                               Vec4<Real>* __restrict__ svel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id[i];
    if (t >= first) return;
    spos[t] = pos[i];
    svel[t] = vel[i];
}

template <class Real>
__global__ void __launch_bounds__(kBlock) restore_untagged_kernel(Vec4<Real>* __restrict__ pos,
                                                                  Vec4<Real>* __restrict__ vel,
                                                                  const uint32_t* __restrict__ id, uint32_t n,
                                                                  uint32_t first, const Vec4<Real>* __restrict__ spos,
                                                                  const Vec4<Real>* __restrict__ svel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id[i];
    if (t >= first) return;
    pos[i] = spos[t];
    vel[i] = svel[t];
}

template <class Real>
__global__ void __launch_bounds__(kBlock) damp_tagged_kernel(Vec4<Real>* __restrict__ vel,
                                                             const uint32_t* __restrict__ id, uint32_t n,
                                                             uint32_t first, Real f) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || id[i] < first) return;
    Vec4<Real> v = vel[i];
    v.x *= f;
    v.y *= f;
    v.z *= f;
    vel[i] = v;
}

template <class Real> __global__ void dt_kernel(DevState<Real>* __restrict__ ds, int op, DtArgs a) {
    DFSPH_PDL_ENTER;
    double* t = ds->dtd;
    StepParams<Real>& p = ds->p;
    if (op == 0) {
        for (int k = 0; k < kDtSlots; ++k) t[k] = a.v[k];
    } else if (op == 1 || op == 2) {
        double hf;
        if (op == 1) {
            hf = a.v[0] > 0.0 ? a.v[0] : t[kDtFixed];
        } else {
            const double vmax2 = ds->ctl[2].sum;
            hf = a.v[0] * 0.4 * (a.v[3] / sqrt(vmax2));
            hf = (a.v[2] < hf) ? a.v[2] : hf;  // std::min(hf, max), NaN as std::min treats it
            hf = (hf < a.v[1]) ? a.v[1] : hf;  // std::max(hf, min)
        }
        const double h = t[kDtH];
        t[kDtHFuture] = hf;
        t[kDtInvHFuture] = 1.0 / hf;
        t[kDtRatio] = h / hf;
        t[kDtRatio2] = (h * h) / (hf * hf);
    } else {  // op 3
        t[kDtHPast] = t[kDtH];
        t[kDtH] = t[kDtHFuture];
        t[kDtInvH] = t[kDtInvHFuture];
    }
    p.h = (Real)t[kDtH];
    p.h_future = (Real)t[kDtHFuture];
    p.inv_h = (Real)t[kDtInvH];
    p.inv_h_future = (Real)t[kDtInvHFuture];
    p.h_ratio_to_past = (Real)t[kDtRatio];
    p.h_ratio_to_past2 = (Real)t[kDtRatio2];
}

}  // namespace

template <class Real> void launch_set_state(DevState<Real>* dst, const DevState<Real>& v, cudaStream_t s) {
    launch_pdl(set_state_kernel<Real>, 1, 1, 0, s, dst, v);
}
template <class Real> void launch_dt(DevState<Real>* d, int op, const DtArgs& a, cudaStream_t s) {
    launch_pdl(dt_kernel<Real>, 1, 1, 0, s, d, op, a);
}

template <class Real>
void launch_unpack_fluid(const float* xyz, const float* vxyz, const float* mass, float default_mass, uint32_t n,
                         Vec4<Real>* pos, Vec4<Real>* vel, Real* kappa, Real* kappaV, uint32_t* id, cudaStream_t s,
                         uint32_t id0) {
    if (n)
        launch_pdl(unpack_fluid_kernel<Real>, grid_for(n), kBlock, 0, s, xyz, vxyz, mass, default_mass, n, pos, vel, kappa,
                                                                 kappaV, id, id0);
}
template <class Real>
void launch_update_fluid(const float* xyz, const float* vxyz, uint32_t n, const uint32_t* id, Vec4<Real>* pos,
                         Vec4<Real>* vel, cudaStream_t s, bool set_vel) {
    if (n) launch_pdl(update_fluid_kernel<Real>, grid_for(n), kBlock, 0, s, xyz, vxyz, n, id, pos, vel, set_vel);
}
template <class Real>
void launch_unpack_boundary(const float* xyz, const float* psi, uint32_t n, Vec4<Real>* bpos, Vec4<Real>* bvel,
                            cudaStream_t s) {
    if (n) launch_pdl(unpack_boundary_kernel<Real>, grid_for(n), kBlock, 0, s, xyz, psi, n, bpos, bvel);
}
template <class Real>
void launch_reorder_boundary(const uint32_t* perm, uint32_t n, const Vec4<Real>* bpos_in, const Vec4<Real>* bvel_in,
                             Vec4<Real>* bpos_out, Vec4<Real>* bvel_out, uint32_t* bid_out, cudaStream_t s) {
    if (n)
        launch_pdl(reorder_boundary_kernel<Real>, grid_for(n), kBlock, 0, s, perm, n, bpos_in, bvel_in, bpos_out, bvel_out,
                                                                     bid_out);
}
template <class Real>
void launch_move_boundary(const float* xyz, const float* vxyz, uint32_t n, const uint32_t* bid, Vec4<Real>* bpos,
                          Vec4<Real>* bvel, cudaStream_t s) {
    if (n) launch_pdl(move_boundary_kernel<Real>, grid_for(n), kBlock, 0, s, xyz, vxyz, n, bid, bpos, bvel);
}
template <class Real>
void launch_rigid_boundary(const float* rest, uint32_t n, const uint32_t* bid, const RigidMotion& m, Vec4<Real>* bpos,
                           Vec4<Real>* bvel, cudaStream_t s) {
    if (n) launch_pdl(rigid_boundary_kernel<Real>, grid_for(n), kBlock, 0, s, rest, n, bid, m, bpos, bvel);
}
template <class Real>
void launch_force_from_fx(const unsigned long long* fx, uint32_t n, Real* out, cudaStream_t s) {
    if (n) launch_pdl(force_from_fx_kernel<Real>, grid_for(n), kBlock, 0, s, fx, n, out);
}
template <class Real>
void launch_save_untagged(const Vec4<Real>* pos, const Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first,
                          Vec4<Real>* spos, Vec4<Real>* svel, cudaStream_t s) {
    if (n) launch_pdl(save_untagged_kernel<Real>, grid_for(n), kBlock, 0, s, pos, vel, id, n, first, spos, svel);
}
template <class Real>
void launch_restore_untagged(Vec4<Real>* pos, Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first,
                             const Vec4<Real>* spos, const Vec4<Real>* svel, cudaStream_t s) {
    if (n) launch_pdl(restore_untagged_kernel<Real>, grid_for(n), kBlock, 0, s, pos, vel, id, n, first, spos, svel);
}
template <class Real>
void launch_damp_tagged(Vec4<Real>* vel, const uint32_t* id, uint32_t n, uint32_t first, Real f, cudaStream_t s) {
    if (n) launch_pdl(damp_tagged_kernel<Real>, grid_for(n), kBlock, 0, s, vel, id, n, first, f);
}
template <class Real, class Out>
void launch_pack_field(const Real* src, int src_stride, int comps, const uint32_t* id, uint32_t n, Out* dst,
                       cudaStream_t s) {
    if (n) launch_pdl(pack_field_kernel<Real, Out>, grid_for(n), kBlock, 0, s, src, src_stride, comps, id, n, dst);
}
void launch_pack_u32(const uint32_t* src, int comps, const uint32_t* id, uint32_t n, uint32_t* dst, cudaStream_t s) {
    if (n) launch_pdl(pack_u32_kernel, grid_for(n), kBlock, 0, s, src, comps, id, n, dst);
}
void launch_unpack_counts(const uint32_t* counts, const uint32_t* id, uint32_t n, uint32_t* dst, cudaStream_t s) {
    if (n) launch_pdl(unpack_counts_kernel, grid_for(n), kBlock, 0, s, counts, id, n, dst);
}

#define DFSPH_INSTANTIATE_IO(R)                                                                                      \
    template void launch_set_state<R>(DevState<R>*, const DevState<R>&, cudaStream_t);                               \
    template void launch_dt<R>(DevState<R>*, int, const DtArgs&, cudaStream_t);                                       \
    template void launch_unpack_fluid<R>(const float*, const float*, const float*, float, uint32_t, Vec4<R>*,        \
                                         Vec4<R>*, R*, R*, uint32_t*, cudaStream_t, uint32_t);                                 \
    template void launch_update_fluid<R>(const float*, const float*, uint32_t, const uint32_t*, Vec4<R>*, Vec4<R>*,  \
                                         cudaStream_t, bool);                                                        \
    template void launch_unpack_boundary<R>(const float*, const float*, uint32_t, Vec4<R>*, Vec4<R>*, cudaStream_t); \
    template void launch_reorder_boundary<R>(const uint32_t*, uint32_t, const Vec4<R>*, const Vec4<R>*, Vec4<R>*,   \
                                             Vec4<R>*, uint32_t*, cudaStream_t);                                     \
    template void launch_move_boundary<R>(const float*, const float*, uint32_t, const uint32_t*, Vec4<R>*, Vec4<R>*, \
                                          cudaStream_t);                                                             \
    template void launch_rigid_boundary<R>(const float*, uint32_t, const uint32_t*, const RigidMotion&, Vec4<R>*,    \
                                           Vec4<R>*, cudaStream_t);                                                  \
    template void launch_force_from_fx<R>(const unsigned long long*, uint32_t, R*, cudaStream_t);                    \
    template void launch_save_untagged<R>(const Vec4<R>*, const Vec4<R>*, const uint32_t*, uint32_t, uint32_t,       \
                                          Vec4<R>*, Vec4<R>*, cudaStream_t);                                         \
    template void launch_restore_untagged<R>(Vec4<R>*, Vec4<R>*, const uint32_t*, uint32_t, uint32_t,                \
                                             const Vec4<R>*, const Vec4<R>*, cudaStream_t);                          \
    template void launch_damp_tagged<R>(Vec4<R>*, const uint32_t*, uint32_t, uint32_t, R, cudaStream_t);             \
    template void launch_pack_field<R, float>(const R*, int, int, const uint32_t*, uint32_t, float*, cudaStream_t);  \
    template void launch_pack_field<R, double>(const R*, int, int, const uint32_t*, uint32_t, double*, cudaStream_t);

DFSPH_INSTANTIATE_IO(float)
DFSPH_INSTANTIATE_IO(double)

}  // namespace dfsph
