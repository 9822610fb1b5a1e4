// solver.cu — the gather kernels of the DFSPH time step.
//
// Reference kernels (SPlisHSPlasH/DFSPH/DFSPH_core_cuda.cu):
//   density + alpha + kappa_v warm start + divergence source  DFSPH_divergence_warmstart_init_kernel :221-237
//   divergence Jacobi (warm start / iteration)                 divergenceSolveParticle :400-480, :495-517
//   divergence residual                                        computeDensityChange :546-614, :618-709, :732-748
//   XSPH viscosity + gravity                                   DFSPH_viscosityXSPH_kernel :1423-1507
//   velocity update + kappa warm-start scaling                 DFSPH_update_vel_kernel :3047-3070
//   pressure Jacobi (warm start / iteration)                   pressureSolveParticle :867-951, :965-980
//   density residual                                           computeDensityAdv :1165-1214, :1217-1243, :1264-1284
//   position update                                            DFSPH_update_pos_kernel :3127-3215
// The residual sums that decide convergence (cub::DeviceReduce::Sum + blocking copy in the
// reference, :774-781 and :1321-1325) are fused into the residual kernels as deterministic FP64
// block reductions whose last block evaluates the loop condition on the device (and, inside a CUDA
// graph, sets the while-node condition), so no host round trip happens per iteration.
#include <type_traits>

#include "dfsph_state.cuh"
#include "io.cuh"

namespace dfsph {

namespace {

// Neighbours per batch in the passes that carry both warm-start candidates.
#ifndef DFSPH_DUAL_BATCH
#define DFSPH_DUAL_BATCH 2
#endif
constexpr int kDualBatch = DFSPH_DUAL_BATCH;

template <class Real> __device__ __forceinline__ Real rmax(Real a, Real b);
template <> __device__ __forceinline__ float rmax<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double rmax<double>(double a, double b) { return fmax(a, b); }
template <class Real> __device__ __forceinline__ Real rmin(Real a, Real b);
template <> __device__ __forceinline__ float rmin<float>(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ double rmin<double>(double a, double b) { return fmin(a, b); }

// |v| > 1e-5 with v in float: identical to the reference's promotion of |v| to double against the
// double literal, because no float lies strictly between 1e-5f and the next float above 1e-5.
__device__ __forceinline__ bool above_eps(float v) { return fabsf(v) > 1.0e-5f; }
__device__ __forceinline__ bool above_eps(double v) { return fabs(v) > kEps; }

__device__ __forceinline__ uint32_t fluid_count(uint32_t c) { return c & 0xFFFFu; }
__device__ __forceinline__ uint32_t boundary_count(uint32_t c) { return c >> 16; }

// Deterministic FP64 sum over the grid, then (last block) the loop decision. The partial of each
// block is reduced in a fixed shuffle pattern and the last block adds the partials in block order.
// kAux also sums a second value (block partials after the first gridDim.x) into ctl->aux.
// A loop pass that ends its loop adds its iteration count to ctl->iter_sum and, if the loop ran out
// of iterations above the tolerance, raises nc_bit in *status (so a step needs no host read to
// report a non-converged solve).
template <int kIsInit, bool kAux = false>
__device__ void reduce_and_decide(double v, double* __restrict__ partials, LoopCtl* __restrict__ ctl, uint32_t n,
                                  double eta, int min_it, int max_it, cudaGraphConditionalHandle handle,
                                  bool use_handle, double aux = 0.0, uint32_t* status = nullptr,
                                  uint32_t nc_bit = 0) {
    __shared__ double warp_sums[kWarpsPerBlock];
    __shared__ double warp_aux[kAux ? kWarpsPerBlock : 1];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if (kAux) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) aux += __shfl_down_sync(0xFFFFFFFFu, aux, o);
    }
    if (lane == 0) {
        warp_sums[warp] = v;
        if (kAux) warp_aux[warp] = aux;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, a = 0.0;
        for (int w = 0; w < kWarpsPerBlock; ++w) s += warp_sums[w];
        partials[blockIdx.x] = s;
        if (kAux) {
            for (int w = 0; w < kWarpsPerBlock; ++w) a += warp_aux[w];
            partials[gridDim.x + blockIdx.x] = a;
        }
        __threadfence();
        const uint32_t t = atomicAdd(&ctl->ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double s = 0.0, a = 0.0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        s += ((volatile double*)partials)[b];
        if (kAux) a += ((volatile double*)partials)[gridDim.x + b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if (kAux) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, o);
    }
    __syncthreads();
    if (lane == 0) {
        warp_sums[warp] = s;
        if (kAux) warp_aux[warp] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kWarpsPerBlock; ++w) tot += warp_sums[w];
        if (kAux) {
            double ta = 0.0;
            for (int w = 0; w < kWarpsPerBlock; ++w) ta += warp_aux[w];
            ctl->aux = ta;
        }
        const double avg = n ? tot / (double)n : 0.0;
        ctl->sum = tot;
        uint32_t cont;
        if (kIsInit) {
            // The init pass fixes the tolerance and bounds of the loop that follows; the loop
            // kernels (possibly replayed from a CUDA graph) read them back from the control block.
            ctl->eta = eta;
            ctl->min_iter = min_it;
            ctl->max_iter = max_it;
            ctl->init_avg = avg;
            ctl->avg = 0.0;
            ctl->iter = 0;
            cont = (max_it > 0) ? 1u : 0u;
        } else {
            const int it = ctl->iter + 1;
            ctl->iter = it;
            ctl->avg = avg;
            cont = ((avg > ctl->eta) || (it < ctl->min_iter)) && (it < ctl->max_iter) ? 1u : 0u;
            if (!cont) {
                ctl->iter_sum += (uint32_t)it;
                if (status && it >= ctl->max_iter && avg > ctl->eta) atomicOr(status, nc_bit);
            }
        }
        ctl->cont = cont;
        ctl->ticket = 0;
        __threadfence();
        if (use_handle) cudaGraphSetConditional(handle, cont);
    }
}

// ---------------------------------------------------------------------------------------------
// Boundary neighbour data (position + psi, and the velocity when the boundary moves).
template <class Real> struct BNbr {
    Vec4<Real> x;
    Real vx, vy, vz;
};
template <class Real>
__device__ __forceinline__ void load_bnbr(BNbr<Real>& b, const Vec4<Real>* __restrict__ bpos,
                                          const Vec4<Real>* __restrict__ bvel, uint32_t j, bool moving) {
    b.x = ld4<Real>(bpos + j);
    if (moving) {
        const Vec4<Real> v = ld4<Real>(bvel + j);
        b.vx = v.x; b.vy = v.y; b.vz = v.z;
    } else {
        b.vx = b.vy = b.vz = Real(0);
    }
}

// Neighbours per gather batch of the residual passes (3) and the density pass (2): at four the
// residual passes spill 16-24 B and the density pass (FP64 density terms) 276 B at the 64-register
// cap. Measured per step against four: -0.3 % / -0.8 % at 1 M particles, -1.2 % each at 250 k.
#ifndef DFSPH_RESID_BATCH
#define DFSPH_RESID_BATCH 3
#endif
constexpr int kResidBatch = DFSPH_RESID_BATCH;
#ifndef DFSPH_DENSITY_BATCH
#define DFSPH_DENSITY_BATCH 2
#endif
constexpr int kDensityBatch = DFSPH_DENSITY_BATCH;

// Sum over fluid then boundary neighbours of m_j (v_i - v_j).grad W_ij, in list order.
template <class Real>
__device__ __forceinline__ Real velocity_divergence(const DevState<Real>* __restrict__ ds, const StepParams<Real>& p,
                                                    uint32_t i, const Vec4<Real>& xi, const Vec4<Real>& vi,
                                                    uint32_t nf, uint32_t nb, const Vec4<Real>* __restrict__ vel) {
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride;
    const Cubic<Real> K = p.kern;
    KSum<Real> s;
    Vec4<Real> xj[kResidBatch], vj[kResidBatch];
    visit_neighbors<kResidBatch>(
        nbr, stride, i, 0, nf, i,
        [&](int u, uint32_t j) {
            xj[u] = ld4<Real>(pos + j);
            vj[u] = ld4<Real>(vel + j);
        },
        [&](int u) {
            Real gx, gy, gz;
            K.gradW(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z, gx, gy, gz);
            s.add(xj[u].w * ((vi.x - vj[u].x) * gx + (vi.y - vj[u].y) * gy + (vi.z - vj[u].z) * gz));
        });
    if (nb) {
        const bool moving = p.boundary_moving != 0;
        BNbr<Real> b[kResidBatch];
        visit_neighbors<kResidBatch>(
            nbr, stride, i, nf, nf + nb, 0u, [&](int u, uint32_t j) { load_bnbr(b[u], ds->bpos, ds->bvel, j, moving); },
            [&](int u) {
                Real gx, gy, gz;
                K.gradW(xi.x - b[u].x.x, xi.y - b[u].x.y, xi.z - b[u].x.z, gx, gy, gz);
                s.add(b[u].x.w * ((vi.x - b[u].vx) * gx + (vi.y - b[u].vy) * gy + (vi.z - b[u].vz) * gz));
            });
    }
    return s.value();
}

// velocity_divergence for two velocity fields in one pass over the neighbours (positions and
// indices loaded once); each sum is accumulated exactly as velocity_divergence would.
template <class Real>
__device__ __forceinline__ void velocity_divergence2(const DevState<Real>* __restrict__ ds, const StepParams<Real>& p,
                                                     uint32_t i, const Vec4<Real>& xi, const Vec4<Real>& via,
                                                     const Vec4<Real>& vib, uint32_t nf, uint32_t nb,
                                                     const Vec4<Real>* __restrict__ vela,
                                                     const Vec4<Real>* __restrict__ velb, Real& outa, Real& outb) {
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride;
    const Cubic<Real> K = p.kern;
    KSum<Real> sa, sb;
    Vec4<Real> xj[kDualBatch], va[kDualBatch], vb[kDualBatch];
    visit_neighbors<kDualBatch>(
        nbr, stride, i, 0, nf, i,
        [&](int u, uint32_t j) {
            xj[u] = ld4<Real>(pos + j);
            va[u] = ld4<Real>(vela + j);
            vb[u] = ld4<Real>(velb + j);
        },
        [&](int u) {
            Real gx, gy, gz;
            K.gradW(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z, gx, gy, gz);
            sa.add(xj[u].w * ((via.x - va[u].x) * gx + (via.y - va[u].y) * gy + (via.z - va[u].z) * gz));
            sb.add(xj[u].w * ((vib.x - vb[u].x) * gx + (vib.y - vb[u].y) * gy + (vib.z - vb[u].z) * gz));
        });
    if (nb) {
        const bool moving = p.boundary_moving != 0;
        BNbr<Real> b[kDualBatch];
        visit_neighbors<kDualBatch>(
            nbr, stride, i, nf, nf + nb, 0u, [&](int u, uint32_t j) { load_bnbr(b[u], ds->bpos, ds->bvel, j, moving); },
            [&](int u) {
                Real gx, gy, gz;
                K.gradW(xi.x - b[u].x.x, xi.y - b[u].x.y, xi.z - b[u].x.z, gx, gy, gz);
                sa.add(b[u].x.w * ((via.x - b[u].vx) * gx + (via.y - b[u].vy) * gy + (via.z - b[u].vz) * gz));
                sb.add(b[u].x.w * ((vib.x - b[u].vx) * gx + (vib.y - b[u].vy) * gy + (vib.z - b[u].vz) * gz));
            });
    }
    outa = sa.value();
    outb = sb.value();
}

// Jacobi velocity correction: sum over fluid neighbours of (k_i + k_j) m_j grad W_ij where
// |k_i + k_j| > eps, plus (when |k_i| > eps) k_i sum over boundary neighbours of psi_b grad W_ib.
// kof(j) returns k_j (a load, possibly transformed). With boundary forces on (kForces, and at run
// time `forces`), each boundary term also adds -m_i k_i psi_b grad W_ib to the boundary particle's force,
// as the reference does for dynamic bodies (DFSPH_core_cuda.cu:467-477, :937-946).
template <class Real, bool kForces = false, class KOf>
__device__ __forceinline__ void jacobi_sum(const DevState<Real>* __restrict__ ds, const StepParams<Real>& p, uint32_t i,
                                           const Vec4<Real>& xi, Real ki, uint32_t nf, uint32_t nb, KOf&& kof,
                                           KSum3<Real>& acc, bool forces = true) {
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride;
    const Cubic<Real> K = p.kern;
    Vec4<Real> xj[kGatherBatch];
    Real kj[kGatherBatch];
    visit_neighbors<kGatherBatch>(
        nbr, stride, i, 0, nf, i,
        [&](int u, uint32_t j) {
            xj[u] = ld4<Real>(pos + j);
            kj[u] = kof(j);
        },
        [&](int u) {
            const Real ks = ki + kj[u];
            if (above_eps(ks)) {
                Real gx, gy, gz;
                K.gradW(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z, gx, gy, gz);
                const Real sc = ks * xj[u].w;
                acc.add(sc * gx, sc * gy, sc * gz);
            }
        });
    if (nb && above_eps(ki)) {
        const Vec4<Real>* __restrict__ bpos = ds->bpos;
        unsigned long long* __restrict__ bf = (kForces && forces) ? ds->bforce : nullptr;
        Vec4<Real> xb[kGatherBatch];
        uint32_t jb[kGatherBatch];
        visit_neighbors<kGatherBatch>(
            nbr, stride, i, nf, nf + nb, 0u,
            [&](int u, uint32_t j) {
                xb[u] = ld4<Real>(bpos + j);
                jb[u] = j;
            },
            [&](int u) {
                Real gx, gy, gz;
                K.gradW(xi.x - xb[u].x, xi.y - xb[u].y, xi.z - xb[u].z, gx, gy, gz);
                const Real sc = ki * xb[u].w;
                acc.add(sc * gx, sc * gy, sc * gz);
                if (kForces && bf) {
                    const Real f = -xi.w * sc;
                    unsigned long long* fb = bf + 3 * (size_t)jb[u];
                    add_force_fx(fb, (double)(f * gx));
                    add_force_fx(fb + 1, (double)(f * gy));
                    add_force_fx(fb + 2, (double)(f * gz));
                }
            });
    }
}

// Two warm-start candidates in one pass over the neighbours: the same sums as jacobi_sum for the
// coefficients ka / kb (the plain and the learned candidate), each accumulated exactly as a
// single-candidate pass would (the gradient is shared). Boundary forces, when on, follow candidate b
// (the one applied in place).
template <class Real, bool kForces = false, class KOfA, class KOfB>
__device__ __forceinline__ void jacobi_sum2(const DevState<Real>* __restrict__ ds, const StepParams<Real>& p,
                                            uint32_t i, const Vec4<Real>& xi, Real kia, Real kib, uint32_t nf,
                                            uint32_t nb, KOfA&& kofa, KOfB&& kofb, KSum3<Real>& acca,
                                            KSum3<Real>& accb) {
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride;
    const Cubic<Real> K = p.kern;
    Vec4<Real> xj[kDualBatch];
    Real kja[kDualBatch], kjb[kDualBatch];
    visit_neighbors<kDualBatch>(
        nbr, stride, i, 0, nf, i,
        [&](int u, uint32_t j) {
            xj[u] = ld4<Real>(pos + j);
            kja[u] = kofa(j);
            kjb[u] = kofb(j);
        },
        [&](int u) {
            const Real ksa = kia + kja[u], ksb = kib + kjb[u];
            const bool ea = above_eps(ksa), eb = above_eps(ksb);
            if (ea || eb) {
                Real gx, gy, gz;
                K.gradW(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z, gx, gy, gz);
                if (ea) {
                    const Real sc = ksa * xj[u].w;
                    acca.add(sc * gx, sc * gy, sc * gz);
                }
                if (eb) {
                    const Real sc = ksb * xj[u].w;
                    accb.add(sc * gx, sc * gy, sc * gz);
                }
            }
        });
    const bool ba = above_eps(kia), bb = above_eps(kib);
    if (nb && (ba || bb)) {
        const Vec4<Real>* __restrict__ bpos = ds->bpos;
        unsigned long long* __restrict__ bf = kForces ? ds->bforce : nullptr;
        Vec4<Real> xb[kDualBatch];
        uint32_t jb[kDualBatch];
        visit_neighbors<kDualBatch>(
            nbr, stride, i, nf, nf + nb, 0u,
            [&](int u, uint32_t j) {
                xb[u] = ld4<Real>(bpos + j);
                jb[u] = j;
            },
            [&](int u) {
                Real gx, gy, gz;
                K.gradW(xi.x - xb[u].x, xi.y - xb[u].y, xi.z - xb[u].z, gx, gy, gz);
                if (ba) {
                    const Real sc = kia * xb[u].w;
                    acca.add(sc * gx, sc * gy, sc * gz);
                }
                if (bb) {
                    const Real sc = kib * xb[u].w;
                    accb.add(sc * gx, sc * gy, sc * gz);
                    if (kForces && bf) {
                        const Real f = -xi.w * sc;
                        unsigned long long* fb = bf + 3 * (size_t)jb[u];
                        add_force_fx(fb, (double)(f * gx));
                        add_force_fx(fb + 1, (double)(f * gy));
                        add_force_fx(fb + 2, (double)(f * gz));
                    }
                }
            });
    }
}

// ---------------------------------------------------------------------------------------------
// density + alpha + divergence source (+ kappa_v warm-start scaling), one pass over the neighbours.
// warm_v and features are runtime flags so that every mode runs the same machine code for the
// density and alpha arithmetic (the learned mode with a plain warm start reproduces the plain mode
// bit for bit).
template <class Real>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) density_alpha_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                               bool warm_v, bool features) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const Vec4<Real>* __restrict__ vel = ds->vel;
    const uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride;
    const Cubic<Real> K = p.kern;

    if (warm_v) ds->kappaV[i] = rmax<Real>(ds->kappaV[i] * p.h_ratio_to_past / Real(2), Real(-0.5));

    const Vec4<Real> xi = pos[i];
    const Vec4<Real> vi = vel[i];
    const uint32_t c = ds->counts[i];
    const uint32_t nf = fluid_count(c), nb = boundary_count(c);
    // rho - rho0 is accumulated directly (rest density first, then the self term and the neighbour
    // terms) so that the density residual rho + h*div - rho0 of the pressure solve never subtracts
    // two numbers of ~1e3 in FP32 (the reference forms rho, then rho + h*div - rho0).
    // FP32 build: each density term m_j W_ij is formed and summed in FP64 (density_term). FP64
    // build: plain terms, compensated sum.
    constexpr bool kF64Terms = std::is_same<Real, float>::value;
    NSum<Real> rho;
    double rho64 = -(double)p.density0;
    KSum<Real> sgk, drho;
    KSum3<Real> gpi;
    rho.add(-p.density0);
    auto add_term = [&](Real rx, Real ry, Real rz, Real m, Real w) {
        if constexpr (kF64Terms) {
            rho64 = __dadd_rn(rho64, density_term(K, rx, ry, rz, m));
        } else {
            rho.add(m * w);
        }
    };
    add_term(Real(0), Real(0), Real(0), xi.w, K.W0);
    auto accumulate = [&](const Vec4<Real>& xj, Real vx, Real vy, Real vz) {
        Real w, gx, gy, gz;
        const Real rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        if constexpr (kF64Terms) K.gradW(rx, ry, rz, gx, gy, gz), w = Real(0);
        else K.W_gradW(rx, ry, rz, w, gx, gy, gz);
        add_term(rx, ry, rz, xj.w, w);
        const Real px = xj.w * gx, py = xj.w * gy, pz = xj.w * gz;
        sgk.add(px * px + py * py + pz * pz);
        gpi.add(px, py, pz);
        drho.add((vi.x - vx) * px + (vi.y - vy) * py + (vi.z - vz) * pz);
    };
    {
        Vec4<Real> xj[kDensityBatch], vj[kDensityBatch];
        visit_neighbors<kDensityBatch>(
            nbr, stride, i, 0, nf, i,
            [&](int u, uint32_t j) {
                xj[u] = ld4<Real>(pos + j);
                vj[u] = ld4<Real>(vel + j);
            },
            [&](int u) { accumulate(xj[u], vj[u].x, vj[u].y, vj[u].z); });
    }
    if (nb) {
        const bool moving = p.boundary_moving != 0;
        BNbr<Real> b[kDensityBatch];
        visit_neighbors<kDensityBatch>(
            nbr, stride, i, nf, nf + nb, 0u, [&](int u, uint32_t j) { load_bnbr(b[u], ds->bpos, ds->bvel, j, moving); },
            [&](int u) { accumulate(b[u].x, b[u].vx, b[u].vy, b[u].vz); });
    }
    const Real gx = gpi.x.value(), gy = gpi.y.value(), gz = gpi.z.value();
    const Real sg = sgk.value() + (gx * gx + gy * gy + gz * gz);
    const Real alpha = -p.inv_h / rmax<Real>(sg, Real(kEps));
    const Real density = kF64Terms ? (Real)rho64 : rho.value();
    ds->factor[i] = alpha;
    ds->density[i] = density;
    uint32_t num = nf;
    if (num < kMinNeighborsForDivergence) num += nb;
    const Real dadv = (num < kMinNeighborsForDivergence) ? Real(0) : rmax<Real>(drho.value(), Real(0));
    ds->densityAdv[i] = dadv;
    if (features) {  // inputs of the warm-start MLP (mlp.cuh)
        float4* f = reinterpret_cast<float4*>(ds->features + (size_t)i * 8);
        f[0] = make_float4((float)(density / p.density0), (float)(dadv * alpha), (float)(nf + nb) * (1.0f / 64.0f),
                           (float)ds->kappaT[i]);
        f[1] = make_float4((float)ds->kappaVT[i], 0.0f, 0.0f, 0.0f);
    }
}

// Divergence warm start (divergenceSolveParticle<true>, only where the source is positive,
// DFSPH_core_cuda.cu:509-512): v_i += h * sum (kv_i + kv_j) m_j grad W_ij + h kv_i sum psi_b grad W_ib.
template <class Real, bool kForces>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) divergence_warm_jacobi_kernel(const DevState<Real>* __restrict__ ds,
                                                                        uint32_t n, const Real* __restrict__ kw,
                                                                        Vec4<Real>* __restrict__ vout) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!(ds->densityAdv[i] > Real(0))) {
        if (vout) vout[i] = ds->vel[i];  // a candidate's velocity buffer holds every particle
        return;
    }
    const StepParams<Real>& p = ds->p;
    const Real* __restrict__ kv = kw ? kw : ds->kappaV;
    const Real ki = kv[i];
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acc;
    jacobi_sum<Real, kForces>(ds, p, i, xi, ki, fluid_count(c), boundary_count(c), [&](uint32_t j) { return kv[j]; },
                              acc, vout == nullptr);  // a candidate pass (vout set) adds no boundary force
    Vec4<Real> v = ds->vel[i];
    v.x += acc.x.value() * p.h;
    v.y += acc.y.value() * p.h;
    v.z += acc.z.value() * p.h;
    (vout ? vout : ds->vel)[i] = v;
}

// Residual pass modes: a loop iteration, the init pass, and the fallback init pass of the learned
// warm start (runs only if the plain candidate's probed residual, ctl[3], beat the learned
// candidate's init residual; it then installs the plain candidate: velocities from velP, warm
// coefficients from the plain array, and redoes the init on them).
constexpr int kLoop = 0, kInitPass = 1, kFallback = 2;

// True in every block of a fallback pass when the plain candidate is to replace the learned one:
// when the learned candidate's sum |r| (its init pass, ctl[slot].aux) exceeds the plain one's
// (probe, ctl[3].sum). Both sums are final before the launch; a NaN also falls back.
template <class Real>
__device__ __forceinline__ bool take_fallback(const DevState<Real>* __restrict__ ds, int slot, uint32_t bit) {
    const double plain = ds->ctl[3].sum, learned = ds->ctl[slot].aux;
    const bool fb = !(learned <= plain);
    if (!fb && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(ds->status + 2, bit);
    return fb;
}

// Divergence residual (computeDensityChange): rho_dot_i = max(sum m_j (v_i - v_j).grad W_ij +
// sum psi_b (v_i - v_b).grad W_ib, 0), 0 with fewer than 20 neighbours. Also stores
// k_i = rho_dot_i * alpha_i for the next Jacobi pass. The init pass additionally zeroes kappa_v
// (DFSPH_divergence_init_kernel, :631-633).
template <class Real, int kMode, bool kKeep>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) divergence_residual_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                     double eta, int min_it, int max_it,
                                                                     cudaGraphConditionalHandle handle,
                                                                     bool use_handle) {
    DFSPH_PDL_ENTER;
    // The init passes receive the tolerance per unit of h (maxErrorV 0.01 rho0 / h): h is the
    // device's (the dt history lives on the device).
    if (kMode != kLoop) eta = eta / ds->dtd[kDtH];
    if (kMode == kFallback && !take_fallback(ds, 0, 1u)) return;  // uniform over the grid
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const Vec4<Real>* __restrict__ vel = kMode == kFallback ? ds->velP : ds->vel;
    double contrib = 0.0, aux = 0.0;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        if (kMode != kLoop) ds->kappaV[i] = Real(0);
        if (kMode == kFallback) {
            ds->vel[i] = vel[i];
            ds->kappaVW[i] = ds->kappaVP[i];
        }
        const uint32_t c = ds->counts[i];
        const uint32_t nf = fluid_count(c), nb = boundary_count(c);
        uint32_t num = nf;
        if (num < kMinNeighborsForDivergence) num += nb;
        Real raw = Real(0);
        if (num >= kMinNeighborsForDivergence) {
            const Vec4<Real> xi = ds->pos[i];
            const Vec4<Real> vi = vel[i];
            raw = velocity_divergence<Real>(ds, p, i, xi, vi, nf, nb, vel);
        }
        const Real dadv = rmax<Real>(raw, Real(0));
        if (kKeep) ds->residV[i] = raw;  // learned warm start only
        aux = fabs((double)raw);
        ds->densityAdv[i] = dadv;
        ds->kcoef[i] = dadv * ds->factor[i];
        contrib = (double)dadv;
    }
    // The learned init pass also sums |r| (unclamped) for the fallback decision.
    reduce_and_decide<kMode != kLoop ? 1 : 0, kKeep && kMode == kInitPass>(
        contrib, ds->partials, ds->ctl + 0, n, eta, min_it, max_it, handle, use_handle, aux, ds->status,
        DFSPH_ST_DIVERGENCE_NOT_CONVERGED);
}

// Divergence Jacobi iteration (divergenceSolveParticle<false>): k_i = rho_dot_i alpha_i,
// kappa_v_i += k_i, v_i += h * [sum (k_i + k_j) m_j grad W_ij + k_i sum psi_b grad W_ib].
template <class Real, bool kForces>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) divergence_jacobi_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                   cudaGraphConditionalHandle handle, bool use_handle) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // Inside a graph while-loop the condition is cleared here and only set again by the last block
    // of the residual pass that follows: a loop can end early but can never spin without bound.
    if (use_handle && i == 0) cudaGraphSetConditional(handle, 0u);
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    const Real* __restrict__ kc = ds->kcoef;
    const Real ki = kc[i];
    ds->kappaV[i] += ki;
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acc;
    jacobi_sum<Real, kForces>(ds, p, i, xi, ki, fluid_count(c), boundary_count(c), [&](uint32_t j) { return kc[j]; },
                              acc);
    Vec4<Real> v = ds->vel[i];
    v.x += acc.x.value() * p.h;
    v.y += acc.y.value() * p.h;
    v.z += acc.z.value() * p.h;
    ds->vel[i] = v;
}

// XSPH viscosity + gravity: a_i = g - sum (inv_h * nu * m_j / rho_j) (v_i - v_j) W_ij over fluid
// neighbours. With kCfl the block maximum of |v + a h|^2 is stored for the CFL time step.
// The viscosity pass gathers position, velocity and density: at four neighbours per batch it spills
// at the 64-register cap; two per batch runs without spills, 14 % faster at 1 M particles.
#ifndef DFSPH_VISC_BATCH
#define DFSPH_VISC_BATCH 2
#endif
constexpr int kViscBatch = DFSPH_VISC_BATCH;
template <class Real, bool kCfl>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) viscosity_kernel(const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float vmag = 0.0f;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        const Vec4<Real>* __restrict__ pos = ds->pos;
        const Vec4<Real>* __restrict__ vel = ds->vel;
        const Real* __restrict__ rho = ds->density;  // rho - rho0
        const Cubic<Real> K = p.kern;
        const Vec4<Real> xi = pos[i];
        const Vec4<Real> vi = vel[i];
        const uint32_t nf = fluid_count(ds->counts[i]);
        const Real cvis = p.inv_h * p.viscosity;
        KSum3<Real> a;
        Vec4<Real> xj[kViscBatch], vj[kViscBatch];
        Real rj[kViscBatch];
        visit_neighbors<kViscBatch>(
            ds->nbr, p.nbr_stride, i, 0, nf, i,
            [&](int u, uint32_t j) {
                xj[u] = ld4<Real>(pos + j);
                vj[u] = ld4<Real>(vel + j);
                rj[u] = p.density0 + rho[j];
            },
            [&](int u) {
                const Real w = K.W(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z);
                const Real sc = cvis * (xj[u].w / rj[u]);
                a.add(-(sc * (vi.x - vj[u].x)) * w, -(sc * (vi.y - vj[u].y)) * w, -(sc * (vi.z - vj[u].z)) * w);
            });
        Vec4<Real> out;
        out.x = p.gx + a.x.value();
        out.y = p.gy + a.y.value();
        out.z = p.gz + a.z.value();
        out.w = Real(0);
        ds->acc[i] = out;
        if (kCfl) {
            const Real ux = vi.x + out.x * p.h, uy = vi.y + out.y * p.h, uz = vi.z + out.z * p.h;
            vmag = (float)(ux * ux + uy * uy + uz * uz);
        }
    }
    if (kCfl) {
        __shared__ float wmax[kWarpsPerBlock];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmag = fmaxf(vmag, __shfl_down_sync(0xFFFFFFFFu, vmag, o));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = vmag;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = 0.0f;
            for (int w = 0; w < kWarpsPerBlock; ++w) m = fmaxf(m, wmax[w]);
            ds->cfl_partials[blockIdx.x] = m;
        }
    }
}

// Maximum of the CFL partials into ctl[2].sum (one block).
template <class Real>
__global__ void __launch_bounds__(kBlock) cfl_reduce_kernel(const DevState<Real>* __restrict__ ds, uint32_t n_blocks) {
    DFSPH_PDL_ENTER;
    float m = 0.0f;
    for (uint32_t b = threadIdx.x; b < n_blocks; b += blockDim.x) m = fmaxf(m, ds->cfl_partials[b]);
    __shared__ float wmax[kWarpsPerBlock];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.0f;
        for (int w = 0; w < kWarpsPerBlock; ++w) r = fmaxf(r, wmax[w]);
        ds->ctl[2].sum = (double)r;
    }
}

// v_i += h a_i (DFSPH_update_vel_kernel); the kappa warm-start scaling of that kernel is applied
// on the fly by the pressure warm start, which is the only reader of the scaled value.
template <class Real>
__global__ void __launch_bounds__(kBlock) update_vel_kernel(const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Real h = ds->p.h;
    Vec4<Real> v = ds->vel[i];
    const Vec4<Real> a = ds->acc[i];
    v.x += h * a.x;
    v.y += h * a.y;
    v.z += h * a.z;
    ds->vel[i] = v;
    ds->kappa[i] = rmax<Real>(ds->kappa[i] * ds->p.h_ratio_to_past2, Real(-0.5));
}

// Pressure warm start (pressureSolveParticle<true>) fused with the velocity update: with
// kFusedVel the particle first applies v_i += h a_i and uses kappa scaled by (h/h_future)^2 and
// clamped at -0.5 (update_vel, :3061-3065), computed for the neighbours on the fly.
template <class Real, bool kFusedVel, bool kForces>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) pressure_warm_jacobi_kernel(const DevState<Real>* __restrict__ ds,
                                                                      uint32_t n, const Real* __restrict__ kw,
                                                                      Vec4<Real>* __restrict__ vout) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    // kw given: final warm-start coefficients; otherwise the reference's kappa, scaled by
    // (h/h_future)^2 and clamped when the velocity update is fused in (update_vel, :3061-3065).
    const bool scale = kFusedVel && kw == nullptr;
    const Real* __restrict__ kap = kw ? kw : ds->kappa;
    const Real r2 = p.h_ratio_to_past2;
    const Real ki = scale ? rmax<Real>(kap[i] * r2, Real(-0.5)) : kap[i];
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acc;
    jacobi_sum<Real, kForces>(ds, p, i, xi, ki, fluid_count(c), boundary_count(c),
                              [&](uint32_t j) { return scale ? rmax<Real>(kap[j] * r2, Real(-0.5)) : kap[j]; }, acc,
                              vout == nullptr);  // a candidate pass (vout set) adds no boundary force
    Vec4<Real> v = ds->vel[i];
    if (kFusedVel) {
        const Vec4<Real> a = ds->acc[i];
        v.x += p.h * a.x;
        v.y += p.h * a.y;
        v.z += p.h * a.z;
    }
    v.x += acc.x.value() * p.h_future;
    v.y += acc.y.value() * p.h_future;
    v.z += acc.z.value() * p.h_future;
    (vout ? vout : ds->vel)[i] = v;
}

// Density residual (computeDensityAdv): rho_adv_i = max(rho_i + h_f * [sum m_j (v_i - v_j).grad W_ij
// + sum psi_b (v_i - v_b).grad W_ib] - rho0, 0); kappa_i += rho_adv_i alpha_i; k_i = rho_adv_i alpha_i.
// kInit first scales alpha by 1/h_future and zeroes kappa (DFSPH_pressure_init_kernel, :1230-1238).
template <class Real, int kMode, bool kKeep>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) pressure_residual_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                   double eta, int min_it, int max_it,
                                                                   cudaGraphConditionalHandle handle,
                                                                   bool use_handle) {
    DFSPH_PDL_ENTER;
    if (kMode == kFallback && !take_fallback(ds, 1, 2u)) return;  // uniform over the grid
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const Vec4<Real>* __restrict__ vel = kMode == kFallback ? ds->velP : ds->vel;
    double contrib = 0.0, aux = 0.0;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        Real alpha = ds->factor[i];  // the fallback pass finds alpha already scaled by its init pass
        Real kap = Real(0);
        if (kMode == kInitPass) {
            alpha *= p.inv_h_future;
            ds->factor[i] = alpha;
        } else if (kMode == kLoop) {
            kap = ds->kappa[i];
        } else {
            ds->vel[i] = vel[i];
            ds->kappaW[i] = ds->kappaP[i];
        }
        const Vec4<Real> xi = ds->pos[i];
        const Vec4<Real> vi = vel[i];
        const uint32_t c = ds->counts[i];
        const Real sdiv = velocity_divergence<Real>(ds, p, i, xi, vi, fluid_count(c), boundary_count(c), vel);
        const Real raw = ds->density[i] + p.h_future * sdiv;  // density[] = rho - rho0
        const Real dadv = rmax<Real>(raw, Real(0));
        if (kKeep) ds->resid[i] = raw;  // learned warm start only
        aux = fabs((double)raw);
        const Real kc = dadv * alpha;
        ds->densityAdv[i] = dadv;
        ds->kcoef[i] = kc;
        ds->kappa[i] = kap + kc;
        contrib = (double)dadv;
    }
    reduce_and_decide<kMode != kLoop ? 1 : 0, kKeep && kMode == kInitPass>(
        contrib, ds->partials, ds->ctl + 1, n, eta, min_it, max_it, handle, use_handle, aux, ds->status,
        DFSPH_ST_PRESSURE_NOT_CONVERGED);
}

// Pressure Jacobi iteration (pressureSolveParticle<false>): v_i += h_f * [sum (k_i + k_j) m_j grad W_ij
// + k_i sum psi_b grad W_ib] with k = rho_adv * alpha.
template <class Real, bool kForces>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) pressure_jacobi_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                 cudaGraphConditionalHandle handle, bool use_handle) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (use_handle && i == 0) cudaGraphSetConditional(handle, 0u);  // see divergence_jacobi_kernel
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    const Real* __restrict__ kc = ds->kcoef;
    const Real ki = kc[i];
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acc;
    jacobi_sum<Real, kForces>(ds, p, i, xi, ki, fluid_count(c), boundary_count(c), [&](uint32_t j) { return kc[j]; },
                              acc);
    Vec4<Real> v = ds->vel[i];
    v.x += acc.x.value() * p.h_future;
    v.y += acc.y.value() * p.h_future;
    v.z += acc.z.value() * p.h_future;
    ds->vel[i] = v;
}

// x_i += h v_i (DFSPH_update_pos_kernel with border damping and wave cancelling off).
template <class Real>
__global__ void __launch_bounds__(kBlock) update_pos_kernel(const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Real h = ds->p.h;
    Vec4<Real> x = ds->pos[i];
    const Vec4<Real> v = ds->vel[i];
    x.x += h * v.x;
    x.y += h * v.y;
    x.z += h * v.z;
    ds->pos[i] = x;
}

// Initial residual of a warm-start candidate whose velocities are `vel`, as sum |r| of the unclamped
// residuals (probe: the sum goes to ctl[3], nothing else is written). which = 0: divergence
// (computeDensityChange), 1: density. The solver's own criterion clamps r at 0 and so cannot see an
// over-pressured candidate (r < 0 everywhere it pushes too hard); |r| sees both directions.
template <class Real, int kWhich>
__global__ void __launch_bounds__(kBlock, kGatherMinBlocks) probe_residual_kernel(const DevState<Real>* __restrict__ ds,
                                                                              uint32_t n,
                                                                              const Vec4<Real>* __restrict__ vel) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double contrib = 0.0;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        const uint32_t c = ds->counts[i];
        const uint32_t nf = fluid_count(c), nb = boundary_count(c);
        if (kWhich == 0) {
            uint32_t num = nf;
            if (num < kMinNeighborsForDivergence) num += nb;
            if (num >= kMinNeighborsForDivergence)
                contrib = fabs((double)velocity_divergence<Real>(ds, p, i, ds->pos[i], vel[i], nf, nb, vel));
        } else {
            const Real sdiv = velocity_divergence<Real>(ds, p, i, ds->pos[i], vel[i], nf, nb, vel);
            contrib = fabs((double)(ds->density[i] + p.h_future * sdiv));
        }
    }
    reduce_and_decide<1>(contrib, ds->partials, ds->ctl + 3, n, 0.0, 0, 1, 0, false);
}

// ---- both warm-start candidates in one pass (learned warm start with the plain fallback) ---------
// Two sets of compensated sums fit the single-candidate passes' 64 registers (4 CTAs per SM) with
// two neighbours per batch: on 2 M particles this beats 2-3 CTAs per SM at batch 2-4 by 1-4 %.
#ifndef DFSPH_DUAL_MIN_BLOCKS
#define DFSPH_DUAL_MIN_BLOCKS 4
#endif
constexpr int kDualMinBlocks = DFSPH_DUAL_MIN_BLOCKS;
// The plain candidate (kappaVP / kappaP) goes to velP, the learned one (kappaVW / kappaW) to vel in
// place; each velocity is the one the single-candidate pass would produce.
template <class Real, bool kForces>
__global__ void __launch_bounds__(kBlock, kDualMinBlocks) divergence_warm_dual_kernel(
    const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!(ds->densityAdv[i] > Real(0))) {
        ds->velP[i] = ds->vel[i];
        return;
    }
    const StepParams<Real>& p = ds->p;
    const Real* __restrict__ ka = ds->kappaVP;
    const Real* __restrict__ kb = ds->kappaVW;
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acca, accb;
    jacobi_sum2<Real, kForces>(ds, p, i, xi, ka[i], kb[i], fluid_count(c), boundary_count(c),
                               [&](uint32_t j) { return ka[j]; }, [&](uint32_t j) { return kb[j]; }, acca, accb);
    const Vec4<Real> v0 = ds->vel[i];
    Vec4<Real> va = v0, vb = v0;
    va.x += acca.x.value() * p.h;
    va.y += acca.y.value() * p.h;
    va.z += acca.z.value() * p.h;
    vb.x += accb.x.value() * p.h;
    vb.y += accb.y.value() * p.h;
    vb.z += accb.z.value() * p.h;
    ds->velP[i] = va;
    ds->vel[i] = vb;
}

template <class Real, bool kFusedVel, bool kForces>
__global__ void __launch_bounds__(kBlock, kDualMinBlocks) pressure_warm_dual_kernel(
    const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    const Real* __restrict__ ka = ds->kappaP;
    const Real* __restrict__ kb = ds->kappaW;
    const Vec4<Real> xi = ds->pos[i];
    const uint32_t c = ds->counts[i];
    KSum3<Real> acca, accb;
    jacobi_sum2<Real, kForces>(ds, p, i, xi, ka[i], kb[i], fluid_count(c), boundary_count(c),
                               [&](uint32_t j) { return ka[j]; }, [&](uint32_t j) { return kb[j]; }, acca, accb);
    Vec4<Real> v = ds->vel[i];
    if (kFusedVel) {
        const Vec4<Real> a = ds->acc[i];
        v.x += p.h * a.x;
        v.y += p.h * a.y;
        v.z += p.h * a.z;
    }
    Vec4<Real> va = v, vb = v;
    va.x += acca.x.value() * p.h_future;
    va.y += acca.y.value() * p.h_future;
    va.z += acca.z.value() * p.h_future;
    vb.x += accb.x.value() * p.h_future;
    vb.y += accb.y.value() * p.h_future;
    vb.z += accb.z.value() * p.h_future;
    ds->velP[i] = va;
    ds->vel[i] = vb;
}

// Init residual pass of both candidates: the learned one (vel) writes the solver's arrays and
// reduces into ctl[slot] (sum of the clamped residuals, aux = sum |r|); the plain one (velP) writes
// dadvP / kcP / rawP and reduces into ctl[3] the same way (separate block partials).
template <class Real>
__global__ void __launch_bounds__(kBlock, kDualMinBlocks) divergence_residual_dual_kernel(
    const DevState<Real>* __restrict__ ds, uint32_t n, double eta, int min_it, int max_it) {
    DFSPH_PDL_ENTER;
    eta = eta / ds->dtd[kDtH];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double cb = 0.0, ab = 0.0, ca = 0.0, aa = 0.0;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        ds->kappaV[i] = Real(0);
        const uint32_t c = ds->counts[i];
        const uint32_t nf = fluid_count(c), nb = boundary_count(c);
        uint32_t num = nf;
        if (num < kMinNeighborsForDivergence) num += nb;
        Real rb = Real(0), ra = Real(0);
        if (num >= kMinNeighborsForDivergence) {
            const Vec4<Real> xi = ds->pos[i];
            velocity_divergence2<Real>(ds, p, i, xi, ds->velP[i], ds->vel[i], nf, nb, ds->velP, ds->vel, ra, rb);
        }
        const Real alpha = ds->factor[i];
        const Real db = rmax<Real>(rb, Real(0)), da = rmax<Real>(ra, Real(0));
        ds->residV[i] = rb;
        ds->densityAdv[i] = db;
        ds->kcoef[i] = db * alpha;
        ds->rawP[i] = ra;
        ds->dadvP[i] = da;
        ds->kcP[i] = da * alpha;
        cb = (double)db;
        ab = fabs((double)rb);
        ca = (double)da;
        aa = fabs((double)ra);
    }
    reduce_and_decide<1, true>(cb, ds->partials, ds->ctl + 0, n, eta, min_it, max_it, 0, false, ab);
    __syncthreads();
    reduce_and_decide<1, true>(ca, ds->partials + 2 * gridDim.x, ds->ctl + 3, n, eta, min_it, max_it, 0, false, aa);
}

template <class Real>
__global__ void __launch_bounds__(kBlock, kDualMinBlocks) pressure_residual_dual_kernel(
    const DevState<Real>* __restrict__ ds, uint32_t n, double eta, int min_it, int max_it) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double cb = 0.0, ab = 0.0, ca = 0.0, aa = 0.0;
    if (i < n) {
        const StepParams<Real>& p = ds->p;
        const Real alpha = ds->factor[i] * p.inv_h_future;
        ds->factor[i] = alpha;
        const Vec4<Real> xi = ds->pos[i];
        const uint32_t c = ds->counts[i];
        const uint32_t nf = fluid_count(c), nb = boundary_count(c);
        Real sa, sb;
        velocity_divergence2<Real>(ds, p, i, xi, ds->velP[i], ds->vel[i], nf, nb, ds->velP, ds->vel, sa, sb);
        const Real rb = ds->density[i] + p.h_future * sb, ra = ds->density[i] + p.h_future * sa;
        const Real db = rmax<Real>(rb, Real(0)), da = rmax<Real>(ra, Real(0));
        const Real kb = db * alpha, ka = da * alpha;
        ds->resid[i] = rb;
        ds->densityAdv[i] = db;
        ds->kcoef[i] = kb;
        ds->kappa[i] = Real(0) + kb;
        ds->rawP[i] = ra;
        ds->dadvP[i] = da;
        ds->kcP[i] = ka;
        cb = (double)db;
        ab = fabs((double)rb);
        ca = (double)da;
        aa = fabs((double)ra);
    }
    reduce_and_decide<1, true>(cb, ds->partials, ds->ctl + 1, n, eta, min_it, max_it, 0, false, ab);
    __syncthreads();
    reduce_and_decide<1, true>(ca, ds->partials + 2 * gridDim.x, ds->ctl + 3, n, eta, min_it, max_it, 0, false, aa);
}

// Keeps the learned candidate unless its sum |r| exceeds the plain one's (or is NaN); otherwise
// installs the plain candidate's velocities, warm coefficients, residual arrays and init sum.
template <class Real>
__global__ void __launch_bounds__(kBlock) select_candidate_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                  int which) {
    DFSPH_PDL_ENTER;
    const int slot = which == 0 ? 0 : 1;
    const double learned = ds->ctl[slot].aux, plain = ds->ctl[3].aux;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (learned <= plain) {
        if (i == 0) atomicOr(ds->status + 2, which == 0 ? 1u : 2u);
        return;
    }
    if (i == 0) {  // (aux, the decision's input, stays: every block reads it)
        LoopCtl* c = ds->ctl + slot;
        c->sum = ds->ctl[3].sum;
        c->init_avg = n ? ds->ctl[3].sum / (double)n : 0.0;
    }
    if (i >= n) return;
    ds->vel[i] = ds->velP[i];
    ds->densityAdv[i] = ds->dadvP[i];
    ds->kcoef[i] = ds->kcP[i];
    if (which == 0) {
        ds->kappaVW[i] = ds->kappaVP[i];
        ds->residV[i] = ds->rawP[i];
    } else {
        ds->kappaW[i] = ds->kappaP[i];
        ds->kappa[i] = Real(0) + ds->kcP[i];  // as the init pass forms it (kappa = 0 + k)
        ds->resid[i] = ds->rawP[i];
    }
}

// Warm-start candidates (see launch_warm_values). kappa <= 0 is pressure, so min() takes the larger
// pressure. The learned candidate raises the reference warm start to `damping` times the predicted
// needed coefficient (the previous step's needed value plus the network's correction, scaled by the
// dt ratio like the reference's warm start, in the reference's range [-0.5, 0]) wherever that is the
// larger pressure, and keeps the reference warm start elsewhere. A clamped-residual Jacobi solve only
// ever adds pressure, so from a warm start between the reference's and the needed pressure it ends
// where the reference's solve ends (the needed pressure, or the reference warm start where that is
// already larger); damping < 1 keeps a prediction error from overshooting the needed pressure.
template <class Real>
__global__ void __launch_bounds__(kBlock) warm_values_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                             int which, bool learned, bool use_pred, Real damping) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    if (i == 0) ds->dtd[which == 0 ? kDtRatioUsedV : kDtRatio2UsedP] = ds->dtd[which == 0 ? kDtRatio : kDtRatio2];
    if (which == 0) {
        const Real plain = rmax<Real>(ds->kappaV[i] * p.h_ratio_to_past / Real(2), Real(-0.5));
        Real use = plain;
        if (learned) {
            const Real corr = use_pred ? (Real)ds->out_scale[1] * (Real)ds->pred[2 * (size_t)i + 1] : Real(0);
            const Real need = rmin<Real>(rmax<Real>((ds->kappaVT[i] + corr) * p.h_ratio_to_past, Real(-0.5)), Real(0));
            use = rmin<Real>(plain, damping * need);
        }
        ds->kappaVP[i] = plain;
        ds->kappaV[i] = use;
        ds->kappaVW[i] = use;
    } else {
        const Real plain = rmax<Real>(ds->kappa[i] * p.h_ratio_to_past2, Real(-0.5));
        Real use = plain;
        if (learned) {
            const Real corr = use_pred ? (Real)ds->out_scale[0] * (Real)ds->pred[2 * (size_t)i] : Real(0);
            const Real need = rmin<Real>(rmax<Real>((ds->kappaT[i] + corr) * p.h_ratio_to_past2, Real(-0.5)), Real(0));
            use = rmin<Real>(plain, damping * need);
        }
        ds->kappaP[i] = plain;
        ds->kappaW[i] = use;
    }
}

// Pressure each solve actually needed, per particle: the applied total (warm start + corrections)
// less one Jacobi estimate of its excess, kept in the reference's range of coefficients [-0.5, 0]
// (kappa <= 0 is pressure; no solve applies tension). A solve only ever adds pressure (its residuals
// are clamped at zero), so an over-pressured warm start passes through unchanged; the unclamped
// final residual r < 0 measures the excess and min(r, 0) * alpha removes it (alpha of the pressure
// solve is already divided by h_future, the divergence solve's alpha is factor * h_future here).
// Free-surface particles have r << 0 from their missing neighbours: the clamp at 0 leaves them
// without pressure rather than under tension.
template <class Real>
__device__ __forceinline__ Real clamp_kappa(Real k) {
    return rmin<Real>(rmax<Real>(k, Real(-0.5)), Real(0));
}
template <class Real>
__device__ __forceinline__ void needed_totals(const DevState<Real>* __restrict__ ds, uint32_t i, bool div_ran,
                                              Real& kt, Real& kvt) {
    const Real f = ds->factor[i];
    kt = clamp_kappa(ds->kappaW[i] + ds->kappa[i] + rmin<Real>(ds->resid[i], Real(0)) * f);
    kvt = div_ran ? clamp_kappa(ds->kappaVW[i] + ds->kappaV[i] +
                                rmin<Real>(ds->residV[i], Real(0)) * (f * ds->p.h_future))
                  : Real(0);
}

// A plain step after a learned one (the cost gate's probe windows): the reference warm start carries
// a solve's corrections only, and after a learned step those miss the learned warm start the solve
// began from; the applied warm start is added back so that the plain step starts from the total.
template <class Real>
__global__ void __launch_bounds__(kBlock) restore_totals_kernel(const DevState<Real>* __restrict__ ds, uint32_t n) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ds->kappa[i] = ds->kappa[i] + ds->kappaW[i];
    ds->kappaV[i] = ds->kappaV[i] + ds->kappaVW[i];
}

template <class Real>
__global__ void __launch_bounds__(kBlock) totals_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                        bool div_ran) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Real kt, kvt;
    needed_totals(ds, i, div_ran, kt, kvt);
    ds->kappaT[i] = kt;
    ds->kappaVT[i] = kvt;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) gather_training_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                 uint32_t batch, uint32_t offset, bool div_ran,
                                                                 float* __restrict__ x, float* __restrict__ t) {
    DFSPH_PDL_ENTER;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= batch) return;
    const double r2 = ds->dtd[kDtRatio2UsedP], hr = ds->dtd[kDtRatioUsedV];  // dt ratios the warm starts used
    const uint32_t i = (uint32_t)(((uint64_t)k * n / batch + offset) % n);
    const float4* f = reinterpret_cast<const float4*>(ds->features + (size_t)i * 8);
    reinterpret_cast<float4*>(x + (size_t)k * 8)[0] = f[0];
    reinterpret_cast<float4*>(x + (size_t)k * 8)[1] = f[1];
    Real kt, kvt;
    needed_totals(ds, i, div_ran, kt, kvt);
    const double tot = (double)kt, totv = (double)kvt;
    t[2 * (size_t)k] = (float)((tot / r2 - (double)ds->kappaT[i]) / (double)ds->out_scale[0]);
    t[2 * (size_t)k + 1] = (float)((totv / hr - (double)ds->kappaVT[i]) / (double)ds->out_scale[1]);
}

}  // namespace

template <class Real>
void launch_density_alpha(const DevState<Real>* d, uint32_t n, bool warm_v, bool features, cudaStream_t s) {
    if (!n) return;
    launch_pdl(density_alpha_kernel<Real>, grid_for(n), kBlock, 0, s, d, n, warm_v && !features, features);
}
template <class Real>
void launch_divergence_warm_jacobi(const DevState<Real>* d, uint32_t n, const Real* kw, Vec4<Real>* vout,
                                   cudaStream_t s, bool forces) {
    if (!n) return;
    if (forces) launch_pdl(divergence_warm_jacobi_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n, kw, vout);
    else launch_pdl(divergence_warm_jacobi_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n, kw, vout);
}
template <class Real>
void launch_probe_residual(const DevState<Real>* d, uint32_t n, int which, const Vec4<Real>* vel, cudaStream_t s) {
    const unsigned g = grid_for(n ? n : 1);
    if (which == 0) launch_pdl(probe_residual_kernel<Real, 0>, g, kBlock, 0, s, d, n, vel);
    else launch_pdl(probe_residual_kernel<Real, 1>, g, kBlock, 0, s, d, n, vel);
}
template <class Real>
void launch_warm_values(const DevState<Real>* d, uint32_t n, int which, bool learned, bool use_pred, double damping,
                        cudaStream_t s) {
    if (n) launch_pdl(warm_values_kernel<Real>, grid_for(n), kBlock, 0, s, d, n, which, learned, use_pred, (Real)damping);
}
template <class Real> void launch_restore_totals(const DevState<Real>* d, uint32_t n, cudaStream_t s) {
    if (n) launch_pdl(restore_totals_kernel<Real>, grid_for(n), kBlock, 0, s, d, n);
}
template <class Real> void launch_totals(const DevState<Real>* d, uint32_t n, bool div_ran, cudaStream_t s) {
    if (n) launch_pdl(totals_kernel<Real>, grid_for(n), kBlock, 0, s, d, n, div_ran);
}
template <class Real>
void launch_gather_training(const DevState<Real>* d, uint32_t n, uint32_t batch, uint32_t offset, bool div_ran, float* x,
                            float* t, cudaStream_t s) {
    if (n && batch) launch_pdl(gather_training_kernel<Real>, grid_for(batch), kBlock, 0, s, d, n, batch, offset, div_ran, x, t);
}
template <class Real>
void launch_divergence_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                                cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s, bool keep) {
    const unsigned g = grid_for(n ? n : 1);
    auto k = init ? (keep ? divergence_residual_kernel<Real, kInitPass, true> : divergence_residual_kernel<Real, kInitPass, false>)
                  : (keep ? divergence_residual_kernel<Real, kLoop, true> : divergence_residual_kernel<Real, kLoop, false>);
    launch_pdl(k, g, kBlock, 0, s, d, n, eta, min_it, max_it, h, use_handle);
}
template <class Real>
void launch_divergence_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                              cudaStream_t s, bool forces) {
    if (!n) return;
    if (forces) launch_pdl(divergence_jacobi_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n, h, use_handle);
    else launch_pdl(divergence_jacobi_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n, h, use_handle);
}
template <class Real> void launch_viscosity(const DevState<Real>* d, uint32_t n, bool cfl, cudaStream_t s) {
    if (!n) return;
    if (cfl) launch_pdl(viscosity_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n);
    else launch_pdl(viscosity_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n);
}
template <class Real> void launch_update_vel(const DevState<Real>* d, uint32_t n, cudaStream_t s) {
    if (n) launch_pdl(update_vel_kernel<Real>, grid_for(n), kBlock, 0, s, d, n);
}
template <class Real>
void launch_pressure_warm_jacobi(const DevState<Real>* d, uint32_t n, bool fused_vel, const Real* kw,
                                 Vec4<Real>* vout, cudaStream_t s, bool forces) {
    if (!n) return;
    const unsigned g = grid_for(n);
    if (forces) {
        if (fused_vel) launch_pdl(pressure_warm_jacobi_kernel<Real, true, true>, g, kBlock, 0, s, d, n, kw, vout);
        else launch_pdl(pressure_warm_jacobi_kernel<Real, false, true>, g, kBlock, 0, s, d, n, kw, vout);
    } else {
        if (fused_vel) launch_pdl(pressure_warm_jacobi_kernel<Real, true, false>, g, kBlock, 0, s, d, n, kw, vout);
        else launch_pdl(pressure_warm_jacobi_kernel<Real, false, false>, g, kBlock, 0, s, d, n, kw, vout);
    }
}
template <class Real>
void launch_pressure_residual(const DevState<Real>* d, uint32_t n, bool init, double eta, int min_it, int max_it,
                              cudaGraphConditionalHandle h, bool use_handle, cudaStream_t s, bool keep) {
    const unsigned g = grid_for(n ? n : 1);
    auto k = init ? (keep ? pressure_residual_kernel<Real, kInitPass, true> : pressure_residual_kernel<Real, kInitPass, false>)
                  : (keep ? pressure_residual_kernel<Real, kLoop, true> : pressure_residual_kernel<Real, kLoop, false>);
    launch_pdl(k, g, kBlock, 0, s, d, n, eta, min_it, max_it, h, use_handle);
}
template <class Real>
void launch_warm_dual(const DevState<Real>* d, uint32_t n, int which, bool fused_vel, cudaStream_t s, bool forces) {
    if (!n) return;
    if (which == 0) {
        if (forces) launch_pdl(divergence_warm_dual_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n);
        else launch_pdl(divergence_warm_dual_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n);
    } else if (fused_vel) {
        if (forces) launch_pdl(pressure_warm_dual_kernel<Real, true, true>, grid_for(n), kBlock, 0, s, d, n);
        else launch_pdl(pressure_warm_dual_kernel<Real, true, false>, grid_for(n), kBlock, 0, s, d, n);
    } else {
        if (forces) launch_pdl(pressure_warm_dual_kernel<Real, false, true>, grid_for(n), kBlock, 0, s, d, n);
        else launch_pdl(pressure_warm_dual_kernel<Real, false, false>, grid_for(n), kBlock, 0, s, d, n);
    }
}
template <class Real>
void launch_residual_dual(const DevState<Real>* d, uint32_t n, int which, double eta, int min_it, int max_it,
                          cudaStream_t s) {
    if (!n) return;
    if (which == 0) launch_pdl(divergence_residual_dual_kernel<Real>, grid_for(n), kBlock, 0, s, d, n, eta, min_it, max_it);
    else launch_pdl(pressure_residual_dual_kernel<Real>, grid_for(n), kBlock, 0, s, d, n, eta, min_it, max_it);
}
template <class Real> void launch_select_candidate(const DevState<Real>* d, uint32_t n, int which, cudaStream_t s) {
    launch_pdl(select_candidate_kernel<Real>, grid_for(n ? n : 1), kBlock, 0, s, d, n, which);
}
template <class Real>
void launch_fallback_residual(const DevState<Real>* d, uint32_t n, int which, double eta, int min_it, int max_it,
                              cudaStream_t s) {
    const unsigned g = grid_for(n ? n : 1);
    if (which == 0)
        launch_pdl(divergence_residual_kernel<Real, kFallback, true>, g, kBlock, 0, s, d, n, eta, min_it, max_it, 0, false);
    else
        launch_pdl(pressure_residual_kernel<Real, kFallback, true>, g, kBlock, 0, s, d, n, eta, min_it, max_it, 0, false);
}
template <class Real>
void launch_pressure_jacobi(const DevState<Real>* d, uint32_t n, cudaGraphConditionalHandle h, bool use_handle,
                            cudaStream_t s, bool forces) {
    if (!n) return;
    if (forces) launch_pdl(pressure_jacobi_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n, h, use_handle);
    else launch_pdl(pressure_jacobi_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n, h, use_handle);
}
template <class Real> void launch_update_pos(const DevState<Real>* d, uint32_t n, cudaStream_t s) {
    if (n) launch_pdl(update_pos_kernel<Real>, grid_for(n), kBlock, 0, s, d, n);
}
template <class Real> void launch_cfl_reduce(const DevState<Real>* d, uint32_t n_blocks, cudaStream_t s) {
    launch_pdl(cfl_reduce_kernel<Real>, 1, kBlock, 0, s, d, n_blocks);
}

#define DFSPH_INSTANTIATE_SOLVER(R)                                                                                  \
    template void launch_density_alpha<R>(const DevState<R>*, uint32_t, bool, bool, cudaStream_t);                  \
    template void launch_divergence_warm_jacobi<R>(const DevState<R>*, uint32_t, const R*, Vec4<R>*, cudaStream_t,  \
                                                   bool);                                                            \
    template void launch_probe_residual<R>(const DevState<R>*, uint32_t, int, const Vec4<R>*, cudaStream_t);        \
    template void launch_warm_values<R>(const DevState<R>*, uint32_t, int, bool, bool, double, cudaStream_t);       \
    template void launch_totals<R>(const DevState<R>*, uint32_t, bool, cudaStream_t);                               \
    template void launch_restore_totals<R>(const DevState<R>*, uint32_t, cudaStream_t);                              \
    template void launch_gather_training<R>(const DevState<R>*, uint32_t, uint32_t, uint32_t, bool, float*, float*, \
                                            cudaStream_t);                                                           \
    template void launch_divergence_residual<R>(const DevState<R>*, uint32_t, bool, double, int, int,               \
                                                cudaGraphConditionalHandle, bool, cudaStream_t, bool);               \
    template void launch_divergence_jacobi<R>(const DevState<R>*, uint32_t, cudaGraphConditionalHandle, bool,       \
                                              cudaStream_t, bool);                                                   \
    template void launch_viscosity<R>(const DevState<R>*, uint32_t, bool, cudaStream_t);                            \
    template void launch_update_vel<R>(const DevState<R>*, uint32_t, cudaStream_t);                                 \
    template void launch_pressure_warm_jacobi<R>(const DevState<R>*, uint32_t, bool, const R*, Vec4<R>*,            \
                                                 cudaStream_t, bool);                                                \
    template void launch_pressure_residual<R>(const DevState<R>*, uint32_t, bool, double, int, int,                 \
                                              cudaGraphConditionalHandle, bool, cudaStream_t, bool);                 \
    template void launch_fallback_residual<R>(const DevState<R>*, uint32_t, int, double, int, int, cudaStream_t);   \
    template void launch_warm_dual<R>(const DevState<R>*, uint32_t, int, bool, cudaStream_t, bool);                  \
    template void launch_residual_dual<R>(const DevState<R>*, uint32_t, int, double, int, int, cudaStream_t);        \
    template void launch_select_candidate<R>(const DevState<R>*, uint32_t, int, cudaStream_t);                       \
    template void launch_pressure_jacobi<R>(const DevState<R>*, uint32_t, cudaGraphConditionalHandle, bool,         \
                                            cudaStream_t, bool);                                                     \
    template void launch_update_pos<R>(const DevState<R>*, uint32_t, cudaStream_t);                                 \
    template void launch_cfl_reduce<R>(const DevState<R>*, uint32_t, cudaStream_t);

DFSPH_INSTANTIATE_SOLVER(float)
DFSPH_INSTANTIATE_SOLVER(double)

}  // namespace dfsph
