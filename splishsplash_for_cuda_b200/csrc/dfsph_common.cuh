// dfsph_common.cuh — types, SPH kernel functions, the canonical neighbour predicate and the
// compensated sums shared by every device kernel of the DFSPH time step.
//
// Everything here is templated on the arithmetic type Real (float = product, double = the FP64
// build of the same kernels used to state each field's FP32 error).
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "../../include/dfsph_c.h"

namespace dfsph {

// ---- programmatic dependent launch -------------------------------------------------------------
// The kernels of a time step are launched with programmatic stream serialisation: the next kernel's
// launch is processed while the previous grid's last blocks finish, instead of after the grid has
// completed (about 2 us per kernel boundary on B200). Every kernel starts with pdl_wait(), which
// blocks until the previous grid has completed and its writes are visible, so the ordering is the
// plain stream order; each block signals its dependents when it ends (PdlTrigger). The attribute is
// left off while a loop body is captured into a graph (g_pdl_off).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
struct PdlTrigger {
    __device__ __forceinline__ ~PdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
};
#define DFSPH_PDL_ENTER \
    pdl_wait();         \
    const PdlTrigger pdl_trigger_guard_ {}

inline thread_local bool g_pdl_off = false;

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = g_pdl_off ? 0 : 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------------------------------------
// Launch shapes. One thread per particle for the gathers (SPlisHSPlasH/DFSPH/DFSPH_define_cuda.h:6
// uses 128); 256 threads keep 8 warps per block and let the FP64 residual reduction use one shared
// array per block.
constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / 32;
// Minimum resident blocks per SM asked of the compiler for the gather kernels (register cap).
#ifndef DFSPH_MIN_BLOCKS
#define DFSPH_MIN_BLOCKS 4
#endif
constexpr int kGatherMinBlocks = DFSPH_MIN_BLOCKS;

// Divergence and pressure minimum iteration counts of the reference GPU loops
// (DFSPH_core_cuda.cu:828 and :1378).
constexpr int kMinItersV = 3;
constexpr int kMinItersP = 2;

// Jacobi coefficient threshold m_eps (DFSPH_define_cuda.h:7); compared in double as the reference
// does (float |k| promoted against the double literal 1.0e-5).
constexpr double kEps = 1.0e-5;

// Neighbour count below which a particle gets no divergence source (DFSPH_core_cuda.cu:340-351).
constexpr uint32_t kMinNeighborsForDivergence = 20;

// ---------------------------------------------------------------------------------------------
// Vector helpers.
template <class Real> struct V3 {
    Real x, y, z;
};
template <class Real> __host__ __device__ inline V3<Real> v3(Real x, Real y, Real z) { return {x, y, z}; }

template <class Real> struct Vec4Traits;
template <> struct Vec4Traits<float> { using type = float4; };
struct alignas(32) double4a { double x, y, z, w; };
template <> struct Vec4Traits<double> { using type = double4a; };
template <class Real> using Vec4 = typename Vec4Traits<Real>::type;

template <class Real> __device__ __forceinline__ Vec4<Real> ld4(const Vec4<Real>* p) { return *p; }
template <> __device__ __forceinline__ float4 ld4<float>(const float4* p) { return __ldg(p); }

// ---------------------------------------------------------------------------------------------
// Compensated (Kahan) accumulation of FP32 sums. For double the same code runs; the compensation
// term is simply tiny.
template <class Real> struct KSum {
    Real s = Real(0), c = Real(0);
    __device__ __forceinline__ void add(Real v) {
        const Real y = v - c;
        const Real t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ Real value() const { return s; }
};
// Neumaier's variant: exact compensation whichever operand is larger. Used for the density
// deviation rho - rho0, a sum whose terms (the rest density, the self term, ~30 neighbour terms of
// up to a few hundred kg/m^3) cancel to a value ~1e3 times smaller than themselves.
template <class Real> struct NSum {
    Real s = Real(0), c = Real(0);
    __device__ __forceinline__ void add(Real v) {
        const Real t = s + v;
        c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
        s = t;
    }
    __device__ __forceinline__ Real value() const { return s + c; }
};
template <class Real> struct KSum3 {
    KSum<Real> x, y, z;
    __device__ __forceinline__ void add(Real a, Real b, Real d) { x.add(a); y.add(b); z.add(d); }
};

// ---------------------------------------------------------------------------------------------
// Boundary forces in 64-bit fixed point: 2^32 units per newton, +-2^31 N range. Each contribution is
// rounded once to 2^-32 N (2.3e-10 N) and added with an integer atomic, so the accumulated force is
// the same whatever the order of the additions (an FP32 atomicAdd sum is not).
constexpr double kForceScale = 4294967296.0;
__device__ __forceinline__ void add_force_fx(unsigned long long* p, double f) {
    atomicAdd(p, (unsigned long long)llrint(f * kForceScale));
}

// ---------------------------------------------------------------------------------------------
// Canonical pair predicate. The reference tests (pos_i - pos_j).squaredNorm() < H*H
// (SPlisHSPlasH/DFSPH/DFSPH_macro_cuda.h:149, squaredNorm at SPlisHSPlasH/Vector.h:137). Its
// rounding depends on how the compiler contracts x*x+y*y+z*z; this library fixes one order with
// explicit round-to-nearest intrinsics so that the device kernels and the CPU oracle decide every
// pair identically: d2 = fma(dz,dz, fma(dy,dy, dx*dx)), strict d2 < H*H.
__device__ __forceinline__ bool pair_within(float xi, float yi, float zi, float xj, float yj, float zj, float H2) {
    const float dx = __fsub_rn(xi, xj), dy = __fsub_rn(yi, yj), dz = __fsub_rn(zi, zj);
    const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    return d2 < H2;
}
__device__ __forceinline__ bool pair_within(double xi, double yi, double zi, double xj, double yj, double zj, double H2) {
    // The FP64 build decides pairs on the FP32-rounded coordinates so that both builds use the same
    // neighbour sets (positions enter both builds as the same float values).
    return pair_within((float)xi, (float)yi, (float)zi, (float)xj, (float)yj, (float)zj, (float)H2);
}

// Cell coordinate along one axis: floor(x / H + offset), the reference's
// (pos / kernelRadius) + gridOffset followed by toFloor (DFSPH_core_cuda.cu:1839-1841,
// SPlisHSPlasH/Vector.h:157), in FP32 with an IEEE division.
__device__ __forceinline__ int cell_coord(float x, float H, int offset) {
    return (int)floorf(__fadd_rn(__fdiv_rn(x, H), (float)offset));
}
__device__ __forceinline__ int cell_coord(double x, double H, int offset) {
    return cell_coord((float)x, (float)H, offset);
}

// 30-bit Morton key of 10-bit cell coordinates (x in the lowest bit of each triple).
__host__ __device__ inline uint32_t spread_bits10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__host__ __device__ inline uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread_bits10(x) | (spread_bits10(y) << 1) | (spread_bits10(z) << 2);
}
__host__ __device__ inline uint32_t compact_bits10(uint32_t v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x000003FFu;
    return v;
}
constexpr uint32_t kEscapedKey = 0xFFFFFFFFu;  // sorts after every valid 30-bit Morton key

// ---------------------------------------------------------------------------------------------
// Cubic spline kernel (SPlisHSPlasH/DFSPH/SPH_kernels.h:20-100, CubicKernelPerso): W and grad W
// with support H, k = 8/(pi H^3), l = 48/(pi H^3); grad W = 0 for |r| <= 1e-6.
//   W(q)      = k (6 q^3 - 6 q^2 + 1)   for q <= 1/2,   2 k (1 - q)^3   for 1/2 < q <= 1
//   grad W(r) = l q (3 q - 2) r / (|r| H)  for q <= 1/2,  -l (1 - q)^2 r / (|r| H)  for 1/2 < q <= 1
// The reference evaluates q = |r| / H and 1 / (|r| H) with two divisions and a square root per pair;
// here one reciprocal square root of |r|^2 and the precomputed 1/H give q and 1/(|r| H) with
// multiplications only (a few ulp from the division form; the CPU oracle keeps the division form
// and the parity tests bound the difference).
template <class Real> struct Cubic {
    Real H, invH, k, l, W0;
    // 1/H^2 and k in FP64 for the density terms of the FP32 build (density_term below); unused by
    // the FP64 build.
    double ih2_d, k_d;
    static __device__ __forceinline__ float rsqrt_(float v) { return rsqrtf(v); }
    static __device__ __forceinline__ double rsqrt_(double v) { return rsqrt(v); }
    __device__ __forceinline__ Real W_of_q(Real q) const {
        if (q <= Real(1)) {
            if (q <= Real(0.5)) {
                const Real q2 = q * q;
                const Real q3 = q2 * q;
                return k * (Real(6) * q3 - Real(6) * q2 + Real(1));
            }
            const Real f = Real(1) - q;
            return k * (Real(2) * f * f * f);
        }
        return Real(0);
    }
    // |r| <= 1e-6 (tested as |r|^2 <= 1e-12, the same cut-off up to rounding) gives grad W = 0 and
    // W = W0 = W(0).
    __device__ __forceinline__ Real W(Real rx, Real ry, Real rz) const {
        const Real r2 = rx * rx + ry * ry + rz * rz;
        if (!(r2 > Real(1e-12))) return W0;
        const Real q = r2 * rsqrt_(r2) * invH;
        return W_of_q(q);
    }
    __device__ __forceinline__ void gradW(Real rx, Real ry, Real rz, Real& gx, Real& gy, Real& gz) const {
        const Real r2 = rx * rx + ry * ry + rz * rz;
        gx = gy = gz = Real(0);
        if (r2 > Real(1e-12)) {
            const Real inv_rl = rsqrt_(r2);
            const Real q = r2 * inv_rl * invH;
            if (q <= Real(1)) {
                const Real c = (q <= Real(0.5)) ? l * q * (Real(3) * q - Real(2)) : l * (-(Real(1) - q) * (Real(1) - q));
                const Real f = c * inv_rl * invH;
                gx = f * rx;
                gy = f * ry;
                gz = f * rz;
            }
        }
    }
    __device__ __forceinline__ void W_gradW(Real rx, Real ry, Real rz, Real& w, Real& gx, Real& gy, Real& gz) const {
        const Real r2 = rx * rx + ry * ry + rz * rz;
        gx = gy = gz = Real(0);
        w = W0;
        if (r2 > Real(1e-12)) {
            const Real inv_rl = rsqrt_(r2);
            const Real q = r2 * inv_rl * invH;
            w = W_of_q(q);
            if (q <= Real(1)) {
                const Real c = (q <= Real(0.5)) ? l * q * (Real(3) * q - Real(2)) : l * (-(Real(1) - q) * (Real(1) - q));
                const Real f = c * inv_rl * invH;
                gx = f * rx;
                gy = f * ry;
                gz = f * rz;
            }
        }
    }
};

// ---------------------------------------------------------------------------------------------
// Density terms m_j W_ij of the FP32 build in double-float arithmetic (unevaluated pairs of FP32
// values, hi + lo, built from error-free transformations: Knuth's TwoSum, Dekker's Fast2Sum and
// the FMA product error). Why: the density deviation rho - rho0 that drives the pressure solve is
// ~1/40 of rho at the most compressed particles, and a plain FP32 term m_j W(q) carries ~5 ulp of
// error (|r|^2 rounding, sqrt and the steep cubic amplify it), i.e. ~1e-4 kg/m^3 on rho and ~4e-6
// relative on rho - rho0, kappa and the velocities it corrects. Forming |r|^2, q, W and m W as
// pairs keeps each term within ~2^-40 of the exact value for the given FP32 coordinates; the sum
// itself stays an FP32 compensated sum (hi parts in Neumaier's sum, lo parts in a plain FP32 sum).
// Every operation is an explicit round-to-nearest intrinsic so nothing is contracted.
// Density term m_j W(r_ij) of the FP32 build, evaluated in native FP64 from the FP32 distance
// components (their squares are exact in FP64): the FP32 build sums rho - rho0 in FP64 from these
// terms, so the density residual keeps the accuracy of the FP64 build where rho ~ rho0 cancels.
// The self term (r = 0) is m k.
// Every FP64 operation is rounded on its own (no contraction), in the order the oracle's FP32
// instance evaluates it, so the two agree bit for bit on the same inputs.
__device__ __forceinline__ double density_term(const Cubic<float>& K, float rx, float ry, float rz, float m) {
    const double dx = rx, dy = ry, dz = rz;
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    const double q2 = __dmul_rn(r2, K.ih2_d);
    if (q2 > 1.0) return 0.0;
    double w = K.k_d;
    if (q2 > 0.0) {
        const double q = __dsqrt_rn(q2);
        if (q <= 0.5) {
            w = __dmul_rn(K.k_d, __dadd_rn(1.0, __dmul_rn(__dmul_rn(6.0, q2), __dadd_rn(q, -1.0))));
        } else {
            const double f = __dadd_rn(1.0, -q);
            w = __dmul_rn(__dmul_rn(2.0, K.k_d), __dmul_rn(__dmul_rn(f, f), f));
        }
    }
    return __dmul_rn(w, (double)m);
}

// ---------------------------------------------------------------------------------------------
// Batched neighbour visit. The neighbours [k0, k1) of particle i are taken kGatherBatch at a time:
// first the batch's indices are loaded (coalesced rows of the interleaved table), then load(u, j)
// issues every gather of the batch, then use(u) consumes them in list order. Keeping a batch of
// independent gathers in flight per thread hides the latency that a one-at-a-time loop exposes,
// while the summation order (and so every result bit) stays that of the plain loop. Slots past the
// end of the list load `fallback` (an in-range index) and are not used.
#ifndef DFSPH_GATHER_BATCH
#define DFSPH_GATHER_BATCH 4
#endif
constexpr int kGatherBatch = DFSPH_GATHER_BATCH;
#ifndef DFSPH_PREFETCH_IDX
#define DFSPH_PREFETCH_IDX 1
#endif
constexpr uint32_t kNoNeighbor = 0xFFFFFFFFu;
// The neighbour-index stream (read once per pass, coalesced: 128 B per warp and list slot, no reuse)
// is read through the read-only path without allocating in L1 (L1::no_allocate), so that the lines it
// would take stay with the neighbours' positions and velocities, which the passes re-read from L1.
// Measured per step: 2.9 % faster at 1 M particles (passes larger than L2), 2.2 % slower at 250 k
// (L2-resident passes); a runtime choice by size cost more in registers than it saved. The asm is
// volatile: a load hoisted out of its condition would read past the list.
#ifndef DFSPH_IDX_NO_ALLOCATE
#define DFSPH_IDX_NO_ALLOCATE 1
#endif
__device__ __forceinline__ uint32_t ld_idx(const uint32_t* p) {
#if DFSPH_IDX_NO_ALLOCATE
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}

template <int B, class Load, class Use>
__device__ __forceinline__ void visit_neighbors(const uint32_t* __restrict__ nbr, uint32_t stride, uint32_t i,
                                                uint32_t k0, uint32_t k1, uint32_t fallback, Load&& load, Use&& use) {
#if DFSPH_PREFETCH_IDX
    // The index loads of the next batch are issued before the gathers of this one, so that their
    // latency (a coalesced stream, usually from DRAM) overlaps the dependent gathers.
    uint32_t jj[B];
#pragma unroll
    for (int u = 0; u < B; ++u) jj[u] = (k0 + u) < k1 ? ld_idx(nbr + (size_t)(k0 + u) * stride + i) : kNoNeighbor;
    for (uint32_t kb = k0; kb < k1; kb += B) {
        uint32_t jn[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const uint32_t k = kb + B + u;
            jn[u] = k < k1 ? ld_idx(nbr + (size_t)k * stride + i) : kNoNeighbor;
        }
#pragma unroll
        for (int u = 0; u < B; ++u) load(u, jj[u] == kNoNeighbor ? fallback : jj[u]);
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (kb + u < k1) use(u);
#pragma unroll
        for (int u = 0; u < B; ++u) jj[u] = jn[u];
    }
#else
    for (uint32_t kb = k0; kb < k1; kb += B) {
        uint32_t jj[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const uint32_t k = kb + u;
            jj[u] = k < k1 ? ld_idx(nbr + (size_t)k * stride + i) : kNoNeighbor;
        }
#pragma unroll
        for (int u = 0; u < B; ++u) load(u, jj[u] == kNoNeighbor ? fallback : jj[u]);
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (kb + u < k1) use(u);
    }
#endif
}

// ---------------------------------------------------------------------------------------------
// Per-launch parameters (passed by value). The dt history mirrors DFSPHCData
// (DFSPH_c_arrays_structure.h:343-354, updateTimeStep/onSimulationStepEnd at .cpp:1100-1118).
template <class Real> struct StepParams {
    Cubic<Real> kern;
    Real H2;              // H*H for the predicate (computed in float for both builds)
    Real density0;
    Real viscosity;
    Real gx, gy, gz;
    Real h, h_future, inv_h, inv_h_future, h_ratio_to_past, h_ratio_to_past2;
    int off_x, off_y, off_z;     // grid offset (cells)
    int dim_x, dim_y, dim_z;     // cell grid extent
    uint32_t n_fluid;
    uint32_t n_boundary;
    uint32_t nbr_stride;         // row stride of the interleaved neighbour table
    uint32_t nbr_cap;            // stored neighbours per particle
    int boundary_moving;         // 1: boundary velocities are read (else zero)
    int bshift;                  // 1: the boundary translated rigidly by (bsx, bsy, bsz) since its binning
    Real bsx, bsy, bsz;
};

// Device-side control block of one solver loop (divergence or pressure).
struct LoopCtl {
    double sum;          // last residual sum over all fluid particles (FP64)
    double avg;          // sum / n
    double eta;          // tolerance (absolute)
    double init_avg;     // residual after the init pass
    int32_t iter;        // iterations done
    int32_t max_iter;
    int32_t min_iter;
    uint32_t cont;       // loop condition for the next iteration
    uint32_t ticket;     // last-block election counter
    uint32_t iter_sum;   // iterations of every loop ended since the counter was last cleared
    double aux;          // second sum of an init pass that reduces two values (learned warm start)
};

}  // namespace dfsph
