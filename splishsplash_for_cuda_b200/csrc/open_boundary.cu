// open_boundary.cu — the simple open boundary of the reference (OpenBoundariesSimple.cu) and the
// stable compaction / exclusive scan it needs.
//
// Reference: OpenBoundariesSimple::init (OpenBoundariesSimple.cu:105-350) keeps the inflow samples
// near the boundary and below the fluid surface; applyOpenBoundary (:495-620) adds a fluid particle
// at every sample with room around it (inflow_with_predefined_positions_kernel, :352-470) and removes
// the particles of the boundary layer above the fluid surface (outflow_basic_kernel, :475-492). The
// shapes are BufferFluidSurface's (BufferFluidSurface.cu:421-900).
//
// Differences by design: new particles are appended in sample order from an exclusive scan of the
// decisions (the reference appends in atomicAdd order, which varies run to run); removal is a stable
// compaction that keeps the survivors' order and renumbers their ids densely; surface arithmetic is
// written with explicit round-to-nearest operations so that no multiply-add is contracted.
#include "open_boundary.cuh"

#include <cmath>

namespace dfsph {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;  // 4096
static_assert(kScanThreads == 1024, "block_exclusive assumes 32 warps");

// |e|^2 summed left to right without contraction (the oracle evaluates the same expression).
__device__ __forceinline__ float sq3(float a, float b, float c) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}
__device__ __forceinline__ double sq3(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// ---- surfaces ------------------------------------------------------------------------------------
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float norm3(F3 a) { return __fsqrt_rn(dot3(a, a)); }
__device__ __forceinline__ F3 f3(const float* v) { return {v[0], v[1], v[2]}; }

// Star outline test for a point at horizontal offset v (v.y = 0) with |v| = nv in
// [radius_internal, radius] (BufferFluidSurface::isinside, case 5).
__device__ bool star_inside(const dfsph_surface& S, F3 v, float nv) {
    const F3 u = {__fdiv_rn(v.x, nv), __fdiv_rn(v.y, nv), __fdiv_rn(v.z, nv)};
    const float alpha = acosf(dot3(u, f3(S.direction)));
    const float alpha0 = __fdiv_rn(__fmul_rn(2.0f, 3.14159265358979f), (float)S.points);
    float k = __fdiv_rn(alpha, alpha0);
    for (uint32_t it = 0; k > 1.0f && it <= S.points; ++it) k = __fsub_rn(k, 1.0f);  // angle modulo one point
    const float x = __fmul_rn(k, alpha0);
    const float half = __fdiv_rn(alpha0, 2.0f);
    float a1 = 0.0f, r1 = S.radius, a2 = __fadd_rn(0.0f, half), r2 = S.radius_internal;
    if (x > half) {
        r1 = S.radius_internal;
        r2 = S.radius;
        a1 = a2;
        a2 = __fadd_rn(a1, half);
    }
    const float x1 = __fmul_rn(r1, cosf(a1)), y1 = __fmul_rn(r1, sinf(a1));
    const float x2 = __fmul_rn(r2, cosf(a2)), y2 = __fmul_rn(r2, sinf(a2));
    const float m = __fdiv_rn(__fsub_rn(y2, y1), __fsub_rn(x2, x1));
    const float c = __fadd_rn(__fmul_rn(-x1, m), y1);
    const float d = __fdiv_rn(c, __fadd_rn(__fmul_rn(-m, cosf(x)), __fmul_rn(1.0f, sinf(x))));
    return nv <= d;
}

// Moller-Trumbore ray / triangle test as BufferFluidSurface.cu:14-47 evaluates it (RayIntersectsTriangle
// <true, false>): FP32 throughout, products and sums in the written order, 1/a in FP64; a ray crossing
// counts when the triangle's plane is not parallel to it (|a| >= 1e-7), the hit lies inside the
// triangle (u, v >= 0, u <= 1, u + v <= 1) and ahead of the point (t > 0).
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ bool ray_hits_triangle_ahead(F3 o, F3 d, F3 v0, F3 v1, F3 v2) {
    const float eps = 1e-7f;
    const F3 e1 = sub3(v1, v0), e2 = sub3(v2, v0);
    const F3 h = cross3(d, e2);
    const float a = dot3(e1, h);
    if (a > -eps && a < eps) return false;
    const float f = (float)__ddiv_rn(1.0, (double)a);
    const F3 s = sub3(o, v0);
    const float u = __fmul_rn(f, dot3(s, h));
    if (u < 0.0f || u > 1.0f) return false;
    const F3 q = cross3(s, e1);
    const float v = __fmul_rn(f, dot3(d, q));
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
    return __fmul_rn(f, dot3(e2, q)) > 0.0f;
}

// MeshPerso::isInside (BufferFluidSurface.cu:224-270): outside the bounding box (vertices and the
// origin, translated) a point is outside; inside it, inside when the ray along the fixed direction
// crosses an odd number of triangles.
__device__ bool mesh_inside(const DevSurface& S, F3 p) {
    const float* c = S.s.center;
    const F3 lo = {__fadd_rn(S.m.bmin[0], c[0]), __fadd_rn(S.m.bmin[1], c[1]), __fadd_rn(S.m.bmin[2], c[2])};
    const F3 hi = {__fadd_rn(S.m.bmax[0], c[0]), __fadd_rn(S.m.bmax[1], c[1]), __fadd_rn(S.m.bmax[2], c[2])};
    if (p.x < lo.x || p.y < lo.y || p.z < lo.z || p.x > hi.x || p.y > hi.y || p.z > hi.z) return false;
    const F3 d = {S.m.dir[0], S.m.dir[1], S.m.dir[2]};
    const F3 off = {c[0], c[1], c[2]};
    uint32_t hits = 0;
    for (uint32_t t = 0; t < S.m.nt; ++t) {
        const float4 a = S.m.tri[3 * (size_t)t], b = S.m.tri[3 * (size_t)t + 1], e = S.m.tri[3 * (size_t)t + 2];
        const F3 v0 = {__fadd_rn(a.x, off.x), __fadd_rn(a.y, off.y), __fadd_rn(a.z, off.z)};
        const F3 v1 = {__fadd_rn(b.x, off.x), __fadd_rn(b.y, off.y), __fadd_rn(b.z, off.z)};
        const F3 v2 = {__fadd_rn(e.x, off.x), __fadd_rn(e.y, off.y), __fadd_rn(e.z, off.z)};
        if (ray_hits_triangle_ahead(p, d, v0, v1, v2)) ++hits;
    }
    return (hits & 1u) != 0u;
}

__device__ bool surface_inside(const DevSurface& D, F3 p) {
    const dfsph_surface& S = D.s;
    bool r = false;
    switch (S.type) {
        case DFSPH_SURFACE_PLANE:
            r = !(dot3(sub3(p, f3(S.origin)), f3(S.normal)) < 0.0f);
            break;
        case DFSPH_SURFACE_CUBOID: {
            const F3 v = sub3(p, f3(S.center));
            r = fabsf(v.x) < S.half_lengths[0] && fabsf(v.y) < S.half_lengths[1] && fabsf(v.z) < S.half_lengths[2];
            break;
        }
        case DFSPH_SURFACE_CYLINDER: {
            F3 v = sub3(p, f3(S.center));
            if (fabsf(v.y) > S.half_lengths[1]) break;
            v.y = 0.0f;
            r = norm3(v) < S.radius;
            break;
        }
        case DFSPH_SURFACE_SPHERE:
            r = norm3(sub3(p, f3(S.center))) < S.radius;
            break;
        case DFSPH_SURFACE_STAR: {
            F3 v = sub3(p, f3(S.center));
            if (fabsf(v.y) > S.half_lengths[1]) break;
            v.y = 0.0f;
            const float nv = norm3(v);
            if (nv < S.radius_internal) r = true;
            else if (nv > S.radius) r = false;
            else r = star_inside(S, v, nv);
            break;
        }
        case DFSPH_SURFACE_MESH:
            r = mesh_inside(D, p);
            break;
        default:
            break;
    }
    return S.reversed ? !r : r;
}

// Inward normal: center - p for the round shapes, zero for planes, cuboids and meshes
// (BufferFluidSurface::getNormal).
__device__ F3 surface_normal(const DevSurface& D, F3 p) {
    const dfsph_surface& S = D.s;
    F3 r = {0.0f, 0.0f, 0.0f};
    if (S.type == DFSPH_SURFACE_CYLINDER || S.type == DFSPH_SURFACE_SPHERE || S.type == DFSPH_SURFACE_STAR)
        r = sub3(f3(S.center), p);
    if (S.reversed) r = {-r.x, -r.y, -r.z};
    if (!(r.x == 0.0f && r.y == 0.0f && r.z == 0.0f)) {
        const float nr = norm3(r);
        r = {__fdiv_rn(r.x, nr), __fdiv_rn(r.y, nr), __fdiv_rn(r.z, nr)};
    }
    return r;
}

template <class Real>
__device__ __forceinline__ bool cell_of(Real x, Real y, Real z, const StepParams<Real>& p, int& cx, int& cy, int& cz) {
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) return false;
    cx = cell_coord(x, p.kern.H, p.off_x);
    cy = cell_coord(y, p.kern.H, p.off_y);
    cz = cell_coord(z, p.kern.H, p.off_z);
    return cx >= 0 && cy >= 0 && cz >= 0 && cx < p.dim_x && cy < p.dim_y && cz < p.dim_z;
}

__device__ __forceinline__ uint32_t lin(int x, int y, int z, const int dx, const int dy) {
    return (uint32_t)x + (uint32_t)dx * ((uint32_t)y + (uint32_t)dy * (uint32_t)z);
}

// ---- scan ----------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one value per thread over the block; returns the block total in *total.
__device__ uint32_t block_exclusive(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inc = warp_inclusive(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {  // 32 warps: one warp total per lane
        const uint32_t w = warp_sums[lane];
        const uint32_t wi = warp_inclusive(w);
        warp_sums[lane] = wi - w;  // exclusive
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                                      uint32_t* __restrict__ sums) {
    DFSPH_PDL_ENTER;
    __shared__ uint32_t tot;
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    block_exclusive(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block: exclusive scan of the tile sums in place, the grand total to *total.
__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(uint32_t* __restrict__ sums, uint32_t tiles,
                                                                 uint32_t* __restrict__ total) {
    DFSPH_PDL_ENTER;
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < tiles; base += kScanTile) {
        const uint32_t i0 = base + threadIdx.x * kScanItems;
        uint32_t v[kScanItems], s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = (i0 + k < tiles) ? sums[i0 + k] : 0u;
            s += v[k];
        }
        uint32_t off = block_exclusive(s, &tot) + carry;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (i0 + k < tiles) {
                sums[i0 + k] = off;
                off += v[k];
            }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                                  const uint32_t* __restrict__ sums,
                                                                  uint32_t* __restrict__ out) {
    DFSPH_PDL_ENTER;
    __shared__ uint32_t tot;
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t off = block_exclusive(s, &tot) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) {
            out[base + k] = off;
            off += v[k];
        }
}

// ---- open boundary kernels -----------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(kBlock) select_kernel(const float4* __restrict__ samples, uint32_t ns,
                                                        DevSurface interior, DevSurface surface,
                                                        StepParams<Real> p, uint32_t* __restrict__ keep) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const float4 s = samples[i];
    const F3 x = {s.x, s.y, s.z};
    int cx, cy, cz;
    keep[i] = (!surface_inside(interior, x) && surface_inside(surface, x) &&
               cell_of<Real>((Real)s.x, (Real)s.y, (Real)s.z, p, cx, cy, cz))
                  ? 1u
                  : 0u;
}

__global__ void __launch_bounds__(kBlock) compact_samples_kernel(const float4* __restrict__ samples,
                                                                 const uint32_t* __restrict__ keep,
                                                                 const uint32_t* __restrict__ rank, uint32_t ns,
                                                                 float4* __restrict__ out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ns && keep[i]) out[rank[i]] = samples[i];
}

__global__ void __launch_bounds__(kBlock) shift_samples_kernel(float4* __restrict__ samples, uint32_t ns, float dx,
                                                               float dy, float dz) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    float4 s = samples[i];
    s.x = __fadd_rn(s.x, dx);
    s.y = __fadd_rn(s.y, dy);
    s.z = __fadd_rn(s.z, dz);
    samples[i] = s;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) inflow_kernel(const DevState<Real>* __restrict__ ds,
                                                        const float4* __restrict__ samples, uint32_t ns,
                                                        float allowed_distance, float allowed_density, Real mass,
                                                        DevSurface boundary, const uint2* __restrict__ ftab,
                                                        const uint2* __restrict__ btab, uint32_t* __restrict__ flag,
                                                        float4* __restrict__ vout) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const StepParams<Real>& p = ds->p;
    const float4 s = samples[i];
    const Real xi = (Real)s.x, yi = (Real)s.y, zi = (Real)s.z;
    int cx, cy, cz;
    uint32_t add = 0;
    float4 vo = make_float4(0.f, 0.f, 0.f, 0.f);
    if (cell_of<Real>(xi, yi, zi, p, cx, cy, cz)) {
        const Vec4<Real>* __restrict__ pos = ds->pos;
        const Vec4<Real>* __restrict__ vel = ds->vel;
        // closest fluid particle of the 27 cells (every particle of the cells, as the reference's
        // structure iteration)
        Real min_d = Real(100);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                    if (X < 0 || Y < 0 || Z < 0 || X >= p.dim_x || Y >= p.dim_y || Z >= p.dim_z) continue;
                    const uint2 r = ftab[lin(X, Y, Z, p.dim_x, p.dim_y)];
                    for (uint32_t j = r.x; j < r.y; ++j) {
                        const Vec4<Real> xj = ld4<Real>(pos + j);
                        const Real d = sqrt(sq3(xi - xj.x, yi - xj.y, zi - xj.z));
                        min_d = d < min_d ? d : min_d;
                    }
                }
        if (min_d > (Real)allowed_distance) {
            Real rho = p.kern.W0 * mass, wsum = Real(0), vx = 0, vy = 0, vz = 0;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                        if (X < 0 || Y < 0 || Z < 0 || X >= p.dim_x || Y >= p.dim_y || Z >= p.dim_z) continue;
                        const uint2 r = ftab[lin(X, Y, Z, p.dim_x, p.dim_y)];
                        for (uint32_t j = r.x; j < r.y; ++j) {
                            const Vec4<Real> xj = ld4<Real>(pos + j);
                            const Real w = p.kern.W(xi - xj.x, yi - xj.y, zi - xj.z) * xj.w;
                            const Vec4<Real> vj = ld4<Real>(vel + j);
                            rho += w;
                            vx += vj.x * w;
                            vy += vj.y * w;
                            vz += vj.z * w;
                            wsum += w;
                        }
                    }
            if (p.n_boundary > 0) {
                const Vec4<Real>* __restrict__ bpos = ds->bpos;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                            if (X < 0 || Y < 0 || Z < 0 || X >= p.dim_x || Y >= p.dim_y || Z >= p.dim_z) continue;
                            const uint2 r = btab[lin(X, Y, Z, p.dim_x, p.dim_y)];
                            for (uint32_t j = r.x; j < r.y; ++j) {
                                const Vec4<Real> xb = ld4<Real>(bpos + j);
                                const Real w = p.kern.W(xi - xb.x, yi - xb.y, zi - xb.z) * xb.w;
                                wsum += w;
                                rho += w;
                            }
                        }
            }
            if (wsum > Real(0)) {
                vx /= wsum;
                vy /= wsum;
                vz /= wsum;
            }
            const F3 nrm = surface_normal(boundary, F3{s.x, s.y, s.z});
            const F3 v3 = {(float)vx, (float)vy, (float)vz};
            add = (!(rho > (Real)allowed_density) && !(dot3(v3, nrm) < 0.0f)) ? 1u : 0u;
            vo = make_float4(v3.x, v3.y, v3.z, 0.f);
        }
    }
    flag[i] = add;
    vout[i] = vo;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) append_kernel(const float4* __restrict__ samples,
                                                        const float4* __restrict__ svel,
                                                        const uint32_t* __restrict__ flag,
                                                        const uint32_t* __restrict__ rank, uint32_t ns, uint32_t n,
                                                        uint32_t capacity, Real mass, Vec4<Real>* __restrict__ pos,
                                                        Vec4<Real>* __restrict__ vel, Real* __restrict__ kappa,
                                                        Real* __restrict__ kappaV, uint32_t* __restrict__ id,
                                                        Real* __restrict__ kT, Real* __restrict__ kVT) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns || !flag[i]) return;
    const uint32_t r = rank[i];
    if (r >= capacity - n) return;  // n <= capacity
    const uint32_t k = n + r;
    const float4 s = samples[i], v = svel[i];
    Vec4<Real> x, u;
    x.x = (Real)s.x;
    x.y = (Real)s.y;
    x.z = (Real)s.z;
    x.w = mass;
    u.x = (Real)v.x;
    u.y = (Real)v.y;
    u.z = (Real)v.z;
    u.w = Real(0);
    pos[k] = x;
    vel[k] = u;
    kappa[k] = Real(0);
    kappaV[k] = Real(0);
    id[k] = k;
    if (kT) kT[k] = Real(0);
    if (kVT) kVT[k] = Real(0);
}

template <class Real>
__global__ void __launch_bounds__(kBlock) outflow_tag_kernel(const Vec4<Real>* __restrict__ pos, uint32_t n,
                                                             DevSurface interior, DevSurface surface,
                                                             uint32_t* __restrict__ alive) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Vec4<Real> x = pos[i];
    const F3 p = {(float)x.x, (float)x.y, (float)x.z};
    alive[i] = (!surface_inside(interior, p) && !surface_inside(surface, p)) ? 0u : 1u;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) compact_fluid_kernel(
    const uint32_t* __restrict__ alive, const uint32_t* __restrict__ dst, uint32_t n,
    const Vec4<Real>* __restrict__ pos_in, const Vec4<Real>* __restrict__ vel_in, const Real* __restrict__ kappa_in,
    const Real* __restrict__ kappaV_in, const uint32_t* __restrict__ id_in, const Real* __restrict__ kT_in,
    const Real* __restrict__ kVT_in, Vec4<Real>* __restrict__ pos_out, Vec4<Real>* __restrict__ vel_out,
    Real* __restrict__ kappa_out, Real* __restrict__ kappaV_out, uint32_t* __restrict__ id_out,
    Real* __restrict__ kT_out, Real* __restrict__ kVT_out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !alive[i]) return;
    const uint32_t k = dst[i];
    pos_out[k] = pos_in[i];
    vel_out[k] = vel_in[i];
    kappa_out[k] = kappa_in[i];
    kappaV_out[k] = kappaV_in[i];
    id_out[k] = id_in[i];
    if (kT_in) kT_out[k] = kT_in[i];
    if (kVT_in) kVT_out[k] = kVT_in[i];
}

// checkParticlesPositions(2) (SPH_other_systems_cuda.cu:1242-1281): a particle with any coordinate
// above the box maximum or below its minimum is removed (NaN coordinates compare false and stay).
template <class Real>
__global__ void __launch_bounds__(kBlock) box_tag_kernel(const Vec4<Real>* __restrict__ pos, uint32_t n, float lo_x,
                                                         float lo_y, float lo_z, float hi_x, float hi_y, float hi_z,
                                                         uint32_t* __restrict__ alive, uint32_t* __restrict__ count) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Vec4<Real> x = pos[i];
    const bool out = x.x > (Real)hi_x || x.y > (Real)hi_y || x.z > (Real)hi_z || x.x < (Real)lo_x ||
                     x.y < (Real)lo_y || x.z < (Real)lo_z;
    alive[i] = out ? 0u : 1u;
    if (out) atomicAdd(count, 1u);
}

__global__ void __launch_bounds__(kBlock) alive_by_id_kernel(const uint32_t* __restrict__ id,
                                                             const uint32_t* __restrict__ alive, uint32_t n,
                                                             uint32_t* __restrict__ out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = id[i];
    if (k < n) out[k] = alive[i];
}

__global__ void __launch_bounds__(kBlock) renumber_kernel(uint32_t* __restrict__ id, uint32_t n,
                                                          const uint32_t* __restrict__ new_id) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) id[i] = new_id[id[i]];
}

}  // namespace

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, uint32_t* total,
                        cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(uint32_t), s);
        return;
    }
    const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    launch_pdl(scan_tile_sums_kernel, tiles, kScanThreads, 0, s, in, n, scratch);
    launch_pdl(scan_sums_kernel, 1, kScanThreads, 0, s, scratch, tiles, total);
    launch_pdl(scan_apply_kernel, tiles, kScanThreads, 0, s, in, n, scratch, out);
}

void mesh_ray_direction(float dir[3]) {
    // the constants are doubles rounded to float, as Vector3d(2.575, 6.19763, 5.986) rounds them;
    // volatile: no contraction, no reassociation
    volatile float x = (float)2.575, y = (float)6.19763, z = (float)5.986;
    volatile float xx = x * x, yy = y * y, zz = z * z;
    volatile float s = xx + yy;
    s = s + zz;
    const float nrm = std::sqrt((float)s);
    dir[0] = x / nrm;
    dir[1] = y / nrm;
    dir[2] = z / nrm;
}

template <class Real>
void launch_open_boundary_select(const float4* samples, uint32_t ns, DevSurface interior, DevSurface fluid_surface,
                                 const StepParams<Real>& p, uint32_t* keep, cudaStream_t s) {
    if (ns) launch_pdl(select_kernel<Real>, grid_for(ns), kBlock, 0, s, samples, ns, interior, fluid_surface, p, keep);
}
void launch_compact_samples(const float4* samples, const uint32_t* keep, const uint32_t* rank, uint32_t ns,
                            float4* out, cudaStream_t s) {
    if (ns) launch_pdl(compact_samples_kernel, grid_for(ns), kBlock, 0, s, samples, keep, rank, ns, out);
}
void launch_shift_samples(float4* samples, uint32_t ns, float dx, float dy, float dz, cudaStream_t s) {
    if (ns) launch_pdl(shift_samples_kernel, grid_for(ns), kBlock, 0, s, samples, ns, dx, dy, dz);
}
template <class Real>
void launch_inflow(const DevState<Real>* d, const float4* samples, uint32_t ns, float allowed_distance,
                   float allowed_density, Real mass, DevSurface boundary, const uint2* fluid_table,
                   const uint2* boundary_table, uint32_t* flag, float4* vel, cudaStream_t s) {
    if (ns)
        launch_pdl(inflow_kernel<Real>, grid_for(ns), kBlock, 0, s, d, samples, ns, allowed_distance, allowed_density, mass,
                                                            boundary, fluid_table, boundary_table, flag, vel);
}
template <class Real>
void launch_append_inflow(const float4* samples, const float4* svel, const uint32_t* flag, const uint32_t* rank,
                          uint32_t ns, uint32_t n, uint32_t capacity, Real mass, Vec4<Real>* pos, Vec4<Real>* vel,
                          Real* kappa, Real* kappaV, uint32_t* id, Real* kappaT, Real* kappaVT, cudaStream_t s) {
    if (ns && n < capacity)
        launch_pdl(append_kernel<Real>, grid_for(ns), kBlock, 0, s, samples, svel, flag, rank, ns, n, capacity, mass, pos, vel,
                                                            kappa, kappaV, id, kappaT, kappaVT);
}
template <class Real>
void launch_outflow_tag(const Vec4<Real>* pos, uint32_t n, DevSurface interior, DevSurface fluid_surface,
                        uint32_t* alive, cudaStream_t s) {
    if (n) launch_pdl(outflow_tag_kernel<Real>, grid_for(n), kBlock, 0, s, pos, n, interior, fluid_surface, alive);
}
template <class Real>
void launch_compact_fluid(const uint32_t* alive, const uint32_t* dst, uint32_t n, const Vec4<Real>* pos_in,
                          const Vec4<Real>* vel_in, const Real* kappa_in, const Real* kappaV_in, const uint32_t* id_in,
                          const Real* kT_in, const Real* kVT_in, Vec4<Real>* pos_out, Vec4<Real>* vel_out,
                          Real* kappa_out, Real* kappaV_out, uint32_t* id_out, Real* kT_out, Real* kVT_out,
                          cudaStream_t s) {
    if (n)
        launch_pdl(compact_fluid_kernel<Real>, grid_for(n), kBlock, 0, s, alive, dst, n, pos_in, vel_in, kappa_in, kappaV_in,
                                                                  id_in, kT_in, kVT_in, pos_out, vel_out, kappa_out,
                                                                  kappaV_out, id_out, kT_out, kVT_out);
}
template <class Real>
void launch_box_tag(const Vec4<Real>* pos, uint32_t n, const float lo[3], const float hi[3], uint32_t* alive,
                    uint32_t* count, cudaStream_t s) {
    if (n)
        launch_pdl(box_tag_kernel<Real>, grid_for(n), kBlock, 0, s, pos, n, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], alive,
                                                            count);
}
void launch_alive_by_id(const uint32_t* id, const uint32_t* alive, uint32_t n, uint32_t* alive_by_id, cudaStream_t s) {
    if (n) launch_pdl(alive_by_id_kernel, grid_for(n), kBlock, 0, s, id, alive, n, alive_by_id);
}
void launch_renumber_ids(uint32_t* id, uint32_t n, const uint32_t* new_id, cudaStream_t s) {
    if (n) launch_pdl(renumber_kernel, grid_for(n), kBlock, 0, s, id, n, new_id);
}

#define DFSPH_INSTANTIATE_OPEN_BOUNDARY(R)                                                                        \
    template void launch_open_boundary_select<R>(const float4*, uint32_t, DevSurface, DevSurface,           \
                                                 const StepParams<R>&, uint32_t*, cudaStream_t);                  \
    template void launch_inflow<R>(const DevState<R>*, const float4*, uint32_t, float, float, R, DevSurface,   \
                                   const uint2*, const uint2*, uint32_t*, float4*, cudaStream_t);                 \
    template void launch_append_inflow<R>(const float4*, const float4*, const uint32_t*, const uint32_t*,         \
                                          uint32_t, uint32_t, uint32_t, R, Vec4<R>*, Vec4<R>*, R*, R*, uint32_t*, \
                                          R*, R*, cudaStream_t);                                                  \
    template void launch_outflow_tag<R>(const Vec4<R>*, uint32_t, DevSurface, DevSurface, uint32_t*,        \
                                        cudaStream_t);                                                            \
    template void launch_compact_fluid<R>(const uint32_t*, const uint32_t*, uint32_t, const Vec4<R>*,             \
                                          const Vec4<R>*, const R*, const R*, const uint32_t*, const R*, const R*, \
                                          Vec4<R>*, Vec4<R>*, R*, R*, uint32_t*, R*, R*, cudaStream_t);       \
    template void launch_box_tag<R>(const Vec4<R>*, uint32_t, const float*, const float*, uint32_t*, uint32_t*,   \
                                    cudaStream_t);

DFSPH_INSTANTIATE_OPEN_BOUNDARY(float)
DFSPH_INSTANTIATE_OPEN_BOUNDARY(double)

}  // namespace dfsph
