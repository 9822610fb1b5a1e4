// neighbors.cu — cell keys, fluid reorder, cell-start table, neighbour lists and boundary psi.
//
// Reference: cuda_neighborsSearch (DFSPH_core_cuda.cu:2651-3024) with
// DFSPH_computeGridIdx_kernel (:1833-1848), DFSPH_CountingSortIds_kernel (:1851-1857),
// cuda_sortData (:2057-2120) and DFSPH_neighborsSearch_kernel<true> (:2219-2517), which iterates
// ITER_NEIGHBORS_FROM_STRUCTURE_LINEAR_ADVANCED (DFSPH_macro_cuda.h:136-155): every particle of the
// 27 cells around the particle's cell is tested with squaredNorm < H^2, self excluded for the fluid.
//
// Differences by design: 30-bit Morton keys sorted by a stable in-house radix sort (sort.cu)
// instead of a dense 256^3 histogram; a cell table sized to the scene's grid, cleared per step;
// neighbour lists with a checked capacity (the reference writes past MAX_NEIGHBOURS = 90 unchecked).
#include "dfsph_state.cuh"

namespace dfsph {

namespace {

template <class Real>
__device__ __forceinline__ bool particle_cell(Real x, Real y, Real z, const StepParams<Real>& p, int& cx, int& cy,
                                              int& cz) {
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) return false;
    cx = cell_coord(x, p.kern.H, p.off_x);
    cy = cell_coord(y, p.kern.H, p.off_y);
    cz = cell_coord(z, p.kern.H, p.off_z);
    return cx >= 0 && cy >= 0 && cz >= 0 && cx < p.dim_x && cy < p.dim_y && cz < p.dim_z;
}

__device__ __forceinline__ uint32_t cell_linear(int cx, int cy, int cz, int dim_x, int dim_y) {
    return (uint32_t)cx + (uint32_t)dim_x * ((uint32_t)cy + (uint32_t)dim_y * (uint32_t)cz);
}

template <class Real>
__global__ void __launch_bounds__(kBlock) cell_keys_kernel(const Vec4<Real>* __restrict__ pos, uint32_t n,
                                                           StepParams<Real> p, uint32_t* __restrict__ keys,
                                                           uint32_t* __restrict__ status, uint32_t* __restrict__ z0,
                                                           size_t w0, uint32_t* __restrict__ z1, size_t w1) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = i; k < w0; k += stride) z0[k] = 0u;  // optional buffers to clear (w = 0: none)
    for (size_t k = i; k < w1; k += stride) z1[k] = 0u;
    if (i >= n) return;
    const Vec4<Real> x = pos[i];
    int cx, cy, cz;
    uint32_t key;
    if (particle_cell(x.x, x.y, x.z, p, cx, cy, cz)) {
        key = morton3((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
    } else {
        key = kEscapedKey;
        const bool finite = isfinite(x.x) && isfinite(x.y) && isfinite(x.z);
        atomicOr(status, finite ? DFSPH_ST_ESCAPED : (DFSPH_ST_NONFINITE | DFSPH_ST_ESCAPED));
    }
    keys[i] = key;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) reorder_fluid_kernel(
    const uint32_t* __restrict__ perm, uint32_t n, const Vec4<Real>* __restrict__ pos_in,
    const Vec4<Real>* __restrict__ vel_in, const Real* __restrict__ kappa_in, const Real* __restrict__ kappaV_in,
    const uint32_t* __restrict__ id_in, Vec4<Real>* __restrict__ pos_out, Vec4<Real>* __restrict__ vel_out,
    Real* __restrict__ kappa_out, Real* __restrict__ kappaV_out, uint32_t* __restrict__ id_out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t j = perm[i];
    if (j >= n) j = i;  // only after a failed sort (flagged in the status word); stay in range
    pos_out[i] = pos_in[j];
    vel_out[i] = vel_in[j];
    kappa_out[i] = kappa_in[j];
    kappaV_out[i] = kappaV_in[j];
    id_out[i] = id_in[j];
}

template <class Real>
__global__ void __launch_bounds__(kBlock) reorder_pair_kernel(const uint32_t* __restrict__ perm, uint32_t n,
                                                              const Real* __restrict__ a_in,
                                                              const Real* __restrict__ b_in, Real* __restrict__ a_out,
                                                              Real* __restrict__ b_out) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t j = perm[i];
    if (j >= n) j = i;
    a_out[i] = a_in[j];
    b_out[i] = b_in[j];
}

// Cell start/end from run boundaries of the sorted keys (replaces the dense histogram scan).
__global__ void __launch_bounds__(kBlock) cell_bounds_kernel(const uint32_t* __restrict__ keys, uint32_t n, int dim_x,
                                                             int dim_y, int dim_z, uint2* __restrict__ table) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = keys[i];
    if (k == kEscapedKey) return;
    const uint32_t cx = compact_bits10(k), cy = compact_bits10(k >> 1), cz = compact_bits10(k >> 2);
    if (cx >= (uint32_t)dim_x || cy >= (uint32_t)dim_y || cz >= (uint32_t)dim_z) return;
    const uint32_t lin = cell_linear((int)cx, (int)cy, (int)cz, dim_x, dim_y);
    if (i == 0 || keys[i - 1] != k) table[lin].x = i;
    if (i == n - 1 || keys[i + 1] != k) table[lin].y = i + 1;
}

// A cell-table run [r.x, r.y) of a set of `limit` particles. Checked builds verify it and raise
// DFSPH_ST_INDEX instead of scanning a run out of range; the unchecked build trusts the table.
__device__ __forceinline__ bool run_in_range(uint2 r, uint32_t limit, uint32_t* status) {
#ifdef DFSPH_CHECKED
    if (r.x > r.y || r.y > limit) {
        atomicOr(status, DFSPH_ST_INDEX);
        return false;
    }
#else
    (void)r;
    (void)limit;
    (void)status;
#endif
    return true;
}

#ifdef DFSPH_CHECKED
// Test hook of the checked build: replaces particle 0's first list entry by `value` (an index past the
// fluid count, inside the allocation), which the validation below must report.
__global__ void corrupt_first_neighbor_kernel(uint32_t* __restrict__ nbr, const uint32_t* __restrict__ counts,
                                              uint32_t value) {
    if (threadIdx.x == 0 && (counts[0] & 0xFFFFu) > 0) nbr[0] = value;
}

// Validation of the lists before any pass gathers through them (checked build): a count past the
// table's capacity, a fluid entry >= n or a boundary entry >= n_boundary raises DFSPH_ST_INDEX and
// empties that particle's list, so no pass reads out of range. The passes themselves are the
// unchecked build's code, so a clean run gives the same bits.
__global__ void __launch_bounds__(kBlock) validate_neighbors_kernel(uint32_t* __restrict__ counts,
                                                                    const uint32_t* __restrict__ nbr, uint32_t n,
                                                                    uint32_t n_boundary, uint32_t stride, uint32_t cap,
                                                                    uint32_t* __restrict__ status) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = counts[i], nf = c & 0xFFFFu, nb = c >> 16;
    bool bad = nf + nb > cap;
    for (uint32_t k = 0; k < nf + nb && !bad; ++k) bad = nbr[(size_t)k * stride + i] >= (k < nf ? n : n_boundary);
    if (bad) {
        atomicOr(status, DFSPH_ST_INDEX);
        counts[i] = 0u;
    }
}
#endif

// One thread per fluid particle: fluid neighbours (self excluded) then boundary neighbours, cells in
// a fixed order (z, y, x from -1 to +1), particles of a cell in sorted order. Lists are written
// interleaved (nbr[k * stride + i]) so that the gathers read them coalesced.
// Appends the candidates [j0, j1) of one cell that lie within H of particle i, in index order (the
// fluid skips i itself). The positions are loaded kScanBatch at a time so that several loads are in
// flight per thread; the tests and appends keep the order of a one-at-a-time loop.
constexpr uint32_t kScanBatch = 4;
template <class Real, bool kFluid>
__device__ __forceinline__ void scan_cell(const Vec4<Real>* __restrict__ src, uint32_t j0, uint32_t j1, uint32_t i,
                                          const Vec4<Real>& xi, Real H2, uint32_t* __restrict__ nbr, uint32_t stride,
                                          uint32_t cap, uint32_t& total, uint32_t& cnt, bool& overflow) {
    for (uint32_t jb = j0; jb < j1; jb += kScanBatch) {
        Vec4<Real> xj[kScanBatch];
#pragma unroll
        for (uint32_t u = 0; u < kScanBatch; ++u) xj[u] = ld4<Real>(src + min(jb + u, j1 - 1));
#pragma unroll
        for (uint32_t u = 0; u < kScanBatch; ++u) {
            const uint32_t j = jb + u;
            if (j < j1 && (!kFluid || j != i) && pair_within(xi.x, xi.y, xi.z, xj[u].x, xj[u].y, xj[u].z, H2)) {
                if (total < cap) {
                    nbr[(size_t)total * stride + i] = j;
                    ++total;
                    ++cnt;
                } else {
                    overflow = true;
                }
            }
        }
    }
}

template <class Real, bool kShift>
__global__ void __launch_bounds__(kBlock) build_neighbors_kernel(const DevState<Real>* __restrict__ ds, uint32_t n,
                                                                 const uint2* __restrict__ ftab,
                                                                 const uint2* __restrict__ btab) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepParams<Real>& p = ds->p;
    const Vec4<Real>* __restrict__ pos = ds->pos;
    const Vec4<Real>* __restrict__ bpos = ds->bpos;
    uint32_t* __restrict__ nbr = ds->nbr;
    const uint32_t stride = p.nbr_stride, cap = p.nbr_cap;
    const Vec4<Real> xi = pos[i];
    int cx, cy, cz;
    uint32_t nf = 0, nb = 0, total = 0;
    bool overflow = false;
    if (particle_cell(xi.x, xi.y, xi.z, p, cx, cy, cz)) {
        const Real H2 = p.H2;
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = cz + dz;
            if (z < 0 || z >= p.dim_z) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = cy + dy;
                if (y < 0 || y >= p.dim_y) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = cx + dx;
                    if (x < 0 || x >= p.dim_x) continue;
                    const uint2 r = ftab[cell_linear(x, y, z, p.dim_x, p.dim_y)];
                    if (!run_in_range(r, n, ds->status)) continue;
                    scan_cell<Real, true>(pos, r.x, r.y, i, xi, H2, nbr, stride, cap, total, nf, overflow);
                }
            }
        }
        if (p.n_boundary > 0 && !kShift) {
            for (int dz = -1; dz <= 1; ++dz) {
                const int z = cz + dz;
                if (z < 0 || z >= p.dim_z) continue;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int y = cy + dy;
                    if (y < 0 || y >= p.dim_y) continue;
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int x = cx + dx;
                        if (x < 0 || x >= p.dim_x) continue;
                        const uint2 r = btab[cell_linear(x, y, z, p.dim_x, p.dim_y)];
                        if (!run_in_range(r, p.n_boundary, ds->status)) continue;
                        scan_cell<Real, false>(bpos, r.x, r.y, i, xi, H2, nbr, stride, cap, total, nb, overflow);
                    }
                }
            }
        }
        if (p.n_boundary > 0 && kShift) {
            // The whole boundary has only translated by s since it was binned: the cells around the
            // binned cell of x_i - s, with one more layer on a side where x_i - s lies within 1e-3 of a
            // cell face (the binned and the current positions differ from s by rounding; the pair test
            // uses the current positions).
            int lo[3], hi[3];
            bool query = true;
            const float q[3] = {__fsub_rn((float)xi.x, (float)p.bsx), __fsub_rn((float)xi.y, (float)p.bsy),
                                __fsub_rn((float)xi.z, (float)p.bsz)};
            const int off[3] = {p.off_x, p.off_y, p.off_z};
            const float Hf = (float)p.kern.H;
            for (int a = 0; a < 3 && query; ++a) {
                const float t = __fadd_rn(__fdiv_rn(q[a], Hf), (float)off[a]);
                if (!(fabsf(t) < 1.0e8f)) {  // also NaN: no boundary neighbours, as off the grid
                    query = false;
                    break;
                }
                const float c = floorf(t), frac = t - c;
                lo[a] = (int)c - 1 - (frac < 1e-3f ? 1 : 0);
                hi[a] = (int)c + 1 + (frac > 1.0f - 1e-3f ? 1 : 0);
            }
            for (int z = query ? lo[2] : 1; query && z <= hi[2]; ++z) {
                if (z < 0 || z >= p.dim_z) continue;
                for (int y = lo[1]; y <= hi[1]; ++y) {
                    if (y < 0 || y >= p.dim_y) continue;
                    for (int x = lo[0]; x <= hi[0]; ++x) {
                        if (x < 0 || x >= p.dim_x) continue;
                        const uint2 r = btab[cell_linear(x, y, z, p.dim_x, p.dim_y)];
                        if (!run_in_range(r, p.n_boundary, ds->status)) continue;
                        scan_cell<Real, false>(bpos, r.x, r.y, i, xi, H2, nbr, stride, cap, total, nb, overflow);
                    }
                }
            }
        }
    }
    if (overflow) atomicOr(ds->status, DFSPH_ST_NEIGHBOR_OVERFLOW);
    ds->counts[i] = nf | (nb << 16);
}

// Akinci boundary psi (FluidModel::computeBoundaryPsi, FluidModel.cpp:233-258):
// psi_b = rho0 / (W0 + sum_{b' != b, |x_b - x_b'| < H} W(x_b - x_b')), accumulated in FP64.
template <class Real>
__global__ void __launch_bounds__(kBlock) boundary_psi_kernel(const Vec4<Real>* __restrict__ bpos_in,
                                                              Vec4<Real>* __restrict__ bpos_out, uint32_t nb,
                                                              StepParams<Real> p, const uint2* __restrict__ btab,
                                                              uint32_t* __restrict__ status) {
    DFSPH_PDL_ENTER;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const Vec4<Real> xb = bpos_in[b];
    int cx, cy, cz;
    const double H = (double)p.kern.H;
    const double k = 8.0 / (3.14159265358979323846 * H * H * H);
    double delta = k;  // W(0)
    if (particle_cell(xb.x, xb.y, xb.z, p, cx, cy, cz)) {
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = cz + dz;
            if (z < 0 || z >= p.dim_z) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = cy + dy;
                if (y < 0 || y >= p.dim_y) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = cx + dx;
                    if (x < 0 || x >= p.dim_x) continue;
                    const uint2 r = btab[cell_linear(x, y, z, p.dim_x, p.dim_y)];
                    if (!run_in_range(r, nb, status)) continue;
                    for (uint32_t j = r.x; j < r.y; ++j) {
                        if (j == b) continue;
                        const Vec4<Real> xj = bpos_in[j];
                        if (pair_within(xb.x, xb.y, xb.z, xj.x, xj.y, xj.z, p.H2)) {
                            const double rx = (double)xb.x - (double)xj.x;
                            const double ry = (double)xb.y - (double)xj.y;
                            const double rz = (double)xb.z - (double)xj.z;
                            const double q = sqrt(rx * rx + ry * ry + rz * rz) / H;
                            double w = 0.0;
                            if (q <= 1.0) {
                                if (q <= 0.5) {
                                    w = k * (6.0 * q * q * q - 6.0 * q * q + 1.0);
                                } else {
                                    const double f = 1.0 - q;
                                    w = k * (2.0 * f * f * f);
                                }
                            }
                            delta += w;
                        }
                    }
                }
            }
        }
    } else {
        atomicOr(status, DFSPH_ST_BOUNDARY_OVERFLOW);
    }
    Vec4<Real> out = xb;
    out.w = (Real)((double)p.density0 / delta);
    bpos_out[b] = out;
}

template <class Real>
__global__ void __launch_bounds__(kBlock) scatter_by_id_kernel(const uint32_t* __restrict__ id, uint32_t n,
                                                               const Real* __restrict__ src, int comps,
                                                               int src_stride, Real* __restrict__ dst) {
    DFSPH_PDL_ENTER;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = id[i];
    for (int c = 0; c < comps; ++c) dst[(size_t)t * comps + c] = src[(size_t)i * src_stride + c];
}

}  // namespace

template <class Real>
void launch_cell_keys(const Vec4<Real>* pos, uint32_t n, const StepParams<Real>& p, uint32_t* keys, uint32_t* status,
                      cudaStream_t s, uint32_t* clear0, size_t words0, uint32_t* clear1, size_t words1) {
    if (n)
        launch_pdl(cell_keys_kernel<Real>, grid_for(n), kBlock, 0, s, pos, n, p, keys, status, clear0, words0, clear1,
                   words1);
}
template <class Real>
void launch_reorder_fluid(const uint32_t* perm, uint32_t n, const Vec4<Real>* pos_in, const Vec4<Real>* vel_in,
                          const Real* kappa_in, const Real* kappaV_in, const uint32_t* id_in, Vec4<Real>* pos_out,
                          Vec4<Real>* vel_out, Real* kappa_out, Real* kappaV_out, uint32_t* id_out, cudaStream_t s) {
    if (n)
        launch_pdl(reorder_fluid_kernel<Real>, grid_for(n), kBlock, 0, s, perm, n, pos_in, vel_in, kappa_in, kappaV_in, id_in,
                                                                  pos_out, vel_out, kappa_out, kappaV_out, id_out);
}
template <class Real>
void launch_reorder_pair(const uint32_t* perm, uint32_t n, const Real* a_in, const Real* b_in, Real* a_out,
                         Real* b_out, cudaStream_t s) {
    if (n) launch_pdl(reorder_pair_kernel<Real>, grid_for(n), kBlock, 0, s, perm, n, a_in, b_in, a_out, b_out);
}
void launch_cell_bounds(const uint32_t* sorted_keys, uint32_t n, int dim_x, int dim_y, int dim_z, uint2* table,
                        cudaStream_t s) {
    if (n) launch_pdl(cell_bounds_kernel, grid_for(n), kBlock, 0, s, sorted_keys, n, dim_x, dim_y, dim_z, table);
}
template <class Real>
void launch_build_neighbors(const DevState<Real>* d, uint32_t n, const uint2* fluid_table, const uint2* boundary_table,
                            cudaStream_t s, bool boundary_shifted) {
    if (!n) return;
    if (boundary_shifted)
        launch_pdl(build_neighbors_kernel<Real, true>, grid_for(n), kBlock, 0, s, d, n, fluid_table, boundary_table);
    else
        launch_pdl(build_neighbors_kernel<Real, false>, grid_for(n), kBlock, 0, s, d, n, fluid_table, boundary_table);
}
void launch_validate_neighbors(uint32_t* counts, const uint32_t* nbr, uint32_t n, uint32_t n_boundary, uint32_t stride,
                               uint32_t cap, uint32_t* status, cudaStream_t s) {
#ifdef DFSPH_CHECKED
    if (n) launch_pdl(validate_neighbors_kernel, grid_for(n), kBlock, 0, s, counts, nbr, n, n_boundary, stride, cap, status);
#else
    (void)counts;
    (void)nbr;
    (void)n;
    (void)n_boundary;
    (void)stride;
    (void)cap;
    (void)status;
    (void)s;
#endif
}
void launch_corrupt_first_neighbor(uint32_t* nbr, const uint32_t* counts, uint32_t value, cudaStream_t s) {
#ifdef DFSPH_CHECKED
    corrupt_first_neighbor_kernel<<<1, 32, 0, s>>>(nbr, counts, value);
#else
    (void)nbr;
    (void)counts;
    (void)value;
    (void)s;
#endif
}
template <class Real>
void launch_boundary_psi(const Vec4<Real>* bpos_in, Vec4<Real>* bpos_out, uint32_t nb, const StepParams<Real>& p,
                         const uint2* boundary_table, uint32_t* status, cudaStream_t s) {
    if (nb) launch_pdl(boundary_psi_kernel<Real>, grid_for(nb), kBlock, 0, s, bpos_in, bpos_out, nb, p, boundary_table, status);
}
template <class Real>
void launch_scatter_by_id(const uint32_t* id, uint32_t n, const Real* src, int comps, int src_stride, Real* dst,
                          cudaStream_t s) {
    if (n) launch_pdl(scatter_by_id_kernel<Real>, grid_for(n), kBlock, 0, s, id, n, src, comps, src_stride, dst);
}

#define DFSPH_INSTANTIATE_NEIGHBORS(R)                                                                               \
    template void launch_cell_keys<R>(const Vec4<R>*, uint32_t, const StepParams<R>&, uint32_t*, uint32_t*,          \
                                      cudaStream_t, uint32_t*, size_t, uint32_t*, size_t);                           \
    template void launch_reorder_fluid<R>(const uint32_t*, uint32_t, const Vec4<R>*, const Vec4<R>*, const R*,       \
                                          const R*, const uint32_t*, Vec4<R>*, Vec4<R>*, R*, R*, uint32_t*,          \
                                          cudaStream_t);                                                             \
    template void launch_build_neighbors<R>(const DevState<R>*, uint32_t, const uint2*, const uint2*, cudaStream_t,   \
                                            bool);                                                                   \
    template void launch_reorder_pair<R>(const uint32_t*, uint32_t, const R*, const R*, R*, R*, cudaStream_t);       \
    template void launch_boundary_psi<R>(const Vec4<R>*, Vec4<R>*, uint32_t, const StepParams<R>&, const uint2*,     \
                                         uint32_t*, cudaStream_t);                                                   \
    template void launch_scatter_by_id<R>(const uint32_t*, uint32_t, const R*, int, int, R*, cudaStream_t);

DFSPH_INSTANTIATE_NEIGHBORS(float)
DFSPH_INSTANTIATE_NEIGHBORS(double)

}  // namespace dfsph
