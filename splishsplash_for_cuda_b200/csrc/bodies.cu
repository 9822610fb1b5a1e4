// bodies.cu — force and torque of the fluid on boundary bodies.
//
// The reference hands the per-particle boundary forces of its dynamic bodies to the host each step
// (DFSPHCData::readDynamicObjectsData, DFSPH_c_arrays_structure.cpp:1177-1193; the forces are the
// atomicAdd of -m_i k_i psi_b grad W_ib in the Jacobi passes, DFSPH_core_cuda.cu:335-337, 804-806)
// and the rigid-body solver sums them. Here the sum is taken on the device: the forces and
// positions are first packed into upload order, so each body is a contiguous range, then one block
// per body reduces its range in a fixed order (deterministic, FP64).
#include "bodies.cuh"
#include "dfsph_common.cuh"

namespace dfsph {

namespace {

constexpr int kWrenchThreads = 256;

__global__ void __launch_bounds__(kWrenchThreads) body_wrench_kernel(const double* __restrict__ pos,
                                                                     const double* __restrict__ force,
                                                                     const uint32_t* __restrict__ first,
                                                                     const uint32_t* __restrict__ count,
                                                                     const double* __restrict__ centers,
                                                                     double* __restrict__ out) {
    DFSPH_PDL_ENTER;
    __shared__ double acc[6][kWrenchThreads];
    const uint32_t b = blockIdx.x;
    const double cx = centers[3 * b], cy = centers[3 * b + 1], cz = centers[3 * b + 2];
    double f[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    const uint32_t lo = first[b], hi = first[b] + count[b];
    for (uint32_t u = lo + threadIdx.x; u < hi; u += kWrenchThreads) {
        const double fx = force[3 * (size_t)u], fy = force[3 * (size_t)u + 1], fz = force[3 * (size_t)u + 2];
        const double rx = pos[3 * (size_t)u] - cx, ry = pos[3 * (size_t)u + 1] - cy, rz = pos[3 * (size_t)u + 2] - cz;
        f[0] += fx;
        f[1] += fy;
        f[2] += fz;
        t[0] += ry * fz - rz * fy;
        t[1] += rz * fx - rx * fz;
        t[2] += rx * fy - ry * fx;
    }
    for (int c = 0; c < 3; ++c) {
        acc[c][threadIdx.x] = f[c];
        acc[3 + c][threadIdx.x] = t[c];
    }
    __syncthreads();
    for (int w = kWrenchThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 6; ++c) acc[c][threadIdx.x] += acc[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 6) out[6 * (size_t)b + threadIdx.x] = acc[threadIdx.x][0];
}

}  // namespace

void launch_body_wrench(const double* pos, const double* force, const uint32_t* first, const uint32_t* count,
                        const double* centers, uint32_t n_bodies, double* out, cudaStream_t s) {
    if (n_bodies) launch_pdl(body_wrench_kernel, n_bodies, kWrenchThreads, 0, s, pos, force, first, count, centers, out);
}

}  // namespace dfsph
