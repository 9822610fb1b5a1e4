// sort.cu — stable LSD radix sort of 32-bit cell keys with 32-bit payloads.
//
// Replaces the reference's per-step counting sort over a dense 256^3 cell histogram
// (DFSPH_core_cuda.cu:1833-1857 atomicAdd ranks + cub::DeviceScan over 16.8 M counters at :1920),
// whose order within a cell depends on atomics. This sort is stable, so the sorted order, the
// neighbour lists and every sum that follows are deterministic run to run.
//
// Design: 8-bit digits; one histogram pass computes all digit histograms; each digit pass is a
// single "onesweep" kernel: a tile ranks its keys stably in shared memory (warp match + per-warp
// digit counters), publishes its per-digit count, and obtains its global exclusive prefix by a
// decoupled look-back over earlier tiles. Tiles take their index from an atomic counter at start,
// so a tile only ever waits on tiles that are already running; every wait is bounded and gives up
// with DFSPH_ST_SORT_TIMEOUT instead of hanging.
#include "dfsph_common.cuh"
#include "sort.cuh"

namespace dfsph {

namespace {
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr int kSpinLimit = 1 << 22;

__global__ void __launch_bounds__(kSortThreads) histogram_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                 int passes, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[4][256];
    for (int t = threadIdx.x; t < 4 * 256; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < passes * 256; t += blockDim.x) {
        const uint32_t v = (&sh[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

// Exclusive scan of each pass's 256-bin histogram (one block of 256 threads).
__global__ void __launch_bounds__(256) scan_kernel(const uint32_t* __restrict__ hist, int passes,
                                                   uint32_t* __restrict__ offsets) {
    __shared__ uint32_t s[256];
    for (int p = 0; p < passes; ++p) {
        const uint32_t v = hist[p * 256 + threadIdx.x];
        s[threadIdx.x] = v;
        __syncthreads();
        for (int d = 1; d < 256; d <<= 1) {
            const uint32_t add = threadIdx.x >= d ? s[threadIdx.x - d] : 0u;
            __syncthreads();
            s[threadIdx.x] += add;
            __syncthreads();
        }
        offsets[p * 256 + threadIdx.x] = s[threadIdx.x] - v;
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }

__global__ void __launch_bounds__(kSortThreads) onesweep_kernel(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, uint32_t n, int shift, const uint32_t* __restrict__ digit_offsets,
    uint32_t* __restrict__ tile_status, uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status_word) {
    __shared__ uint32_t warp_hist[kSortWarps][256];
    __shared__ uint32_t digit_base[256];
    __shared__ uint32_t s_tile;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kSortWarps * 256; t += kSortThreads) (&warp_hist[0][0])[t] = 0;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kSortTile + warp * (kSortItems * 32);

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
    const uint32_t lanemask_lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + r * 32 + lane;
        const bool valid = idx < n;
        key[r] = valid ? kin[idx] : 0u;
        val[r] = valid ? (vin ? vin[idx] : idx) : 0u;
        const uint32_t d = valid ? ((key[r] >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t prior = valid ? warp_hist[warp][d] : 0u;
        __syncwarp();
        if (valid && (peers & lanemask_lt) == 0) warp_hist[warp][d] = prior + __popc(peers);
        __syncwarp();
        rank[r] = prior + __popc(peers & lanemask_lt);
    }
    __syncthreads();

    // Per digit: exclusive prefix over warps, tile total, then the decoupled look-back.
    {
        const int d = threadIdx.x;  // kSortThreads == 256 digits
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = warp_hist[w][d];
            warp_hist[w][d] = total;
            total += c;
        }
        uint32_t* my = tile_status + (size_t)tile * 256 + d;
        uint32_t exclusive = 0;
        if (tile == 0) {
            st_volatile(my, kFlagPrefix | total);
        } else {
            st_volatile(my, kFlagAggregate | total);
            int look = (int)tile - 1;
            int spins = 0;
            while (look >= 0) {
                const uint32_t v = ld_volatile(tile_status + (size_t)look * 256 + d);
                const uint32_t flag = v & ~kCountMask;
                if (flag == 0) {
                    if (++spins > kSpinLimit) {
                        atomicOr(status_word, DFSPH_ST_SORT_TIMEOUT);
                        break;
                    }
                    if (spins > 16) __nanosleep(64);
                    continue;
                }
                exclusive += v & kCountMask;
                if (flag == kFlagPrefix) break;
                --look;
            }
            st_volatile(my, kFlagPrefix | ((exclusive + total) & kCountMask));
        }
        digit_base[d] = digit_offsets[d] + exclusive;
    }
    __syncthreads();

#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[r] >> shift) & 255u;
            const uint32_t pos = digit_base[d] + warp_hist[warp][d] + rank[r];
            if (pos < n) {  // only false after a timed-out look-back; never write out of range
                kout[pos] = key[r];
                vout[pos] = val[r];
            }
        }
    }
}
}  // namespace

size_t radix_sort_workspace_words(uint32_t n_max, int passes) {
    const size_t tiles = (n_max + kSortTile - 1) / kSortTile;
    return 4 + 1024 + 1024 + (size_t)passes * tiles * 256;
}

// Sorts (keys_a, vals_a) by key. Pass p reads buffer set (p even ? a : b) and writes the other;
// the first pass takes iota payloads when iota_values is set. The result is returned through
// *keys_out / *vals_out and lies in set a after an even number of passes, else in set b.
void radix_sort_pairs(SortBuffers& b, uint32_t n, int passes, bool iota_values, cudaStream_t stream,
                      uint32_t* status_word, uint64_t* launch_counter, uint32_t** keys_out, uint32_t** vals_out) {
    if (n == 0 || passes == 0) {
        *keys_out = b.keys_a;
        *vals_out = b.vals_a;
        return;
    }
    const size_t tiles = (n + kSortTile - 1) / kSortTile;
    // workspace: [0,4) tile counters, [4,1028) histograms, [1028,2052) digit offsets, then tile status
    uint32_t* counters = b.workspace;
    uint32_t* hist = b.workspace + 4;
    uint32_t* offsets = hist + 1024;
    uint32_t* status = offsets + 1024;
    cudaMemsetAsync(b.workspace, 0, radix_sort_workspace_words(n, passes) * sizeof(uint32_t), stream);
    int hist_blocks = (int)((n + kSortThreads * 16 - 1) / (kSortThreads * 16));
    if (hist_blocks > 148 * 4) hist_blocks = 148 * 4;
    if (hist_blocks < 1) hist_blocks = 1;
    histogram_kernel<<<hist_blocks, kSortThreads, 0, stream>>>(b.keys_a, n, passes, hist);
    scan_kernel<<<1, 256, 0, stream>>>(hist, passes, offsets);
    *launch_counter += 2;
    for (int p = 0; p < passes; ++p) {
        const bool even = (p & 1) == 0;
        const uint32_t* kin = even ? b.keys_a : b.keys_b;
        const uint32_t* vin = (p == 0 && iota_values) ? nullptr : (even ? b.vals_a : b.vals_b);
        uint32_t* kout = even ? b.keys_b : b.keys_a;
        uint32_t* vout = even ? b.vals_b : b.vals_a;
        onesweep_kernel<<<(unsigned)tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, 8 * p, offsets + p * 256,
                                                                   status + (size_t)p * tiles * 256, counters + p,
                                                                   status_word);
        *launch_counter += 1;
    }
    const bool in_a = (passes & 1) == 0;
    *keys_out = in_a ? b.keys_a : b.keys_b;
    *vals_out = in_a ? b.vals_a : b.vals_b;
}

}  // namespace dfsph
