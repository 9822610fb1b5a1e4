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
#include <string>

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

// Digits are taken from key & key_mask (all ones for the solver's keys).
__global__ void __launch_bounds__(kSortThreads) histogram_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                 int passes, uint32_t key_mask,
                                                                 uint32_t* __restrict__ hist) {
    DFSPH_PDL_ENTER;
    __shared__ uint32_t sh[4][256];
    for (int t = threadIdx.x; t < 4 * 256; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i] & key_mask;
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
    DFSPH_PDL_ENTER;
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
    uint32_t* __restrict__ vout, uint32_t n, int shift, uint32_t key_mask, const uint32_t* __restrict__ digit_offsets,
    uint32_t* __restrict__ tile_status, uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status_word,
    uint32_t withheld_tile) {
    DFSPH_PDL_ENTER;
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
        const uint32_t d = valid ? (((key[r] & key_mask) >> shift) & 255u) : 256u;
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
        // A withheld tile (failure-detection tests only) never publishes: its successors' bounded
        // look-back runs out and raises DFSPH_ST_SORT_TIMEOUT.
        const bool publish = tile != withheld_tile;
        if (tile == 0) {
            if (publish) st_volatile(my, kFlagPrefix | total);
        } else {
            if (publish) st_volatile(my, kFlagAggregate | total);
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
            if (publish) st_volatile(my, kFlagPrefix | ((exclusive + total) & kCountMask));
        }
        digit_base[d] = digit_offsets[d] + exclusive;
    }
    __syncthreads();

#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = ((key[r] & key_mask) >> shift) & 255u;
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
                      uint32_t* status_word, uint64_t* launch_counter, uint32_t** keys_out, uint32_t** vals_out,
                      uint32_t withheld_tile, bool workspace_cleared) {
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
    if (!workspace_cleared)
        cudaMemsetAsync(b.workspace, 0, radix_sort_workspace_words(n, passes) * sizeof(uint32_t), stream);
    int hist_blocks = (int)((n + kSortThreads * 16 - 1) / (kSortThreads * 16));
    if (hist_blocks > 148 * 4) hist_blocks = 148 * 4;
    if (hist_blocks < 1) hist_blocks = 1;
    launch_pdl(histogram_kernel, hist_blocks, kSortThreads, 0, stream, b.keys_a, n, passes, 0xFFFFFFFFu, hist);
    launch_pdl(scan_kernel, 1, 256, 0, stream, hist, passes, offsets);
    *launch_counter += 2;
    for (int p = 0; p < passes; ++p) {
        const bool even = (p & 1) == 0;
        const uint32_t* kin = even ? b.keys_a : b.keys_b;
        const uint32_t* vin = (p == 0 && iota_values) ? nullptr : (even ? b.vals_a : b.vals_b);
        uint32_t* kout = even ? b.keys_b : b.keys_a;
        uint32_t* vout = even ? b.vals_b : b.vals_a;
        launch_pdl(onesweep_kernel, (unsigned)tiles, kSortThreads, 0, stream, kin, vin, kout, vout, n, 8 * p, 0xFFFFFFFFu,
                   offsets + p * 256,
                                                                   status + (size_t)p * tiles * 256, counters + p,
                                                                   status_word, withheld_tile);
        *launch_counter += 1;
    }
    const bool in_a = (passes & 1) == 0;
    *keys_out = in_a ? b.keys_a : b.keys_b;
    *vals_out = in_a ? b.vals_a : b.vals_b;
}

// ---------------------------------------------------------------------------------------------------
// Allocation-free variant of the cell-key sort.
//
// Some callers cannot allocate device memory at all: code that runs inside a host that owns every
// allocation (a simulation framework with its own pool, a plugin that is handed device buffers and
// must not grow the process's footprint, or code running where cudaMalloc would synchronise the
// device). dfsph_sort_cell_keys_noalloc serves them: the caller passes the input keys and the output
// buffers, and the sort's scratch (digit histograms, look-back tile flags, one ping-pong key/payload
// pair) lives in the file-scope device array below, of a fixed maximum size. Every GPU that loads
// this library holds the array until the process exits.
namespace {
constexpr uint32_t kNoAllocMaxKeys = 1u << 18;  // 262,144 keys per call
constexpr size_t kNoAllocTiles = (kNoAllocMaxKeys + kSortTile - 1) / kSortTile;
// layout (32-bit words): [0,4) tile counters, [4,8) status word, [8,1032) digit histograms,
// [1032,2056) digit offsets, then 4 passes of tile look-back flags, then the ping-pong keys and
// payloads. Everything before the ping-pong pair is cleared at the start of every call.
constexpr size_t kNoAllocCounters = 0, kNoAllocStatus = 4, kNoAllocHist = 8, kNoAllocOffsets = 1032;
constexpr size_t kNoAllocTileFlags = 2056;
constexpr size_t kNoAllocClearWords = kNoAllocTileFlags + 4 * kNoAllocTiles * 256;
constexpr size_t kNoAllocWords = kNoAllocClearWords + 2 * (size_t)kNoAllocMaxKeys;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

int noalloc_fail(int code, const std::string& msg) {
    set_global_error(msg);  // reported by dfsph_last_error(NULL)
    return code;
}
}  // namespace

}  // namespace dfsph

extern "C" int dfsph_sort_cell_keys_noalloc(const uint32_t* keys_in, uint32_t* keys_out, uint32_t* perm_out,
                                            uint32_t n, int key_bits, void* stream) {
    using namespace dfsph;
    if (n > kNoAllocMaxKeys)
        return noalloc_fail(DFSPH_E_INVALID, "dfsph_sort_cell_keys_noalloc: n = " + std::to_string(n) +
                                                 " exceeds the maximum of " + std::to_string(kNoAllocMaxKeys) + " keys");
    if (key_bits < 1 || key_bits > 32) return noalloc_fail(DFSPH_E_INVALID, "key_bits must be in [1, 32]");
    if (n == 0) return DFSPH_OK;
    if (!keys_in || !keys_out || !perm_out) return noalloc_fail(DFSPH_E_INVALID, "null device buffer");
    // The passes read the input while they write the outputs (an odd pass count writes the caller's
    // buffers on the first pass): overlapping buffers would race.
    const auto overlap = [n](const void* a, const void* b) {
        const uintptr_t pa = (uintptr_t)a, pb = (uintptr_t)b, len = (uintptr_t)n * sizeof(uint32_t);
        return pa < pb + len && pb < pa + len;
    };
    if (overlap(keys_in, keys_out) || overlap(keys_in, perm_out) || overlap(keys_out, perm_out))
        return noalloc_fail(DFSPH_E_INVALID, "keys_in, keys_out and perm_out must not overlap");
    cudaStream_t s = (cudaStream_t)stream;
    // The call ends with a copy into host memory and a wait, neither of which a stream capture admits.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return noalloc_fail(DFSPH_E_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
        return noalloc_fail(DFSPH_E_STATE, "dfsph_sort_cell_keys_noalloc cannot run under stream capture");
    // Device address of the scratch array on the current device (the host-side name
    // g_noalloc_scratch is only a stand-in and must never be handed to a kernel). Looked up on every
    // call, a host-side lookup, so that it stays valid after a device reset reloads the module.
    void* sym = nullptr;
    e = cudaGetSymbolAddress(&sym, g_noalloc_scratch);
    if (e != cudaSuccess) return noalloc_fail(DFSPH_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    uint32_t* scratch = (uint32_t*)sym;
    const int passes = (key_bits + 7) / 8;
    const uint32_t key_mask = key_bits == 32 ? 0xFFFFFFFFu : ((1u << key_bits) - 1u);
    const size_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* counters = scratch + kNoAllocCounters;
    uint32_t* status = scratch + kNoAllocStatus;
    uint32_t* hist = scratch + kNoAllocHist;
    uint32_t* offsets = scratch + kNoAllocOffsets;
    uint32_t* flags = scratch + kNoAllocTileFlags;
    uint32_t* pk = scratch + kNoAllocClearWords;  // ping-pong keys
    uint32_t* pv = pk + kNoAllocMaxKeys;           // ping-pong payloads
    e = cudaMemsetAsync(scratch, 0, kNoAllocClearWords * sizeof(uint32_t), s);
    if (e != cudaSuccess) return noalloc_fail(DFSPH_E_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    int hist_blocks = (int)((n + kSortThreads * 16 - 1) / (kSortThreads * 16));
    if (hist_blocks > 148 * 4) hist_blocks = 148 * 4;
    launch_pdl(histogram_kernel, hist_blocks, kSortThreads, 0, s, keys_in, n, passes, key_mask, hist);
    launch_pdl(scan_kernel, 1, 256, 0, s, hist, passes, offsets);
    // The last pass must write the caller's buffers: with an odd pass count the first pass writes
    // them, with an even count the first pass writes the scratch pair.
    const uint32_t* kin = keys_in;
    const uint32_t* vin = nullptr;  // iota payloads on the first pass
    bool to_out = (passes & 1) == 1;
    for (int p = 0; p < passes; ++p) {
        uint32_t* kout = to_out ? keys_out : pk;
        uint32_t* vout = to_out ? perm_out : pv;
        launch_pdl(onesweep_kernel, (unsigned)tiles, kSortThreads, 0, s, kin, vin, kout, vout, n, 8 * p, key_mask,
                   offsets + p * 256, flags + (size_t)p * tiles * 256, counters + p, status, kNoWithheldTile);
        kin = kout;
        vin = vout;
        to_out = !to_out;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(DFSPH_E_CUDA, std::string("sort launch: ") + cudaGetErrorString(e));
    uint32_t st = 0;
    e = cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return noalloc_fail(DFSPH_E_CUDA, std::string("sort: ") + cudaGetErrorString(e));
    if (st & DFSPH_ST_SORT_TIMEOUT) return noalloc_fail(DFSPH_E_DEVICE, "sort look-back gave up (output unspecified)");
    return DFSPH_OK;
}
