// sort.cuh — interface of the in-house stable radix sort (sort.cu).
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace dfsph {

struct SortBuffers {
    uint32_t* keys_a = nullptr;
    uint32_t* vals_a = nullptr;
    uint32_t* keys_b = nullptr;
    uint32_t* vals_b = nullptr;
    uint32_t* workspace = nullptr;  // radix_sort_workspace_words(n_max, 4) words
};

size_t radix_sort_workspace_words(uint32_t n_max, int passes);

// Message slot of dfsph_last_error(NULL): errors of calls that have no context (dfsph_create and
// the allocation-free entry points). Thread-local.
void set_global_error(const std::string& msg);
// withheld_tile: a tile id whose look-back flags are never published (failure-detection tests: its
// successors' bounded waits run out and set DFSPH_ST_SORT_TIMEOUT; the output is then unspecified
// but every write stays in range). kNoWithheldTile in normal use.
constexpr uint32_t kNoWithheldTile = 0xFFFFFFFFu;
// workspace_cleared: the caller has already zeroed radix_sort_workspace_words(n, passes) words of
// the workspace on this stream (otherwise the sort clears them itself).
void radix_sort_pairs(SortBuffers& b, uint32_t n, int passes, bool iota_values, cudaStream_t stream,
                      uint32_t* status_word, uint64_t* launch_counter, uint32_t** keys_out, uint32_t** vals_out,
                      uint32_t withheld_tile = kNoWithheldTile, bool workspace_cleared = false);

}  // namespace dfsph
