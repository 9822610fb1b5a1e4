// mma_phases.h — parity bookkeeping of the mbarrier that tracks a CTA's tensor-core MMA groups.
//
// Each tcgen05.commit arrives once on the barrier, completing one phase; a wait names the parity of
// the phase it waits for. The forward kernel waits on every group it commits, with an iteration
// limit. When a wait gives up, the group it waited for may still be running and writing the CTA's
// tensor memory, so before the memory is freed the issuing thread waits (again bounded) for exactly
// that group: the parity recorded when the group was committed. Plain C++ so that the bookkeeping can
// be checked on the host (tests/cpp/mma_phase_check.cpp) for a give-up at every stage.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace dfsph {

struct MmaPhases {
    uint32_t phase = 0;           // parity of the next committed group's phase
    bool inflight = false;        // a committed group not yet seen complete by this thread
    uint32_t inflight_phase = 0;  // its parity

    // A group was committed (call before waiting on `phase`).
    __host__ __device__ void committed() {
        inflight = true;
        inflight_phase = phase;
    }
    // The wait on `phase` for the last committed group returned: done = it completed.
    __host__ __device__ void waited(bool done) {
        if (done) inflight = false;
        phase ^= 1u;
    }
    // Parity to drain before freeing the tensor memory, if anything is still in flight.
    __host__ __device__ bool drain(uint32_t& parity) const {
        parity = inflight_phase;
        return inflight;
    }
};

}  // namespace dfsph
