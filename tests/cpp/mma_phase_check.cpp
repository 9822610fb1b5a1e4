// Host check of the forward kernel's MMA barrier bookkeeping (csrc/mma_phases.h): thread 0 of a CTA
// runs tiles of three committed MMA groups (one per layer) and waits on each with a limit. For a
// give-up at every stage of every tile, every wait must name the parity of the group it waits for,
// and the drain before the tensor memory is freed must name the group that was not seen complete
// (and nothing when every group completed). Exit code 0 = all cases pass.
#include <cstdio>

#include "../../splishsplash_for_cuda_b200/csrc/mma_phases.h"

static int run(int tiles, int fail_at) {
    dfsph::MmaPhases ph;
    int commit = 0;
    bool ok = true;
    for (int t = 0; t < tiles && ok; ++t)
        for (int stage = 0; stage < 3 && ok; ++stage) {  // stages 2 and 3 only after a completed stage
            ph.committed();
            if (ph.phase != (uint32_t)(commit & 1)) {
                std::printf("tile %d stage %d: waits on parity %u, group %d has parity %d\n", t, stage, ph.phase,
                            commit, commit & 1);
                return 1;
            }
            const bool done = commit != fail_at;
            ph.waited(done);
            ok = done;
            ++commit;
        }
    uint32_t parity = 0;
    const bool pending = ph.drain(parity);
    if (fail_at < 3 * tiles) {
        if (!pending || parity != (uint32_t)(fail_at & 1)) {
            std::printf("give-up at group %d: drain %d parity %u, expected parity %d\n", fail_at, pending, parity,
                        fail_at & 1);
            return 1;
        }
    } else if (pending) {
        std::printf("no give-up: nothing may be drained\n");
        return 1;
    }
    return 0;
}

int main() {
    int bad = 0, cases = 0;
    for (int tiles = 1; tiles <= 4; ++tiles)
        for (int fail_at = 0; fail_at <= 3 * tiles; ++fail_at, ++cases) bad += run(tiles, fail_at);
    std::printf("%d of %d cases pass\n", cases - bad, cases);
    return bad ? 1 : 0;
}
