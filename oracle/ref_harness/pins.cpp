// pins.cpp — runs pieces of the reference's own GPU-path code on the host (test infrastructure):
// the FP32 cubic kernel SPH::CubicKernelPerso (SPlisHSPlasH/DFSPH/SPH_kernels.h:20-100) and the
// neighbour iteration macros ITER_NEIGHBORS_INIT_CELL_COMPUTATION /
// ITER_NEIGHBORS_FROM_STRUCTURE_LINEAR_ADVANCED (SPlisHSPlasH/DFSPH/DFSPH_macro_cuda.h:113-155) over a
// dense 256^3 cell table built the way cuda_neighborsSearchInternal_sortParticlesId does
// (DFSPH_core_cuda.cu:1833-1920: cell id of floor(x/H + offset), per-cell counts, exclusive scan,
// scatter of particle ids). The headers are included from the reference tree; their __host__
// __device__ functions compile as host code. Output feeds the oracle pins in tests/.
#include <cstdint>
#include <cstring>
#include <vector>

#include "SPH_kernels.h"
#include "DFSPH_macro_cuda.h"

using SPH::Vector3d;
using SPH::Vector3i;

namespace {
struct CellTable {
    unsigned int* cell_start_end;
    unsigned int* p_id_sorted;
};

// Dense cell table of a point set, as the reference builds it (counting sort of ids by cell).
void build_table(const std::vector<Vector3d>& pts, float H, const Vector3i& off, std::vector<unsigned int>& start_end,
                 std::vector<unsigned int>& sorted) {
    const size_t cells = (size_t)CELL_COUNT;
    std::vector<unsigned int> hist(cells + 1, 0), cid(pts.size()), rank(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) {
        Vector3d p = (pts[i] / H) + off;
        p.toFloor();
        cid[i] = COMPUTE_CELL_INDEX((int)p.x, (int)p.y, (int)p.z);
        rank[i] = hist[cid[i]]++;
    }
    start_end.assign(cells + 1, 0);
    unsigned int acc = 0;
    for (size_t c = 0; c <= cells; ++c) {
        start_end[c] = acc;
        acc += hist[c];
    }
    sorted.assign(pts.size(), 0);
    for (size_t i = 0; i < pts.size(); ++i) sorted[start_end[cid[i]] + rank[i]] = (unsigned int)i;
}
}  // namespace

extern "C" {

// W(r) and the x component of grad W((r, 0, 0)) of the reference FP32 cubic kernel of support H.
int ref_cubic_values(float H, const float* r, uint32_t n, float* w, float* gx) {
    SPH::CubicKernelPerso k;
    k.setRadius(H);
    for (uint32_t i = 0; i < n; ++i) {
        w[i] = k.W(r[i]);
        gx[i] = k.gradW(Vector3d(r[i], 0.0f, 0.0f)).x;
    }
    return 0;
}

// Neighbour lists of every fluid particle through the reference macros: fluid neighbours (self
// excluded), then boundary neighbours. counts[2 i] / counts[2 i + 1]; lists[i * row + k].
// Returns -1 if a coordinate falls outside the 256^3 table.
int ref_neighbor_lists(const float* fluid, uint32_t n, const float* boundary, uint32_t nb, float H, const int* offset,
                       uint32_t* counts, uint32_t* lists, uint32_t row) {
    const Vector3i gridOffset(offset[0], offset[1], offset[2]);
    std::vector<Vector3d> fp(n), bp(nb);
    for (uint32_t i = 0; i < n; ++i) fp[i] = Vector3d(fluid[3 * i], fluid[3 * i + 1], fluid[3 * i + 2]);
    for (uint32_t i = 0; i < nb; ++i) bp[i] = Vector3d(boundary[3 * i], boundary[3 * i + 1], boundary[3 * i + 2]);
    for (const auto* set : {&fp, &bp})
        for (const auto& p : *set) {
            Vector3d c = (p / H) + gridOffset;
            if (c.x < 1 || c.y < 1 || c.z < 1 || c.x >= CELL_ROW_LENGTH - 1 || c.y >= CELL_ROW_LENGTH - 1 ||
                c.z >= CELL_ROW_LENGTH - 1)
                return -1;
        }
    std::vector<unsigned int> fse, fsorted, bse, bsorted;
    build_table(fp, H, gridOffset, fse, fsorted);
    build_table(bp, H, gridOffset, bse, bsorted);
    CellTable ft{fse.data(), fsorted.data()}, bt{bse.data(), bsorted.data()};
    const CellTable* fluidSet = &ft;
    const CellTable* boundarySet = &bt;
    const Vector3d* fpos = fp.data();
    const Vector3d* bpos = bp.data();
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t nf = 0, nbc = 0;
        uint32_t* out = lists + (size_t)i * row;
        {
            ITER_NEIGHBORS_INIT_CELL_COMPUTATION(fp[i], H, gridOffset);
            unsigned int successive_cells_count = (x > 0) ? 3 : 2;
            x = (x > 0) ? x - 1 : x;
            ITER_NEIGHBORS_FROM_STRUCTURE_LINEAR_ADVANCED(fluidSet, fpos, {
                if (j != i) {
                    if (nf < row) out[nf] = j;
                    ++nf;
                }
            });
        }
        {
            ITER_NEIGHBORS_INIT_CELL_COMPUTATION(fp[i], H, gridOffset);
            unsigned int successive_cells_count = (x > 0) ? 3 : 2;
            x = (x > 0) ? x - 1 : x;
            ITER_NEIGHBORS_FROM_STRUCTURE_LINEAR_ADVANCED(boundarySet, bpos, {
                if (nf + nbc < row) out[nf + nbc] = j;
                ++nbc;
            });
        }
        counts[2 * (size_t)i] = nf;
        counts[2 * (size_t)i + 1] = nbc;
    }
    return 0;
}

}  // extern "C"
