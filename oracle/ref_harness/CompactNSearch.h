// CompactNSearch.h — this project's own implementation of the CompactNSearch API that the reference
// CPU solver is written against (test infrastructure: used only to build the reference TimeStepDFSPH
// harness under oracle/_ref/). The reference pins CompactNSearch at commit
// 1d9cf800ab4cbb2af956577b99fdd355c16181ba (CMakeLists.txt:75-83) as an ExternalProject that is not
// vendored; its published behaviour is restated here: fixed-radius neighbour search between point
// sets, a uniform grid of cell size r, neighbours j of point i in set a within set b when
// |x_i - x_j|^2 < r^2 (a point is never its own neighbour), per-pair activation flags, and a z-order
// sort of dynamic point sets applied to caller arrays with sort_field(). Call sites:
// SPlisHSPlasH/FluidModel.h:125-141, FluidModel.cpp:159-313, TimeStep.cpp:205-209.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <numeric>
#include <utility>
#include <vector>

namespace CompactNSearch {

using Real = double;

class NeighborhoodSearch;

class PointSet {
public:
    PointSet(Real const* x, std::size_t n, bool dynamic) : m_x(x), m_n(n), m_dynamic(dynamic) {}

    std::size_t n_points() const { return m_n; }
    bool is_dynamic() const { return m_dynamic; }
    Real const* GetPoints() const { return m_x; }

    // Number of neighbours of point i of this set found in point set `point_set`.
    std::size_t n_neighbors(unsigned int point_set, unsigned int i) const {
        return point_set < m_neighbors.size() && i < m_neighbors[point_set].size()
                   ? m_neighbors[point_set][i].size()
                   : 0;
    }
    unsigned int neighbor(unsigned int point_set, unsigned int i, unsigned int k) const {
        return m_neighbors[point_set][i][k];
    }

    // Reorders a per-point caller array by the last z_sort() of this set.
    template <typename T> void sort_field(T* lst) const {
        if (m_sort_table.empty()) return;
        std::vector<T> tmp(lst, lst + m_sort_table.size());
        for (std::size_t i = 0; i < m_sort_table.size(); ++i) lst[i] = tmp[m_sort_table[i]];
    }

    // Composition of every z_sort() so far: original index of the point now at slot i.
    const std::vector<unsigned int>& original_index() const { return m_original; }

private:
    friend class NeighborhoodSearch;
    Real const* m_x;
    std::size_t m_n;
    bool m_dynamic;
    std::vector<std::vector<std::vector<unsigned int>>> m_neighbors;  // [other set][point] -> list
    std::vector<unsigned int> m_sort_table;
    std::vector<unsigned int> m_original;
};

class NeighborhoodSearch {
public:
    explicit NeighborhoodSearch(Real r, bool erase_empty_cells = false) : m_r(r) { (void)erase_empty_cells; }

    Real radius() const { return m_r; }
    void set_radius(Real r) { m_r = r; }

    unsigned int add_point_set(Real const* x, std::size_t n, bool is_dynamic = true, bool search_neighbors = true,
                               bool find_neighbors = true) {
        m_sets.emplace_back(x, n, is_dynamic);
        const std::size_t k = m_sets.size();
        std::vector<std::vector<bool>> act(k, std::vector<bool>(k, false));
        for (std::size_t i = 0; i + 1 < k; ++i)
            for (std::size_t j = 0; j + 1 < k; ++j) act[i][j] = m_active[i][j];
        for (std::size_t j = 0; j < k; ++j) {
            act[k - 1][j] = search_neighbors;
            act[j][k - 1] = find_neighbors;
        }
        m_active = act;
        m_sets.back().m_original.resize(n);
        std::iota(m_sets.back().m_original.begin(), m_sets.back().m_original.end(), 0u);
        return (unsigned int)(k - 1);
    }

    void resize_point_set(unsigned int i, Real const* x, std::size_t n) {
        m_sets[i].m_x = x;
        m_sets[i].m_n = n;
        m_sets[i].m_original.resize(n);
    }

    void set_active(unsigned int i, unsigned int j, bool active) { m_active[i][j] = active; }
    void set_active(unsigned int i, bool search_neighbors = true, bool find_neighbors = true) {
        for (std::size_t j = 0; j < m_sets.size(); ++j) {
            m_active[i][j] = search_neighbors;
            m_active[j][i] = find_neighbors;
        }
    }
    void set_active(bool active) {
        for (auto& row : m_active) std::fill(row.begin(), row.end(), active);
    }
    bool is_active(unsigned int i, unsigned int j) const { return m_active[i][j]; }

    std::size_t n_point_sets() const { return m_sets.size(); }
    PointSet const& point_set(unsigned int i) const { return m_sets[i]; }
    PointSet& point_set(unsigned int i) { return m_sets[i]; }
    std::vector<PointSet> const& point_sets() const { return m_sets; }

    // Z-order (Morton) sort of every dynamic point set by its grid cell; callers apply the
    // permutation to their arrays with sort_field().
    void z_sort() {
        for (auto& ps : m_sets) {
            if (!ps.m_dynamic || ps.m_n == 0) continue;
            std::vector<std::pair<uint64_t, unsigned int>> keys(ps.m_n);
            for (std::size_t i = 0; i < ps.m_n; ++i) keys[i] = {morton(cell_of(ps.m_x + 3 * i)), (unsigned int)i};
            std::stable_sort(keys.begin(), keys.end(),
                             [](const auto& a, const auto& b) { return a.first < b.first; });
            ps.m_sort_table.resize(ps.m_n);
            std::vector<unsigned int> orig(ps.m_n);
            for (std::size_t i = 0; i < ps.m_n; ++i) {
                ps.m_sort_table[i] = keys[i].second;
                orig[i] = ps.m_original[keys[i].second];
            }
            ps.m_original = orig;
        }
    }

    void find_neighbors(bool points_changed = true) {
        (void)points_changed;
        const std::size_t k = m_sets.size();
        std::vector<std::vector<std::pair<uint64_t, unsigned int>>> grid(k);
        for (std::size_t b = 0; b < k; ++b) {
            bool needed = false;
            for (std::size_t a = 0; a < k; ++a) needed = needed || m_active[a][b];
            if (needed) grid[b] = build_grid(m_sets[b]);
        }
        const Real r2 = m_r * m_r;
        for (std::size_t a = 0; a < k; ++a) {
            PointSet& pa = m_sets[a];
            pa.m_neighbors.assign(k, {});
            for (std::size_t b = 0; b < k; ++b) {
                if (!m_active[a][b]) continue;
                auto& lists = pa.m_neighbors[b];
                lists.assign(pa.m_n, {});
                const PointSet& pb = m_sets[b];
                const auto& gb = grid[b];
#pragma omp parallel for schedule(dynamic, 512)
                for (int64_t ii = 0; ii < (int64_t)pa.m_n; ++ii) {
                    const unsigned int i = (unsigned int)ii;
                    const Real* xi = pa.m_x + 3 * (std::size_t)i;
                    const auto c = cell_of(xi);
                    auto& out = lists[i];
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                const uint64_t key = pack({c[0] + dx, c[1] + dy, c[2] + dz});
                                auto lo = std::lower_bound(gb.begin(), gb.end(), std::make_pair(key, 0u));
                                for (auto it = lo; it != gb.end() && it->first == key; ++it) {
                                    const unsigned int j = it->second;
                                    if (a == b && i == j) continue;
                                    const Real* xj = pb.m_x + 3 * (std::size_t)j;
                                    const Real ddx = xi[0] - xj[0], ddy = xi[1] - xj[1], ddz = xi[2] - xj[2];
                                    if (ddx * ddx + ddy * ddy + ddz * ddz < r2) out.push_back(j);
                                }
                            }
                }
            }
        }
    }

private:
    struct Cell {
        int v[3];
        int operator[](int a) const { return v[a]; }
    };
    Cell cell_of(const Real* x) const {
        Cell c;
        for (int a = 0; a < 3; ++a) c.v[a] = (int)std::floor(x[a] / m_r);
        return c;
    }
    static uint64_t pack(const Cell& c) {
        return ((uint64_t)(uint32_t)(c[0] + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(c[1] + (1 << 20)) << 21) |
               (uint64_t)(uint32_t)(c[2] + (1 << 20));
    }
    static uint64_t spread(uint64_t v) {
        v &= 0x1FFFFF;
        v = (v | (v << 32)) & 0x1F00000000FFFFull;
        v = (v | (v << 16)) & 0x1F0000FF0000FFull;
        v = (v | (v << 8)) & 0x100F00F00F00F00Full;
        v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
        v = (v | (v << 2)) & 0x1249249249249249ull;
        return v;
    }
    static uint64_t morton(const Cell& c) {
        return spread((uint64_t)(c[0] + (1 << 20))) | (spread((uint64_t)(c[1] + (1 << 20))) << 1) |
               (spread((uint64_t)(c[2] + (1 << 20))) << 2);
    }
    std::vector<std::pair<uint64_t, unsigned int>> build_grid(const PointSet& ps) const {
        std::vector<std::pair<uint64_t, unsigned int>> g(ps.m_n);
        for (std::size_t i = 0; i < ps.m_n; ++i) g[i] = {pack(cell_of(ps.m_x + 3 * i)), (unsigned int)i};
        std::sort(g.begin(), g.end());
        return g;
    }

    Real m_r;
    std::vector<PointSet> m_sets;
    std::vector<std::vector<bool>> m_active;
};

}  // namespace CompactNSearch
