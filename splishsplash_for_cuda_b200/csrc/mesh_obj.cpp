// mesh_obj.cpp — Wavefront OBJ reader for the triangle meshes of the open boundary's mesh surfaces
// (the reference reads them with OBJ_Loader in MeshPerso::loadFromFile, BufferFluidSurface.cu:119-216).
// Only the geometry is read: `v x y z` records and `f` records whose vertex references may be
// `i`, `i/t`, `i//n` or `i/t/n`, 1-based or negative (relative to the vertices read so far);
// polygons are split into fans from their first vertex. Other records (vt, vn, o, g, s, usemtl,
// mtllib, comments) are skipped. Host code; no GPU is needed.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "dfsph_c.h"

namespace {

// The vertex index of one face reference ("12", "12/3", "12//7", "-1/2/3"), 0-based; false when it
// does not name a vertex read so far.
bool face_index(const std::string& tok, size_t nv, uint32_t* out) {
    const size_t slash = tok.find('/');
    const std::string head = tok.substr(0, slash);
    if (head.empty()) return false;
    char* end = nullptr;
    const long long k = std::strtoll(head.c_str(), &end, 10);
    if (end == head.c_str() || *end != '\0' || k == 0) return false;
    const long long i = k > 0 ? k - 1 : (long long)nv + k;
    if (i < 0 || (size_t)i >= nv) return false;
    *out = (uint32_t)i;
    return true;
}

}  // namespace

extern "C" int dfsph_read_obj(const char* path, float* vertices, uint32_t vertex_capacity, uint32_t* n_vertices,
                              uint32_t* triangles, uint32_t triangle_capacity, uint32_t* n_triangles) {
    if (!path || !n_vertices || !n_triangles) return DFSPH_E_INVALID;
    std::ifstream in(path);
    if (!in) return DFSPH_E_INVALID;
    std::vector<float> v;
    std::vector<uint32_t> t;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string kind;
        if (!(ls >> kind)) continue;
        if (kind == "v") {
            float x, y, z;  // read as float directly (rounded once, as OBJ_Loader's std::stof does)
            if (!(ls >> x >> y >> z)) return DFSPH_E_INVALID;
            v.push_back(x);
            v.push_back(y);
            v.push_back(z);
        } else if (kind == "f") {
            std::vector<uint32_t> poly;
            std::string tok;
            while (ls >> tok) {
                uint32_t i;
                if (!face_index(tok, v.size() / 3, &i)) return DFSPH_E_INVALID;
                poly.push_back(i);
            }
            if (poly.size() < 3) return DFSPH_E_INVALID;
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                t.push_back(poly[0]);
                t.push_back(poly[k]);
                t.push_back(poly[k + 1]);
            }
        }
    }
    const size_t nv = v.size() / 3, nt = t.size() / 3;
    if (nv > UINT32_MAX || nt > UINT32_MAX) return DFSPH_E_INVALID;
    *n_vertices = (uint32_t)nv;
    *n_triangles = (uint32_t)nt;
    if (vertices) {
        if (vertex_capacity < nv) return DFSPH_E_INVALID;
        std::memcpy(vertices, v.data(), v.size() * sizeof(float));
    }
    if (triangles) {
        if (triangle_capacity < nt) return DFSPH_E_INVALID;
        std::memcpy(triangles, t.data(), t.size() * sizeof(uint32_t));
    }
    return DFSPH_OK;
}
