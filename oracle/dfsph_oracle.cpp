// dfsph_oracle.cpp — CPU ORACLE (test infrastructure only, never part of the product).
//
// A plain C++ restatement of the reference GPU DFSPH time step, used by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker. It is templated on
// the arithmetic type: the FP64 instance is the "truth" the FP32 device kernels are compared
// against; the FP32 instance states the error budget of plain FP32 arithmetic.
//
// Followed reference code (paths inside scarensac/SPlisHSPlasH_for_cuda):
//   cubic kernel W / grad W            SPlisHSPlasH/DFSPH/SPH_kernels.h:20-100
//   neighbour predicate, 27 cells      SPlisHSPlasH/DFSPH/DFSPH_macro_cuda.h:136-155 (strict d^2 < H^2, self excluded)
//   cell = floor(x / H + offset)       SPlisHSPlasH/DFSPH/DFSPH_core_cuda.cu:1833-1848
//   grid offset -(floor(min/H) - 5)    SPlisHSPlasH/DFSPH/DFSPH_c_arrays_structure.cpp:1050-1098
//   boundary psi                       SPlisHSPlasH/FluidModel.cpp:233-258
//   density, alpha, kappa_v warm start SPlisHSPlasH/DFSPH/DFSPH_core_cuda.cu:221-237 (+ :336 alpha)
//   divergence solve                   DFSPH_core_cuda.cu:400-480, 495-517, 546-614, 618-709, 785-861
//   XSPH viscosity + gravity           DFSPH_core_cuda.cu:1423-1507
//   dt bookkeeping                     DFSPH_c_arrays_structure.cpp:1100-1118
//   velocity update                    DFSPH_core_cuda.cu:3047-3070
//   pressure solve                     DFSPH_core_cuda.cu:867-951, 965-980, 1165-1243, 1264-1284, 1338-1419
//   position update                    DFSPH_core_cuda.cu:3127-3215 (damping and wave cancelling off)
//   CFL                                DFSPH_core_cuda.cu:3321-3394
//   simple open boundary               OpenBoundariesSimple.cu:105-350 (init), 352-470 (inflow),
//                                      475-492 (outflow), 495-620 (apply); surfaces
//                                      BufferFluidSurface.cu:421-900 (isinside, getNormal)
//
// The pair predicate is the canonical FP32 form shared with the device code:
// d2 = fma(dz, dz, fma(dy, dy, dx*dx)) on float coordinates, then d2 < H*H (H*H rounded to float).
// Compile with -ffp-contract=off so nothing else is contracted.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace {

constexpr double kEps = 1.0e-5;
constexpr uint32_t kMinNeighbors = 20;

inline bool pair_within(float xi, float yi, float zi, float xj, float yj, float zj, float H2) {
    const float dx = xi - xj, dy = yi - yj, dz = zi - zj;
    const float d2 = std::fmaf(dz, dz, std::fmaf(dy, dy, dx * dx));
    return d2 < H2;
}

inline int cell_coord(float x, float H, int off) { return (int)std::floor((x / H) + (float)off); }

template <class Real> struct Kahan {
    Real s = 0, c = 0;
    void add(Real v) {
        const Real y = v - c;
        const Real t = s + y;
        c = (t - s) - y;
        s = t;
    }
    Real value() const { return s; }
};

template <class Real> struct Neumaier {
    Real s = 0, c = 0;
    void add(Real v) {
        const Real t = s + v;
        c += (std::fabs(s) >= std::fabs(v)) ? ((s - t) + v) : ((v - t) + s);
        s = t;
    }
    Real value() const { return s + c; }
};

template <class Real> struct Cubic {
    Real H = 0, k = 0, l = 0, W0 = 0;
    void set(double Hd) {
        H = (Real)Hd;
        k = (Real)(8.0 / (M_PI * Hd * Hd * Hd));
        l = (Real)(48.0 / (M_PI * Hd * Hd * Hd));
        W0 = k;
    }
    Real W_of_q(Real q) const {
        if (q <= Real(1)) {
            if (q <= Real(0.5)) {
                const Real q2 = q * q, q3 = q2 * q;
                return k * (Real(6) * q3 - Real(6) * q2 + Real(1));
            }
            const Real f = Real(1) - q;
            return k * (Real(2) * f * f * f);
        }
        return Real(0);
    }
    Real W(Real rx, Real ry, Real rz) const { return W_of_q(std::sqrt(rx * rx + ry * ry + rz * rz) / H); }
    void gradW(Real rx, Real ry, Real rz, Real& gx, Real& gy, Real& gz) const {
        const Real rl = std::sqrt(rx * rx + ry * ry + rz * rz);
        const Real q = rl / H;
        gx = gy = gz = 0;
        if (q <= Real(1) && (double)rl > 1.0e-6) {
            const Real s = Real(1) / (rl * H);
            Real c;
            if (q <= Real(0.5)) c = l * q * (Real(3) * q - Real(2));
            else {
                const Real f = Real(1) - q;
                c = l * (-f * f);
            }
            gx = c * (rx * s);
            gy = c * (ry * s);
            gz = c * (rz * s);
        }
    }
};

// Density terms m_j W_ij of the FP32 instance, evaluated in FP64 from the FP32 distance components
// and summed in FP64, as the device's density_term (dfsph_common.cuh). The FP64 instance evaluates
// the terms with its kernel.
struct DensityTerms {
    double ih2 = 0, k = 0;
    void set(double H) {
        ih2 = 1.0 / (H * H);
        k = 8.0 / (M_PI * H * H * H);
    }
    double term(float rx, float ry, float rz, float m) const {
        const double dx = rx, dy = ry, dz = rz;
        const double q2 = (dx * dx + dy * dy + dz * dz) * ih2;
        if (q2 > 1.0) return 0.0;
        double w = k;
        if (q2 > 0.0) {
            const double q = std::sqrt(q2);
            if (q <= 0.5) {
                w = k * (1.0 + 6.0 * q2 * (q - 1.0));
            } else {
                const double f = 1.0 - q;
                w = 2.0 * k * (f * f * f);
            }
        }
        return w * (double)m;
    }
};

// Layout of the C ABI's dfsph_surface (restated; BufferFluidSurface's fields).
struct Surface {
    int32_t type, reversed;
    float origin[3], normal[3], center[3], half_lengths[3];
    float radius, radius_internal;
    uint32_t points;
    float direction[3];
};

// BufferFluidSurface::isinside / getNormal in FP32, each expression evaluated left to right.
float sdot(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
float snorm(const float* a) { return std::sqrt(sdot(a, a)); }

// Triangle meshes of type-3 surfaces by id (MeshPerso, BufferFluidSurface.cu:49-410): triangles as
// vertex triples, the box of the vertices and the origin, the ray direction.
struct OracleMesh {
    std::vector<float> tri;  // 9 per triangle
    float bmin[3] = {0.f, 0.f, 0.f}, bmax[3] = {0.f, 0.f, 0.f};
};
OracleMesh g_meshes[8];

void ray_direction(float d[3]) {  // normalise((2.575, 6.19763, 5.986)) in FP32, each operation rounded
    const float x = (float)2.575, y = (float)6.19763, z = (float)5.986;
    const float n = std::sqrt(x * x + y * y + z * z);
    d[0] = x / n;
    d[1] = y / n;
    d[2] = z / n;
}
void scross(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
// RayIntersectsTriangle<true, false> (BufferFluidSurface.cu:14-47) followed by the t > 0 test of
// MeshPerso::isInside.
bool ray_hits_ahead(const float* o, const float* d, const float* v0, const float* v1, const float* v2) {
    const float eps = 1e-7f;
    float e1[3], e2[3], h[3], s[3], q[3];
    for (int a = 0; a < 3; ++a) {
        e1[a] = v1[a] - v0[a];
        e2[a] = v2[a] - v0[a];
    }
    scross(d, e2, h);
    const float a = sdot(e1, h);
    if (a > -eps && a < eps) return false;
    const float f = (float)(1.0 / (double)a);
    for (int k = 0; k < 3; ++k) s[k] = o[k] - v0[k];
    const float u = f * sdot(s, h);
    if (u < 0.0f || u > 1.0f) return false;
    scross(s, e1, q);
    const float v = f * sdot(d, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    return f * sdot(e2, q) > 0.0f;
}
bool mesh_inside(const Surface& S, const float* p) {
    const OracleMesh& m = g_meshes[S.points];
    for (int a = 0; a < 3; ++a)
        if (p[a] < m.bmin[a] + S.center[a]) return false;
    for (int a = 0; a < 3; ++a)
        if (p[a] > m.bmax[a] + S.center[a]) return false;
    float d[3];
    ray_direction(d);
    uint32_t hits = 0;
    const size_t nt = m.tri.size() / 9;
    for (size_t t = 0; t < nt; ++t) {
        float v[9];
        for (int k = 0; k < 9; ++k) v[k] = m.tri[9 * t + k] + S.center[k % 3];
        if (ray_hits_ahead(p, d, v, v + 3, v + 6)) ++hits;
    }
    return (hits & 1u) != 0u;
}

bool surface_inside(const Surface& S, const float* p) {
    bool r = false;
    float v[3];
    switch (S.type) {
        case 3:
            r = S.points < 8 && mesh_inside(S, p);
            break;
        case 0:
            for (int a = 0; a < 3; ++a) v[a] = p[a] - S.origin[a];
            r = !(sdot(v, S.normal) < 0.0f);
            break;
        case 1:
            for (int a = 0; a < 3; ++a) v[a] = std::fabs(p[a] - S.center[a]);
            r = v[0] < S.half_lengths[0] && v[1] < S.half_lengths[1] && v[2] < S.half_lengths[2];
            break;
        case 2:
        case 5: {
            for (int a = 0; a < 3; ++a) v[a] = p[a] - S.center[a];
            if (std::fabs(v[1]) > S.half_lengths[1]) break;
            v[1] = 0.0f;
            const float nv = snorm(v);
            if (S.type == 2) {
                r = nv < S.radius;
                break;
            }
            if (nv < S.radius_internal) {
                r = true;
            } else if (nv > S.radius) {
                r = false;
            } else {
                const float u[3] = {v[0] / nv, v[1] / nv, v[2] / nv};
                const float alpha = std::acos(sdot(u, S.direction));
                const float alpha0 = (2.0f * 3.14159265358979f) / (float)S.points;
                float k = alpha / alpha0;
                for (uint32_t it = 0; k > 1.0f && it <= S.points; ++it) k -= 1.0f;
                const float x = k * alpha0;
                const float half = alpha0 / 2.0f;
                float a1 = 0.0f, r1 = S.radius, a2 = 0.0f + half, r2 = S.radius_internal;
                if (x > half) {
                    r1 = S.radius_internal;
                    r2 = S.radius;
                    a1 = a2;
                    a2 = a1 + half;
                }
                const float x1 = r1 * std::cos(a1), y1 = r1 * std::sin(a1);
                const float x2 = r2 * std::cos(a2), y2 = r2 * std::sin(a2);
                const float m = (y2 - y1) / (x2 - x1);
                const float c = -x1 * m + y1;
                const float d = c / (-m * std::cos(x) + 1.0f * std::sin(x));
                r = nv <= d;
            }
            break;
        }
        case 4:
            for (int a = 0; a < 3; ++a) v[a] = p[a] - S.center[a];
            r = snorm(v) < S.radius;
            break;
        default:
            break;
    }
    return S.reversed ? !r : r;
}

void surface_normal(const Surface& S, const float* p, float* out) {
    out[0] = out[1] = out[2] = 0.0f;
    if (S.type == 2 || S.type == 4 || S.type == 5)
        for (int a = 0; a < 3; ++a) out[a] = S.center[a] - p[a];
    if (S.reversed)
        for (int a = 0; a < 3; ++a) out[a] = -out[a];
    if (!(out[0] == 0.0f && out[1] == 0.0f && out[2] == 0.0f)) {
        const float nr = snorm(out);
        for (int a = 0; a < 3; ++a) out[a] = out[a] / nr;
    }
}

struct Params {
    double particle_radius, density0, viscosity, gravitation[3], time_step;
    int32_t max_iterations;
    double max_error;
    int32_t max_iterations_v;
    double max_error_v;
    int32_t enable_divergence_solver, cfl_method;
    double cfl_factor, cfl_max_time_step, cfl_min_time_step;
    uint32_t neighbor_capacity;
    int32_t brute_force;  // 1: O(N^2) neighbour search instead of the cell grid
};

template <class Real> struct Oracle {
    Params prm{};
    Cubic<Real> K;
    DensityTerms DT;
    float Hf = 0, H2f = 0;
    int off[3] = {0, 0, 0}, dim[3] = {0, 0, 0};
    bool grid = false;
    // fluid (original order)
    uint32_t n = 0;
    std::vector<Real> x, v, m, rho, alpha, dadv, kap, kapv, a, kc;
    // Warm starts applied and last unclamped residuals of the step's two solves, for the coefficients
    // each solve needed (the learned warm start's training targets and network inputs).
    std::vector<Real> kw_p, kw_v, raw_p, raw_v;
    bool div_ran = false;
    // boundary
    uint32_t nb = 0;
    std::vector<Real> bx, bv, psi;
    // Force of the fluid on each boundary particle, summed over the Jacobi passes of a step
    // (DFSPH_core_cuda.cu:467-477, :937-946: -m_i k_i psi_b grad W_ib), when enabled.
    bool bforce_on = false;
    std::vector<double> bF;
    bool boundary_moving = false;
    // neighbours
    std::vector<std::vector<uint32_t>> nf, nbd;
    bool overflow = false;
    // dt history
    double h = 0, h_future = 0, h_past = 0, inv_h = 0, inv_h_future = 0, h_ratio = 1, h_ratio2 = 1;
    double time_step = 0;
    int last_iters = 0, last_iters_v = 0;
    double last_err = 0, last_err_v = 0, init_err = 0, init_err_v = 0;

    void init(const Params& p) {
        prm = p;
        K.set((double)(float)(4.0 * p.particle_radius));
        DT.set((double)(float)(4.0 * p.particle_radius));
        Hf = (float)(4.0 * p.particle_radius);
        H2f = Hf * Hf;
        time_step = p.time_step;
        reset_dt();
    }
    // ---- simple open boundary ------------------------------------------------------------------
    bool ob_ready = false;
    Surface ob_b{}, ob_i{}, ob_s{};
    std::vector<float> ob_x;  // kept samples

    void ob_init(const Surface& b, const Surface& in, const Surface& sf, const float* xyz, uint32_t ns) {
        ob_b = b;
        ob_i = in;
        ob_s = sf;
        ob_x.clear();
        for (uint32_t i = 0; i < ns; ++i) {
            const float* p = xyz + 3 * (size_t)i;
            int cx, cy, cz;
            if (!surface_inside(in, p) && surface_inside(sf, p) && cell_of(p[0], p[1], p[2], cx, cy, cz))
                ob_x.insert(ob_x.end(), p, p + 3);
        }
        ob_ready = true;
    }

    void ob_shift(const float* d) {
        for (Surface* S : {&ob_b, &ob_i, &ob_s}) {
            float* c = (S->type == 0) ? S->origin : S->center;
            for (int a = 0; a < 3; ++a) c[a] += d[a];
        }
        for (size_t k = 0; k < ob_x.size(); ++k) ob_x[k] += d[k % 3];
    }

    float inflow_mass = 0.0f;  // mass of the particles the inflow adds: the first uploaded particle's

    // applyOpenBoundary: inflow decisions against the current fluid (all of them, in sample order),
    // then the outflow over every particle, new ones included.
    void ob_apply(double allowed_distance, double allowed_density, bool inflow, bool outflow, uint32_t capacity,
                  uint32_t& added, uint32_t& removed, bool& clipped) {
        added = removed = 0;
        clipped = false;
        const Real mass = (Real)inflow_mass;
        if (inflow && !ob_x.empty()) {
            const std::vector<float> fp = fpos(), fb = fbpos();
            const Buckets bf = bucket(fp, n), bbk = bucket(fb, nb);
            const uint32_t ns = (uint32_t)(ob_x.size() / 3);
            std::vector<float> newx, newv;
            for (uint32_t i = 0; i < ns; ++i) {
                const float* sp = &ob_x[3 * (size_t)i];
                const Real xi = sp[0], yi = sp[1], zi = sp[2];
                Real min_d = Real(100);
                bool any_cell = false;
                for_cells(sp[0], sp[1], sp[2], [&](size_t c) {
                    any_cell = true;
                    for (uint32_t t = bf.start[c]; t < bf.start[c + 1]; ++t) {
                        const uint32_t j = bf.items[t];
                        const Real ex = xi - x[3 * j], ey = yi - x[3 * j + 1], ez = zi - x[3 * j + 2];
                        const Real dd = std::sqrt(ex * ex + ey * ey + ez * ez);
                        min_d = dd < min_d ? dd : min_d;
                    }
                });
                if (!any_cell || !(min_d > (Real)(float)allowed_distance)) continue;
                Real rho0 = K.W0 * mass, wsum = 0, vx = 0, vy = 0, vz = 0;
                for_cells(sp[0], sp[1], sp[2], [&](size_t c) {
                    for (uint32_t t = bf.start[c]; t < bf.start[c + 1]; ++t) {
                        const uint32_t j = bf.items[t];
                        const Real w = K.W(xi - x[3 * j], yi - x[3 * j + 1], zi - x[3 * j + 2]) * m[j];
                        rho0 += w;
                        vx += v[3 * j] * w;
                        vy += v[3 * j + 1] * w;
                        vz += v[3 * j + 2] * w;
                        wsum += w;
                    }
                });
                for_cells(sp[0], sp[1], sp[2], [&](size_t c) {
                    for (uint32_t t = bbk.start[c]; t < bbk.start[c + 1]; ++t) {
                        const uint32_t j = bbk.items[t];
                        const Real w = K.W(xi - bx[3 * j], yi - bx[3 * j + 1], zi - bx[3 * j + 2]) * psi[j];
                        wsum += w;
                        rho0 += w;
                    }
                });
                if (wsum > Real(0)) {
                    vx /= wsum;
                    vy /= wsum;
                    vz /= wsum;
                }
                float nrm[3];
                surface_normal(ob_b, sp, nrm);
                const float vf[3] = {(float)vx, (float)vy, (float)vz};
                if (rho0 > (Real)(float)allowed_density || sdot(vf, nrm) < 0.0f) continue;
                newx.insert(newx.end(), sp, sp + 3);
                newv.insert(newv.end(), vf, vf + 3);
            }
            uint32_t want = (uint32_t)(newx.size() / 3);
            added = std::min<uint32_t>(want, capacity > n ? capacity - n : 0);
            clipped = added < want;
            for (uint32_t k = 0; k < added; ++k) {
                for (int a3 = 0; a3 < 3; ++a3) {
                    x.push_back((Real)newx[3 * k + a3]);
                    v.push_back((Real)newv[3 * k + a3]);
                    a.push_back(0);
                }
                m.push_back(mass);
                for (auto* vec : {&rho, &alpha, &dadv, &kap, &kapv, &kc}) vec->push_back(0);
            }
            n += added;
            nf.resize(n);
            nbd.resize(n);
        }
        if (outflow && n) {
            removed = compact([&](uint32_t i) {
                const float p[3] = {(float)x[3 * i], (float)x[3 * i + 1], (float)x[3 * i + 2]};
                return surface_inside(ob_i, p) || surface_inside(ob_s, p);
            });
        }
    }

    // Keeps the particles with keep(i), in order; returns how many were removed.
    template <class Keep> uint32_t compact(Keep&& keep) {
        uint32_t w = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (!keep(i)) continue;
            if (w != i) {
                for (int a3 = 0; a3 < 3; ++a3) {
                    x[3 * w + a3] = x[3 * i + a3];
                    v[3 * w + a3] = v[3 * i + a3];
                    a[3 * w + a3] = a[3 * i + a3];
                }
                for (auto* vec : {&m, &rho, &alpha, &dadv, &kap, &kapv, &kc}) (*vec)[w] = (*vec)[i];
            }
            ++w;
        }
        const uint32_t removed = n - w;
        n = w;
        x.resize(3 * (size_t)n);
        v.resize(3 * (size_t)n);
        a.resize(3 * (size_t)n);
        for (auto* vec : {&m, &rho, &alpha, &dadv, &kap, &kapv, &kc}) vec->resize(n);
        nf.resize(n);
        nbd.resize(n);
        return removed;
    }

    uint32_t remove_out_of_box() {
        const uint32_t r = compact([&](uint32_t i) {
            bool out = false;
            for (int a3 = 0; a3 < 3; ++a3)
                out = out || x[3 * i + a3] > (Real)bb_hi[a3] || x[3 * i + a3] < (Real)bb_lo[a3];
            return !out;
        });
        escaped_removed += r;
        return r;
    }

    void reset_dt() {
        h = h_future = h_past = time_step;
        inv_h = inv_h_future = 1.0 / time_step;
        h_ratio = h_ratio2 = 1.0;
    }

    // domain box (initGridOffset's boundingBoxMin / Max) and the end-of-step removal of the
    // particles outside it (checkParticlesPositions(2), SPH_other_systems_cuda.cu:1242-1328)
    float bb_lo[3] = {0, 0, 0}, bb_hi[3] = {0, 0, 0};
    bool remove_escaped = true;
    uint64_t escaped_removed = 0;

    void set_grid(const float mn[3], const float mx[3]) {
        for (int a3 = 0; a3 < 3; ++a3) {
            bb_lo[a3] = mn[a3];
            bb_hi[a3] = mx[a3];
            const int fmin = (int)std::floor(mn[a3] / Hf);
            const int fmax = (int)std::floor(mx[a3] / Hf);
            off[a3] = -(fmin - 5);
            dim[a3] = fmax + off[a3] + 6;
        }
        grid = true;
    }

    bool cell_of(float px, float py, float pz, int& cx, int& cy, int& cz) const {
        if (!(std::isfinite(px) && std::isfinite(py) && std::isfinite(pz))) return false;
        cx = cell_coord(px, Hf, off[0]);
        cy = cell_coord(py, Hf, off[1]);
        cz = cell_coord(pz, Hf, off[2]);
        return cx >= 0 && cy >= 0 && cz >= 0 && cx < dim[0] && cy < dim[1] && cz < dim[2];
    }

    // Cell buckets of a point set (particles of a cell in increasing index).
    struct Buckets {
        std::vector<uint32_t> start, items;
    };
    Buckets bucket(const std::vector<float>& p, uint32_t count) const {
        Buckets b;
        const size_t cells = (size_t)dim[0] * dim[1] * dim[2];
        std::vector<uint32_t> cnt(cells + 1, 0), cid(count, UINT32_MAX);
        for (uint32_t i = 0; i < count; ++i) {
            int cx, cy, cz;
            if (cell_of(p[3 * i], p[3 * i + 1], p[3 * i + 2], cx, cy, cz)) {
                cid[i] = (uint32_t)(cx + dim[0] * (cy + dim[1] * cz));
                cnt[cid[i] + 1]++;
            }
        }
        for (size_t c = 0; c < cells; ++c) cnt[c + 1] += cnt[c];
        b.start = cnt;
        b.items.assign(cnt[cells], 0);
        std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
        for (uint32_t i = 0; i < count; ++i)
            if (cid[i] != UINT32_MAX) b.items[fill[cid[i]]++] = i;
        return b;
    }

    std::vector<float> fpos() const {
        std::vector<float> f(3 * (size_t)n);
        for (size_t i = 0; i < f.size(); ++i) f[i] = (float)x[i];
        return f;
    }
    std::vector<float> fbpos() const {
        std::vector<float> f(3 * (size_t)nb);
        for (size_t i = 0; i < f.size(); ++i) f[i] = (float)bx[i];
        return f;
    }

    template <class F> void for_cells(float px, float py, float pz, F&& f) const {
        int cx, cy, cz;
        if (!cell_of(px, py, pz, cx, cy, cz)) return;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                    if (X < 0 || Y < 0 || Z < 0 || X >= dim[0] || Y >= dim[1] || Z >= dim[2]) continue;
                    f((size_t)(X + dim[0] * (Y + dim[1] * Z)));
                }
    }

    void neighbors() {
        if (bforce_on) bF.assign(3 * (size_t)nb, 0.0);
        const std::vector<float> fp = fpos(), fb = fbpos();
        nf.assign(n, {});
        nbd.assign(n, {});
        overflow = false;
        if (prm.brute_force) {
            for (uint32_t i = 0; i < n; ++i) {
                int cx, cy, cz;
                if (!cell_of(fp[3 * i], fp[3 * i + 1], fp[3 * i + 2], cx, cy, cz)) continue;
                for (uint32_t j = 0; j < n; ++j)
                    if (j != i && pair_within(fp[3 * i], fp[3 * i + 1], fp[3 * i + 2], fp[3 * j], fp[3 * j + 1],
                                              fp[3 * j + 2], H2f))
                        nf[i].push_back(j);
                for (uint32_t j = 0; j < nb; ++j)
                    if (pair_within(fp[3 * i], fp[3 * i + 1], fp[3 * i + 2], fb[3 * j], fb[3 * j + 1], fb[3 * j + 2],
                                    H2f))
                        nbd[i].push_back(j);
            }
        } else {
            const Buckets bf = bucket(fp, n), bbk = bucket(fb, nb);
#pragma omp parallel for schedule(dynamic, 256)
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                const uint32_t i = (uint32_t)ii;
                const float xi = fp[3 * i], yi = fp[3 * i + 1], zi = fp[3 * i + 2];
                for_cells(xi, yi, zi, [&](size_t c) {
                    for (uint32_t t = bf.start[c]; t < bf.start[c + 1]; ++t) {
                        const uint32_t j = bf.items[t];
                        if (j != i && pair_within(xi, yi, zi, fp[3 * j], fp[3 * j + 1], fp[3 * j + 2], H2f))
                            nf[i].push_back(j);
                    }
                });
                for_cells(xi, yi, zi, [&](size_t c) {
                    for (uint32_t t = bbk.start[c]; t < bbk.start[c + 1]; ++t) {
                        const uint32_t j = bbk.items[t];
                        if (pair_within(xi, yi, zi, fb[3 * j], fb[3 * j + 1], fb[3 * j + 2], H2f)) nbd[i].push_back(j);
                    }
                });
            }
        }
        const uint32_t cap = prm.neighbor_capacity;
        for (uint32_t i = 0; i < n; ++i) {
            if (nf[i].size() + nbd[i].size() > cap) {
                overflow = true;
                if (nf[i].size() > cap) nf[i].resize(cap);
                nbd[i].resize(std::min<size_t>(nbd[i].size(), cap - nf[i].size()));
            }
        }
    }

    // psi_b = rho0 / (W0 + sum_{b' != b} W(x_b - x_b')) in FP64 (FluidModel::computeBoundaryPsi).
    void compute_psi() {
        const std::vector<float> fb = fbpos();
        const Buckets bbk = bucket(fb, nb);
        const double H = (double)Hf;
        const double k = 8.0 / (M_PI * H * H * H);
        psi.assign(nb, 0);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t bb = 0; bb < (int64_t)nb; ++bb) {
            const uint32_t b = (uint32_t)bb;
            const float xb = fb[3 * b], yb = fb[3 * b + 1], zb = fb[3 * b + 2];
            double delta = k;
            for_cells(xb, yb, zb, [&](size_t c) {
                for (uint32_t t = bbk.start[c]; t < bbk.start[c + 1]; ++t) {
                    const uint32_t j = bbk.items[t];
                    if (j == b || !pair_within(xb, yb, zb, fb[3 * j], fb[3 * j + 1], fb[3 * j + 2], H2f)) continue;
                    const double rx = (double)xb - fb[3 * j], ry = (double)yb - fb[3 * j + 1],
                                 rz = (double)zb - fb[3 * j + 2];
                    const double q = std::sqrt(rx * rx + ry * ry + rz * rz) / H;
                    double w = 0;
                    if (q <= 1.0) {
                        if (q <= 0.5) w = k * (6.0 * q * q * q - 6.0 * q * q + 1.0);
                        else {
                            const double f = 1.0 - q;
                            w = k * (2.0 * f * f * f);
                        }
                    }
                    delta += w;
                }
            });
            psi[b] = (Real)(prm.density0 / delta);
        }
    }

    // ---- passes ---------------------------------------------------------------------------------
    Real bvel(uint32_t j, int c) const { return boundary_moving ? bv[3 * j + c] : Real(0); }

    void density_alpha(bool warm_v) {
        const Real hr = (Real)h_ratio, invh = (Real)inv_h;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            if (warm_v) kapv[i] = std::max<Real>(kapv[i] * hr / Real(2), Real(-0.5));
            // rho - rho0 accumulated directly (the device kernels do the same; see density_alpha_kernel)
            Neumaier<Real> r;
            double r64 = -(double)(Real)prm.density0;
            Kahan<Real> sgk, dr, gx, gy, gz;
            r.add((Real)-prm.density0);
            auto add_term = [&](Real rx, Real ry, Real rz, Real mj, Real w) {
                if (sizeof(Real) == 4) {
                    r64 += DT.term((float)rx, (float)ry, (float)rz, (float)mj);
                } else {
                    r.add(mj * w);
                }
            };
            add_term(0, 0, 0, m[i], K.W0);
            const Real xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
            const Real vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
            for (uint32_t j : nf[i]) {
                const Real rx = xi - x[3 * j], ry = yi - x[3 * j + 1], rz = zi - x[3 * j + 2];
                Real w = K.W(rx, ry, rz), g0, g1, g2;
                K.gradW(rx, ry, rz, g0, g1, g2);
                add_term(rx, ry, rz, m[j], w);
                const Real px = m[j] * g0, py = m[j] * g1, pz = m[j] * g2;
                sgk.add(px * px + py * py + pz * pz);
                gx.add(px); gy.add(py); gz.add(pz);
                dr.add((vx - v[3 * j]) * px + (vy - v[3 * j + 1]) * py + (vz - v[3 * j + 2]) * pz);
            }
            for (uint32_t j : nbd[i]) {
                const Real rx = xi - bx[3 * j], ry = yi - bx[3 * j + 1], rz = zi - bx[3 * j + 2];
                Real w = K.W(rx, ry, rz), g0, g1, g2;
                K.gradW(rx, ry, rz, g0, g1, g2);
                add_term(rx, ry, rz, psi[j], w);
                const Real px = psi[j] * g0, py = psi[j] * g1, pz = psi[j] * g2;
                sgk.add(px * px + py * py + pz * pz);
                gx.add(px); gy.add(py); gz.add(pz);
                dr.add((vx - bvel(j, 0)) * px + (vy - bvel(j, 1)) * py + (vz - bvel(j, 2)) * pz);
            }
            const Real Gx = gx.value(), Gy = gy.value(), Gz = gz.value();
            const Real sg = sgk.value() + (Gx * Gx + Gy * Gy + Gz * Gz);
            alpha[i] = -invh / std::max<Real>(sg, (Real)kEps);
            rho[i] = sizeof(Real) == 4 ? (Real)r64 : r.value();  // rho - rho0
            uint32_t num = (uint32_t)nf[i].size();
            if (num < kMinNeighbors) num += (uint32_t)nbd[i].size();
            dadv[i] = (num < kMinNeighbors) ? Real(0) : std::max<Real>(dr.value(), Real(0));
        }
    }

    // Jacobi velocity correction with coefficient k (per particle); dt is h or h_future.
    template <class KF, class Skip>
    void jacobi(KF&& kof, Real dt, Skip&& skip, bool forces = true) {
        std::vector<Real> dv(3 * (size_t)n, 0);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            if (skip(i)) continue;
            const Real ki = kof(i);
            const Real xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
            Kahan<Real> ax, ay, az;
            for (uint32_t j : nf[i]) {
                const Real ks = ki + kof(j);
                if (std::fabs((double)ks) > kEps) {
                    Real g0, g1, g2;
                    K.gradW(xi - x[3 * j], yi - x[3 * j + 1], zi - x[3 * j + 2], g0, g1, g2);
                    const Real s = ks * m[j];
                    ax.add(s * g0); ay.add(s * g1); az.add(s * g2);
                }
            }
            if (std::fabs((double)ki) > kEps) {
                for (uint32_t j : nbd[i]) {
                    Real g0, g1, g2;
                    K.gradW(xi - bx[3 * j], yi - bx[3 * j + 1], zi - bx[3 * j + 2], g0, g1, g2);
                    const Real s = ki * psi[j];
                    ax.add(s * g0); ay.add(s * g1); az.add(s * g2);
                    if (bforce_on && forces) {
                        const double f = -(double)m[i] * (double)s;
#pragma omp atomic
                        bF[3 * (size_t)j] += f * (double)g0;
#pragma omp atomic
                        bF[3 * (size_t)j + 1] += f * (double)g1;
#pragma omp atomic
                        bF[3 * (size_t)j + 2] += f * (double)g2;
                    }
                }
            }
            dv[3 * i] = ax.value() * dt;
            dv[3 * i + 1] = ay.value() * dt;
            dv[3 * i + 2] = az.value() * dt;
        }
        for (uint32_t i = 0; i < n; ++i)
            if (!skip(i))
                for (int c = 0; c < 3; ++c) v[3 * i + c] += dv[3 * i + c];
    }

    // sum_j m_j (v_i - v_j).grad W_ij + sum_b psi_b (v_i - v_b).grad W_ib
    Real velocity_divergence(uint32_t i) const {
        const Real xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
        const Real vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
        Kahan<Real> s;
        for (uint32_t j : nf[i]) {
            Real g0, g1, g2;
            K.gradW(xi - x[3 * j], yi - x[3 * j + 1], zi - x[3 * j + 2], g0, g1, g2);
            s.add(m[j] * ((vx - v[3 * j]) * g0 + (vy - v[3 * j + 1]) * g1 + (vz - v[3 * j + 2]) * g2));
        }
        for (uint32_t j : nbd[i]) {
            Real g0, g1, g2;
            K.gradW(xi - bx[3 * j], yi - bx[3 * j + 1], zi - bx[3 * j + 2], g0, g1, g2);
            s.add(psi[j] * ((vx - bvel(j, 0)) * g0 + (vy - bvel(j, 1)) * g1 + (vz - bvel(j, 2)) * g2));
        }
        return s.value();
    }

    double divergence_residual(bool init) {
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            if (init) kapv[i] = 0;
            uint32_t num = (uint32_t)nf[i].size();
            if (num < kMinNeighbors) num += (uint32_t)nbd[i].size();
            raw_v[i] = (num < kMinNeighbors) ? Real(0) : velocity_divergence(i);
            dadv[i] = std::max<Real>(raw_v[i], Real(0));
            kc[i] = dadv[i] * alpha[i];
        }
        double sum = 0;
        for (uint32_t i = 0; i < n; ++i) sum += (double)dadv[i];
        return n ? sum / n : 0.0;
    }

    int divergence_solve(int max_iter, double max_error) {
        if (n == 0) {
            last_iters_v = 0;
            last_err_v = 0;
            return 0;
        }
        density_alpha(true);
        kw_v = kapv;
        raw_v.assign(n, Real(0));
        div_ran = true;
        jacobi([&](uint32_t j) { return kapv[j]; }, (Real)h, [&](uint32_t i) { return !(dadv[i] > Real(0)); });
        init_err_v = divergence_residual(true);
        const double eta = max_error * 0.01 * prm.density0 / h;
        int it = 0;
        double avg = 0;
        while (((avg > eta) || (it < 3)) && (it < max_iter)) {
            for (uint32_t i = 0; i < n; ++i) kapv[i] += kc[i];
            jacobi([&](uint32_t j) { return kc[j]; }, (Real)h, [](uint32_t) { return false; });
            avg = divergence_residual(false);
            ++it;
        }
        last_iters_v = it;
        last_err_v = avg;
        return it;
    }

    void viscosity() {
        const Real cvis = (Real)inv_h * (Real)prm.viscosity;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            const Real xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
            const Real vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
            Kahan<Real> ax, ay, az;
            for (uint32_t j : nf[i]) {
                const Real w = K.W(xi - x[3 * j], yi - x[3 * j + 1], zi - x[3 * j + 2]);
                const Real s = cvis * (m[j] / ((Real)prm.density0 + rho[j]));
                ax.add(-(s * (vx - v[3 * j])) * w);
                ay.add(-(s * (vy - v[3 * j + 1])) * w);
                az.add(-(s * (vz - v[3 * j + 2])) * w);
            }
            a[3 * i] = (Real)prm.gravitation[0] + ax.value();
            a[3 * i + 1] = (Real)prm.gravitation[1] + ay.value();
            a[3 * i + 2] = (Real)prm.gravitation[2] + az.value();
        }
    }

    double cfl_max_speed2() const {
        double m2 = 0;
        for (uint32_t i = 0; i < n; ++i) {
            double s = 0;
            for (int c = 0; c < 3; ++c) {
                const Real u = v[3 * i + c] + a[3 * i + c] * (Real)h;
                s += (double)(u * u);
            }
            m2 = std::max(m2, s);
        }
        return m2;
    }

    void update_time_step(double hf) {
        h_future = hf;
        inv_h_future = 1.0 / hf;
        h_ratio = h / hf;
        h_ratio2 = (h * h) / (hf * hf);
    }

    void update_vel() {
        for (uint32_t i = 0; i < n; ++i) {
            for (int c = 0; c < 3; ++c) v[3 * i + c] += (Real)h * a[3 * i + c];
            kap[i] = std::max<Real>(kap[i] * (Real)h_ratio2, Real(-0.5));
        }
    }

    double pressure_residual(bool init) {
        const Real hf = (Real)h_future;
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            if (init) {
                alpha[i] *= (Real)inv_h_future;
                kap[i] = 0;
            }
            raw_p[i] = rho[i] + hf * velocity_divergence(i);  // rho[] = rho - rho0
            dadv[i] = std::max<Real>(raw_p[i], Real(0));
            kc[i] = dadv[i] * alpha[i];
            kap[i] += kc[i];
        }
        double sum = 0;
        for (uint32_t i = 0; i < n; ++i) sum += (double)dadv[i];
        return n ? sum / n : 0.0;
    }

    int pressure_solve(int max_iter, double max_error) {
        if (n == 0) {
            last_iters = 0;
            last_err = 0;
            return 0;
        }
        kw_p = kap;
        raw_p.assign(n, Real(0));
        jacobi([&](uint32_t j) { return kap[j]; }, (Real)h_future, [](uint32_t) { return false; });
        init_err = pressure_residual(true);
        const double eta = max_error * 0.01 * prm.density0;
        int it = 0;
        double avg = 0;
        while (((avg > eta) || (it < 2)) && (it < max_iter)) {
            jacobi([&](uint32_t j) { return kc[j]; }, (Real)h_future, [](uint32_t) { return false; });
            avg = pressure_residual(false);
            ++it;
        }
        last_iters = it;
        last_err = avg;
        return it;
    }

    void update_pos() {
        for (size_t k = 0; k < 3 * (size_t)n; ++k) x[k] += (Real)h * v[k];
    }

    void on_step_end() {
        h_past = h;
        h = h_future;
        inv_h = inv_h_future;
    }

    // Pressure (which = 0) or divergence (1) coefficient the last solve needed, per particle
    // (needed_totals of the device's solver.cu): the applied total, warm start plus corrections, less
    // one Jacobi estimate min(r, 0) alpha of its excess, clamped to [-0.5, 0]. alpha here is the
    // pressure solve's alpha / h_future; the divergence solve's alpha is that times h_future.
    double needed(int which, uint32_t i) const {
        auto clampk = [](double k) { return std::min(std::max(k, -0.5), 0.0); };
        if (which == 0) {
            if (kw_p.size() != n || raw_p.size() != n) return 0.0;
            return clampk((double)(kw_p[i] + kap[i] + std::min<Real>(raw_p[i], Real(0)) * alpha[i]));
        }
        if (!div_ran || kw_v.size() != n || raw_v.size() != n) return 0.0;
        return clampk((double)(kw_v[i] + kapv[i] + std::min<Real>(raw_v[i], Real(0)) * (alpha[i] * (Real)h_future)));
    }

    // dfsph_dynamic_window_stabilize (DynamicWindow::stabilizeFluid method 0, DynamicWindow.cu:
    // 3160-3700): `iters` steps of the fixed step `dt` with the warm starts cleared before and after;
    // the particles before `first` keep their positions and velocities, the others' velocities are
    // multiplied by `damping` before each position update; the dt history is restored afterwards.
    void stabilize(uint32_t iters, double dt, double damping, uint32_t first) {
        const double sh = h, shf = h_future, shp = h_past, sih = inv_h, sihf = inv_h_future, sr = h_ratio,
                     sr2 = h_ratio2;
        h = h_future = dt;
        inv_h = inv_h_future = 1.0 / dt;
        h_ratio = h_ratio2 = 1.0;
        std::fill(kap.begin(), kap.end(), Real(0));
        std::fill(kapv.begin(), kapv.end(), Real(0));
        first = std::min(first, n);
        const std::vector<Real> sx(x.begin(), x.begin() + 3 * (size_t)first), sv(v.begin(), v.begin() + 3 * (size_t)first);
        for (uint32_t it = 0; it < iters; ++it) {
            neighbors();
            if (prm.enable_divergence_solver) divergence_solve(prm.max_iterations_v, prm.max_error_v);
            else density_alpha(false);
            viscosity();
            update_vel();
            pressure_solve(prm.max_iterations, prm.max_error);
            if (damping < 1.0)
                for (size_t k = 3 * (size_t)first; k < 3 * (size_t)n; ++k) v[k] *= (Real)damping;
            update_pos();
            std::copy(sx.begin(), sx.end(), x.begin());
            std::copy(sv.begin(), sv.end(), v.begin());
            on_step_end();
        }
        std::fill(kap.begin(), kap.end(), Real(0));
        std::fill(kapv.begin(), kapv.end(), Real(0));
        h = sh; h_future = shf; h_past = shp; inv_h = sih; inv_h_future = sihf; h_ratio = sr; h_ratio2 = sr2;
    }

    void step() {
        div_ran = false;
        neighbors();
        if (prm.enable_divergence_solver) divergence_solve(prm.max_iterations_v, prm.max_error_v);
        else {
            density_alpha(false);
            last_iters_v = 0;
            last_err_v = 0;
        }
        viscosity();
        if (prm.cfl_method) {
            double hn = prm.cfl_factor * 0.4 * (2.0 * prm.particle_radius / std::sqrt(cfl_max_speed2()));
            hn = std::min(hn, prm.cfl_max_time_step);
            hn = std::max(hn, prm.cfl_min_time_step);
            update_time_step(hn);
        } else {
            update_time_step(time_step);
        }
        update_vel();
        pressure_solve(prm.max_iterations, prm.max_error);
        update_pos();
        on_step_end();
        if (remove_escaped) remove_out_of_box();
    }
};

struct Handle {
    int precision;
    Oracle<float> f;
    Oracle<double> d;
};

template <class O> void set_fluid(O& o, const float* xyz, const float* vxyz, const float* mass, uint32_t n) {
    using Real = typename std::remove_reference<decltype(o.x[0])>::type;
    o.n = n;
    o.x.assign(3 * (size_t)n, 0);
    o.v.assign(3 * (size_t)n, 0);
    o.m.assign(n, 0);
    const double d = 2.0 * o.prm.particle_radius;
    const float default_mass = (float)(0.8 * d * d * d * o.prm.density0);  // FluidModel.cpp:104
    for (size_t k = 0; k < 3 * (size_t)n; ++k) {
        o.x[k] = (Real)xyz[k];
        o.v[k] = vxyz ? (Real)vxyz[k] : Real(0);
    }
    for (uint32_t i = 0; i < n; ++i) o.m[i] = (Real)(mass ? mass[i] : default_mass);
    o.inflow_mass = (n && mass) ? mass[0] : default_mass;  // the new particles' mass (fluid->mass[0])
    for (auto* vec : {&o.rho, &o.alpha, &o.dadv, &o.kap, &o.kapv, &o.kc}) vec->assign(n, 0);
    o.a.assign(3 * (size_t)n, 0);
    o.nf.assign(n, {});
    o.nbd.assign(n, {});
    o.reset_dt();
}

template <class O> int set_boundary(O& o, const float* xyz, const float* psi, uint32_t n, const double* grid_box) {
    using Real = typename std::remove_reference<decltype(o.x.data()[0])>::type;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (grid_box && grid_box[0] < grid_box[3] && grid_box[1] < grid_box[4] && grid_box[2] < grid_box[5]) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = (float)grid_box[a];
            mx[a] = (float)grid_box[3 + a];
        }
    } else {
        if (n == 0) return -1;
        for (uint32_t i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::min(mn[a], xyz[3 * i + a]);
                mx[a] = std::max(mx[a], xyz[3 * i + a]);
            }
    }
    o.set_grid(mn, mx);
    o.nb = n;
    o.bx.assign(3 * (size_t)n, 0);
    o.bv.assign(3 * (size_t)n, 0);
    for (size_t k = 0; k < 3 * (size_t)n; ++k) o.bx[k] = (Real)xyz[k];
    o.boundary_moving = false;
    if (psi) {
        o.psi.assign(n, 0);
        for (uint32_t i = 0; i < n; ++i) o.psi[i] = (Real)psi[i];
    } else {
        o.compute_psi();
    }
    return 0;
}

}  // namespace

extern "C" {

// Field ids follow include/dfsph_c.h (DFSPH_F_*).
void* oracle_create(int precision, const Params* p) {
    if (!p || (precision != 32 && precision != 64)) return nullptr;
    auto* h = new Handle();
    h->precision = precision;
    if (precision == 32) h->f.init(*p);
    else h->d.init(*p);
    return h;
}

void oracle_destroy(void* handle) { delete (Handle*)handle; }

#define ORACLE_DO(h, expr) (((Handle*)(h))->precision == 32 ? ([&](auto& o) { return expr; })(((Handle*)(h))->f) \
                                                            : ([&](auto& o) { return expr; })(((Handle*)(h))->d))

int oracle_set_boundary(void* h, const float* xyz, const float* psi, uint32_t n, const double* grid_box) {
    return ORACLE_DO(h, set_boundary(o, xyz, psi, n, grid_box));
}

int oracle_set_boundary_velocity(void* h, const float* xyz, const float* vxyz) {
    return ORACLE_DO(h, ([&] {
        for (size_t k = 0; k < 3 * (size_t)o.nb; ++k) {
            o.bx[k] = xyz[k];
            o.bv[k] = vxyz ? vxyz[k] : 0.0f;
        }
        o.boundary_moving = true;
        return 0;
    })());
}

int oracle_set_fluid(void* h, const float* xyz, const float* vxyz, const float* mass, uint32_t n) {
    return ORACLE_DO(h, (set_fluid(o, xyz, vxyz, mass, n), 0));
}

// Overwrites positions (and velocities) keeping warm starts and dt history.
int oracle_update_fluid(void* h, const double* xyz, const double* vxyz) {
    return ORACLE_DO(h, ([&] {
        for (size_t k = 0; k < 3 * (size_t)o.n; ++k) {
            o.x[k] = xyz[k];
            if (vxyz) o.v[k] = vxyz[k];
        }
        return 0;
    })());
}

int oracle_step(void* h, int32_t* iters, int32_t* iters_v, double* err, double* err_v) {
    return ORACLE_DO(h, ([&] {
        o.step();
        if (iters) *iters = o.last_iters;
        if (iters_v) *iters_v = o.last_iters_v;
        if (err) *err = o.last_err;
        if (err_v) *err_v = o.last_err_v;
        return (int)o.overflow;
    })());
}

int oracle_open_boundary_init(void* h, const Surface* b, const Surface* in, const Surface* sf, const float* xyz,
                              uint32_t ns, uint32_t* kept) {
    return ORACLE_DO(h, ([&] {
        o.ob_init(*b, *in, *sf, xyz, ns);
        if (kept) *kept = (uint32_t)(o.ob_x.size() / 3);
        return 0;
    })());
}

int oracle_open_boundary_apply(void* h, double dist, double rho, int inflow, int outflow, uint32_t capacity,
                               uint32_t* added, uint32_t* removed) {
    return ORACLE_DO(h, ([&] {
        uint32_t ad = 0, rm = 0;
        bool clipped = false;
        o.ob_apply(dist, rho, inflow != 0, outflow != 0, capacity, ad, rm, clipped);
        if (added) *added = ad;
        if (removed) *removed = rm;
        return clipped ? 1 : 0;
    })());
}

int oracle_open_boundary_shift(void* h, const float* d) { return ORACLE_DO(h, (o.ob_shift(d), 0)); }

// Removes the fluid particles with a coordinate outside [lo, hi] (compared as the device's box tag,
// open_boundary.cu box_tag_kernel), keeping the order of the others; the dynamic window's removal
// behind a moved window.
int oracle_dynamic_window_stabilize(void* h, uint32_t iters, double dt, double damping, uint32_t first) {
    return ORACLE_DO(h, (o.stabilize(iters, dt, damping, first), 0));
}

int oracle_remove_outside_box(void* h, const float* lo, const float* hi, uint32_t* removed) {
    return ORACLE_DO(h, ([&] {
        using R = typename std::remove_reference<decltype(o.x[0])>::type;
        const uint32_t r = o.compact([&](uint32_t i) {
            for (int a = 0; a < 3; ++a) {
                const R c = o.x[3 * i + a];
                if (c > (R)hi[a] || c < (R)lo[a]) return false;
            }
            return true;
        });
        if (removed) *removed = r;
        return 0;
    })());
}

// inside[i] and normal[3 i..] of the restated BufferFluidSurface::isinside / getNormal.
int oracle_set_surface_mesh(uint32_t id, const float* v, uint32_t nv, const uint32_t* t, uint32_t nt) {
    if (id >= 8 || nt == 0) return -1;
    OracleMesh& m = g_meshes[id];
    m = OracleMesh{};
    for (uint32_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) {
            const float x = v[3 * (size_t)i + a];
            if (m.bmin[a] > x) m.bmin[a] = x;
            if (m.bmax[a] < x) m.bmax[a] = x;
        }
    m.tri.resize(9 * (size_t)nt);
    for (size_t k = 0; k < 3 * (size_t)nt; ++k) {
        if (t[k] >= nv) return -1;
        for (int a = 0; a < 3; ++a) m.tri[3 * k + a] = v[3 * (size_t)t[k] + a];
    }
    return 0;
}

int oracle_surface_eval(const Surface* s, const float* p, uint32_t n, uint8_t* inside, float* normal) {
    for (uint32_t i = 0; i < n; ++i) {
        inside[i] = surface_inside(*s, p + 3 * (size_t)i) ? 1 : 0;
        surface_normal(*s, p + 3 * (size_t)i, normal + 3 * (size_t)i);
    }
    return 0;
}

// Piecewise phases, mirroring the C ABI of the device library.
int oracle_neighbors(void* h) { return ORACLE_DO(h, (o.neighbors(), (int)o.overflow)); }
int oracle_divergence_solve(void* h, int max_iter, double max_error) {
    return ORACLE_DO(h, o.divergence_solve(max_iter, max_error));
}
int oracle_density_alpha(void* h, int warm_v) { return ORACLE_DO(h, (o.density_alpha(warm_v != 0), 0)); }
int oracle_external_forces(void* h) { return ORACLE_DO(h, (o.viscosity(), 0)); }
int oracle_update_time_step(void* h, double hf) { return ORACLE_DO(h, (o.update_time_step(hf), 0)); }
int oracle_update_vel(void* h) { return ORACLE_DO(h, (o.update_vel(), 0)); }
int oracle_pressure_solve(void* h, int max_iter, double max_error) {
    return ORACLE_DO(h, o.pressure_solve(max_iter, max_error));
}
int oracle_update_pos(void* h) { return ORACLE_DO(h, (o.update_pos(), 0)); }
int oracle_on_step_end(void* h) { return ORACLE_DO(h, (o.on_step_end(), 0)); }

int oracle_get(void* h, int field, double* out) {
    return ORACLE_DO(h, ([&] {
        auto put = [&](const auto& vec) {
            for (size_t k = 0; k < vec.size(); ++k) out[k] = (double)vec[k];
            return 0;
        };
        switch (field) {
            case 0: return put(o.x);
            case 1: return put(o.v);
            case 2: return put(o.m);
            case 3: {  // density = rho0 + (rho - rho0)
                for (size_t k = 0; k < o.rho.size(); ++k) out[k] = o.prm.density0 + (double)o.rho[k];
                return 0;
            }
            case 4: return put(o.alpha);
            case 5: return put(o.dadv);
            case 6: return put(o.kap);
            case 7: return put(o.kapv);
            case 8: return put(o.a);
            case 10: return put(o.psi);
            case 11: return put(o.bx);
            case 14: return o.bforce_on ? put(o.bF) : -1;
            case 20:  // needed pressure coefficient of the last solve (not a C ABI field)
            case 21:  // needed divergence coefficient
                for (uint32_t i = 0; i < o.n; ++i) out[i] = o.needed(field - 20, i);
                return 0;
            default: return -1;
        }
    })());
}

int oracle_get_scalar(void* h, const char* key, double* out) {
    return ORACLE_DO(h, ([&] {
        const std::string k(key);
        if (k == "h") *out = o.h;
        else if (k == "h_future") *out = o.h_future;
        else if (k == "h_past") *out = o.h_past;
        else if (k == "inv_h") *out = o.inv_h;
        else if (k == "iterations") *out = o.last_iters;
        else if (k == "iterations_v") *out = o.last_iters_v;
        else if (k == "density_error") *out = o.last_err;
        else if (k == "divergence_error") *out = o.last_err_v;
        else if (k == "init_density_error") *out = o.init_err;
        else if (k == "init_divergence_error") *out = o.init_err_v;
        else if (k == "grid_offset_x") *out = o.off[0];
        else if (k == "grid_offset_y") *out = o.off[1];
        else if (k == "grid_offset_z") *out = o.off[2];
        else if (k == "grid_dim_x") *out = o.dim[0];
        else if (k == "grid_dim_y") *out = o.dim[1];
        else if (k == "grid_dim_z") *out = o.dim[2];
        else if (k == "n") *out = o.n;
        else if (k == "escaped_removed") *out = (double)o.escaped_removed;
        else return -1;
        return 0;
    })());
}

int oracle_set_scalar(void* h, const char* key, double v) {
    return ORACLE_DO(h, ([&] {
        const std::string k(key);
        if (k == "h") o.h = v;
        else if (k == "h_future") o.h_future = v;
        else if (k == "inv_h") o.inv_h = v;
        else if (k == "time_step") o.time_step = v;
        else if (k == "boundary_forces") {
            o.bforce_on = v != 0;
            if (o.bforce_on) o.bF.assign(3 * (size_t)o.nb, 0.0);
        }
        else if (k == "remove_escaped") o.remove_escaped = v != 0;
        else return -1;
        return 0;
    })());
}

// counts[2*i] fluid, counts[2*i+1] boundary; lists[i*row + k] fluid ids then boundary indices.
int oracle_get_neighbors(void* h, uint32_t* counts, uint32_t* lists, uint32_t row) {
    return ORACLE_DO(h, ([&] {
        for (uint32_t i = 0; i < o.n; ++i) {
            counts[2 * (size_t)i] = (uint32_t)o.nf[i].size();
            counts[2 * (size_t)i + 1] = (uint32_t)o.nbd[i].size();
            size_t k = 0;
            for (uint32_t j : o.nf[i])
                if (k < row) lists[(size_t)i * row + k++] = j;
            for (uint32_t j : o.nbd[i])
                if (k < row) lists[(size_t)i * row + k++] = j;
        }
        return 0;
    })());
}

// Kernel function values for the pin against the reference CubicKernelPerso.
int oracle_kernel_values(double H, const double* r, uint32_t count, int precision, double* w, double* dw) {
    if (precision == 32) {
        Cubic<float> K;
        K.set(H);
        for (uint32_t i = 0; i < count; ++i) {
            float g0, g1, g2;
            w[i] = K.W((float)r[i], 0.0f, 0.0f);
            K.gradW((float)r[i], 0.0f, 0.0f, g0, g1, g2);
            dw[i] = g0;
        }
    } else {
        Cubic<double> K;
        K.set(H);
        for (uint32_t i = 0; i < count; ++i) {
            double g0, g1, g2;
            w[i] = K.W(r[i], 0.0, 0.0);
            K.gradW(r[i], 0.0, 0.0, g0, g1, g2);
            dw[i] = g0;
        }
    }
    return 0;
}

}  // extern "C"
