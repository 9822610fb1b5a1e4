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
    float Hf = 0, H2f = 0;
    int off[3] = {0, 0, 0}, dim[3] = {0, 0, 0};
    bool grid = false;
    // fluid (original order)
    uint32_t n = 0;
    std::vector<Real> x, v, m, rho, alpha, dadv, kap, kapv, a, kc;
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
        Hf = (float)(4.0 * p.particle_radius);
        H2f = Hf * Hf;
        time_step = p.time_step;
        reset_dt();
    }
    void reset_dt() {
        h = h_future = h_past = time_step;
        inv_h = inv_h_future = 1.0 / time_step;
        h_ratio = h_ratio2 = 1.0;
    }

    void set_grid(const float mn[3], const float mx[3]) {
        for (int a3 = 0; a3 < 3; ++a3) {
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
            Kahan<Real> sgk, dr, gx, gy, gz;
            r.add((Real)-prm.density0);
            r.add(m[i] * K.W0);
            const Real xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
            const Real vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
            for (uint32_t j : nf[i]) {
                const Real rx = xi - x[3 * j], ry = yi - x[3 * j + 1], rz = zi - x[3 * j + 2];
                Real w = K.W(rx, ry, rz), g0, g1, g2;
                K.gradW(rx, ry, rz, g0, g1, g2);
                r.add(m[j] * w);
                const Real px = m[j] * g0, py = m[j] * g1, pz = m[j] * g2;
                sgk.add(px * px + py * py + pz * pz);
                gx.add(px); gy.add(py); gz.add(pz);
                dr.add((vx - v[3 * j]) * px + (vy - v[3 * j + 1]) * py + (vz - v[3 * j + 2]) * pz);
            }
            for (uint32_t j : nbd[i]) {
                const Real rx = xi - bx[3 * j], ry = yi - bx[3 * j + 1], rz = zi - bx[3 * j + 2];
                Real w = K.W(rx, ry, rz), g0, g1, g2;
                K.gradW(rx, ry, rz, g0, g1, g2);
                r.add(psi[j] * w);
                const Real px = psi[j] * g0, py = psi[j] * g1, pz = psi[j] * g2;
                sgk.add(px * px + py * py + pz * pz);
                gx.add(px); gy.add(py); gz.add(pz);
                dr.add((vx - bvel(j, 0)) * px + (vy - bvel(j, 1)) * py + (vz - bvel(j, 2)) * pz);
            }
            const Real Gx = gx.value(), Gy = gy.value(), Gz = gz.value();
            const Real sg = sgk.value() + (Gx * Gx + Gy * Gy + Gz * Gz);
            alpha[i] = -invh / std::max<Real>(sg, (Real)kEps);
            rho[i] = r.value();  // rho - rho0
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
            dadv[i] = (num < kMinNeighbors) ? Real(0) : std::max<Real>(velocity_divergence(i), Real(0));
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
            dadv[i] = std::max<Real>(rho[i] + hf * velocity_divergence(i), Real(0));  // rho[] = rho - rho0
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

    void step() {
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
