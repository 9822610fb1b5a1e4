/* dfsph.hpp — C++ facade over the C ABI (dfsph_c.h) with the shape of the reference's host classes,
 * for C++ callers that used SPH::DFSPHCUDA / SPH::DFSPHCData / the cuda_* host functions.
 *
 *   reference                                          here
 *   SPH::DFSPHCUDA : TimeStep (DFSPH_CUDA.h:85-110,    dfsph::DFSPHCUDA: step(), reset(),
 *     TimeStep.h:70-103)                                 get/set of the TimeStep parameters,
 *                                                        getIterationCount(V), m_data
 *   SPH::DFSPHCData (DFSPH_c_arrays_structure.h:297)    dfsph::DFSPHCData: updateTimeStep,
 *                                                        onSimulationStepEnd, readDynamicData,
 *                                                        getFluidParticlesCount, h / h_future / h_past
 *   cuda_* host functions (DFSPH_core_cuda.h:27-74)     dfsph::cuda_* with the same arguments
 *   SPH::TimeStepDFSPH (TimeStepDFSPH.h:20-48)          dfsph::TimeStepDFSPH: the same TimeStep
 *                                                        interface on the device time step
 *   SceneLoader::readScene (SceneLoader.cpp:39-320)     dfsph::SceneData::load (dfsph_scene_load)
 *
 * Header-only; link with libdfsph_b200.so. Errors throw dfsph::Error (code + dfsph_last_error
 * message) where the reference calls exit(). The scene is given as plain arrays (the reference builds
 * it from a FluidModel: fluid positions / velocities and the boundary samples).
 */
#ifndef DFSPH_HPP
#define DFSPH_HPP

#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "dfsph_c.h"

namespace dfsph {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(const dfsph_ctx* ctx, int code) {
    if (code != DFSPH_OK) {
        const char* m = dfsph_last_error(ctx);
        throw Error(code, "DFSPH error " + std::to_string(code) + ": " + (m ? m : ""));
    }
}

/* The reference's viscosity choices (TimeStep.h:16); the device time step implements XSPH. */
enum class ViscosityMethods { None = 0, Standard, XSPH, Bender2017, Peer2015, Peer2016 };

/* State accessors of one context (the parts of SPH::DFSPHCData callers use). Non-owning. */
class DFSPHCData {
public:
    explicit DFSPHCData(dfsph_ctx* ctx = nullptr) : ctx_(ctx) {}

    unsigned int getFluidParticlesCount() const {
        uint32_t n = 0;
        check(ctx_, dfsph_num_fluid(ctx_, &n));
        return n;
    }
    /* DFSPHCData::readDynamicData (DFSPH_c_arrays_structure.cpp:1120-1150): positions and
     * velocities, 3 floats per particle in particle-id order. */
    void readDynamicData(std::vector<float>& pos, std::vector<float>& vel) const {
        const size_t n = getFluidParticlesCount();
        pos.resize(3 * n);
        vel.resize(3 * n);
        check(ctx_, dfsph_read_dynamic_data(ctx_, pos.data(), vel.data()));
    }
    void updateTimeStep(double h_future) { check(ctx_, dfsph_update_time_step(ctx_, h_future)); }
    void onSimulationStepEnd() { check(ctx_, dfsph_on_step_end(ctx_)); }
    double h() const { return param("h"); }
    double h_future() const { return param("h_future"); }
    double h_past() const { return param("h_past"); }
    double get_current_timestep() const { return h(); }
    /* checkParticlesPositions(mode): 0 counts, 2 counts and removes the particles outside the box. */
    int checkParticlesPositions(int mode = 2) {
        uint32_t c = 0;
        check(ctx_, dfsph_check_particles_positions(ctx_, mode, &c));
        return (int)c;
    }
    dfsph_ctx* handle() const { return ctx_; }

private:
    double param(const char* key) const {
        double v = 0;
        check(ctx_, dfsph_get_param(ctx_, key, &v));
        return v;
    }
    dfsph_ctx* ctx_;
};

/* A reference JSON scene read by the library (dfsph_scene_load): the solver parameters and the
 * particle arrays (SceneLoader::readScene + the scene part of DemoBase::buildModel). */
struct SceneData {
    dfsph_scene scene{};
    std::vector<float> fluid, fluid_vel, boundary;  // fluid_vel empty when the scene gives none

    static SceneData load(const std::string& json_path) {
        SceneData d;
        dfsph_scene_file* f = nullptr;
        check(nullptr, dfsph_scene_load(json_path.c_str(), &d.scene, &f));
        uint32_t n = 0, nb = 0;
        int has_vel = 0;
        int code = dfsph_scene_file_counts(f, &n, &nb, &has_vel);
        if (code == DFSPH_OK) {
            d.fluid.resize(3 * (size_t)n);
            d.boundary.resize(3 * (size_t)nb);
            if (has_vel) d.fluid_vel.resize(3 * (size_t)n);
            code = dfsph_scene_file_fluid(f, d.fluid.data(), has_vel ? d.fluid_vel.data() : nullptr);
        }
        if (code == DFSPH_OK) code = dfsph_scene_file_boundary(f, d.boundary.data());
        dfsph_scene_file_free(f);
        check(nullptr, code);
        return d;
    }
};

/* SPH::DFSPHCUDA over one context. The arrays passed to the constructor are kept for reset(). */
class DFSPHCUDA {
public:
    /* From a reference JSON scene (its learnedWarmStart block is applied by
     * dfsph_create_from_scene_file; here the learned mode is set with set()). */
    explicit DFSPHCUDA(const std::string& scene_json) : DFSPHCUDA(SceneData::load(scene_json)) {}
    explicit DFSPHCUDA(const SceneData& d) : DFSPHCUDA(d.scene, d.fluid, d.boundary, d.fluid_vel) {}
    DFSPHCUDA(const dfsph_scene& scene, std::vector<float> fluid_xyz, std::vector<float> boundary_xyz,
              std::vector<float> fluid_vel = {}, std::vector<float> boundary_psi = {})
        : fluid_(std::move(fluid_xyz)), vel_(std::move(fluid_vel)), boundary_(std::move(boundary_xyz)),
          psi_(std::move(boundary_psi)) {
        if (fluid_.size() % 3 || boundary_.size() % 3 || (!vel_.empty() && vel_.size() != fluid_.size()) ||
            (!psi_.empty() && psi_.size() * 3 != boundary_.size()))
            throw Error(DFSPH_E_INVALID, "DFSPHCUDA: array sizes do not match");
        dfsph_scene s = scene;
        radius_ = scene.particle_radius;
        if (s.fluid_capacity < fluid_.size() / 3) s.fluid_capacity = (uint32_t)(fluid_.size() / 3);
        if (s.boundary_capacity < boundary_.size() / 3) s.boundary_capacity = (uint32_t)(boundary_.size() / 3);
        check(nullptr, dfsph_create(&s, &ctx_));
        m_data = DFSPHCData(ctx_);
        try {
            reset();
        } catch (...) {
            dfsph_destroy(ctx_);
            throw;
        }
    }
    ~DFSPHCUDA() { dfsph_destroy(ctx_); }
    DFSPHCUDA(const DFSPHCUDA&) = delete;
    DFSPHCUDA& operator=(const DFSPHCUDA&) = delete;

    /* DFSPHCUDA::step (DFSPH_CUDA.cpp:82-794). */
    void step() {
        check(ctx_, dfsph_step(ctx_, &stats_));
        m_iterations = (unsigned)stats_.iterations;
        m_iterationsV = (unsigned)stats_.iterations_v;
    }
    /* DFSPHCUDA::reset (DFSPH_CUDA.cpp:796-817): the boundary and fluid given at construction. */
    void reset() {
        check(ctx_, dfsph_set_boundary(ctx_, boundary_.data(), psi_.empty() ? nullptr : psi_.data(),
                                       (uint32_t)(boundary_.size() / 3)));
        check(ctx_, dfsph_upload_fluid(ctx_, fluid_.data(), vel_.empty() ? nullptr : vel_.data(), nullptr,
                                       (uint32_t)(fluid_.size() / 3)));
        m_iterations = m_iterationsV = 0;
    }

    unsigned int getIterationCount() const { return m_iterations; }
    unsigned int getIterationCountV() const { return m_iterationsV; }
    bool getEnableDivergenceSolver() const { return get("enable_divergence_solver") != 0; }
    void setEnableDivergenceSolver(bool v) { set("enable_divergence_solver", v ? 1 : 0); }
    unsigned int getCflMethod() const { return (unsigned)get("cfl_method"); }
    void setCflMethod(unsigned int v) { set("cfl_method", v); }
    double getCflFactor() const { return get("cfl_factor"); }
    void setCflFactor(double v) { set("cfl_factor", v); }
    double getCflMaxTimeStepSize() const { return get("cfl_max_time_step"); }
    void setCflMaxTimeStepSize(double v) { set("cfl_max_time_step", v); }
    double getMaxError() const { return get("max_error"); }
    void setMaxError(double v) { set("max_error", v); }
    unsigned int getMaxIterations() const { return (unsigned)get("max_iterations"); }
    void setMaxIterations(unsigned int v) { set("max_iterations", v); }
    double getMaxErrorV() const { return get("max_error_v"); }
    void setMaxErrorV(double v) { set("max_error_v", v); }
    unsigned int getMaxIterationsV() const { return (unsigned)get("max_iterations_v"); }
    void setMaxIterationsV(unsigned int v) { set("max_iterations_v", v); }
    ViscosityMethods getViscosityMethod() const { return ViscosityMethods::XSPH; }
    void setViscosityMethod(ViscosityMethods v) {
        if (v != ViscosityMethods::XSPH)
            throw Error(DFSPH_E_INVALID, "only the XSPH viscosity is implemented by the device time step");
    }
    double getViscosity() const { return get("viscosity"); }
    void setViscosity(double v) { set("viscosity", v); }

    /* ---- the host-side operations of the reference's DFSPHCUDA (DFSPH_CUDA.cpp:1885-1979, 3889-4210) */

    /* DFSPHCData::fluid_files_folder: where handleSimulationSave / handleSimulationLoad write and read. */
    std::string fluid_files_folder = "file_data/";
    /* handleSimulationSave: the fluid (with general_data.txt) and the boundary in the reference's text
     * format. Dynamic bodies are ranges of the boundary here, so save_solids adds nothing of its own. */
    void handleSimulationSave(bool save_liquid, bool save_solids, bool save_boundaries) {
        (void)save_solids;
        const int what = (save_liquid ? DFSPH_SNAP_FLUID : 0) | (save_boundaries ? DFSPH_SNAP_BOUNDARY : 0);
        if (what) check(ctx_, dfsph_save_snapshot(ctx_, fluid_files_folder.c_str(), what));
    }
    /* handleSimulationLoad (dynamic bodies: as handleSimulationSave). */
    void handleSimulationLoad(bool load_liquid, bool load_liquid_velocities, bool load_solids,
                              bool load_solids_velocities, bool load_boundaries) {
        (void)load_solids;
        (void)load_solids_velocities;
        const int what = (load_liquid ? DFSPH_SNAP_FLUID : 0) | (load_boundaries ? DFSPH_SNAP_BOUNDARY : 0);
        if (what)
            check(ctx_, dfsph_load_snapshot(ctx_, fluid_files_folder.c_str(), what, load_liquid_velocities ? 1 : 0));
    }
    /* zeroFluidVelocities (DFSPHCData::zeroFluidVelocities): positions kept, velocities zero. */
    void zeroFluidVelocities() {
        std::vector<float> x, v;
        m_data.readDynamicData(x, v);
        if (!x.empty()) check(ctx_, dfsph_update_fluid(ctx_, x.data(), nullptr));
    }
    /* getFluidLevel / handleFLuidLevelControl (DFSPH_CUDA.cpp:4150-4160; dfsph_fluid_level,
     * dfsph_fluid_level_control). */
    double getFluidLevel() const {
        double v = -1;
        check(ctx_, dfsph_fluid_level(ctx_, &v));
        return v;
    }
    void handleFLuidLevelControl(double level) {
        if (level > 0) check(ctx_, dfsph_fluid_level_control(ctx_, level, nullptr, nullptr));
    }
    /* updateTimeStepDuration: the time step used while the CFL condition is off. */
    void updateTimeStepDuration(double duration) { set("time_step", duration); }
    /* applyOpenBoundaries (DFSPH_CUDA.cpp:3889-3986) with the reference's thresholds (1.75 r,
     * 700 kg/m^3, :3903-3906) once dfsph_open_boundary_init has set the surfaces and samples. */
    void applyOpenBoundaries() {
        check(ctx_, dfsph_open_boundary_apply(ctx_, 1.75 * radius_, 700.0, 1, 1, nullptr, nullptr));
    }
    /* The dynamic window (DynamicWindowInterface): its box and walls, then handleSimulationMovement
     * (DFSPH_CUDA.cpp:4142-4147: movements of more than 0.5 m shift it, with the open boundary's inflow
     * thresholds for the newly covered region) and getSimulationCenter (the box's centre). */
    void dynamicWindowInit(const double lo[3], const double hi[3], uint32_t wall_first, uint32_t wall_count,
                           const std::vector<float>& rest_xyz) {
        check(ctx_, dfsph_dynamic_window_init(ctx_, lo, hi, wall_first, wall_count, rest_xyz.data(),
                                              (uint32_t)(rest_xyz.size() / 3)));
        for (int a = 0; a < 3; ++a) window_center_[a] = 0.5 * (lo[a] + hi[a]);
    }
    void handleSimulationMovement(const double movement[3]) {
        const double m2 = movement[0] * movement[0] + movement[1] * movement[1] + movement[2] * movement[2];
        if (m2 > 0.25)
            check(ctx_, dfsph_dynamic_window_shift(ctx_, movement, 1.75 * radius_, 700.0, nullptr, nullptr));
    }
    std::array<double, 3> getSimulationCenter() const {
        double d[3] = {0, 0, 0};
        if (dfsph_dynamic_window_displacement(ctx_, d) != DFSPH_OK) d[0] = d[1] = d[2] = 0.0;
        return {window_center_[0] + d[0], window_center_[1] + d[1], window_center_[2] + d[2]};
    }
    /* Dynamic bodies as ranges of the boundary (upload order): the centre of their samples as
     * uploaded (rest_position) and their current position, for updateRigidBodies and
     * getFluidImpactOnDynamicBodies (which needs set("boundary_forces", 1)). */
    struct DynamicBody {
        uint32_t first, count;
        std::array<double, 3> position;
        std::array<double, 3> rest_position;
        std::array<double, 4> q{{1.0, 0.0, 0.0, 0.0}};  // orientation (w, x, y, z), unit
    };
    std::vector<DynamicBody> dynamic_bodies;
    void addDynamicBody(uint32_t first, uint32_t count, const std::array<double, 3>& center) {
        dynamic_bodies.push_back({first, count, center, center, {{1.0, 0.0, 0.0, 0.0}}});
    }
    /* DFSPHCUDA::is_dynamic_bodies_paused / handleDynamicBodiesPause (DFSPH_CUDA.cpp:1860-1883,
     * DFSPHCData::pause_solids): pausing sets every dynamic body's particle velocities (and so its
     * rigid velocity field) to zero, keeping its pose. */
    bool is_dynamic_bodies_paused = false;
    void handleDynamicBodiesPause(bool pause) {
        is_dynamic_bodies_paused = pause;
        if (!pause) return;
        const std::array<double, 3> zero{{0.0, 0.0, 0.0}};
        for (DynamicBody& body : dynamic_bodies) apply_pose(body, body.position, body.q, zero, zero);
    }
    /* The state the reference's rigid-body solver hands back each step (DynamicBody: position,
     * velocity, orientation q = (w, x, y, z), angular velocity). */
    struct DynamicBodyState {
        std::array<double, 3> position, velocity, angular_velocity;
        std::array<double, 4> q;
    };
    /* updateRigidBodies (DFSPHCData::update_solids; update_dynamicObject_UnifiedParticleSet_cuda,
     * DFSPH_core_cuda.cu:3407-3449): body b's samples go to R(q) (x0 - rest) + position with the rigid
     * velocity field v + w x (x - position), on the device. */
    void updateRigidBodies(const std::vector<DynamicBodyState>& states) {
        if (states.size() != dynamic_bodies.size()) throw Error(DFSPH_E_INVALID, "one state per dynamic body");
        for (size_t b = 0; b < states.size(); ++b)
            apply_pose(dynamic_bodies[b], states[b].position, states[b].q, states[b].velocity,
                       states[b].angular_velocity);
    }
    /* updateRigidBodiesStatefromFile (DFSPHCData::update_solids_from_file, DFSPH_c_arrays_structure.cpp:
     * 1445-1479): waits for `solids_files_folder` + "update_solids.txt", reads per dynamic body its
     * position, velocity, orientation (x y z w) and angular velocity (13 numbers), applies them as
     * updateRigidBodies does and removes the file. The reference waits without limit; this wait gives
     * up after timeout_s seconds (Error DFSPH_E_STATE). */
    std::string solids_files_folder;
    void updateRigidBodiesStatefromFile(double timeout_s = 60.0) {
        const std::string path = solids_files_folder + "update_solids.txt";
        std::ifstream f;
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            f.open(path);
            if (f.is_open()) break;
            if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s)
                throw Error(DFSPH_E_STATE, "no " + path + " within the time limit");
            std::this_thread::sleep_for(std::chrono::milliseconds(100));
        }
        std::vector<DynamicBodyState> states(dynamic_bodies.size());
        for (DynamicBodyState& st : states) {
            double qx, qy, qz, qs;
            f >> st.position[0] >> st.position[1] >> st.position[2] >> st.velocity[0] >> st.velocity[1] >>
                st.velocity[2] >> qx >> qy >> qz >> qs >> st.angular_velocity[0] >> st.angular_velocity[1] >>
                st.angular_velocity[2];
            if (!f) throw Error(DFSPH_E_INVALID, "truncated " + path);
            st.q = {{qs, qx, qy, qz}};
        }
        f.close();
        updateRigidBodies(states);
        std::remove(path.c_str());
    }
    /* updateRigidBodiesStateToFile (DFSPHCData::update_solids_to_file, UnifiedParticleSet::
     * write_forces_to_file, DFSPH_c_arrays_structure.cpp:1422-1443, 681-712): per dynamic body i,
     * "solid_forces_file_<i>.txt" holds its particle count, then one line per particle with its
     * position in the body frame and the fluid's force on it; "solids_file.txt" the number of bodies;
     * all in `solids_files_folder` (needs set("boundary_forces", 1)). */
    void updateRigidBodiesStateToFile() {
        std::vector<double> f, x;
        boundary_force_and_position(f, x);
        std::remove((solids_files_folder + "solids_file.txt").c_str());
        for (size_t b = 0; b < dynamic_bodies.size(); ++b) {
            const DynamicBody& body = dynamic_bodies[b];
            if ((uint64_t)body.first + body.count > f.size() / 3)
                throw Error(DFSPH_E_INVALID, "dynamic body beyond the boundary");
            double R[9];
            rotation(body.q, R);
            std::ostringstream oss;
            oss << body.count << std::endl;
            for (uint32_t i = body.first; i < body.first + body.count; ++i) {
                double d[3], x0[3];
                for (int a = 0; a < 3; ++a) d[a] = x[3 * (size_t)i + a] - body.position[a];
                for (int a = 0; a < 3; ++a) x0[a] = R[a] * d[0] + R[3 + a] * d[1] + R[6 + a] * d[2];  // R^T d
                oss << (float)x0[0] << " " << (float)x0[1] << " " << (float)x0[2] << " ";
                oss << (float)f[3 * (size_t)i] << " " << (float)f[3 * (size_t)i + 1] << " " << (float)f[3 * (size_t)i + 2]
                    << " ";
                oss << std::endl;
            }
            const std::string name = solids_files_folder + "solid_forces_file_" + std::to_string(b) + ".txt";
            std::remove(name.c_str());
            std::ofstream out(name, std::ios_base::app);
            if (!out) throw Error(DFSPH_E_INVALID, "cannot write " + name);
            out << oss.str();
        }
        std::ofstream main(solids_files_folder + "solids_file.txt");
        if (!main) throw Error(DFSPH_E_INVALID, "cannot write " + solids_files_folder + "solids_file.txt");
        main << dynamic_bodies.size();
    }
    /* getFluidImpactOnDynamicBodies (compute_fluid_impact_on_dynamic_body_kernel,
     * DFSPH_memory_management_cuda.cu:688-705): per body, the sum of its particles' fluid forces
     * multiplied component-wise by the body's reduction factor, and the moment of those forces about
     * the body's position; appended to sph_forces / sph_moments, summed in FP64 on the host. */
    void getFluidImpactOnDynamicBodies(std::vector<std::array<double, 3>>& sph_forces,
                                       std::vector<std::array<double, 3>>& sph_moments,
                                       const std::vector<std::array<double, 3>>& reduction_factors) {
        std::vector<double> f, x;
        boundary_force_and_position(f, x);
        const size_t nb = f.size() / 3;
        for (size_t b = 0; b < dynamic_bodies.size(); ++b) {
            const DynamicBody& body = dynamic_bodies[b];
            if ((uint64_t)body.first + body.count > nb) throw Error(DFSPH_E_INVALID, "dynamic body beyond the boundary");
            const std::array<double, 3> r =
                b < reduction_factors.size() ? reduction_factors[b] : std::array<double, 3>{1.0, 1.0, 1.0};
            std::array<double, 3> F{0, 0, 0}, M{0, 0, 0};
            for (uint32_t i = body.first; i < body.first + body.count; ++i) {
                const double fx = f[3 * (size_t)i] * r[0], fy = f[3 * (size_t)i + 1] * r[1], fz = f[3 * (size_t)i + 2] * r[2];
                const double px = x[3 * (size_t)i] - body.position[0], py = x[3 * (size_t)i + 1] - body.position[1],
                             pz = x[3 * (size_t)i + 2] - body.position[2];
                F[0] += fx;
                F[1] += fy;
                F[2] += fz;
                M[0] += py * fz - pz * fy;
                M[1] += pz * fx - px * fz;
                M[2] += px * fy - py * fx;
            }
            sph_forces.push_back(F);
            sph_moments.push_back(M);
        }
    }

    /* getFluidBoyancyOnDynamicBodies (compute_fluid_Boyancy_on_dynamic_body_cuda,
     * DFSPH_memory_management_cuda.cu:729-776): per body, the vertical component of its particles'
     * fluid forces as the buoyancy (0, sum F_y, 0) and the point where it applies, the particles'
     * positions weighted by |F_y|; both zero when no particle feels a vertical force. */
    void getFluidBoyancyOnDynamicBodies(std::vector<std::array<double, 3>>& forces,
                                        std::vector<std::array<double, 3>>& pts_appli) {
        std::vector<double> f, x;
        boundary_force_and_position(f, x);
        for (const DynamicBody& body : dynamic_bodies) {
            if ((uint64_t)body.first + body.count > f.size() / 3)
                throw Error(DFSPH_E_INVALID, "dynamic body beyond the boundary");
            double fy = 0, wsum = 0, p[3] = {0, 0, 0};
            for (uint32_t i = body.first; i < body.first + body.count; ++i) {
                const double b = f[3 * (size_t)i + 1], a = std::fabs(b);
                if (a > 0) {
                    wsum += a;
                    fy += b;
                    for (int k = 0; k < 3; ++k) p[k] += x[3 * (size_t)i + k] * a;
                }
            }
            if (std::fabs(fy) > 0) {
                forces.push_back({0.0, fy, 0.0});
                pts_appli.push_back({p[0] / wsum, p[1] / wsum, p[2] / wsum});
            } else {
                forces.push_back({0.0, 0.0, 0.0});
                pts_appli.push_back({0.0, 0.0, 0.0});
            }
        }
    }

    const dfsph_step_stats& lastStats() const { return stats_; }
    dfsph_ctx* handle() const { return ctx_; }
    /* Any dfsph_set_param / dfsph_get_param key (e.g. "learned_warm_start", "boundary_forces"). */
    double get(const char* key) const {
        double v = 0;
        check(ctx_, dfsph_get_param(ctx_, key, &v));
        return v;
    }
    void set(const char* key, double v) { check(ctx_, dfsph_set_param(ctx_, key, v)); }

    DFSPHCData m_data;
    unsigned int m_iterations = 0, m_iterationsV = 0;

private:
    // Rotation matrix (row-major) of the unit quaternion q = (w, x, y, z).
    static void rotation(const std::array<double, 4>& q, double R[9]) {
        const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
        const double M[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy),
                             2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx),
                             2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)};
        for (int k = 0; k < 9; ++k) R[k] = M[k];
    }
    // update_dynamicObject_UnifiedParticleSet_cuda (DFSPH_core_cuda.cu:3407-3449) for one body: its
    // samples go to R(q) (x0 - rest) + position with the rigid velocity field v + w x (x - position),
    // on the device; the body keeps the pose.
    void apply_pose(DynamicBody& body, const std::array<double, 3>& position, const std::array<double, 4>& q,
                    const std::array<double, 3>& velocity, const std::array<double, 3>& om) {
        const double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!(len > 0)) throw Error(DFSPH_E_INVALID, "quaternion must be non-zero");
        const std::array<double, 4> u{{q[0] / len, q[1] / len, q[2] / len, q[3] / len}};
        double R[9];
        rotation(u, R);
        const std::array<double, 3>& c = body.rest_position;
        double arm[3], p[3], v[3];  // x = R x0 + p with p = position - R c; v passed about p
        for (int i = 0; i < 3; ++i) arm[i] = R[3 * i] * c[0] + R[3 * i + 1] * c[1] + R[3 * i + 2] * c[2];
        for (int i = 0; i < 3; ++i) p[i] = position[i] - arm[i];
        v[0] = velocity[0] - (om[1] * arm[2] - om[2] * arm[1]);
        v[1] = velocity[1] - (om[2] * arm[0] - om[0] * arm[2]);
        v[2] = velocity[2] - (om[0] * arm[1] - om[1] * arm[0]);
        check(ctx_, dfsph_move_boundary_rigid(ctx_, body.first, body.count, u.data(), p, v, om.data()));
        body.position = position;
        body.q = u;
    }
    // The fluid's force on every boundary particle during the last step and the particles' positions,
    // 3 FP64 values each in upload order.
    void boundary_force_and_position(std::vector<double>& f, std::vector<double>& x) const {
        double v = 0;
        check(ctx_, dfsph_get_param(ctx_, "num_boundary", &v));
        const size_t nb = (size_t)v;
        f.assign(3 * nb, 0.0);
        x.assign(3 * nb, 0.0);
        if (!nb) return;
        check(ctx_, dfsph_download(ctx_, DFSPH_F_BOUNDARY_FORCE, DFSPH_DTYPE_F64, f.data(), f.size(), DFSPH_ORDER_ID));
        check(ctx_, dfsph_download(ctx_, DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F64, x.data(), x.size(), DFSPH_ORDER_ID));
    }

    dfsph_ctx* ctx_ = nullptr;
    dfsph_step_stats stats_{};
    std::vector<float> fluid_, vel_, boundary_, psi_;
    double radius_ = 0.0;
    double window_center_[3] = {0.0, 0.0, 0.0};
};

/* SPH::TimeStepDFSPH (TimeStepDFSPH.h:20-48), the reference's CPU solver class, on the device time
 * step: the same public methods (step, reset, get/setEnableDivergenceSolver and the TimeStep
 * parameters of TimeStep.h:70-103), so code written against TimeStepDFSPH runs unchanged apart from
 * its construction, which takes the scene (arrays or a JSON scene file) instead of a FluidModel. */
class TimeStepDFSPH : public DFSPHCUDA {
public:
    using DFSPHCUDA::DFSPHCUDA;
};

/* The host functions of DFSPH_core_cuda.h:27-74 (same arguments; RealCuda -> double). */
inline int cuda_divergenceSolve(DFSPHCData& data, const unsigned int maxIter, const double maxError) {
    int32_t it = 0;
    check(data.handle(), dfsph_divergence_solve(data.handle(), maxIter, maxError, &it));
    return it;
}
inline int cuda_pressureSolve(DFSPHCData& data, const unsigned int maxIter, const double maxError) {
    int32_t it = 0;
    check(data.handle(), dfsph_pressure_solve(data.handle(), maxIter, maxError, &it));
    return it;
}
inline void cuda_neighborsSearch(DFSPHCData& data, bool need_sort = true) {
    check(data.handle(), dfsph_neighbors_search(data.handle(), need_sort ? 1 : 0));
}
inline void cuda_externalForces(DFSPHCData& data) { check(data.handle(), dfsph_external_forces(data.handle())); }
inline void cuda_update_vel(DFSPHCData& data) { check(data.handle(), dfsph_update_vel(data.handle())); }
inline void cuda_update_pos(DFSPHCData& data) { check(data.handle(), dfsph_update_pos(data.handle())); }
inline void cuda_CFL(DFSPHCData& data, const double minTimeStepSize, double m_cflFactor, double m_cflMaxTimeStepSize) {
    check(data.handle(), dfsph_cfl(data.handle(), minTimeStepSize, m_cflFactor, m_cflMaxTimeStepSize));
}

}  // namespace dfsph

#endif /* DFSPH_HPP */
