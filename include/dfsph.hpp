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

#include <cstdint>
#include <stdexcept>
#include <string>
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

    dfsph_ctx* ctx_ = nullptr;
    dfsph_step_stats stats_{};
    std::vector<float> fluid_, vel_, boundary_, psi_;
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
