/*
 * dfsph_c.h — C ABI of the B200-native DFSPH time step.
 *
 * One context (dfsph_ctx) holds the whole device state of one fluid set and one boundary set, the
 * way SPH::DFSPHCData does in the reference (SPlisHSPlasH/DFSPH/DFSPH_c_arrays_structure.h:297-496),
 * and exposes the seven host functions that SPH::DFSPHCUDA::step() calls
 * (SPlisHSPlasH/DFSPH/DFSPH_CUDA.cpp:82-794, declared in SPlisHSPlasH/DFSPH/DFSPH_core_cuda.h:27-74),
 * plus a fused dfsph_step() that runs them in the reference order on the context's own stream.
 *
 * Conventions
 *  - Every entry point returns an int status: DFSPH_OK (0) or a negative DFSPH_E_* code. The
 *    reference has no error channel (gpuAssert -> exit(), DFSPH_macro_cuda.h:22-29); this ABI never
 *    exits and never traps. dfsph_last_error() gives a message for the last failing call.
 *  - Host arrays are plain C arrays owned by the caller; every copy is explicit. Positions and
 *    velocities are packed xyz triples (3 floats per particle).
 *  - Particle order: the solver re-sorts particles every step (cell-sorted order). Unlike the
 *    reference, each particle keeps a stable id (its index at upload); downloads are returned in
 *    id order unless DFSPH_ORDER_SORTED is asked for.
 *  - A context is used by one host thread at a time; several contexts may coexist.
 */
#ifndef DFSPH_C_H
#define DFSPH_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFSPH_ABI_VERSION 1

/* Opaque solver context (one fluid set + one boundary set on one device). */
typedef struct dfsph_ctx dfsph_ctx;

/* ---- status codes ---------------------------------------------------------------------------- */
#define DFSPH_OK 0
#define DFSPH_E_INVALID (-1)  /* bad argument (null pointer, size out of range, unknown key)      */
#define DFSPH_E_CUDA (-2)     /* a CUDA runtime call failed; see dfsph_last_error()               */
#define DFSPH_E_STATE (-3)    /* call out of order (e.g. step before any fluid was uploaded)      */
#define DFSPH_E_NOMEM (-4)    /* device allocation failed                                         */
#define DFSPH_E_DEVICE (-5)   /* the device status word reports a fault of the data (see below)   */

/* ---- device status word bits (dfsph_status) ---------------------------------------------------- */
#define DFSPH_ST_NEIGHBOR_OVERFLOW 0x1u  /* a particle had more neighbours than neighbor_capacity   */
#define DFSPH_ST_NONFINITE 0x2u          /* a fluid position was NaN/Inf                            */
#define DFSPH_ST_ESCAPED 0x4u            /* a fluid particle left the cell grid                     */
#define DFSPH_ST_PRESSURE_NOT_CONVERGED 0x8u    /* pressure solve stopped at max_iterations         */
#define DFSPH_ST_DIVERGENCE_NOT_CONVERGED 0x10u /* divergence solve stopped at max_iterations_v     */
#define DFSPH_ST_SORT_TIMEOUT 0x20u      /* a bounded wait in the radix sort gave up (no hang)      */
#define DFSPH_ST_BOUNDARY_OVERFLOW 0x40u /* a boundary particle had too many boundary neighbours    */
#define DFSPH_ST_FLUID_CAPACITY 0x80u    /* an open-boundary inflow was cut at fluid_capacity        */
#define DFSPH_ST_MMA_TIMEOUT 0x100u      /* a bounded wait for the warm-start network's tensor-core MMA
                                            gave up (no hang; that call's predictions are unspecified) */
#define DFSPH_ST_INDEX 0x200u            /* checked build only: a neighbour-list entry, a list count or a
                                            cell-table run was out of range; it was not read (the run is
                                            skipped, the particle's list emptied) */

/* ---- scene / solver parameters ---------------------------------------------------------------- */
/* Mirrors the "Configuration" keys of the reference JSON scene (Utilities/SceneLoader.cpp:39-160)
 * and the solver members of SPH::TimeStep (SPlisHSPlasH/TimeStep.h:26-34). */
typedef struct dfsph_scene {
    double particle_radius;       /* r; kernel support radius = 4 r (FluidModel::setParticleRadius) */
    double density0;              /* rest density rho0                                                */
    double viscosity;             /* XSPH coefficient (Viscosity_XSPH)                                */
    double gravitation[3];        /* m/s^2                                                            */
    double time_step;             /* initial dt (TimeManager::getTimeStepSize)                        */
    int32_t max_iterations;       /* pressure solve cap (m_maxIterations)                             */
    double max_error;             /* pressure tolerance, percent of rho0 (m_maxError)                 */
    int32_t max_iterations_v;     /* divergence solve cap (m_maxIterationsV)                          */
    double max_error_v;           /* divergence tolerance, percent (m_maxErrorV)                      */
    int32_t enable_divergence_solver; /* m_enableDivergenceSolver                                    */
    int32_t cfl_method;           /* 0: fixed dt; 1: CFL (TimeStep::updateTimeStepSizeCFL semantics) */
    double cfl_factor;            /* m_cflFactor                                                      */
    double cfl_max_time_step;     /* m_cflMaxTimeStepSize                                             */
    double cfl_min_time_step;     /* lower clamp of the CFL dt (reference passes 0.0001)              */
    uint32_t fluid_capacity;      /* max fluid particles held by the context                          */
    uint32_t boundary_capacity;   /* max boundary particles                                           */
    uint32_t neighbor_capacity;   /* stored neighbours per fluid particle (fluid + boundary)          */
    int32_t precision;            /* 32: FP32 kernels (product); 64: FP64 build of the same kernels   */
    int32_t device;               /* CUDA device ordinal                                              */
    int32_t use_graphs;           /* 1: solver loops run as CUDA-graph while-loops (no host sync)     */
    double grid_min[3];           /* optional domain box for the cell grid; used when grid_min <      */
    double grid_max[3];           /*   grid_max on every axis, otherwise the boundary bounding box    */
} dfsph_scene;

/* ---- scene files (reference JSON format) --------------------------------------------------------- */
/* A reference JSON scene read by the library (Utilities/SceneLoader.cpp:39-320 keys: Configuration,
 * FluidBlocks in dense mode, FluidModels and RigidBodies with .bgeo particle files, box walls sampled
 * as a single-layer lattice of spacing 2r; extension keys seed, jitter, precision, learnedWarmStart),
 * so that C and C++ callers need no other reader. Replaces SceneLoader::readScene + the scene part of
 * DemoBase::buildModel (Demos/Common/DemoBase.cpp:539-603). */
typedef struct dfsph_scene_file dfsph_scene_file;
/* Reads json_path; scene (nullable) receives the solver parameters with capacities equal to the
 * particle counts. *out must be released with dfsph_scene_file_free. Errors: DFSPH_E_INVALID with
 * the reason in dfsph_last_error(NULL). */
int dfsph_scene_load(const char* json_path, dfsph_scene* scene, dfsph_scene_file** out);
int dfsph_scene_file_counts(const dfsph_scene_file* f, uint32_t* n_fluid, uint32_t* n_boundary, int* has_velocity);
/* 3 floats per particle; vxyz (nullable) is zero where the scene gives no velocity. */
int dfsph_scene_file_fluid(const dfsph_scene_file* f, float* xyz, float* vxyz);
int dfsph_scene_file_boundary(const dfsph_scene_file* f, float* xyz);
void dfsph_scene_file_free(dfsph_scene_file* f);
/* dfsph_scene_load + dfsph_create + dfsph_set_boundary + dfsph_upload_fluid, and the scene's
 * learnedWarmStart block applied (DemoBase::buildModel + DFSPHCUDA(FluidModel*), DFSPH_CUDA.cpp:38). */
int dfsph_create_from_scene_file(const char* json_path, dfsph_ctx** out);

/* ---- per-step statistics ---------------------------------------------------------------------- */
typedef struct dfsph_step_stats {
    int32_t iterations;           /* pressure iterations (TimeStep::getIterationCount)               */
    int32_t iterations_v;         /* divergence iterations (TimeStep::getIterationCountV)            */
    double density_error;         /* final mean (rho_adv - rho0)^+ of the pressure solve [kg/m^3]    */
    double divergence_error;      /* final mean clamped divergence of the divergence solve           */
    double h;                     /* dt used by this step                                            */
    double h_future;              /* dt chosen for the next step                                     */
    uint32_t status;              /* DFSPH_ST_* bits raised during the step                          */
    uint32_t num_fluid;           /* fluid particles                                                 */
    double ms_total;              /* device time of the step (CUDA events), 0 if timing is off       */
    uint32_t warm_start;          /* learned warm start used: bit 0 divergence, bit 1 pressure       */
    uint32_t trained;             /* 1 if the warm-start network was trained at the end of the step  */
} dfsph_step_stats;

/* ---- fields for upload / download -------------------------------------------------------------- */
enum dfsph_field {
    DFSPH_F_POSITION = 0,   /* 3 per particle */
    DFSPH_F_VELOCITY = 1,   /* 3 */
    DFSPH_F_MASS = 2,       /* 1 */
    DFSPH_F_DENSITY = 3,    /* 1: rho from the density+alpha pass of the last step              */
    DFSPH_F_FACTOR = 4,     /* 1: alpha (DFSPH factor); after a pressure solve it holds alpha/h_f */
    DFSPH_F_DENSITY_ADV = 5,/* 1: last clamped residual (rho_adv - rho0)^+ or divergence         */
    DFSPH_F_KAPPA = 6,      /* 1: pressure warm-start accumulator                                 */
    DFSPH_F_KAPPA_V = 7,    /* 1: divergence warm-start accumulator                               */
    DFSPH_F_ACCELERATION = 8, /* 3: non-pressure acceleration (gravity + XSPH)                     */
    DFSPH_F_ID = 9,         /* 1 (uint32 in a float/double container is not allowed: use dtype 2) */
    DFSPH_F_BOUNDARY_PSI = 10,      /* 1 per boundary particle: Akinci psi (boundary "mass")      */
    DFSPH_F_BOUNDARY_POSITION = 11, /* 3 per boundary particle                                     */
    DFSPH_F_NEIGHBOR_COUNTS = 12,   /* 2 per fluid particle: fluid count, boundary count (dtype 2)  */
    DFSPH_F_BOUNDARY_VELOCITY = 13, /* 3 per boundary particle (zero for a static boundary)         */
    DFSPH_F_BOUNDARY_FORCE = 14,    /* 3 per boundary particle: force of the fluid during the last step
                                       (set_param "boundary_forces" 1; DFSPH_core_cuda.cu:467-477) */
    DFSPH_F_FEATURES = 15           /* 5 per fluid particle, f32 only, learned mode: the warm-start
                                       network's inputs from the last density + alpha pass,
                                       (rho - rho0)/rho0, rho_dot * alpha, neighbours / 64, and the
                                       previous step's needed kappa and kappa_v (no reference
                                       counterpart) */
};
#define DFSPH_DTYPE_F32 0
#define DFSPH_DTYPE_F64 1
#define DFSPH_DTYPE_U32 2
#define DFSPH_ORDER_ID 0
#define DFSPH_ORDER_SORTED 1

/* ---- lifetime ---------------------------------------------------------------------------------- */

/* Fills *scene with the reference defaults (SPH::TimeStep::TimeStep, TimeStep.cpp:23-44; CFL off as
 * in DFSPH_CUDA.cpp:299) and this library's capacities. */
int dfsph_scene_defaults(dfsph_scene* scene);

/* Replaces DFSPHCData::DFSPHCData(FluidModel*) (DFSPH_c_arrays_structure.cpp:852-944): allocates
 * every device buffer for the capacities in *scene and a private CUDA stream. */
int dfsph_create(const dfsph_scene* scene, dfsph_ctx** out);

/* Replaces DFSPHCData::~DFSPHCData (DFSPH_c_arrays_structure.cpp:946-973). Null is accepted. */
int dfsph_destroy(dfsph_ctx* ctx);

/* Message of the last failing call on ctx (or of the last failing dfsph_create when ctx is null). */
const char* dfsph_last_error(const dfsph_ctx* ctx);

/* ---- state upload (DFSPHCData::reset, DFSPH_c_arrays_structure.cpp:975-1048) -------------------- */

/* Static boundary particles (Akinci samples). Replaces boundaries_data->reset + initGridOffset +
 * the boundary neighbour structure (DFSPH_c_arrays_structure.cpp:1005-1015, 1050-1098). The grid
 * offset follows initGridOffset: offset = -(floor(min/H) - 5). When psi is null the Akinci psi
 * (FluidModel::computeBoundaryPsi, FluidModel.cpp:233-258) is computed on the device in FP64;
 * otherwise the given per-particle psi is used as boundary mass, as the reference uploads it. */
int dfsph_set_boundary(dfsph_ctx* ctx, const float* xyz, const float* psi, uint32_t n);

/* Moves the boundary: new positions (and velocities, nullable = zero) for the same n particles in
 * the order of dfsph_set_boundary. psi is kept. The boundary cell structure is rebuilt. */
int dfsph_move_boundary(dfsph_ctx* ctx, const float* xyz, const float* vxyz);

/* Rigid motion of one body of the boundary, on the device (update_dynamicObject_UnifiedParticleSet_cuda,
 * SPlisHSPlasH/DFSPH/DFSPH_core_cuda.cu:3426-3449): the particles of upload indices
 * [first, first + count) go to x = R(q) x0 + position with velocity angular_velocity x (x - position)
 * + velocity, where x0 is each particle's position as given to dfsph_set_boundary (its rest frame)
 * and q = (w, x, y, z) a rotation quaternion (normalised here). Null pointers mean the identity /
 * zero. psi is kept, the other particles keep their state, and the boundary cell structure is
 * rebuilt; no particle data crosses the host link. A pure translation of the whole boundary (first 0,
 * count all, no rotation) that stays within half a cell of the positions the boundary was last binned
 * at is not re-binned: the neighbour search then looks the boundary up at each fluid particle's
 * position minus the translation (one more cell layer near cell faces) and tests the pairs at the
 * current positions, so the neighbour sets are the same; only the order of the boundary entries in a
 * list may differ. */
int dfsph_move_boundary_rigid(dfsph_ctx* ctx, uint32_t first, uint32_t count, const double* q, const double* position,
                              const double* velocity, const double* angular_velocity);

/* Fluid particles (fluid_data->reset<FluidModel>). vxyz may be null (zero velocity). mass may be
 * null: every particle then gets the reference default mass 0.8 * rho0 * (2r)^3
 * (FluidModel::initMasses, FluidModel.cpp:94-107). Particles that the open boundary or the dynamic
 * window add later get the first uploaded particle's mass (the reference gives them fluid->mass[0],
 * OpenBoundariesSimple.cu:457); parameter "inflow_mass" reads or overrides it. Resets kappa,
 * kappa_v and the dt history (h = h_future = h_past = time_step, h_ratio = 1) and assigns ids
 * 0..n-1 in upload order. */
int dfsph_upload_fluid(dfsph_ctx* ctx, const float* xyz, const float* vxyz, const float* mass, uint32_t n);

/* Overwrites positions and velocities of the current n particles (given in id order) but keeps
 * their warm-start accumulators and the dt history: the host-in-the-loop way to edit a running
 * simulation without resetting it (the write-side counterpart of DFSPHCData::readDynamicData,
 * DFSPH_c_arrays_structure.cpp:1120; the reference has no fluid upload between steps). vxyz null sets the velocities
 * to zero. The copies are asynchronous: from page-locked host memory the buffers must stay unchanged
 * until the next call that waits (dfsph_step with stats, a read, dfsph_synchronize). The velocities
 * travel on a second stream and are applied inside the next step's binning, after its sort, or by
 * whichever other call on the context comes first, so every call sees the new state. */
int dfsph_update_fluid(dfsph_ctx* ctx, const float* xyz, const float* vxyz);

/* Copies a field to host memory. n_elems is the capacity of out in elements of dtype; the call
 * fails with DFSPH_E_INVALID if it is too small. order: DFSPH_ORDER_ID or DFSPH_ORDER_SORTED. */
int dfsph_download(dfsph_ctx* ctx, int field, int dtype, void* out, size_t n_elems, int order);

/* DFSPHCData::readDynamicData (DFSPH_c_arrays_structure.cpp:1120-1150): positions and velocities
 * (3 floats per particle each, particle-id order; either may be null) with a single wait. */
int dfsph_read_dynamic_data(dfsph_ctx* ctx, float* xyz, float* vxyz);

/* Neighbour lists of every fluid particle, in id space: counts[2*id] fluid, counts[2*id+1]
 * boundary; lists[id*cap + k] holds fluid neighbour ids first, then boundary indices (in the order
 * given to dfsph_set_boundary). cap is the row length of lists and must be >= neighbor_capacity. */
int dfsph_get_neighbors(dfsph_ctx* ctx, uint32_t* counts, uint32_t* lists, uint32_t cap);

/* ---- one time step ----------------------------------------------------------------------------- */

/* DFSPHCUDA::step() (DFSPH_CUDA.cpp:82-794) without rendering, dynamic bodies, open boundaries or
 * the dynamic window: neighbour search -> divergence solve -> XSPH + gravity -> dt update ->
 * velocity update -> pressure solve -> position update -> onSimulationStepEnd. The whole step runs on
 * the device, dt updates (CFL) included. With stats the call waits for the step and fills them; with
 * stats null it only enqueues the step and returns (no read-back): dfsph_synchronize waits, and
 * dfsph_status / dfsph_get_param ("iterations_sum", "iterations_v_sum", "h", ...) read the results
 * (non-converged solves raise their status bits on the device). */
int dfsph_step(dfsph_ctx* ctx, dfsph_step_stats* stats);

/* DFSPHCData::checkParticlesPositions (DFSPH_c_arrays_structure.cpp:1599, SPH_other_systems_cuda.cu:
 * 1242-1328): counts the fluid particles with a coordinate outside the domain box (the boundary's
 * bounding box, or grid_min / grid_max when given); mode 2 also removes them, keeping the order of
 * the others and renumbering their ids densely; mode 0 only counts (the reference's mode 1 exits).
 * A step called with stats ends with mode 2, as DFSPHCUDA::step does (DFSPH_CUDA.cpp:456), unless
 * the parameter "remove_escaped" is 0; an asynchronous step (stats null) leaves them (a particle that
 * leaves the cell grid is flagged DFSPH_ST_ESCAPED and keeps moving without neighbours). */
int dfsph_check_particles_positions(dfsph_ctx* ctx, int mode, uint32_t* count);

/* The seven host functions of DFSPH_core_cuda.h:27-74, for callers that drive the step themselves. */
int dfsph_neighbors_search(dfsph_ctx* ctx, int sort);                     /* cuda_neighborsSearch */
int dfsph_divergence_solve(dfsph_ctx* ctx, uint32_t max_iter, double max_error, int32_t* iters);
int dfsph_external_forces(dfsph_ctx* ctx);                                /* cuda_externalForces  */
int dfsph_update_time_step(dfsph_ctx* ctx, double h_future);              /* updateTimeStep       */
int dfsph_cfl(dfsph_ctx* ctx, double min_dt, double cfl_factor, double max_dt); /* cuda_CFL       */
int dfsph_update_vel(dfsph_ctx* ctx);                                     /* cuda_update_vel      */
int dfsph_pressure_solve(dfsph_ctx* ctx, uint32_t max_iter, double max_error, int32_t* iters);
int dfsph_update_pos(dfsph_ctx* ctx);                                     /* cuda_update_pos      */
int dfsph_on_step_end(dfsph_ctx* ctx);                                    /* onSimulationStepEnd  */

/* ---- parameters -------------------------------------------------------------------------------- */
/* Keys: "viscosity", "density0", "max_error", "max_error_v", "max_iterations", "max_iterations_v",
 * "enable_divergence_solver", "cfl_method", "cfl_factor", "cfl_max_time_step", "cfl_min_time_step",
 * "time_step" (sets the dt the next dt update uses), "gravitation_x|y|z", "use_graphs",
 * "h", "h_future", "h_past", "inv_h" (dt history of DFSPHCData), "timing" (1: record CUDA events),
 * "iterations_sum" (setting it clears the counters; reading it gives the pressure iterations of all
 * solves since, "iterations_v_sum" the divergence iterations),
 * "remove_escaped" (1, default: a step with stats removes particles outside the domain box),
 * "escaped_removed" (read-only: particles removed that way so far),
 * "boundary_forces" (1: accumulate the fluid's force on every boundary particle in each Jacobi pass,
 * -m_i k_i psi_b grad W_ib summed over both solves of a step, as the reference does for dynamic
 * bodies; cleared by each neighbour search; summed with 64-bit fixed-point atomics in units of
 * 2^-32 N, so the sums do not depend on the order), "inflow_mass" (the mass of particles the open
 * boundary and the dynamic window add; default: the first uploaded particle's),
 * "sort_withhold_tile" (failure-detection tests: the fluid sort's tile with this id never publishes
 * its look-back flags, so the bounded waits of the tiles after it run out, about a second, and the
 * step reports DFSPH_ST_SORT_TIMEOUT with an unspecified particle order; -1 turns it off),
 * "boundary_shift_active" (read-only: 1 while a translation of the whole boundary by
 * dfsph_move_boundary_rigid, less than half a cell since the boundary was last binned, is applied by
 * querying the binned cells at the shifted position instead of re-binning).
 *
 * Learned warm start (no reference counterpart; off by default, dfsph_step only):
 * "learned_warm_start" (1: on), "warm_start_probe" (1: per solve, keep the learned candidate only if
 * its initial residual sum |rho_adv - rho0| (divergence: |rho_dot|) is not above the plain
 * candidate's, default 1), "warm_start_damping" (in (0, 1]: the learned warm start raises the
 * reference's to at most this fraction of the predicted needed pressure, default 0.95),
 * "train_interval" (steps between online trainings, default 50; 0: never), "train_start" (first
 * training step, default 1), "train_iters" (Adam steps per training, default 20), "train_batch"
 * (particles per training batch, 1..65536, default 4096), "learning_rate" (default 1e-3), "mlp_seed"
 * (re-initialises the network).
 * Cost gate of the learned warm start: "learned_gate" (1: the learned passes run only while the plain
 * warm start needs at least "gate_margin" iterations per step, pressure + divergence, above the
 * solves' minimum counts, default 1; setting the key restarts the schedule with a probe), measured on
 * plain steps: a probe of 2 settling + "gate_window" (default 10) steps after every "gate_period"
 * (default 200) learned steps, or every "gate_recheck" (default 50) steps while gated off. One host
 * read of the iteration counters per decision.
 * Read-only: "mlp_ready", "mlp_trainings", "mlp_adam_steps", "mlp_loss" (last batch loss),
 * "learned_solves_v|p" (solves that had a learned candidate), "learned_kept_v|p" (solves that kept it),
 * "gate_learned_steps", "gate_plain_steps" (steps the gate ran with and without the learned passes),
 * "gate_last_excess" (iterations per step above the minimum at the last decision; -1 before any). */
int dfsph_set_param(dfsph_ctx* ctx, const char* key, double value);
int dfsph_get_param(dfsph_ctx* ctx, const char* key, double* value);

/* Device status word (DFSPH_ST_* bits accumulated since the last clear); clear != 0 resets it. */
int dfsph_status(dfsph_ctx* ctx, uint32_t* status, int clear);

/* Number of fluid particles currently held. */
int dfsph_num_fluid(dfsph_ctx* ctx, uint32_t* n);

/* Waits for all work queued on the context's stream. */
int dfsph_synchronize(dfsph_ctx* ctx);

/* Number of kernel launches the library issued on this context since creation (for accounting). */
int dfsph_launch_count(dfsph_ctx* ctx, uint64_t* launches);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own work or events
 * with the solver's. */
int dfsph_get_stream(dfsph_ctx* ctx, void** stream);

/* Kernels that dfsph_time_kernel can time (no reference counterpart: measurement support). */
enum dfsph_kernel_id {
    DFSPH_K_NEIGHBOR_BUILD = 0,
    DFSPH_K_DENSITY_ALPHA = 1,
    DFSPH_K_DIVERGENCE_JACOBI = 2,
    DFSPH_K_DIVERGENCE_RESIDUAL = 3,
    DFSPH_K_VISCOSITY = 4,
    DFSPH_K_PRESSURE_WARM_JACOBI = 5,
    DFSPH_K_PRESSURE_RESIDUAL = 6,
    DFSPH_K_PRESSURE_JACOBI = 7,
    DFSPH_K_UPDATE_POS = 8,
    DFSPH_K_SORT_REORDER = 9,
    DFSPH_K_COUNT = 10
};

/* Launches one kernel of the step `reps` times on the current state with CUDA events around each
 * launch and returns the mean device time per launch in ms. The launches modify the state (the
 * Jacobi kernels move velocities), so call it only when the simulation will not continue, e.g. at
 * the end of a benchmark. */
int dfsph_time_kernel(dfsph_ctx* ctx, int kernel, int reps, double* ms_per_launch);

/* ---- snapshots in the reference's text format ----------------------------------------------------
 * DFSPHCUDA::handleSimulationSave / handleSimulationLoad (SPlisHSPlasH/DFSPH/DFSPH_CUDA.cpp:1885-1979)
 * with UnifiedParticleSet::write_to_file / load_from_file (DFSPH_c_arrays_structure.cpp:424-600):
 * dir/fluid_file.txt and dir/boundaries_file.txt hold a header line "N has_factor_computation
 * velocity_impacted_by_fluid_solver is_dynamic_object" ("N 1 1 0" for the fluid, "N 0 0 0" for a
 * static boundary) and one line "mass x y z vx vy vz" per particle (the boundary's mass column is its
 * psi); dir/general_data.txt holds the time step. Values are written with 9 significant digits (the
 * reference writes 6; both read either). Loading a boundary recomputes psi, as the reference does
 * (computeRigidBodiesParticlesMass); loading the fluid sets h = h_future = h_past to the stored step
 * and clears the warm starts (the format does not hold them). what: DFSPH_SNAP_FLUID |
 * DFSPH_SNAP_BOUNDARY. dir must exist. */
#define DFSPH_SNAP_FLUID 1
#define DFSPH_SNAP_BOUNDARY 2
int dfsph_save_snapshot(dfsph_ctx* ctx, const char* dir, int what);
int dfsph_load_snapshot(dfsph_ctx* ctx, const char* dir, int what, int load_velocities);

/* Partio particle files (Houdini BGEO version 5, gzip-compressed), the format of the reference's
 * PartioReaderWriter (Utilities/PartioReaderWriter.cpp:8-66, 189-231).
 * dfsph_export_bgeo replaces partioExport (Demos/StaticBoundaryDemo/main.cpp:485-496): the fluid's
 * positions, velocities, pscale = particle radius and id = particle id, in particle-id order.
 * dfsph_bgeo_write / dfsph_bgeo_read need no context (and no GPU): write count particles (vxyz may be
 * null: no velocity attribute; radius 0: no pscale attribute); read positions and velocities
 * (zeros when the file has none, untransformed) of a compressed or plain file. With xyz null,
 * dfsph_bgeo_read only stores the particle count; otherwise capacity (particles) must hold it
 * (DFSPH_E_INVALID if not). has_velocity (may be null) is set to 1 when the file has velocities.
 * Errors of the context-free calls are reported by dfsph_last_error(NULL). */
int dfsph_export_bgeo(dfsph_ctx* ctx, const char* path);
int dfsph_bgeo_write(const char* path, const float* xyz, const float* vxyz, uint64_t count, float radius);
int dfsph_bgeo_read(const char* path, float* xyz, float* vxyz, uint64_t capacity, uint64_t* count,
                    int* has_velocity);

/* ---- simple open boundary (OpenBoundariesSimpleInterface, OpenBoundariesSimple.{h,cu}) ----------
 * Surfaces are the reference's BufferFluidSurface shapes (BufferFluidSurface.cu:421-900) with its
 * type numbers. "Inside" follows isinside(): plane
 * (x - origin) . normal >= 0; cuboid |x - center| < half_lengths component-wise; cylinder (axis y)
 * |dy| <= half_lengths[1] and horizontal distance < radius; sphere distance < radius; star (axis y,
 * `points` linear-sided points, the first along `direction`) |dy| <= half_lengths[1] and inside the
 * star outline between radius_internal and radius; mesh (3): the closed triangle mesh registered
 * with dfsph_set_surface_mesh under the id `points`, translated by `center` (MeshPerso, :49-410):
 * outside the box of its vertices and the origin (translated) a point is outside, inside that box it
 * is inside when the ray from it along normalise(2.575, 6.19763, 5.986) crosses an odd number of
 * triangles ahead of it (Moller-Trumbore with the reference's 1e-7 parallel cut-off, :14-47).
 * reversed != 0 swaps inside and outside. The normal used by the inflow is center - x (cylinder,
 * sphere, star; negated when reversed, normalised) and zero for planes, cuboids and meshes. All
 * surface arithmetic is FP32 (1/a of the ray test in FP64, as the reference divides 1.0 by it). */
#define DFSPH_SURFACE_PLANE 0
#define DFSPH_SURFACE_CUBOID 1
#define DFSPH_SURFACE_CYLINDER 2
#define DFSPH_SURFACE_MESH 3
#define DFSPH_SURFACE_SPHERE 4
#define DFSPH_SURFACE_STAR 5
#define DFSPH_MAX_SURFACE_MESHES 8
typedef struct dfsph_surface {
    int32_t type;            /* DFSPH_SURFACE_*                                                   */
    int32_t reversed;        /* != 0: inside and outside swapped                                  */
    float origin[3];         /* plane: a point of the plane                                       */
    float normal[3];         /* plane: the side of the normal is inside                           */
    float center[3];         /* cuboid, cylinder, sphere, star                                    */
    float half_lengths[3];   /* cuboid; cylinder and star use [1] (half height along y)           */
    float radius;            /* cylinder, sphere; star: outer radius                              */
    float radius_internal;   /* star: inner radius                                                */
    uint32_t points;         /* star: number of points (>= 1)                                     */
    float direction[3];      /* star: direction of the first point (horizontal)                   */
} dfsph_surface;

/* Registers (or replaces) the triangle mesh `mesh_id` (< DFSPH_MAX_SURFACE_MESHES) for surfaces of
 * type DFSPH_SURFACE_MESH: n_vertices positions (xyz[3 n]) and n_triangles vertex-index triples. The
 * mesh should be closed. Surfaces already given to dfsph_open_boundary_init see the new mesh from
 * their next use. Errors: DFSPH_E_INVALID for an index out of range or no triangles. */
int dfsph_set_surface_mesh(dfsph_ctx* ctx, uint32_t mesh_id, const float* vertices, uint32_t n_vertices,
                           const uint32_t* triangles, uint32_t n_triangles);
/* Wavefront OBJ reader for such meshes (the reference loads them with OBJ_Loader, MeshPerso::
 * loadFromFile): `v x y z` vertices and `f` faces (indices 1-based or negative, `i/t/n` forms),
 * polygons split into fans from their first vertex; other records are skipped. With null arrays only
 * the counts are returned; otherwise the capacities must hold them. No GPU is needed. */
int dfsph_read_obj(const char* path, float* vertices, uint32_t vertex_capacity, uint32_t* n_vertices,
                   uint32_t* triangles, uint32_t triangle_capacity, uint32_t* n_triangles);

/* OpenBoundariesSimpleInterface::init (OpenBoundariesSimple.cu:105-350): boundary is the simulation
 * boundary, interior a slightly smaller copy (the reference uses 3 r less), fluid_surface the
 * fluid's free surface (inside = below it). Of the n_samples inflow sample positions (a fluid at
 * rest sampled in the same boundary, xyz[3 n]) the context keeps those outside `interior`, inside
 * `fluid_surface` and inside the cell grid; n_kept (may be null) receives their count. Calling it
 * again replaces the previous set. */
int dfsph_open_boundary_init(dfsph_ctx* ctx, const dfsph_surface* boundary, const dfsph_surface* interior,
                             const dfsph_surface* fluid_surface, const float* sample_xyz, uint32_t n_samples,
                             uint32_t* n_kept);
/* OpenBoundariesSimpleInterface::applyOpenBoundary (OpenBoundariesSimple.cu:495-620), called between
 * steps. Inflow (use_inflow): every sample with no fluid particle of the 27 cells around it closer
 * than allowed_distance becomes a fluid particle, with the kernel-and-mass-weighted velocity of its
 * fluid neighbours (boundary neighbours add weight but no velocity), unless its density estimate
 * exceeds allowed_density or that velocity points out of the boundary (v . normal < 0); new
 * particles get the default fluid mass, kappa = kappa_v = 0 and the next ids, in sample order.
 * allowed_distance and allowed_density must be > 0 when use_inflow != 0 (the reference exits
 * otherwise). Outflow (use_outflow): particles outside `interior` and outside `fluid_surface` are
 * removed; the remaining ids are renumbered densely in their previous order. Inflow beyond
 * fluid_capacity is cut and raises DFSPH_ST_FLUID_CAPACITY. added / removed (may be null) receive
 * the counts. Synchronises the context's stream. */
int dfsph_open_boundary_apply(dfsph_ctx* ctx, double allowed_distance, double allowed_density, int use_inflow,
                              int use_outflow, uint32_t* added, uint32_t* removed);
/* The kept inflow samples (xyz[3 capacity]; xyz null: only the count), in sample order. */
int dfsph_open_boundary_samples(dfsph_ctx* ctx, float* xyz, uint32_t capacity, uint32_t* count);
/* Moves the three surfaces and the samples by delta[3] (the reference applies the dynamic window's
 * displacement this way, OpenBoundariesSimple.cu:527-553). */
int dfsph_open_boundary_shift(dfsph_ctx* ctx, const float* delta);

/* ---- dynamic window (own design after DynamicWindowInterface, SPlisHSPlasH/DFSPH/DynamicWindow.h:
 * 31-200, driven like DFSPHCUDA::applyDynamicWindow, DFSPH_CUDA.cpp:3988-4139) ---------------------
 * The simulated region is the box [lo, hi] walled by the boundary particles [wall_first, wall_first +
 * wall_count) (upload order, given to dfsph_set_boundary in the window's initial place); rest_xyz are
 * n_rest positions of a fluid at rest tiling the window (the reference's rest-fluid file). The cell
 * grid does not move: the scene's grid box must cover the window's whole path.
 * dfsph_dynamic_window_shift moves the window by displacement[3], between steps: the walls translate
 * rigidly on the device; fluid particles outside the moved box are removed (ids renumbered densely in
 * their previous order); the rest samples move with the window and those in the region it newly
 * covers become fluid particles by the open boundary's inflow rule (no fluid particle closer than
 * allowed_distance, density estimate at most allowed_density, velocity the kernel-weighted velocity of
 * the fluid around it, kappa = kappa_v = 0, the next ids in sample order); the domain box of the
 * end-of-step removal moves with the window. The reference's tagging by density levels and its
 * damped stabilisation iterations are not reproduced: the pressure solve of the next step takes the
 * seam. added / removed (nullable) receive the counts; synchronises the context's stream. */
int dfsph_dynamic_window_init(dfsph_ctx* ctx, const double* lo, const double* hi, uint32_t wall_first,
                              uint32_t wall_count, const float* rest_xyz, uint32_t n_rest);
int dfsph_dynamic_window_shift(dfsph_ctx* ctx, const double* displacement, double allowed_distance,
                               double allowed_density, uint32_t* added, uint32_t* removed);
/* DFSPHCData::computeFluidLevel (find_fluid_height_cuda, SPH_other_systems_cuda.cu:149-260): per
 * column of cells (x, z), the cells are read from the top down until at least three particles have
 * been seen and the column's height is the middle one of the three highest (a lone splash does not
 * count); *level is the highest column's (-1: no column holds three particles). Computed on the host
 * from the device's binning; synchronises the context's stream. */
int dfsph_fluid_level(dfsph_ctx* ctx, double* level);
/* DFSPHCData::handleFLuidLevelControl (control_fluid_height_cuda, :414-547), between steps; nothing
 * when the level is within 5 cm of target (> 0). Above it, the particles above target are removed
 * (stable, ids renumbered densely). Below it, a lattice of new particles (spacing 2r, layers 0.8 * 2r
 * apart, floor((target - level) / 2r) + 1 layers) spanning the domain box taken from the first and
 * last ten boundary particles in the reference's boundary order (shrunk by 2r) is placed, outside the
 * box's central third in x or z, each point lifted to its column's highest fluid particle + 2.5 r;
 * appended at rest with the inflow mass, in lattice order (ids n, n + 1, ...); past fluid_capacity
 * the rest is dropped and DFSPH_ST_FLUID_CAPACITY set. *removed / *added (nullable) receive the
 * counts. */
int dfsph_fluid_level_control(dfsph_ctx* ctx, double target, uint32_t* removed, uint32_t* added);

/* DynamicWindowInterface::stabilizeFluid, method 0 (DynamicWindow.cu:3160-3700), between steps after
 * dfsph_dynamic_window_shift: `iterations` steps of the fixed time step `time_step` (the reference's
 * default: 5 steps of 3 ms) with kappa and kappa_v cleared before and after; each runs the neighbour
 * search, the divergence solve, viscosity and gravity, the pressure solve with the velocity update,
 * multiplies the velocities of the particles the last shift added by `damping` (in [0, 1]; 1: none)
 * and updates the positions. With tagged_only the other particles keep their positions and velocities
 * (they act as neighbours only); particles count as added by the last shift until the fluid is
 * compacted or uploaded again, and particles appended after the shift (open-boundary inflow, a fluid
 * level raise) count with them. The dt history is restored afterwards. Synchronises the context's
 * stream. */
int dfsph_dynamic_window_stabilize(dfsph_ctx* ctx, uint32_t iterations, double time_step, double damping,
                                   int tagged_only);
/* Total displacement of the window since dfsph_dynamic_window_init. */
int dfsph_dynamic_window_displacement(dfsph_ctx* ctx, double* displacement);

/* Force and torque of the fluid on boundary bodies during the last step (needs "boundary_forces" 1):
 * the per-particle forces the reference hands to its rigid-body solver (readDynamicObjectsData,
 * DFSPH_c_arrays_structure.cpp:1177-1193), summed on the device. Body b is the range
 * [first[b], first[b] + count[b]) of the boundary particles in the order given to dfsph_set_boundary;
 * force_torque[6 b + 0..2] receives the force, [6 b + 3..5] the torque about centers[3 b..3 b + 2]
 * (FP64, deterministic). Bodies move with dfsph_move_boundary. */
int dfsph_body_wrench(dfsph_ctx* ctx, uint32_t n_bodies, const uint32_t* first, const uint32_t* count,
                      const double* centers, double* force_torque);

/* Binary checkpoint of the complete solver state (no reference counterpart; the text snapshot above
 * drops the warm starts and the particle order): particles in their current internal order with
 * kappa and kappa_v, the boundary with psi, the dt history, the grid, the scene parameters and, when
 * the learned warm start is on, its totals, network weights, Adam state, scales and cost-gate
 * schedule. Loading into a context created with at least the same capacities, the same
 * neighbor_capacity and precision resumes bit-identically. Files of format versions 1 to 3 (no
 * gate schedule, no network-usefulness state, no inflow mass) still load. */
int dfsph_checkpoint_save(dfsph_ctx* ctx, const char* path);
int dfsph_checkpoint_load(dfsph_ctx* ctx, const char* path);

/* ---- learned warm-start network (no reference counterpart) -------------------------------------
 * A per-particle MLP, inputs x[8] = [(rho - rho0)/rho0, rho_dot * alpha, neighbours / 64,
 * kappa_total_prev, kappa_v_total_prev, 0, 0, 0] (each multiplied by in_scale[i]), two hidden layers
 * of 64 ReLU units, outputs y[2] = corrections to the previous step's total kappa and kappa_v in units
 * of out_scale. Parameters, FP32, row-major [out][in]: W1[64][8] b1[64] W2[64][64] b2[64] W3[2][64]
 * b3[2]. Inference runs on BF16 tensor cores with FP32 accumulation; training in FP32. Batches of
 * host data hold at most 65536 samples. The loss is the mean over samples of the summed squared
 * output errors. */
#define DFSPH_MLP_INPUTS 8
#define DFSPH_MLP_OUTPUTS 2
#define DFSPH_MLP_PARAMS 4866
int dfsph_mlp_get_params(dfsph_ctx* ctx, float* params, size_t n);
/* Loads weights (resets the Adam moments) and marks the network ready for the warm start. */
int dfsph_mlp_set_params(dfsph_ctx* ctx, const float* params, size_t n);
int dfsph_mlp_get_scales(dfsph_ctx* ctx, float* in_scale, float* out_scale);
/* Sets the input / output scales (otherwise set from the first online training batch). */
int dfsph_mlp_set_scales(dfsph_ctx* ctx, const float* in_scale, const float* out_scale);
/* y[2 i + o] = network output o of sample i (tensor-core inference path). */
int dfsph_mlp_forward(dfsph_ctx* ctx, const float* x, uint32_t n, float* y);
/* Gradient of the loss of targets t[2 i + o] w.r.t. the parameters (FP32), without an update;
 * grad (DFSPH_MLP_PARAMS floats) and loss may be null. */
int dfsph_mlp_gradient(dfsph_ctx* ctx, const float* x, const float* t, uint32_t n, float* grad, double* loss);
/* iters Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) on one batch; loss = loss before the last step. */
int dfsph_mlp_train(dfsph_ctx* ctx, const float* x, const float* t, uint32_t n, int32_t iters, double learning_rate,
                    double* loss);
/* Re-initialises the weights from a seed (He-uniform hidden layers, zero output layer and biases),
 * clears the scales and the Adam state; the warm start is plain until the next training. */
int dfsph_mlp_reset(dfsph_ctx* ctx, uint32_t seed);

/* Allocation-free stable sort of cell keys (no counterpart in the reference: it exists for callers
 * that may not allocate device memory, e.g. a host framework that owns every allocation or a plugin
 * handed fixed device buffers). All pointers are device pointers owned by the caller and must not
 * overlap (DFSPH_E_INVALID otherwise): keys_in[n] is read, keys_out[n] receives the input keys,
 * unchanged, in ascending order of their low key_bits bits (1..32; the bits above are carried but
 * do not order), and perm_out[n] the original index of each (equal low bits keep their input order).
 * The call performs no cudaMalloc/cudaFree: its scratch is a fixed device array built into the
 * library (about 2.6 MB on every GPU that loads it, held until the process exits) and n is limited
 * to 262,144 keys (larger n returns DFSPH_E_INVALID with a message in dfsph_last_error(NULL)). Each
 * call looks up that array's device address on the current device. Every call reuses the same
 * array: calls that overlap on the GPU (other streams, other threads) race and must be serialised by
 * the caller. The call runs on `stream` (a cudaStream_t, NULL = legacy default stream) and returns
 * after the sort has finished; it ends with a host wait, so it cannot be made while the stream is
 * being captured into a graph (DFSPH_E_STATE). */
int dfsph_sort_cell_keys_noalloc(const uint32_t* keys_in, uint32_t* keys_out, uint32_t* perm_out, uint32_t n,
                                 int key_bits, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DFSPH_C_H */
