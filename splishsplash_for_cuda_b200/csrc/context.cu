// context.cu — the solver context behind the C ABI (include/dfsph_c.h).
//
// Solver<Real> owns every device buffer of one fluid set and one static/moving boundary set (what
// SPH::DFSPHCData + UnifiedParticleSet + NeighborsSearchDataSet own in the reference,
// DFSPH_c_arrays_structure.h:36-496) and drives the time step of DFSPHCUDA::step()
// (DFSPH_CUDA.cpp:82-794) on one private stream. Nothing here is a global or a function-local
// static, so several contexts may coexist (the reference keeps statics in cuda_neighborsSearch
// and cuda_CFL, DFSPH_core_cuda.cu:2653-2663, :3333-3348, and is one instance per process).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "bgeo.h"
#include "bodies.cuh"
#include "dfsph_state.cuh"
#include "io.cuh"
#include "mlp.cuh"
#include "open_boundary.cuh"
#include "sort.cuh"

struct dfsph_ctx;

namespace dfsph {

static thread_local std::string g_create_error;

void set_global_error(const std::string& msg) { g_create_error = msg; }

#define DF_CUDA(call)                                                                             \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
            return (e_ == cudaErrorMemoryAllocation) ? DFSPH_E_NOMEM : DFSPH_E_CUDA;               \
        }                                                                                         \
    } while (0)

#define DF_CHECK(cond, code, msg) \
    do {                          \
        if (!(cond)) {            \
            err = (msg);          \
            return (code);        \
        }                         \
    } while (0)

#define DF_TRY(expr)           \
    do {                       \
        int r_ = (expr);       \
        if (r_ != DFSPH_OK) {  \
            return r_;         \
        }                      \
    } while (0)

template <class Real> class Solver {
public:
    explicit Solver(std::string& e) : err(e) {}
    ~Solver() { release(); }

    std::string& err;
    dfsph_scene sc{};
    cudaStream_t stream = nullptr;
    // Velocities given to update_fluid travel on a copy stream and are applied inside the next
    // step's neighbour search, after the neighbour build (the key pass, the sort, the reorder and
    // the build do not read them; the reorder moves stale values that the flush overwrites in the
    // new order): their upload overlaps those passes. Any other call applies them first
    // (flush_pending).
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_vel_ready = nullptr, ev_vel_free = nullptr;
    bool pending_vel = false;
    // Mass of the particles the open boundary and the dynamic window add: the first uploaded
    // particle's (the reference gives new particles fluid->mass[0], OpenBoundariesSimple.cu:457).
    float inflow_mass = 0.0f;
    float new_particle_mass() const {
        if (inflow_mass > 0.0f) return inflow_mass;
        const double d = 2.0 * sc.particle_radius;  // nothing uploaded yet: FluidModel's default
        return (float)(0.8 * d * d * d * sc.density0);
    }
    uint32_t Nc = 0, Bc = 0, cap = 0, stride = 0;
    uint32_t n = 0, nb = 0;
    int cur = 0;
    bool grid_ready = false;
    bool boundary_moving = false;
    int key_passes = 4;
    uint32_t sort_withheld_tile = kNoWithheldTile;  // failure-detection test hook (see sort.cuh)
    int off[3] = {0, 0, 0}, dim[3] = {0, 0, 0};

    DevState<Real> hs{};
    DevState<Real>* ds = nullptr;

    Vec4<Real>* pos[2] = {nullptr, nullptr};
    Vec4<Real>* vel[2] = {nullptr, nullptr};
    Real* kappa[2] = {nullptr, nullptr};
    Real* kappaV[2] = {nullptr, nullptr};
    uint32_t* id[2] = {nullptr, nullptr};
    Real *density = nullptr, *factor = nullptr, *densityAdv = nullptr, *kcoef = nullptr;
    Vec4<Real>* acc = nullptr;
    uint32_t *counts = nullptr, *nbr = nullptr;
    SortBuffers sb;
    uint2* ftab = nullptr;
    uint2* btab = nullptr;
    size_t cells = 0;
    Vec4<Real>* bpos[2] = {nullptr, nullptr};
    Vec4<Real>* bvel[2] = {nullptr, nullptr};
    float* brest = nullptr;  // boundary positions as given to set_boundary (upload order), for rigid moves
    unsigned long long* bforce_fx = nullptr;  // boundary forces, fixed-point sums (converted into bforce)
    Real* bforce = nullptr;  // boundary forces (4 per particle, sorted order), allocated when enabled
    bool boundary_forces = false;
    // Rigid translation of the whole boundary without re-binning: bin_rigid when the binned positions
    // are the rest positions translated by bin_p; bshift_d the translation since (used while every
    // component stays below one cell); bshifted when it is not zero.
    bool bin_rigid = false, bshifted = false;
    double bin_p[3] = {0.0, 0.0, 0.0}, bshift_d[3] = {0.0, 0.0, 0.0};
    uint32_t* bid = nullptr;
    double* partials = nullptr;
    LoopCtl* ctl = nullptr;
    uint32_t* status = nullptr;  // [0] main word, [1] scratch
    float* cfl_partials = nullptr;
    float* stage = nullptr;      // upload staging: 7 floats per particle of max(Nc, Bc)
    void* dl = nullptr;          // download staging: 3 doubles per particle of max(Nc, Bc)
    LoopCtl* h_ctl = nullptr;    // pinned mirror of ctl[0..2]
    uint32_t* h_status = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timing = false;
    uint64_t launches = 0;

    // dt history (DFSPHCData h, h_future, h_past, h_ratio_to_past(2), invH, invH_future). The device
    // block dtd is authoritative (the dt updates of a step run on the device); these are host mirrors,
    // refreshed by every read-back (collect, pull_dt) and pushed by push_dt.
    double h = 0, h_future = 0, h_past = 0, inv_h = 0, inv_h_future = 0, h_ratio = 1, h_ratio2 = 1;
    double time_step = 0;
    double* dtd = nullptr;
    double* h_dt = nullptr;  // pinned mirror of dtd
    bool dt_stale = false;   // the device changed dtd since the last read-back
    bool use_graphs = true;
    cudaGraphExec_t g_loop[2] = {nullptr, nullptr};  // [0] divergence, [1] pressure
    uint32_t g_loop_n[2] = {0, 0};
    int g_loop_u[2] = {0, 0};  // iterations laid out before the while node
    bool g_loop_keep = false;  // the loop graphs store unclamped residuals (learned warm start)
    bool vel_updated = false;  // dfsph_update_vel ran since the last external-force pass

    int last_iters = 0, last_iters_v = 0;
    double last_err = 0, last_err_v = 0;

    // Learned warm start (mlp.cuh). The network buffers are allocated on first use, the
    // per-particle buffers when the mode is first enabled; the plain path touches neither.
    static constexpr uint32_t kMaxTrainBatch = 1u << 16;
    bool learned = false, mlp_ready = false, scales_set = false, probe = true;
    // Ablation of the learned warm start: the needed-coefficient base with the network's correction
    // fixed at zero (no inference, no training).
    bool base_only = false;
    bool last_lp = false;  // the previous dfsph_step ran the learned passes
    // The network's correction is applied only while it predicts better than no correction: each
    // training round first evaluates the current network on the round's fresh batch (data it has not
    // trained on) and keeps its correction on for the next rounds if that loss is below
    // useful_ratio x the loss of predicting zero (the batch's mean squared target).
    bool net_useful = false;
    double useful_ratio = 0.8, zero_loss = 0.0, heldout_loss = 0.0;
    double* h_loss = nullptr;  // pinned copy of the first training step's loss
    // Test hook of the checked build: the next neighbour search writes index n + corrupt_neighbor - 1
    // into particle 0's list (0: off).
    uint32_t corrupt_neighbor = 0;
    Real* kappaT[2] = {nullptr, nullptr};
    Real* kappaVT[2] = {nullptr, nullptr};
    Real *kappaW = nullptr, *kappaVW = nullptr, *kappaP = nullptr, *kappaVP = nullptr;
    Vec4<Real>* velP = nullptr;
    Real *resid = nullptr, *residV = nullptr;
    Real *dadvP = nullptr, *kcP = nullptr, *rawP = nullptr;  // plain candidate of the dual init pass
    float *features = nullptr, *pred = nullptr, *tx = nullptr, *tt = nullptr;
    MlpDev mlp{};
    MlpScales h_scales{};
    uint32_t mlp_seed = 1234567u;
    int train_interval = 50, train_start = 1, train_iters = 20;
    uint32_t train_batch = 4096;
    double lr = 1e-3;
    double damping = 0.95;  // learned warm start: at most damping x the predicted needed coefficient
    int adam_t = 0;
    uint64_t lsteps = 0, trainings = 0, kept_v = 0, kept_p = 0, solves_v = 0, solves_p = 0;
    uint32_t forced_warm = 0;             // learned candidates used without a probe this step
    // Cost gate of the learned warm start. The learned passes (features, inference, both candidates,
    // training) cost about one to two gather passes per step, so they pay only while the plain warm
    // start leaves at least gate_margin iterations (pressure + divergence per step) above the solves'
    // minimum counts. The gate measures the plain solver on plain steps: a probe window of
    // kGateSettle + gate_window plain steps (the first kGateSettle unmeasured: the plain warm start
    // recovers from a learned step) after every gate_period learned steps, or every gate_recheck
    // steps while it keeps the learned passes off.
    static constexpr int kGateSettle = 2;
    bool gate = false;
    int gate_period = 200, gate_window = 10, gate_recheck = 50;
    double gate_margin = 1.0;
    enum GatePhase { kGateSettling = 0, kGateProbe, kGateLearned, kGatePlain };
    int gate_phase = kGateLearned, gate_left = 0, gate_len = 0;
    uint32_t gate_it0 = 0, gate_itv0 = 0;
    uint64_t gate_learned_steps = 0, gate_plain_steps = 0;
    double gate_last_excess = -1.0;
    bool step_trained = false;

    // simple open boundary (OpenBoundariesSimple): surfaces, kept inflow samples and their scratch
    bool ob_ready = false;
    dfsph_surface ob_boundary{}, ob_interior{}, ob_surface{};
    float4* ob_samples = nullptr;  // kept samples (x, y, z, 0)
    float4* ob_vel = nullptr;      // per-sample candidate velocity (also the upload staging of init)
    uint32_t* ob_flag = nullptr;
    uint32_t* ob_rank = nullptr;
    uint32_t* ob_scan = nullptr;   // scan scratch for max(sample capacity, fluid capacity) inputs
    uint32_t* ob_total = nullptr;  // device scan totals
    uint32_t* h_ob = nullptr;      // pinned copy of a scan total
    uint32_t ob_ns = 0, ob_cap = 0;
    uint32_t ob_scan_inputs = 0;   // inputs ob_scan was sized for

    // dynamic window: the window box and its total displacement, the walls that move with it, and
    // the rest-fluid samples (in the window's current place) with their scratch
    bool dw_ready = false;
    // ids >= dw_first_new were added by the last window shift or appended since (the stabilisation's
    // tagged particles; none once the fluid is compacted or uploaded again); dw_spos / dw_svel keep
    // the others' state
    uint32_t dw_first_new = 0;
    Vec4<Real>* dw_spos = nullptr;
    Vec4<Real>* dw_svel = nullptr;
    double dw_lo[3] = {0, 0, 0}, dw_hi[3] = {0, 0, 0}, dw_disp[3] = {0, 0, 0};
    uint32_t dw_wall_first = 0, dw_wall_count = 0, dw_ns = 0, dw_cap = 0;
    float4* dw_samples = nullptr;  // rest samples, moved with the window
    float4* dw_sel = nullptr;      // the samples of the newly covered region
    float4* dw_vel = nullptr;      // their candidate velocities
    uint32_t* dw_flag = nullptr;
    uint32_t* dw_rank = nullptr;

    // end-of-step removal of particles outside the domain box (checkParticlesPositions(2))
    float bb_lo[3] = {0, 0, 0}, bb_hi[3] = {0, 0, 0};
    bool remove_escaped = true;
    uint64_t escaped_removed = 0;

    // ------------------------------------------------------------------------------------------
    template <class T> int dalloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        DF_CUDA(cudaMalloc((void**)p, count * sizeof(T)));
        return DFSPH_OK;
    }

    int init(const dfsph_scene& s) {
        sc = s;
        DF_CHECK(s.fluid_capacity > 0, DFSPH_E_INVALID, "fluid_capacity must be > 0");
        DF_CHECK(s.neighbor_capacity > 0 && s.neighbor_capacity < 65536, DFSPH_E_INVALID,
                 "neighbor_capacity must be in [1, 65535]");
        DF_CHECK(s.particle_radius > 0, DFSPH_E_INVALID, "particle_radius must be > 0");
        DF_CHECK(s.time_step > 0, DFSPH_E_INVALID, "time_step must be > 0");
        DF_CUDA(cudaSetDevice(s.device));
        DF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        Nc = s.fluid_capacity;
        Bc = std::max<uint32_t>(s.boundary_capacity, 1);
        cap = s.neighbor_capacity;
        stride = (Nc + 31u) & ~31u;
        for (int b = 0; b < 2; ++b) {
            DF_TRY(dalloc(&pos[b], Nc));
            DF_TRY(dalloc(&vel[b], Nc));
            DF_TRY(dalloc(&kappa[b], Nc));
            DF_TRY(dalloc(&kappaV[b], Nc));
            DF_TRY(dalloc(&id[b], Nc));
            DF_TRY(dalloc(&bpos[b], Bc));
            DF_TRY(dalloc(&bvel[b], Bc));
        }
        DF_TRY(dalloc(&density, Nc));
        DF_TRY(dalloc(&factor, Nc));
        DF_TRY(dalloc(&densityAdv, Nc));
        DF_TRY(dalloc(&kcoef, Nc));
        DF_TRY(dalloc(&acc, Nc));
        DF_TRY(dalloc(&counts, Nc));
        DF_TRY(dalloc(&nbr, (size_t)cap * stride));
        DF_TRY(dalloc(&bid, Bc));
        DF_TRY(dalloc(&brest, (size_t)Bc * 3));
        const uint32_t nmax = std::max(Nc, Bc);
        DF_TRY(dalloc(&sb.keys_a, nmax));
        DF_TRY(dalloc(&sb.keys_b, nmax));
        DF_TRY(dalloc(&sb.vals_a, nmax));
        DF_TRY(dalloc(&sb.vals_b, nmax));
        DF_TRY(dalloc(&sb.workspace, radix_sort_workspace_words(nmax, 4)));
        DF_TRY(dalloc(&partials, 4 * ((size_t)grid_for(nmax) + 1)));  // two pairs of sums per block at most
        DF_TRY(dalloc(&cfl_partials, grid_for(nmax) + 1));
        DF_TRY(dalloc(&ctl, 4));
        DF_TRY(dalloc(&status, 4));
        DF_TRY(dalloc(&stage, (size_t)nmax * 7));
        DF_CUDA(cudaMalloc(&dl, (size_t)nmax * 3 * sizeof(double)));
        DF_CUDA(cudaMalloc((void**)&ds, sizeof(DevState<Real>)));
        DF_CUDA(cudaMallocHost((void**)&h_ctl, 3 * sizeof(LoopCtl)));
        DF_CUDA(cudaMallocHost((void**)&h_status, 4 * sizeof(uint32_t)));
        DF_TRY(dalloc(&dtd, kDtSlots));
        DF_CUDA(cudaMallocHost((void**)&h_dt, kDtSlots * sizeof(double)));
        DF_CUDA(cudaMemsetAsync(ctl, 0, 4 * sizeof(LoopCtl), stream));
        DF_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(uint32_t), stream));
        DF_CUDA(cudaMemsetAsync(counts, 0, Nc * sizeof(uint32_t), stream));
        DF_CUDA(cudaEventCreate(&ev0));
        DF_CUDA(cudaEventCreate(&ev1));
        DF_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
        DF_CUDA(cudaEventCreateWithFlags(&ev_vel_ready, cudaEventDisableTiming));
        DF_CUDA(cudaEventCreateWithFlags(&ev_vel_free, cudaEventDisableTiming));
        time_step = s.time_step;
        use_graphs = s.use_graphs != 0;
        DF_TRY(sync_state());
        reset_dt();
        return DFSPH_OK;
    }

    void release() {
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        if (stream) cudaStreamSynchronize(stream);
        for (int k = 0; k < 2; ++k)
            if (g_loop[k]) cudaGraphExecDestroy(g_loop[k]);
        auto f = [](void* p) {
            if (p) cudaFree(p);
        };
        for (int b = 0; b < 2; ++b) {
            f(pos[b]); f(vel[b]); f(kappa[b]); f(kappaV[b]); f(id[b]); f(bpos[b]); f(bvel[b]);
        }
        f(density); f(factor); f(densityAdv); f(kcoef); f(acc); f(counts); f(nbr); f(bid); f(bforce); f(bforce_fx);
        f(sb.keys_a); f(sb.keys_b); f(sb.vals_a); f(sb.vals_b); f(sb.workspace);
        f(partials); f(cfl_partials); f(ctl); f(status); f(stage); f(dl); f(ds); f(ftab); f(btab);
        for (int b = 0; b < 2; ++b) {
            f(kappaT[b]); f(kappaVT[b]);
        }
        f(kappaW); f(kappaVW); f(kappaP); f(kappaVP); f(velP); f(resid); f(residV); f(features); f(pred); f(tx);
        f(dadvP); f(kcP); f(rawP);
        f(tt);
        f(mlp.params); f(mlp.adam_m); f(mlp.adam_v); f(mlp.grad); f(mlp.partials);
        f(mlp.w1_bf16); f(mlp.w2_bf16); f(mlp.w3_bf16); f(mlp.scales); f(mlp.loss);
        f(ob_samples); f(ob_vel); f(ob_flag); f(ob_rank); f(ob_scan); f(ob_total); f(wrench_buf);
        f(brest); f(dw_samples); f(dw_sel); f(dw_vel); f(dw_flag); f(dw_rank); f(dw_spos); f(dw_svel);
        for (MeshSlot& m : meshes) {
            f(m.tri);
            m = MeshSlot{};
        }
        if (h_ob) cudaFreeHost(h_ob);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (h_status) cudaFreeHost(h_status);
        if (h_dt) cudaFreeHost(h_dt);
        if (h_loss) cudaFreeHost(h_loss);
        f(dtd);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (ev_vel_ready) cudaEventDestroy(ev_vel_ready);
        if (ev_vel_free) cudaEventDestroy(ev_vel_free);
        stream = nullptr;
    }

    void reset_dt() {
        h = h_future = h_past = time_step;
        inv_h = inv_h_future = 1.0 / time_step;
        h_ratio = h_ratio2 = 1.0;
        push_dt();
    }

    // Host mirrors -> device dt block (and the Real copies the kernels read).
    void push_dt() {
        DtArgs a{};
        a.v[kDtH] = h; a.v[kDtHFuture] = h_future; a.v[kDtHPast] = h_past; a.v[kDtInvH] = inv_h;
        a.v[kDtInvHFuture] = inv_h_future; a.v[kDtRatio] = h_ratio; a.v[kDtRatio2] = h_ratio2;
        a.v[kDtFixed] = time_step; a.v[kDtRatioUsedV] = h_ratio; a.v[kDtRatio2UsedP] = h_ratio2;
        launch_dt<Real>(ds, 0, a, stream);
        launches += 1;
        dt_stale = false;
    }
    void mirror_dt() {
        h = h_dt[kDtH]; h_future = h_dt[kDtHFuture]; h_past = h_dt[kDtHPast]; inv_h = h_dt[kDtInvH];
        inv_h_future = h_dt[kDtInvHFuture]; h_ratio = h_dt[kDtRatio]; h_ratio2 = h_dt[kDtRatio2];
        dt_stale = false;
    }
    int pull_dt() {
        if (!dt_stale) return DFSPH_OK;
        DF_CUDA(cudaMemcpyAsync(h_dt, dtd, kDtSlots * sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        mirror_dt();
        return DFSPH_OK;
    }

    // Parameters of the kernels derived from the scene and the dt history.
    StepParams<Real> params() const {
        StepParams<Real> p{};
        const float Hf = (float)(4.0 * sc.particle_radius);
        const double H = (double)Hf;
        p.kern.H = (Real)Hf;
        p.kern.invH = (Real)(1.0 / H);
        p.kern.k = (Real)(8.0 / (M_PI * H * H * H));
        p.kern.l = (Real)(48.0 / (M_PI * H * H * H));
        p.kern.W0 = p.kern.k;
        p.kern.ih2_d = 1.0 / (H * H);
        p.kern.k_d = 8.0 / (M_PI * H * H * H);
        p.H2 = (Real)(Hf * Hf);
        p.density0 = (Real)sc.density0;
        p.viscosity = (Real)sc.viscosity;
        p.gx = (Real)sc.gravitation[0];
        p.gy = (Real)sc.gravitation[1];
        p.gz = (Real)sc.gravitation[2];
        p.h = (Real)h;
        p.h_future = (Real)h_future;
        p.inv_h = (Real)inv_h;
        p.inv_h_future = (Real)inv_h_future;
        p.h_ratio_to_past = (Real)h_ratio;
        p.h_ratio_to_past2 = (Real)h_ratio2;
        p.off_x = off[0]; p.off_y = off[1]; p.off_z = off[2];
        p.dim_x = dim[0]; p.dim_y = dim[1]; p.dim_z = dim[2];
        p.n_fluid = n;
        p.n_boundary = nb;
        p.nbr_stride = stride;
        p.nbr_cap = cap;
        p.boundary_moving = boundary_moving ? 1 : 0;
        p.bshift = bshifted ? 1 : 0;
        p.bsx = (Real)bshift_d[0];
        p.bsy = (Real)bshift_d[1];
        p.bsz = (Real)bshift_d[2];
        return p;
    }

    int sync_state() {
        hs.p = params();
        hs.pos = pos[cur];
        hs.vel = vel[cur];
        hs.kappa = kappa[cur];
        hs.kappaV = kappaV[cur];
        hs.id = id[cur];
        hs.density = density;
        hs.factor = factor;
        hs.densityAdv = densityAdv;
        hs.kcoef = kcoef;
        hs.acc = acc;
        hs.counts = counts;
        hs.nbr = nbr;
        hs.bpos = bpos[0];
        hs.bvel = bvel[0];
        hs.partials = partials;
        hs.ctl = ctl;
        hs.status = status;
        hs.cfl_partials = cfl_partials;
        hs.dtd = dtd;
        hs.bforce = boundary_forces ? bforce_fx : nullptr;
        hs.features = features;
        hs.pred = pred;
        hs.kappaT = kappaT[cur];
        hs.kappaVT = kappaVT[cur];
        hs.dadvP = dadvP;
        hs.kcP = kcP;
        hs.rawP = rawP;
        hs.kappaW = kappaW;
        hs.kappaVW = kappaVW;
        hs.kappaP = kappaP;
        hs.kappaVP = kappaVP;
        hs.velP = velP;
        hs.resid = resid;
        hs.residV = residV;
        hs.out_scale = mlp.scales ? reinterpret_cast<const float*>(reinterpret_cast<const char*>(mlp.scales) +
                                                                  offsetof(MlpScales, out_scale))
                                  : nullptr;
        launch_set_state<Real>(ds, hs, stream);
        launches += 1;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // Cell grid from a bounding box, following DFSPHCData::initGridOffset
    // (DFSPH_c_arrays_structure.cpp:1050-1098): offset = -(floor(min / H) - 5).
    int set_grid(const float mn[3], const float mx[3]) {
        const float H = (float)(4.0 * sc.particle_radius);
        int o[3], dm[3];
        for (int a = 0; a < 3; ++a) {  // validated first: a rejected box leaves the grid unchanged
            DF_CHECK(std::isfinite(mn[a]) && std::isfinite(mx[a]) && mx[a] >= mn[a], DFSPH_E_INVALID,
                     "invalid grid bounding box");
            const int fmin = (int)std::floor(mn[a] / H);
            const int fmax = (int)std::floor(mx[a] / H);
            o[a] = -(fmin - 5);
            dm[a] = fmax + o[a] + 6;
            DF_CHECK(dm[a] <= 1024, DFSPH_E_INVALID,
                     "domain too large: more than 1024 cells of size 4r along one axis");
        }
        for (int a = 0; a < 3; ++a) {
            off[a] = o[a];
            dim[a] = dm[a];
            bb_lo[a] = mn[a];  // initGridOffset keeps the box as boundingBoxMin / Max
            bb_hi[a] = mx[a];
        }
        return alloc_grid();
    }

    // Cell tables for the current off / dim (also used when a checkpoint restores them).
    int alloc_grid() {
        // Digit passes of the key sort: the highest bit a valid Morton key can set (axis a's top bit
        // lands on key bit 3 (bits_a - 1) + a), plus one so that the escaped-particle key (all ones)
        // still sorts after every valid key in the bits sorted.
        int key_bits = 1;
        for (int a = 0; a < 3; ++a) {
            int bits = 1;
            while ((1 << bits) < dim[a]) ++bits;
            key_bits = std::max(key_bits, 3 * (bits - 1) + a + 1);
        }
        key_passes = std::min(4, (key_bits + 1 + 7) / 8);
        const size_t c = (size_t)dim[0] * dim[1] * dim[2];
        if (c != cells) {
            if (ftab) cudaFree(ftab);
            if (btab) cudaFree(btab);
            ftab = btab = nullptr;
            DF_TRY(dalloc(&ftab, c));
            DF_TRY(dalloc(&btab, c));
            cells = c;
        }
        DF_CUDA(cudaMemsetAsync(btab, 0, cells * sizeof(uint2), stream));
        grid_ready = true;
        return DFSPH_OK;
    }

    static void bbox(const float* xyz, uint32_t count, float mn[3], float mx[3]) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = INFINITY;
            mx[a] = -INFINITY;
        }
        for (uint32_t i = 0; i < count; ++i)
            for (int a = 0; a < 3; ++a) {
                const float v = xyz[3 * (size_t)i + a];
                if (std::isfinite(v)) {
                    mn[a] = std::min(mn[a], v);
                    mx[a] = std::max(mx[a], v);
                }
            }
    }

    bool scene_grid(float mn[3], float mx[3]) const {
        for (int a = 0; a < 3; ++a)
            if (!(sc.grid_min[a] < sc.grid_max[a])) return false;
        for (int a = 0; a < 3; ++a) {
            mn[a] = (float)sc.grid_min[a];
            mx[a] = (float)sc.grid_max[a];
        }
        return true;
    }

    // Sorts the boundary set in place by cell key and rebuilds its cell table.
    int sort_boundary(bool compute_psi) {
        const StepParams<Real> p = params();
        launch_cell_keys<Real>(bpos[1], nb, p, sb.keys_a, status + 1, stream);
        uint32_t *skeys, *perm;
        radix_sort_pairs(sb, nb, key_passes, true, stream, status, &launches, &skeys, &perm);
        launch_reorder_boundary<Real>(perm, nb, bpos[1], bvel[1], bpos[0], bvel[0], bid, stream);
        DF_CUDA(cudaMemsetAsync(btab, 0, cells * sizeof(uint2), stream));
        launch_cell_bounds(skeys, nb, dim[0], dim[1], dim[2], btab, stream);
        launches += 3;
        if (compute_psi) {
            launch_boundary_psi<Real>(bpos[0], bpos[1], nb, p, btab, status, stream);
            DF_CUDA(cudaMemcpyAsync(bpos[0], bpos[1], (size_t)nb * sizeof(Vec4<Real>), cudaMemcpyDeviceToDevice,
                                    stream));
            launches += 1;
        }
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int set_boundary(const float* xyz, const float* psi, uint32_t count) {
        DF_CHECK(count <= Bc, DFSPH_E_INVALID, "boundary count exceeds boundary_capacity");
        DF_CHECK(count == 0 || xyz, DFSPH_E_INVALID, "null boundary positions");
        float mn[3], mx[3];
        if (!scene_grid(mn, mx)) {
            DF_CHECK(count > 0, DFSPH_E_INVALID, "empty boundary and no grid box in the scene");
            bbox(xyz, count, mn, mx);
        }
        DF_TRY(set_grid(mn, mx));
        nb = count;
        boundary_moving = false;
        if (count) {
            DF_CUDA(cudaMemcpyAsync(stage, xyz, (size_t)count * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
            DF_CUDA(cudaMemcpyAsync(brest, stage, (size_t)count * 3 * sizeof(float), cudaMemcpyDeviceToDevice, stream));
            if (psi)
                DF_CUDA(cudaMemcpyAsync(stage + (size_t)count * 3, psi, (size_t)count * sizeof(float),
                                        cudaMemcpyHostToDevice, stream));
            launch_unpack_boundary<Real>(stage, psi ? stage + (size_t)count * 3 : nullptr, count, bpos[1], bvel[1],
                                         stream);
            launches += 1;
            DF_TRY(sort_boundary(psi == nullptr));
        }
        bin_rigid = true;  // binned at the rest positions
        bshifted = false;
        for (int a = 0; a < 3; ++a) bin_p[a] = bshift_d[a] = 0.0;
        invalidate_graphs();
        DF_TRY(sync_state());
        DF_CUDA(cudaStreamSynchronize(stream));
        return DFSPH_OK;
    }

    int move_boundary(const float* xyz, const float* vxyz) {
        DF_CHECK(nb > 0, DFSPH_E_STATE, "no boundary set");
        DF_CHECK(xyz, DFSPH_E_INVALID, "null boundary positions");
        DF_CUDA(cudaMemcpyAsync(stage, xyz, (size_t)nb * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (vxyz)
            DF_CUDA(cudaMemcpyAsync(stage + (size_t)nb * 3, vxyz, (size_t)nb * 3 * sizeof(float),
                                    cudaMemcpyHostToDevice, stream));
        // positions in original order -> staging set [1] in original order, then re-sort
        launch_move_boundary<Real>(stage, vxyz ? stage + (size_t)nb * 3 : nullptr, nb, bid, bpos[0], bvel[0], stream);
        // bring the moved set back to original order in [1]: slot i holds original bid[i]
        launch_pack_field<Real, Real>((const Real*)bpos[0], 4, 4, bid, nb, (Real*)bpos[1], stream);
        launch_pack_field<Real, Real>((const Real*)bvel[0], 4, 4, bid, nb, (Real*)bvel[1], stream);
        launches += 3;
        boundary_moving = true;
        DF_TRY(sort_boundary(false));
        bin_rigid = bshifted = false;
        return sync_state();
    }

    // update_dynamicObject_UnifiedParticleSet_cuda (DFSPH_core_cuda.cu:3426-3449) for the boundary
    // particles of upload indices [first, first + count): x = R(q) x0 + position with x0 the
    // positions given to set_boundary, v = angular_velocity x (x - position) + velocity. Every
    // argument stays on the device path (no host copy of the particles); the cell structure is rebuilt.
    int move_boundary_rigid(uint32_t first, uint32_t count, const double* q, const double* position,
                            const double* velocity, const double* angular_velocity) {
        DF_CHECK(nb > 0, DFSPH_E_STATE, "no boundary set");
        DF_CHECK(first <= nb && count <= nb - first, DFSPH_E_INVALID, "boundary range out of bounds");
        RigidMotion m{};
        double w = 1, x = 0, y = 0, z = 0;
        if (q) {
            const double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            DF_CHECK(len > 0 && std::isfinite(len), DFSPH_E_INVALID, "quaternion must be finite and non-zero");
            w = q[0] / len; x = q[1] / len; y = q[2] / len; z = q[3] / len;
        }
        const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                             2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                             2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)};
        for (int k = 0; k < 9; ++k) m.R[k] = R[k];
        for (int k = 0; k < 3; ++k) {
            m.p[k] = position ? position[k] : 0.0;
            m.v[k] = velocity ? velocity[k] : 0.0;
            m.w[k] = angular_velocity ? angular_velocity[k] : 0.0;
            DF_CHECK(std::isfinite(m.p[k]) && std::isfinite(m.v[k]) && std::isfinite(m.w[k]), DFSPH_E_INVALID,
                     "rigid motion must be finite");
        }
        m.first = first;
        m.count = count;
        if (!count) return DFSPH_OK;
        if (!boundary_moving) DF_CUDA(cudaMemsetAsync(bvel[0], 0, (size_t)nb * sizeof(Vec4<Real>), stream));
        launch_rigid_boundary<Real>(brest, nb, bid, m, bpos[0], bvel[0], stream);
        // A translation of the whole boundary keeps the binning while it stays within a cell of the
        // binned positions: the neighbour search queries the binned cells at x_i minus the shift.
        bool pure = first == 0 && count == nb;
        for (int k = 0; k < 9; ++k) pure = pure && m.R[k] == (k % 4 == 0 ? 1.0 : 0.0);
        const double Hd = 4.0 * sc.particle_radius;
        double d[3];
        bool near = pure && bin_rigid;
        for (int a = 0; a < 3; ++a) {
            d[a] = m.p[a] - bin_p[a];
            near = near && std::fabs(d[a]) < 0.5 * Hd;
        }
        boundary_moving = true;
        if (near) {
            for (int a = 0; a < 3; ++a) bshift_d[a] = d[a];
            bshifted = d[0] != 0.0 || d[1] != 0.0 || d[2] != 0.0;
            launches += 1;
            return sync_state();
        }
        launch_pack_field<Real, Real>((const Real*)bpos[0], 4, 4, bid, nb, (Real*)bpos[1], stream);
        launch_pack_field<Real, Real>((const Real*)bvel[0], 4, 4, bid, nb, (Real*)bvel[1], stream);
        launches += 3;
        DF_TRY(sort_boundary(false));
        bin_rigid = pure;
        bshifted = false;
        for (int a = 0; a < 3; ++a) {
            bin_p[a] = pure ? m.p[a] : 0.0;
            bshift_d[a] = 0.0;
        }
        return sync_state();
    }

    // Re-bins the boundary at its current positions when a rigid translation has been left pending
    // (before anything other than the neighbour search reads the boundary's cell table or order).
    int bin_boundary_now() {
        if (!bshifted) return DFSPH_OK;
        launch_pack_field<Real, Real>((const Real*)bpos[0], 4, 4, bid, nb, (Real*)bpos[1], stream);
        launch_pack_field<Real, Real>((const Real*)bvel[0], 4, 4, bid, nb, (Real*)bvel[1], stream);
        launches += 2;
        DF_TRY(sort_boundary(false));
        for (int a = 0; a < 3; ++a) {
            bin_p[a] += bshift_d[a];
            bshift_d[a] = 0.0;
        }
        bshifted = false;
        return sync_state();
    }

    int upload_fluid(const float* xyz, const float* vxyz, const float* mass, uint32_t count) {
        DF_CHECK(count <= Nc, DFSPH_E_INVALID, "fluid count exceeds fluid_capacity");
        DF_CHECK(count == 0 || xyz, DFSPH_E_INVALID, "null fluid positions");
        if (!grid_ready) {
            float mn[3], mx[3];
            if (!scene_grid(mn, mx)) {
                DF_CHECK(count > 0, DFSPH_E_INVALID, "no boundary, no fluid and no grid box");
                bbox(xyz, count, mn, mx);
                const float H = (float)(4.0 * sc.particle_radius);
                for (int a = 0; a < 3; ++a) {
                    mn[a] -= 20.0f * H;
                    mx[a] += 20.0f * H;
                }
            }
            DF_TRY(set_grid(mn, mx));
        }
        if (count != n) invalidate_graphs();
        n = count;
        cur = 0;
        dw_first_new = count;
        last_lp = false;  // the uploaded state carries no learned warm start
        {
            const double d = 2.0 * sc.particle_radius;
            inflow_mass = (count && mass) ? mass[0] : (float)(0.8 * d * d * d * sc.density0);
        }
        if (count) {
            float* sx = stage;
            float* sv = stage + (size_t)count * 3;
            float* sm = stage + (size_t)count * 6;
            DF_CUDA(cudaMemcpyAsync(sx, xyz, (size_t)count * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
            if (vxyz)
                DF_CUDA(cudaMemcpyAsync(sv, vxyz, (size_t)count * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
            if (mass)
                DF_CUDA(cudaMemcpyAsync(sm, mass, (size_t)count * sizeof(float), cudaMemcpyHostToDevice, stream));
            // FluidModel::initMasses (FluidModel.cpp:94-107): 0.8 * rho0 * (2r)^3
            const double d = 2.0 * sc.particle_radius;
            const float default_mass = (float)(0.8 * d * d * d * sc.density0);
            launch_unpack_fluid<Real>(sx, vxyz ? sv : nullptr, mass ? sm : nullptr, default_mass, count, pos[0], vel[0],
                                      kappa[0], kappaV[0], id[0], stream);
            launches += 1;
            DF_CUDA(cudaMemsetAsync(counts, 0, (size_t)count * sizeof(uint32_t), stream));
        }
        if (kappaT[0]) DF_TRY(clear_totals());
        lsteps = 0;
        reset_dt();
        DF_TRY(sync_state());
        DF_CUDA(cudaStreamSynchronize(stream));
        return DFSPH_OK;
    }

    int update_fluid(const float* xyz, const float* vxyz) {
        DF_CHECK(xyz, DFSPH_E_INVALID, "null fluid positions");
        if (!n) return DFSPH_OK;
        float* sx = stage;
        float* sv = stage + (size_t)n * 3;
        DF_CUDA(cudaMemcpyAsync(sx, xyz, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (!vxyz) {  // positions, velocities zero
            launch_update_fluid<Real>(sx, nullptr, n, id[cur], pos[cur], vel[cur], stream, true);
            launches += 1;
            return DFSPH_OK;
        }
        launch_update_fluid<Real>(sx, nullptr, n, id[cur], pos[cur], vel[cur], stream, false);
        // the staging area is free once the work queued so far has run
        DF_CUDA(cudaEventRecord(ev_vel_free, stream));
        DF_CUDA(cudaStreamWaitEvent(copy_stream, ev_vel_free, 0));
        DF_CUDA(cudaMemcpyAsync(sv, vxyz, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, copy_stream));
        DF_CUDA(cudaEventRecord(ev_vel_ready, copy_stream));
        pending_vel = true;
        launches += 1;
        return DFSPH_OK;
    }

    // Applies velocities uploaded by update_fluid (in id order) to the current particle order.
    int flush_pending() {
        if (!pending_vel) return DFSPH_OK;
        pending_vel = false;
        DF_CUDA(cudaStreamWaitEvent(stream, ev_vel_ready, 0));
        launch_update_fluid<Real>(nullptr, stage + (size_t)n * 3, n, id[cur], pos[cur], vel[cur], stream, true);
        launches += 1;
        return DFSPH_OK;
    }
    // Every entry point but the step applies pending velocities first.
    int enter() { return flush_pending(); }
    int synchronize_all() {
        DF_TRY(flush_pending());
        DF_CUDA(cudaStreamSynchronize(copy_stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        return DFSPH_OK;
    }

    // ------------------------------------------------------------------------------------------
    // cuda_neighborsSearch: keys -> stable radix sort -> reorder (double buffer) -> cell table ->
    // neighbour lists. The particle order is always refreshed (the reference's sort flag is kept in
    // the signature; unsorted searching is not offered).
    int neighbors_search() {
        DF_CHECK(grid_ready, DFSPH_E_STATE, "no grid: set a boundary or upload fluid first");
        // forces on the boundary are per step (the reference clears them when it moves the dynamic
        // bodies at the start of a step, DFSPH_core_cuda.cu:3413)
        if (boundary_forces && nb)
            DF_CUDA(cudaMemsetAsync(bforce_fx, 0, (size_t)nb * 3 * sizeof(unsigned long long), stream));
        if (!n) return DFSPH_OK;
        DF_TRY(bin_fluid(true));
        launch_build_neighbors<Real>(ds, n, ftab, btab, stream, bshifted);
        launches += 1;
        DF_TRY(flush_pending());  // velocities uploaded during the binning and the build
        if (corrupt_neighbor) {  // checked builds only (the key is rejected otherwise); one search
            launch_corrupt_first_neighbor(nbr, counts, n + corrupt_neighbor - 1u, stream);
            corrupt_neighbor = 0;
            launches += 1;
        }
        if (kCheckedBuild) {
            launch_validate_neighbors(counts, nbr, n, nb, stride, cap, status, stream);
            launches += 1;
        }
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // Cell keys -> stable radix sort -> reorder (double buffer) -> cell table of the fluid. With
    // defer_velocities the caller applies velocities pending from update_fluid afterwards.
    int bin_fluid(bool defer_velocities = false) {
        if (!n) {
            DF_CUDA(cudaMemsetAsync(ftab, 0, cells * sizeof(uint2), stream));
            return sync_state();
        }
        const StepParams<Real> p = params();
        // the key pass also clears the fluid cell table and the sort's workspace (no memsets between
        // the kernels of the step)
        launch_cell_keys<Real>(pos[cur], n, p, sb.keys_a, status, stream, (uint32_t*)ftab, 2 * cells, sb.workspace,
                               radix_sort_workspace_words(n, key_passes));
        uint32_t *skeys, *perm;
        radix_sort_pairs(sb, n, key_passes, true, stream, status, &launches, &skeys, &perm, sort_withheld_tile, true);
        if (!defer_velocities) DF_TRY(flush_pending());  // velocities uploaded during the key pass and the sort
        const int nx = 1 - cur;
        launch_reorder_fluid<Real>(perm, n, pos[cur], vel[cur], kappa[cur], kappaV[cur], id[cur], pos[nx], vel[nx],
                                   kappa[nx], kappaV[nx], id[nx], stream);
        if (learned) {
            launch_reorder_pair<Real>(perm, n, kappaT[cur], kappaVT[cur], kappaT[nx], kappaVT[nx], stream);
            launches += 1;
        }
        cur = nx;
        launch_cell_bounds(skeys, n, dim[0], dim[1], dim[2], ftab, stream);
        DF_TRY(sync_state());
        launches += 3;
        return DFSPH_OK;
    }

    // ------------------------------------------------------------------------------------------
    // Simple open boundary (OpenBoundariesSimple.cu).
    // Triangle meshes of DFSPH_SURFACE_MESH surfaces, by id.
    struct MeshSlot {
        float4* tri = nullptr;  // 3 per triangle
        uint32_t nt = 0, cap = 0;
        float bmin[3] = {0.f, 0.f, 0.f}, bmax[3] = {0.f, 0.f, 0.f};
    };
    MeshSlot meshes[DFSPH_MAX_SURFACE_MESHES];

    int set_surface_mesh(uint32_t id, const float* v, uint32_t nv, const uint32_t* t, uint32_t nt) {
        DF_CHECK(id < DFSPH_MAX_SURFACE_MESHES, DFSPH_E_INVALID, "mesh id beyond DFSPH_MAX_SURFACE_MESHES");
        DF_CHECK(nt > 0 && v && t, DFSPH_E_INVALID, "a mesh needs vertices and at least one triangle");
        for (size_t k = 0; k < 3 * (size_t)nt; ++k)
            DF_CHECK(t[k] < nv, DFSPH_E_INVALID, "triangle vertex index out of range");
        for (size_t k = 0; k < 3 * (size_t)nv; ++k)
            DF_CHECK(std::isfinite(v[k]), DFSPH_E_INVALID, "mesh vertices must be finite");
        MeshSlot& m = meshes[id];
        if (nt > m.cap) {
            if (m.tri) DF_CUDA(cudaFree(m.tri));
            m.tri = nullptr;
            m.cap = 0;
            DF_TRY(dalloc(&m.tri, 3 * (size_t)nt));
            m.cap = nt;
        }
        // MeshPerso::loadFromFile (BufferFluidSurface.cu:150-165): the box starts at the origin
        for (int a = 0; a < 3; ++a) m.bmin[a] = m.bmax[a] = 0.0f;
        for (uint32_t i = 0; i < nv; ++i)
            for (int a = 0; a < 3; ++a) {
                const float x = v[3 * (size_t)i + a];
                if (m.bmin[a] > x) m.bmin[a] = x;
                if (m.bmax[a] < x) m.bmax[a] = x;
            }
        std::vector<float4> h(3 * (size_t)nt);
        for (size_t k = 0; k < 3 * (size_t)nt; ++k) {
            const float* p = v + 3 * (size_t)t[k];
            h[k] = make_float4(p[0], p[1], p[2], 0.f);
        }
        DF_CUDA(cudaMemcpyAsync(m.tri, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        m.nt = nt;
        return DFSPH_OK;
    }
    DevSurface dev_surface(const dfsph_surface& s) const {
        DevSurface d = plain_surface(s);
        if (s.type == DFSPH_SURFACE_MESH && s.points < DFSPH_MAX_SURFACE_MESHES) {
            const MeshSlot& m = meshes[s.points];
            d.m.tri = m.tri;
            d.m.nt = m.nt;
            for (int a = 0; a < 3; ++a) {
                d.m.bmin[a] = m.bmin[a];
                d.m.bmax[a] = m.bmax[a];
            }
            mesh_ray_direction(d.m.dir);
        }
        return d;
    }

    bool surface_valid(const dfsph_surface& S) const {
        switch (S.type) {
            case DFSPH_SURFACE_PLANE:
            case DFSPH_SURFACE_CUBOID:
            case DFSPH_SURFACE_CYLINDER:
            case DFSPH_SURFACE_SPHERE:
                return true;
            case DFSPH_SURFACE_STAR:
                return S.points >= 1;
            case DFSPH_SURFACE_MESH:
                return S.points < DFSPH_MAX_SURFACE_MESHES && meshes[S.points].nt > 0;
            default:
                return false;
        }
    }

    int open_boundary_init(const dfsph_surface* bnd, const dfsph_surface* interior, const dfsph_surface* surf,
                           const float* xyz, uint32_t ns, uint32_t* n_kept) {
        DF_CHECK(bnd && interior && surf, DFSPH_E_INVALID, "null surface");
        DF_CHECK(surface_valid(*bnd) && surface_valid(*interior) && surface_valid(*surf), DFSPH_E_INVALID,
                 "unsupported surface (types: plane 0, cuboid 1, cylinder 2, mesh 3 with a registered mesh id, "
                 "sphere 4, star 5 with points >= 1)");
        DF_CHECK(xyz || ns == 0, DFSPH_E_INVALID, "null sample positions");
        DF_CHECK(grid_ready, DFSPH_E_STATE, "no grid: set a boundary or upload fluid first");
        if (ns > ob_cap || !ob_total) {
            for (void* q : {(void*)ob_samples, (void*)ob_vel, (void*)ob_flag, (void*)ob_rank, (void*)ob_scan})
                if (q) cudaFree(q);
            ob_samples = ob_vel = nullptr;
            ob_flag = ob_rank = ob_scan = nullptr;
            ob_cap = std::max(ns, ob_cap);
            DF_TRY(dalloc(&ob_samples, ob_cap));
            DF_TRY(dalloc(&ob_vel, ob_cap));
            DF_TRY(dalloc(&ob_flag, ob_cap));
            DF_TRY(dalloc(&ob_rank, ob_cap));
            ob_scan_inputs = std::max(ob_cap, Nc);
            DF_TRY(dalloc(&ob_scan, scan_scratch_words(ob_scan_inputs)));
            if (!ob_total) DF_TRY(dalloc(&ob_total, 2));
            if (!h_ob) DF_CUDA(cudaMallocHost((void**)&h_ob, 2 * sizeof(uint32_t)));
        }
        DF_TRY(ensure_scan_scratch(std::max(dw_cap, ns)));
        ob_boundary = *bnd;
        ob_interior = *interior;
        ob_surface = *surf;
        ob_ns = 0;
        if (ns) {
            std::vector<float4> h(ns);
            for (uint32_t i = 0; i < ns; ++i) h[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
            DF_CUDA(cudaMemcpyAsync(ob_vel, h.data(), (size_t)ns * sizeof(float4), cudaMemcpyHostToDevice, stream));
            launch_open_boundary_select<Real>(ob_vel, ns, dev_surface(ob_interior), dev_surface(ob_surface), params(),
                                              ob_flag, stream);
            exclusive_scan_u32(ob_flag, ob_rank, ns, ob_scan, ob_total, stream);
            launch_compact_samples(ob_vel, ob_flag, ob_rank, ns, ob_samples, stream);
            DF_CUDA(cudaMemcpyAsync(h_ob, ob_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            DF_CUDA(cudaGetLastError());
            ob_ns = h_ob[0];
            launches += 5;
        }
        ob_ready = true;
        if (n_kept) *n_kept = ob_ns;
        return DFSPH_OK;
    }

    int open_boundary_samples(float* xyz, uint32_t capacity, uint32_t* count) {
        DF_CHECK(count, DFSPH_E_INVALID, "null count");
        DF_CHECK(ob_ready, DFSPH_E_STATE, "open boundary not initialised (dfsph_open_boundary_init)");
        *count = ob_ns;
        if (!xyz) return DFSPH_OK;
        DF_CHECK(capacity >= ob_ns, DFSPH_E_INVALID, "capacity below the sample count");
        std::vector<float4> h(ob_ns);
        if (ob_ns) {
            DF_CUDA(cudaMemcpyAsync(h.data(), ob_samples, (size_t)ob_ns * sizeof(float4), cudaMemcpyDeviceToHost,
                                    stream));
            DF_CUDA(cudaStreamSynchronize(stream));
        }
        for (uint32_t i = 0; i < ob_ns; ++i) {
            xyz[3 * i] = h[i].x;
            xyz[3 * i + 1] = h[i].y;
            xyz[3 * i + 2] = h[i].z;
        }
        return DFSPH_OK;
    }

    int open_boundary_shift(const float* delta) {
        DF_CHECK(delta, DFSPH_E_INVALID, "null delta");
        DF_CHECK(ob_ready, DFSPH_E_STATE, "open boundary not initialised (dfsph_open_boundary_init)");
        for (dfsph_surface* S : {&ob_boundary, &ob_interior, &ob_surface}) {
            float* c = (S->type == DFSPH_SURFACE_PLANE) ? S->origin : S->center;
            for (int a = 0; a < 3; ++a) c[a] += delta[a];
        }
        launch_shift_samples(ob_samples, ob_ns, delta[0], delta[1], delta[2], stream);
        launches += ob_ns ? 1 : 0;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // Stable removal of the particles with alive[i] == 0 (dst = exclusive scan of alive, kept
    // survivors): the state moves to the other buffer; ids stay dense and keep their relative order.
    int compact_fluid(const uint32_t* alive, const uint32_t* dst, uint32_t kept) {
        dw_first_new = kept;  // ids are renumbered: nothing counts as added by the window any more
        const int nx = 1 - cur;
        launch_compact_fluid<Real>(alive, dst, n, pos[cur], vel[cur], kappa[cur], kappaV[cur], id[cur],
                                   learned ? kappaT[cur] : nullptr, learned ? kappaVT[cur] : nullptr, pos[nx],
                                   vel[nx], kappa[nx], kappaV[nx], id[nx], learned ? kappaT[nx] : nullptr,
                                   learned ? kappaVT[nx] : nullptr, stream);
        uint32_t* alive_by_id = sb.keys_b;
        uint32_t* new_id = sb.vals_b;
        launch_alive_by_id(id[cur], alive, n, alive_by_id, stream);
        exclusive_scan_u32(alive_by_id, new_id, n, ob_scan, ob_total + 1, stream);
        launch_renumber_ids(id[nx], kept, new_id, stream);
        cur = nx;
        n = kept;
        launches += 6;
        return DFSPH_OK;
    }

    int ensure_scan_scratch(uint32_t inputs = 0) {
        inputs = std::max(inputs, std::max(ob_cap, Nc));
        if (ob_scan && inputs > ob_scan_inputs) {
            cudaFree(ob_scan);
            ob_scan = nullptr;
        }
        if (!ob_scan) {
            DF_TRY(dalloc(&ob_scan, scan_scratch_words(inputs)));
            ob_scan_inputs = inputs;
        }
        if (!ob_total) DF_TRY(dalloc(&ob_total, 2));
        if (!h_ob) DF_CUDA(cudaMallocHost((void**)&h_ob, 2 * sizeof(uint32_t)));
        return DFSPH_OK;
    }

    // checkParticlesPositions (DFSPH_c_arrays_structure.cpp:1599, SPH_other_systems_cuda.cu:1283-1328):
    // counts the fluid particles outside the domain box; mode 2 also removes them (stable).
    int check_particles_positions(int mode, uint32_t* count) {
        DF_CHECK(mode == 0 || mode == 2, DFSPH_E_INVALID, "mode must be 0 (count) or 2 (remove)");
        uint32_t c = 0;
        if (n && grid_ready) {
            DF_TRY(ensure_scan_scratch());
            DF_CUDA(cudaMemsetAsync(status + 3, 0, sizeof(uint32_t), stream));
            launch_box_tag<Real>(pos[cur], n, bb_lo, bb_hi, sb.keys_a, status + 3, stream);
            DF_CUDA(cudaMemcpyAsync(h_status + 3, status + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            c = h_status[3];
            launches += 1;
            if (mode == 2 && c) DF_TRY(remove_tagged(c));
        }
        if (count) *count = c;
        return DFSPH_OK;
    }

    // Removes the c particles whose sb.keys_a flag is 0.
    int remove_tagged(uint32_t c) {
        DF_TRY(ensure_scan_scratch());
        exclusive_scan_u32(sb.keys_a, sb.vals_a, n, ob_scan, ob_total, stream);
        launches += 3;
        DF_TRY(compact_fluid(sb.keys_a, sb.vals_a, n - c));
        escaped_removed += c;
        invalidate_graphs();
        DF_TRY(sync_state());
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // ---- dynamic window (after DynamicWindowInterface, DynamicWindow.h:31-200, driven like
    // DFSPHCUDA::applyDynamicWindow, DFSPH_CUDA.cpp:3988-4139) ------------------------------------
    int dynamic_window_init(const double* lo, const double* hi, uint32_t wall_first, uint32_t wall_count,
                            const float* xyz, uint32_t ns) {
        DF_CHECK(lo && hi, DFSPH_E_INVALID, "null window box");
        DF_CHECK(lo[0] < hi[0] && lo[1] < hi[1] && lo[2] < hi[2], DFSPH_E_INVALID, "empty window box");
        DF_CHECK(wall_first <= nb && wall_count <= nb - wall_first, DFSPH_E_INVALID, "wall range out of bounds");
        DF_CHECK(xyz || ns == 0, DFSPH_E_INVALID, "null rest samples");
        DF_CHECK(grid_ready, DFSPH_E_STATE, "no grid: set a boundary first");
        if (ns > dw_cap) {
            for (void* q : {(void*)dw_samples, (void*)dw_sel, (void*)dw_vel, (void*)dw_flag, (void*)dw_rank})
                if (q) cudaFree(q);
            dw_samples = dw_sel = dw_vel = nullptr;
            dw_flag = dw_rank = nullptr;
            dw_cap = ns;
            DF_TRY(dalloc(&dw_samples, dw_cap));
            DF_TRY(dalloc(&dw_sel, dw_cap));
            DF_TRY(dalloc(&dw_vel, dw_cap));
            DF_TRY(dalloc(&dw_flag, dw_cap));
            DF_TRY(dalloc(&dw_rank, dw_cap));
        }
        DF_TRY(ensure_scan_scratch(std::max(dw_cap, Nc)));
        if (ns) {
            std::vector<float4> h(ns);
            for (uint32_t i = 0; i < ns; ++i) h[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
            DF_CUDA(cudaMemcpyAsync(dw_samples, h.data(), (size_t)ns * sizeof(float4), cudaMemcpyHostToDevice, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
        }
        for (int a = 0; a < 3; ++a) {
            dw_lo[a] = lo[a];
            dw_hi[a] = hi[a];
            dw_disp[a] = 0.0;
        }
        dw_wall_first = wall_first;
        dw_wall_count = wall_count;
        dw_ns = ns;
        dw_ready = true;
        return DFSPH_OK;
    }

    // Moves the window by d: (1) its walls translate rigidly to their set_boundary place + the total
    // displacement (on the device); (2) fluid particles outside the moved box are removed (stable
    // compaction, ids renumbered); (3) the rest samples move with the window, and those in the region
    // the window newly covers become fluid particles by the open boundary's inflow rule (no fluid
    // particle closer than allowed_distance, density estimate at most allowed_density; velocity the
    // kernel-weighted velocity of the fluid around it). The domain box of the end-of-step removal moves
    // with the window. The cell grid stays where it is: it must cover the window's whole path.
    int dynamic_window_shift(const double* d, double allowed_distance, double allowed_density, uint32_t* added,
                             uint32_t* removed) {
        DF_CHECK(dw_ready, DFSPH_E_STATE, "dynamic window not initialised (dfsph_dynamic_window_init)");
        DF_CHECK(d && std::isfinite(d[0]) && std::isfinite(d[1]) && std::isfinite(d[2]), DFSPH_E_INVALID,
                 "displacement must be finite");
        DF_CHECK(allowed_distance > 0 && allowed_density > 0, DFSPH_E_INVALID,
                 "the window's inflow needs allowed_distance > 0 and allowed_density > 0");
        double old_lo[3], old_hi[3];
        for (int a = 0; a < 3; ++a) {
            old_lo[a] = dw_lo[a] + dw_disp[a];
            old_hi[a] = dw_hi[a] + dw_disp[a];
            dw_disp[a] += d[a];
            bb_lo[a] += (float)d[a];
            bb_hi[a] += (float)d[a];
        }
        if (dw_wall_count) DF_TRY(move_boundary_rigid(dw_wall_first, dw_wall_count, nullptr, dw_disp, nullptr, nullptr));
        DF_TRY(bin_boundary_now());  // the inflow below reads the boundary's cell table
        // (2) removal outside the moved box
        uint32_t n_rm = 0;
        if (n) {
            float lo[3], hi[3];
            for (int a = 0; a < 3; ++a) {
                lo[a] = (float)(dw_lo[a] + dw_disp[a]);
                hi[a] = (float)(dw_hi[a] + dw_disp[a]);
            }
            DF_CUDA(cudaMemsetAsync(status + 3, 0, sizeof(uint32_t), stream));
            launch_box_tag<Real>(pos[cur], n, lo, hi, sb.keys_a, status + 3, stream);
            DF_CUDA(cudaMemcpyAsync(h_status + 3, status + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            launches += 1;
            n_rm = h_status[3];
            if (n_rm) {
                exclusive_scan_u32(sb.keys_a, sb.vals_a, n, ob_scan, ob_total, stream);
                launches += 3;
                DF_TRY(compact_fluid(sb.keys_a, sb.vals_a, n - n_rm));
            }
        }
        // (3) the samples of the newly covered region: outside the previous box, inside the grid
        uint32_t n_add = 0;
        bool clipped = false;
        if (dw_ns) {
            launch_shift_samples(dw_samples, dw_ns, (float)d[0], (float)d[1], (float)d[2], stream);
            dfsph_surface prev{};
            prev.type = DFSPH_SURFACE_CUBOID;
            dfsph_surface all{};  // every point: the half space below y = 3e38
            all.type = DFSPH_SURFACE_PLANE;
            all.origin[1] = 3.0e38f;
            all.normal[1] = -1.0f;
            for (int a = 0; a < 3; ++a) {
                prev.center[a] = (float)(0.5 * (old_lo[a] + old_hi[a]));
                prev.half_lengths[a] = (float)(0.5 * (old_hi[a] - old_lo[a]));
            }
            launch_open_boundary_select<Real>(dw_samples, dw_ns, plain_surface(prev), plain_surface(all), params(), dw_flag,
                                              stream);
            exclusive_scan_u32(dw_flag, dw_rank, dw_ns, ob_scan, ob_total, stream);
            launch_compact_samples(dw_samples, dw_flag, dw_rank, dw_ns, dw_sel, stream);
            DF_CUDA(cudaMemcpyAsync(h_ob, ob_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            const uint32_t nsel = h_ob[0];
            launches += 5;
            if (nsel) {
                DF_TRY(bin_fluid());
                const Real mass = (Real)new_particle_mass();
                dfsph_surface box{};
                box.type = DFSPH_SURFACE_CUBOID;
                for (int a = 0; a < 3; ++a) {
                    box.center[a] = (float)(0.5 * (dw_lo[a] + dw_hi[a]) + dw_disp[a]);
                    box.half_lengths[a] = (float)(0.5 * (dw_hi[a] - dw_lo[a]));
                }
                launch_inflow<Real>(ds, dw_sel, nsel, (float)allowed_distance, (float)allowed_density, mass,
                                    plain_surface(box), ftab, btab, dw_flag, dw_vel, stream);
                exclusive_scan_u32(dw_flag, dw_rank, nsel, ob_scan, ob_total, stream);
                DF_CUDA(cudaMemcpyAsync(h_ob, ob_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
                DF_CUDA(cudaStreamSynchronize(stream));
                const uint32_t want = h_ob[0];
                n_add = std::min<uint32_t>(want, Nc - n);
                clipped = n_add < want;
                launch_append_inflow<Real>(dw_sel, dw_vel, dw_flag, dw_rank, nsel, n, Nc, mass, pos[cur], vel[cur],
                                           kappa[cur], kappaV[cur], id[cur], learned ? kappaT[cur] : nullptr,
                                           learned ? kappaVT[cur] : nullptr, stream);
                n += n_add;
                launches += 5;
            }
        }
        dw_first_new = n - n_add;
        if (n_add || n_rm) invalidate_graphs();
        DF_TRY(sync_state());
        if (clipped) {
            uint32_t st = 0;
            DF_CUDA(cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            st |= DFSPH_ST_FLUID_CAPACITY;
            DF_CUDA(cudaMemcpyAsync(status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        if (added) *added = n_add;
        if (removed) *removed = n_rm;
        return DFSPH_OK;
    }

    // DynamicWindowInterface::stabilizeFluid, method 0 (DynamicWindow.cu:3160-3700: the fluid simulated
    // for a few steps of a fixed time step with the warm starts cleared before and after, restricted
    // to the tagged particles, their velocities damped before each position update). Here the tagged
    // particles are the ones the last shift added; the others, with tagged_only, keep their positions
    // and velocities (they take part as neighbours). Each iteration is the plain step's sequence:
    // neighbour search, divergence solve, viscosity and gravity, pressure solve with the velocity
    // update, damping, position update. The dt history is restored afterwards (the reference sets the
    // previous time step again).
    int dynamic_window_stabilize(uint32_t iterations, double step, double damping, int tagged_only) {
        DF_CHECK(dw_ready, DFSPH_E_STATE, "dynamic window not initialised (dfsph_dynamic_window_init)");
        DF_CHECK(step > 0 && std::isfinite(step), DFSPH_E_INVALID, "stabilisation time step must be finite and > 0");
        DF_CHECK(damping >= 0 && damping <= 1, DFSPH_E_INVALID, "damping must be in [0, 1]");
        if (!n || !iterations) return DFSPH_OK;
        const uint32_t first = tagged_only ? std::min(dw_first_new, n) : 0u;
        std::vector<double> saved(kDtSlots);
        DF_CUDA(cudaMemcpyAsync(saved.data(), dtd, kDtSlots * sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        DtArgs a{};
        for (int k = 0; k < kDtSlots; ++k) a.v[k] = saved[k];
        a.v[kDtH] = a.v[kDtHFuture] = step;
        a.v[kDtInvH] = a.v[kDtInvHFuture] = 1.0 / step;
        a.v[kDtRatio] = a.v[kDtRatio2] = 1.0;
        launch_dt<Real>(ds, 0, a, stream);
        DF_CUDA(cudaMemsetAsync(kappa[cur], 0, (size_t)n * sizeof(Real), stream));
        DF_CUDA(cudaMemsetAsync(kappaV[cur], 0, (size_t)n * sizeof(Real), stream));
        launches += 1;
        if (first) {
            if (!dw_spos) {
                DF_TRY(dalloc(&dw_spos, Nc));
                DF_TRY(dalloc(&dw_svel, Nc));
            }
            launch_save_untagged<Real>(pos[cur], vel[cur], id[cur], n, first, dw_spos, dw_svel, stream);
            launches += 1;
        }
        for (uint32_t it = 0; it < iterations; ++it) {
            DF_TRY(neighbors_search());
            if (sc.enable_divergence_solver) {
                DF_TRY(divergence_solve(sc.max_iterations_v, sc.max_error_v));
            } else {
                launch_density_alpha<Real>(ds, n, false, false, stream);
                launches += 1;
            }
            DF_TRY(external_forces(false));
            DF_TRY(pressure_solve(sc.max_iterations, sc.max_error, true));
            if (damping < 1.0) {
                launch_damp_tagged<Real>(vel[cur], id[cur], n, first, (Real)damping, stream);
                launches += 1;
            }
            DF_TRY(update_pos());
            if (first) {
                launch_restore_untagged<Real>(pos[cur], vel[cur], id[cur], n, first, dw_spos, dw_svel, stream);
                launches += 1;
            }
            DF_TRY(on_step_end());
        }
        DF_CUDA(cudaMemsetAsync(kappa[cur], 0, (size_t)n * sizeof(Real), stream));
        DF_CUDA(cudaMemsetAsync(kappaV[cur], 0, (size_t)n * sizeof(Real), stream));
        for (int k = 0; k < kDtSlots; ++k) a.v[k] = saved[k];
        launch_dt<Real>(ds, 0, a, stream);
        launches += 1;
        dt_stale = true;
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // DFSPHCData::computeFluidLevel (find_fluid_height_cuda, SPH_other_systems_cuda.cu:144-260): per
    // column of cells (x, z), the cells are read from the top down until at least three particles
    // have been seen; the column's height is the middle one of the three highest (a lone splash
    // particle above the surface does not count); the level is the highest column's. Columns of
    // fewer than three particles count -2; no such column at all gives -1; particles off the grid are
    // not read. On the host, from the positions and the cells of the device's binning (FP32,
    // floor(x / H + offset)). `tops` (nullable) receives each column's highest particle in its top
    // occupied cell (find_column_max_height_kernel, :292-318), keyed by column_key.
    static int64_t column_key(int cx, int cz) { return (int64_t)cz * (int64_t)(1 << 30) + cx; }
    int fluid_level(double* out, std::unordered_map<int64_t, float>* tops = nullptr) {
        DF_CHECK(out, DFSPH_E_INVALID, "null output");
        *out = -1.0;
        if (!n || !grid_ready) return DFSPH_OK;
        std::vector<Vec4<Real>> hp(n);
        DF_CUDA(cudaMemcpyAsync(hp.data(), pos[cur], (size_t)n * sizeof(Vec4<Real>), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        const float H = (float)(4.0 * sc.particle_radius);
        struct Cell {
            int64_t column;
            int32_t y;
            Real h;
        };
        std::vector<Cell> cells;
        cells.reserve(n);
        for (const Vec4<Real>& q : hp) {
            const float x = (float)q.x, y = (float)q.y, z = (float)q.z;
            if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z))) continue;
            const int cx = (int)std::floor(x / H + (float)off[0]), cy = (int)std::floor(y / H + (float)off[1]),
                      cz = (int)std::floor(z / H + (float)off[2]);
            if (cx < 0 || cy < 0 || cz < 0 || cx >= dim[0] || cy >= dim[1] || cz >= dim[2]) continue;  // off the grid
            cells.push_back({column_key(cx, cz), cy, q.y});
        }
        std::sort(cells.begin(), cells.end(), [](const Cell& a, const Cell& b) {
            return a.column != b.column ? a.column < b.column : a.y > b.y;
        });
        double level = -1.0;
        for (size_t a = 0; a < cells.size();) {
            size_t b = a;
            while (b < cells.size() && cells[b].column == cells[a].column) ++b;
            if (tops) {  // the top occupied cell's highest particle
                float t = -2.0f;
                for (size_t c = a; c < b && cells[c].y == cells[a].y; ++c) t = std::max(t, (float)cells[c].h);
                (*tops)[cells[a].column] = t;
            }
            Real top[3] = {Real(-2), Real(-2), Real(-2)};  // ascending, as the reference keeps them
            int count = 0;
            for (size_t c = a; c < b;) {
                size_t e = c;
                while (e < b && cells[e].y == cells[c].y) ++e;  // one cell
                for (size_t k = c; k < e; ++k) {
                    ++count;
                    int sup = -1;
                    for (int m = 0; m < 3; ++m)
                        if (cells[k].h > top[m]) sup = m;
                    if (sup > -1) {
                        for (int m = 0; m < sup; ++m) top[m] = top[m + 1];
                        top[sup] = cells[k].h;
                    }
                }
                c = e;
                if (count > 2) break;
            }
            const double col = count > 2 ? (double)top[1] : -2.0;
            if (col > level) level = col;
            a = b;
        }
        *out = level;
        return DFSPH_OK;
    }

    // DFSPHCData::handleFLuidLevelControl (control_fluid_height_cuda, SPH_other_systems_cuda.cu:
    // 414-547): nothing when the level is within 5 cm of the target. Above it, the particles above the
    // target are removed (y > target, the target rounded to FP32; stable compaction, ids renumbered
    // densely). Below it, new particles are placed above the fluid near the walls (raise_fluid_level).
    int fluid_level_control(double target, uint32_t* removed, uint32_t* added) {
        if (removed) *removed = 0;
        if (added) *added = 0;
        if (!(target > 0) || !n) return DFSPH_OK;
        double level = 0;
        std::unordered_map<int64_t, float> tops;
        DF_TRY(fluid_level(&level, &tops));
        if (std::fabs(level - target) < 0.05) return DFSPH_OK;
        if (level < target) return raise_fluid_level(target, level, tops, added);
        DF_TRY(ensure_scan_scratch());
        const float lo[3] = {-3.0e38f, -3.0e38f, -3.0e38f}, hi[3] = {3.0e38f, (float)target, 3.0e38f};
        DF_CUDA(cudaMemsetAsync(status + 3, 0, sizeof(uint32_t), stream));
        launch_box_tag<Real>(pos[cur], n, lo, hi, sb.keys_a, status + 3, stream);
        DF_CUDA(cudaMemcpyAsync(h_status + 3, status + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        launches += 1;
        const uint32_t n_rm = h_status[3];
        if (n_rm) {
            exclusive_scan_u32(sb.keys_a, sb.vals_a, n, ob_scan, ob_total, stream);
            launches += 3;
            DF_TRY(compact_fluid(sb.keys_a, sb.vals_a, n - n_rm));
            invalidate_graphs();
            DF_TRY(sync_state());
            DF_CUDA(cudaStreamSynchronize(stream));
            DF_CUDA(cudaGetLastError());
        }
        if (removed) *removed = n_rm;
        return DFSPH_OK;
    }

    // The raising branch of control_fluid_height_cuda (SPH_other_systems_cuda.cu:486-545) with
    // get_min_max_pos_kernel (:282-304) and place_additional_particles_right_above_kernel (:321-408),
    // in the reference's FP32/FP64 operation order. The domain box: component-wise min (max) of the
    // first (last) ten boundary particles in the reference's boundary order (stable by linear cell
    // index x + 256 z + 65536 y, from the boundary's current positions), shrunk by 2r. A lattice of
    // spacing 2r spans the box (layers 0.8 * 2r apart, odd layers shifted by r in x and z) with
    // floor((target - level) / 2r) + 1 layers; only the points outside the central third of the box
    // (in x or z) are kept, and each is lifted to its column's highest particle + 2.5 r (a column
    // without fluid counts -2). Appended in lattice order (the reference's atomic counter gives an
    // arbitrary order), velocity zero, the inflow mass; past fluid_capacity the rest is dropped and
    // DFSPH_ST_FLUID_CAPACITY is set.
    int raise_fluid_level(double target, double level, const std::unordered_map<int64_t, float>& tops,
                          uint32_t* added) {
        DF_CHECK(nb > 0, DFSPH_E_STATE, "raising the fluid level needs the boundary (the domain's extent)");
        std::vector<float> b((size_t)nb * 3);
        DF_TRY(download(DFSPH_F_BOUNDARY_POSITION, DFSPH_DTYPE_F32, b.data(), b.size(), DFSPH_ORDER_ID));
        const float H = (float)(4.0 * sc.particle_radius);
        std::vector<std::array<int, 3>> key(nb);
        for (uint32_t k = 0; k < nb; ++k)
            for (int a = 0; a < 3; ++a) key[k][a] = (int)std::floor(b[3 * k + a] / H + (float)off[a]);
        std::vector<uint32_t> order(nb);
        for (uint32_t k = 0; k < nb; ++k) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t p, uint32_t q) {
            const auto &kp = key[p], &kq = key[q];
            if (kp[1] != kq[1]) return kp[1] < kq[1];
            if (kp[2] != kq[2]) return kp[2] < kq[2];
            return kp[0] < kq[0];
        });
        float mn[3], mx[3];
        for (int a = 0; a < 3; ++a) {
            mn[a] = b[3 * order[0] + a];
            mx[a] = b[3 * order[nb - 1] + a];
        }
        for (uint32_t k = 0; k < 10 && k < nb; ++k)
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::min(mn[a], b[3 * order[k] + a]);
                mx[a] = std::max(mx[a], b[3 * order[nb - 1 - k] + a]);
            }
        const float r = (float)sc.particle_radius, p = r * 2.0f;
        for (int a = 0; a < 3; ++a) {
            mn[a] += 2.0f * r;
            mx[a] -= 2.0f * r;
        }
        float width[3], count_w[3], border[3];
        for (int a = 0; a < 3; ++a) {
            width[a] = mx[a] - mn[a];
            count_w[a] = std::floor(std::fabs(width[a]) / p) + 1.0f;  // the kernel's |width|
            border[a] = a == 1 ? 0.0f : width[a] / 3.0f;
        }
        // the lattice size as the host computes it (from width itself, y from the missing height)
        const float host_x = std::floor(width[0] / p) + 1.0f, host_z = std::floor(width[2] / p) + 1.0f;
        const float layers = std::floor(((float)target - (float)level) / p) + 1.0f;
        const float want_f = host_x * layers * host_z;
        if (!(want_f >= 1.0f)) return DFSPH_OK;  // the reference stops the program here
        DF_CHECK(want_f < 2.0e9f, DFSPH_E_INVALID, "fluid level control: lattice too large");
        const int want = (int)want_f;
        const bool bordered = border[0] * border[0] + border[2] * border[2] > 0.0f;
        std::vector<float> xyz;
        for (int id = 0; id < want; ++id) {
            const int row = (int)((float)id / count_w[0]);
            const int lev = (int)((float)row / count_w[2]);
            float lx = ((float)id - (float)row * count_w[0]) * p;
            float ly = (float)((double)lev * ((double)p * 0.80));
            float lz = ((float)row - (float)lev * count_w[2]) * p;
            if (lev & 1) {
                lx += p / 2.0f;
                lz += p / 2.0f;
            }
            const float tx = mn[0] + lx, tz = mn[2] + lz;
            if (bordered && !(tx < mn[0] + border[0] || tz < mn[2] + border[2] || tx > mx[0] - border[0] ||
                              tz > mx[2] - border[2]))
                continue;
            const int cx = (int)std::floor(tx / H + (float)off[0]), cz = (int)std::floor(tz / H + (float)off[2]);
            const auto it = tops.find(column_key(cx, cz));
            const float top = it == tops.end() ? -2.0f : it->second;
            const float y0 = (float)((double)(top + p) + (double)p / 4.0);
            xyz.push_back(mn[0] + lx);
            xyz.push_back(y0 + ly);
            xyz.push_back(mn[2] + lz);
        }
        const uint32_t kept = (uint32_t)(xyz.size() / 3);
        const uint32_t n_add = std::min<uint32_t>(kept, Nc - n);
        if (n_add) {
            DF_CUDA(cudaMemcpyAsync(stage, xyz.data(), (size_t)n_add * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
            launch_unpack_fluid<Real>(stage, nullptr, nullptr, new_particle_mass(), n_add, pos[cur] + n, vel[cur] + n,
                                      kappa[cur] + n, kappaV[cur] + n, id[cur] + n, stream, n);
            if (learned && kappaT[cur]) {
                DF_CUDA(cudaMemsetAsync(kappaT[cur] + n, 0, (size_t)n_add * sizeof(Real), stream));
                DF_CUDA(cudaMemsetAsync(kappaVT[cur] + n, 0, (size_t)n_add * sizeof(Real), stream));
            }
            launches += 1;
            n += n_add;
            invalidate_graphs();
            DF_TRY(sync_state());
        }
        if (n_add < kept) {
            uint32_t st = 0;
            DF_CUDA(cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            st |= DFSPH_ST_FLUID_CAPACITY;
            DF_CUDA(cudaMemcpyAsync(status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        if (added) *added = n_add;
        return DFSPH_OK;
    }

    int dynamic_window_state(double* displacement) {
        DF_CHECK(displacement, DFSPH_E_INVALID, "null output");
        DF_CHECK(dw_ready, DFSPH_E_STATE, "dynamic window not initialised (dfsph_dynamic_window_init)");
        for (int a = 0; a < 3; ++a) displacement[a] = dw_disp[a];
        return DFSPH_OK;
    }

    int open_boundary_apply(double allowed_distance, double allowed_density, bool inflow, bool outflow,
                            uint32_t* added, uint32_t* removed) {
        DF_CHECK(ob_ready, DFSPH_E_STATE, "open boundary not initialised (dfsph_open_boundary_init)");
        DF_TRY(bin_boundary_now());  // the inflow reads the boundary's cell table
        if (inflow)
            DF_CHECK(allowed_distance > 0 && allowed_density > 0, DFSPH_E_INVALID,
                     "open boundary inflow needs allowed_distance > 0 and allowed_density > 0");
        uint32_t n_add = 0, n_rm = 0;
        bool clipped = false;
        const uint32_t n0 = n;
        if (inflow && ob_ns) {
            DF_TRY(bin_fluid());
            const Real mass = (Real)new_particle_mass();
            launch_inflow<Real>(ds, ob_samples, ob_ns, (float)allowed_distance, (float)allowed_density, mass,
                                dev_surface(ob_boundary), ftab, btab, ob_flag, ob_vel, stream);
            exclusive_scan_u32(ob_flag, ob_rank, ob_ns, ob_scan, ob_total, stream);
            DF_CUDA(cudaMemcpyAsync(h_ob, ob_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            const uint32_t want = h_ob[0];
            n_add = std::min<uint32_t>(want, Nc - n);
            clipped = n_add < want;
            launch_append_inflow<Real>(ob_samples, ob_vel, ob_flag, ob_rank, ob_ns, n, Nc, mass, pos[cur], vel[cur],
                                       kappa[cur], kappaV[cur], id[cur], learned ? kappaT[cur] : nullptr,
                                       learned ? kappaVT[cur] : nullptr, stream);
            n += n_add;
            launches += 5;
        }
        if (outflow && n) {
            uint32_t* alive = sb.keys_a;
            uint32_t* dst = sb.vals_a;
            launch_outflow_tag<Real>(pos[cur], n, dev_surface(ob_interior), dev_surface(ob_surface), alive, stream);
            exclusive_scan_u32(alive, dst, n, ob_scan, ob_total, stream);
            DF_CUDA(cudaMemcpyAsync(h_ob, ob_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            const uint32_t kept = h_ob[0];
            n_rm = n - kept;
            launches += 4;
            if (n_rm) DF_TRY(compact_fluid(alive, dst, kept));
        }
        if (n != n0) {
            invalidate_graphs();
            DF_TRY(sync_state());
        }
        if (clipped) {
            uint32_t st = 0;
            DF_CUDA(cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            st |= DFSPH_ST_FLUID_CAPACITY;
            DF_CUDA(cudaMemcpyAsync(status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        if (added) *added = n_add;
        if (removed) *removed = n_rm;
        return DFSPH_OK;
    }

    int invalidate_graphs() {
        for (int k = 0; k < 2; ++k) {
            if (g_loop[k]) cudaGraphExecDestroy(g_loop[k]);
            g_loop[k] = nullptr;
            g_loop_n[k] = 0;
            g_loop_u[k] = 0;
        }
        return DFSPH_OK;
    }

    // Loop graph: the first u iterations (those the loop always runs: u = min(minimum iterations,
    // max_iter)) as plain kernel nodes, then a while node whose body is one more Jacobi pass +
    // residual pass. Every residual's last block sets the condition (it = iterations so far:
    // continue while the mean residual is above the tolerance or it < the minimum, and it <
    // max_iter); the condition is 0 at each launch, so with u = max_iter the while node never runs.
    int build_loop_graph(int kind, int u) {
        cudaGraph_t g = nullptr;
        DF_CUDA(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle handle;
        DF_CUDA(cudaGraphConditionalHandleCreate(&handle, g, u > 0 ? 0u : 1u, cudaGraphCondAssignDefault));
        auto iteration = [&]() {
            if (kind == 0) {
                launch_divergence_jacobi<Real>(ds, n, handle, true, stream, boundary_forces);
                launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, handle, true, stream, g_loop_keep);
            } else {
                launch_pressure_jacobi<Real>(ds, n, handle, true, stream, boundary_forces);
                launch_pressure_residual<Real>(ds, n, false, 0.0, 0, 0, handle, true, stream, g_loop_keep);
            }
        };
        g_pdl_off = true;  // graph kernel edges need no programmatic launch
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        std::vector<cudaGraphNode_t> lead;
        if (u > 0) {
            DF_CUDA(cudaStreamBeginCaptureToGraph(stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < u; ++k) iteration();
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t* cdeps = nullptr;
            size_t nc = 0;
            const cudaError_t ei = cudaStreamGetCaptureInfo(stream, &cs, nullptr, nullptr, &cdeps, &nc);
            if (ei == cudaSuccess) lead.assign(cdeps, cdeps + nc);
            cudaGraph_t captured = nullptr;
            const cudaError_t ee = cudaStreamEndCapture(stream, &captured);
            if (ei != cudaSuccess || ee != cudaSuccess || lead.empty()) {
                g_pdl_off = false;
                cudaGraphDestroy(g);
                err = "loop graph capture failed";
                return DFSPH_E_CUDA;
            }
            deps = lead.data();
            ndeps = lead.size();
        }
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        cudaError_t e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                iteration();
                cudaGraph_t captured = nullptr;
                e = cudaStreamEndCapture(stream, &captured);
            }
        }
        g_pdl_off = false;
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        DF_CUDA(e);
        g_loop[kind] = exec;
        g_loop_n[kind] = n;
        g_loop_u[kind] = u;
        return DFSPH_OK;
    }

    // Runs the iterations of one solver loop after its init pass. Graph mode: one graph launch,
    // no host round trip. Host mode: one small readback per iteration (what the reference does).
    int run_loop(int kind, int max_iter, bool keep = false) {
        if (max_iter <= 0) return DFSPH_OK;
        if (use_graphs) {
            if (keep != g_loop_keep) {
                DF_TRY(invalidate_graphs());
                g_loop_keep = keep;
            }
            const int u = std::min(kind == 0 ? kMinItersV : kMinItersP, max_iter);
            if (!g_loop[kind] || g_loop_n[kind] != n || g_loop_u[kind] != u) {
                if (g_loop[kind]) cudaGraphExecDestroy(g_loop[kind]);
                g_loop[kind] = nullptr;
                DF_TRY(build_loop_graph(kind, u));
            }
            DF_CUDA(cudaGraphLaunch(g_loop[kind], stream));
            launches += 1;
            return DFSPH_OK;
        }
        uint32_t cont = 1;
        while (cont) {
            if (kind == 0) {
                launch_divergence_jacobi<Real>(ds, n, 0, false, stream, boundary_forces);
                launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream, keep);
            } else {
                launch_pressure_jacobi<Real>(ds, n, 0, false, stream, boundary_forces);
                launch_pressure_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream, keep);
            }
            launches += 2;
            DF_CUDA(cudaMemcpyAsync(h_ctl + kind, ctl + kind, sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            cont = h_ctl[kind].cont;
        }
        return DFSPH_OK;
    }

    // cuda_divergenceSolve (DFSPH_core_cuda.cu:785-861). lp: learned warm start (dfsph_step only).
    int divergence_solve(int max_iter, double max_error, bool lp = false) {
        if (!n) return DFSPH_OK;
        const double eta = max_error * 0.01 * sc.density0;  // divided by the device's h in the init pass
        if (!lp) {
            launch_density_alpha<Real>(ds, n, true, false, stream);
            launch_divergence_warm_jacobi<Real>(ds, n, nullptr, nullptr, stream, boundary_forces);
            launch_divergence_residual<Real>(ds, n, true, eta, kMinItersV, max_iter, 0, false, stream);
            launches += 3;
        } else {
            const bool infer = mlp_ready && !base_only && net_useful, use = mlp_ready || base_only;
            launch_density_alpha<Real>(ds, n, false, true, stream);
            if (infer) launch_mlp_forward(mlp, features, n, pred, status, stream);
            launch_warm_values<Real>(ds, n, 0, use, infer, damping, stream);
            launches += infer ? 3 : 2;
            if (use && probe) {  // both candidates per pass, then the selection
                launch_warm_dual<Real>(ds, n, 0, false, stream, boundary_forces);
                launch_residual_dual<Real>(ds, n, 0, eta, kMinItersV, max_iter, stream);
                launch_select_candidate<Real>(ds, n, 0, stream);
                launches += 3;
            } else {
                launch_divergence_warm_jacobi<Real>(ds, n, kappaVW, nullptr, stream, boundary_forces);
                launch_divergence_residual<Real>(ds, n, true, eta, kMinItersV, max_iter, 0, false, stream, true);
                launches += 2;
            }
            if (use && !probe) forced_warm |= 1u;
            if (use) ++solves_v;
        }
        DF_TRY(run_loop(0, max_iter, lp));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // cuda_pressureSolve (DFSPH_core_cuda.cu:1338-1419); with fused_vel the velocity update of
    // cuda_update_vel is applied inside the warm-start pass.
    int pressure_solve(int max_iter, double max_error, bool fused_vel, bool lp = false) {
        if (!n) return DFSPH_OK;
        const double eta = max_error * 0.01 * sc.density0;
        if (!lp) {
            launch_pressure_warm_jacobi<Real>(ds, n, fused_vel, nullptr, nullptr, stream, boundary_forces);
            launch_pressure_residual<Real>(ds, n, true, eta, kMinItersP, max_iter, 0, false, stream);
            launches += 2;
        } else {
            const bool infer = mlp_ready && !base_only && net_useful, use = mlp_ready || base_only;
            launch_warm_values<Real>(ds, n, 1, use, infer, damping, stream);
            launches += 1;
            if (use && probe) {
                launch_warm_dual<Real>(ds, n, 1, fused_vel, stream, boundary_forces);
                launch_residual_dual<Real>(ds, n, 1, eta, kMinItersP, max_iter, stream);
                launch_select_candidate<Real>(ds, n, 1, stream);
                launches += 3;
            } else {
                launch_pressure_warm_jacobi<Real>(ds, n, fused_vel, kappaW, nullptr, stream, boundary_forces);
                launch_pressure_residual<Real>(ds, n, true, eta, kMinItersP, max_iter, 0, false, stream, true);
                launches += 2;
            }
            if (use && !probe) forced_warm |= 2u;
            if (use) ++solves_p;
        }
        DF_TRY(run_loop(1, max_iter, lp));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int external_forces(bool cfl) {
        if (!n) return DFSPH_OK;
        launch_viscosity<Real>(ds, n, cfl, stream);
        launches += 1;
        vel_updated = false;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // DFSPHCData::updateTimeStep (DFSPH_c_arrays_structure.cpp:1100-1112), on the device; hf <= 0
    // takes the fixed time step.
    int update_time_step(double hf) {
        DF_CHECK(hf > 0 && std::isfinite(hf), DFSPH_E_INVALID, "time step must be finite and > 0");
        DtArgs a{};
        a.v[0] = hf;
        launch_dt<Real>(ds, 1, a, stream);
        launches += 1;
        dt_stale = true;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // cuda_CFL (DFSPH_core_cuda.cu:3321-3394): dt = cfl * 0.4 * 2r / sqrt(max |v + a h|^2), clamped,
    // reduced and applied on the device (no host round trip).
    int cfl(double min_dt, double factor_, double max_dt) {
        launch_cfl_reduce<Real>(ds, n ? grid_for(n) : 0, stream);
        DtArgs a{};
        a.v[0] = factor_;
        a.v[1] = min_dt;
        a.v[2] = max_dt;
        a.v[3] = 2.0 * sc.particle_radius;
        launch_dt<Real>(ds, 2, a, stream);
        launches += 2;
        dt_stale = true;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int update_vel() {
        if (!n) return DFSPH_OK;
        launch_update_vel<Real>(ds, n, stream);
        launches += 1;
        vel_updated = true;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int update_pos() {
        if (!n) return DFSPH_OK;
        launch_update_pos<Real>(ds, n, stream);
        launches += 1;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int on_step_end() {
        launch_dt<Real>(ds, 3, DtArgs{}, stream);
        launches += 1;
        dt_stale = true;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // Reads the loop control blocks and the status word (one synchronisation).
    int collect(bool div_ran, int max_iter_v, int max_iter) {
        DF_CUDA(cudaMemcpyAsync(h_ctl, ctl, 2 * sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(h_status, status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(h_dt, dtd, kDtSlots * sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        mirror_dt();
        last_iters = n ? h_ctl[1].iter : 0;
        last_err = h_ctl[1].avg;
        last_iters_v = (div_ran && n) ? h_ctl[0].iter : 0;
        last_err_v = div_ran ? h_ctl[0].avg : 0.0;
        if (use_graphs) launches += 2ull * (uint64_t)(last_iters + last_iters_v);
        uint32_t st = h_status[0];
        if (n && last_iters >= max_iter && max_iter > 0 && last_err > h_ctl[1].eta)
            st |= DFSPH_ST_PRESSURE_NOT_CONVERGED;
        if (div_ran && n && last_iters_v >= max_iter_v && max_iter_v > 0 && last_err_v > h_ctl[0].eta)
            st |= DFSPH_ST_DIVERGENCE_NOT_CONVERGED;
        h_status[0] = st;
        return DFSPH_OK;
    }

    int gate_sums(uint32_t& it, uint32_t& itv) {
        LoopCtl c[2];
        DF_CUDA(cudaMemcpyAsync(c, ctl, 2 * sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        it = c[1].iter_sum;
        itv = c[0].iter_sum;
        return DFSPH_OK;
    }

    // Advances the gate's schedule by one step; use_learned says whether this step runs the learned
    // passes. One host read of the iteration counters per phase change.
    int gate_step(bool& use_learned) {
        if (gate_left <= 0) {
            if (gate_phase == kGateLearned) {  // probe: settle, then measure the plain solver
                gate_phase = kGateSettling;
                gate_left = kGateSettle;
            } else if (gate_phase == kGateSettling) {
                DF_TRY(gate_sums(gate_it0, gate_itv0));
                gate_phase = kGateProbe;
                gate_left = gate_len = std::max(gate_window, 1);
            } else {  // a measured plain phase ended: decide
                uint32_t it, itv;
                DF_TRY(gate_sums(it, itv));
                const bool div = sc.enable_divergence_solver != 0;
                const double dp = (double)(it - gate_it0) / gate_len, dv = (double)(itv - gate_itv0) / gate_len;
                const double minp = std::min(kMinItersP, sc.max_iterations);
                const double minv = std::min(kMinItersV, sc.max_iterations_v);
                gate_last_excess = (dp - minp) + (div ? dv - minv : 0.0);
                if (gate_last_excess >= gate_margin) {
                    gate_phase = kGateLearned;
                    gate_left = std::max(gate_period, 1);
                } else {
                    gate_phase = kGatePlain;
                    gate_left = gate_len = std::max(gate_recheck, 1);
                    gate_it0 = it;
                    gate_itv0 = itv;
                }
            }
        }
        use_learned = gate_phase == kGateLearned;
        --gate_left;
        ++(use_learned ? gate_learned_steps : gate_plain_steps);
        return DFSPH_OK;
    }

    int step(dfsph_step_stats* st) {
        DF_CHECK(grid_ready, DFSPH_E_STATE, "step before any boundary or fluid upload");
        if (!n) DF_TRY(flush_pending());
        bool lp = learned && n > 0;
        if (lp && gate) DF_TRY(gate_step(lp));
        if (timing) DF_CUDA(cudaEventRecord(ev0, stream));
        forced_warm = 0;
        step_trained = false;
        if (lp) DF_CUDA(cudaMemsetAsync(status + 2, 0, sizeof(uint32_t), stream));
        if (learned && !lp && last_lp && n) {  // the gate's first plain step after learned ones
            launch_restore_totals<Real>(ds, n, stream);
            launches += 1;
        }
        last_lp = lp;
        DF_TRY(neighbors_search());
        const bool div = sc.enable_divergence_solver != 0;
        if (div) {
            DF_TRY(divergence_solve(sc.max_iterations_v, sc.max_error_v, lp));
        } else if (n) {
            launch_density_alpha<Real>(ds, n, false, lp, stream);
            launches += 1;
            if (lp) {  // no divergence solve: its warm-start arrays stay zero
                DF_CUDA(cudaMemsetAsync(kappaVW, 0, (size_t)n * sizeof(Real), stream));
                DF_CUDA(cudaMemsetAsync(kappaV[cur], 0, (size_t)n * sizeof(Real), stream));
                if (mlp_ready && !base_only && net_useful) {
                    launch_mlp_forward(mlp, features, n, pred, status, stream);
                    launches += 1;
                }
            }
        }
        const bool use_cfl = sc.cfl_method != 0;
        DF_TRY(external_forces(use_cfl));
        if (use_cfl) {
            DF_TRY(cfl(sc.cfl_min_time_step, sc.cfl_factor, sc.cfl_max_time_step));
        } else {
            DF_TRY(update_time_step(time_step));
        }
        DF_TRY(pressure_solve(sc.max_iterations, sc.max_error, true, lp));
        DF_TRY(update_pos());
        if (lp) {
            const bool due = train_interval > 0 &&
                             (lsteps == (uint64_t)train_start ||
                              (lsteps > (uint64_t)train_start && (lsteps - train_start) % train_interval == 0));
            if (due && train_iters > 0 && !base_only) DF_TRY(train_online(div));
            launch_totals<Real>(ds, n, div, stream);
            launches += 1;
            ++lsteps;
        }
        DF_TRY(on_step_end());
        if (timing) DF_CUDA(cudaEventRecord(ev1, stream));
        if (!st) return DFSPH_OK;  // asynchronous step: nothing read back, the host does not wait
        // DFSPHCUDA::step ends with checkParticlesPositions(2) (DFSPH_CUDA.cpp:456): the count comes
        // back with the status words; the removal itself runs only when there is something to remove.
        const bool tag = remove_escaped && n > 0;
        if (tag) {
            DF_TRY(ensure_scan_scratch());
            DF_CUDA(cudaMemsetAsync(status + 3, 0, sizeof(uint32_t), stream));
            launch_box_tag<Real>(pos[cur], n, bb_lo, bb_hi, sb.keys_a, status + 3, stream);
            launches += 1;
        }
        DF_TRY(collect(div, sc.max_iterations_v, sc.max_iterations));
        if (tag && h_status[3]) DF_TRY(remove_tagged(h_status[3]));
        if (lp) {
            const uint32_t w = (h_status[2] | forced_warm) & 3u;
            if (w & 1u) ++kept_v;
            if (w & 2u) ++kept_p;
        }
        if (st) {
            st->iterations = last_iters;
            st->iterations_v = last_iters_v;
            st->density_error = last_err;
            st->divergence_error = last_err_v;
            st->h = h_past;  // after onSimulationStepEnd: the step's dt is h_past, the next one h
            st->h_future = h;
            st->status = h_status[0];
            st->num_fluid = n;
            st->warm_start = lp ? ((h_status[2] | forced_warm) & 3u) : 0u;
            st->trained = step_trained ? 1u : 0u;
            st->ms_total = 0.0;
            if (timing) {
                float ms = 0.0f;
                DF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
                st->ms_total = ms;
            }
        }
        return DFSPH_OK;
    }

    // ------------------------------------------------------------------------------------------
    // Learned warm start: buffers, training, host-facing network calls.
    int ensure_mlp() {
        if (mlp.params) return DFSPH_OK;
        DF_TRY(dalloc(&mlp.params, kMlpParams));
        DF_TRY(dalloc(&mlp.adam_m, kMlpParams));
        DF_TRY(dalloc(&mlp.adam_v, kMlpParams));
        DF_TRY(dalloc(&mlp.grad, kMlpParams));
        DF_TRY(dalloc(&mlp.partials, mlp_partials_floats(kMaxTrainBatch)));
        DF_TRY(dalloc(&mlp.w1_bf16, kMlpHidden * 16));
        DF_TRY(dalloc(&mlp.w2_bf16, kMlpHidden * kMlpHidden));
        DF_TRY(dalloc(&mlp.w3_bf16, 8 * kMlpHidden));
        DF_TRY(dalloc(&mlp.scales, 1));
        DF_TRY(dalloc(&mlp.loss, 1));
        DF_TRY(dalloc(&tx, (size_t)kMaxTrainBatch * kMlpIn));
        DF_TRY(dalloc(&tt, (size_t)kMaxTrainBatch * kMlpOut));
        DF_TRY(mlp_reset(mlp_seed));
        return sync_state();
    }

    int upload_scales() {
        DF_CUDA(cudaMemcpyAsync(mlp.scales, &h_scales, sizeof(MlpScales), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaStreamSynchronize(stream));  // h_scales may change right after
        return DFSPH_OK;
    }

    int mlp_reset(uint32_t seed) {
        mlp_seed = seed;
        for (int i = 0; i < kMlpIn; ++i) h_scales.in_scale[i] = i < 5 ? 1.0f : 0.0f;
        for (int o = 0; o < kMlpOut; ++o) h_scales.out_scale[o] = 1.0f;
        DF_TRY(upload_scales());
        launch_mlp_init(mlp, seed, stream);
        launch_mlp_pack(mlp, stream);
        DF_CUDA(cudaMemsetAsync(mlp.loss, 0, sizeof(double), stream));
        launches += 2;
        adam_t = 0;
        mlp_ready = false;
        net_useful = false;
        scales_set = false;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int clear_totals() {
        for (int b = 0; b < 2; ++b) {
            DF_CUDA(cudaMemsetAsync(kappaT[b], 0, (size_t)Nc * sizeof(Real), stream));
            DF_CUDA(cudaMemsetAsync(kappaVT[b], 0, (size_t)Nc * sizeof(Real), stream));
        }
        return DFSPH_OK;
    }

    int enable_learned(bool on) {
        if (on && !learned) {
            DF_TRY(ensure_mlp());
            if (!kappaT[0]) {
                for (int b = 0; b < 2; ++b) {
                    DF_TRY(dalloc(&kappaT[b], Nc));
                    DF_TRY(dalloc(&kappaVT[b], Nc));
                }
                DF_TRY(dalloc(&kappaW, Nc));
                DF_TRY(dalloc(&kappaVW, Nc));
                DF_TRY(dalloc(&kappaP, Nc));
                DF_TRY(dalloc(&kappaVP, Nc));
                DF_TRY(dalloc(&velP, Nc));
                DF_TRY(dalloc(&resid, Nc));
                DF_TRY(dalloc(&residV, Nc));
                DF_TRY(dalloc(&dadvP, Nc));
                DF_TRY(dalloc(&kcP, Nc));
                DF_TRY(dalloc(&rawP, Nc));
                DF_TRY(dalloc(&features, (size_t)Nc * kMlpIn));
                DF_TRY(dalloc(&pred, (size_t)Nc * kMlpOut));
            }
            DF_TRY(clear_totals());
            lsteps = 0;
        }
        learned = on;
        return sync_state();
    }

    // Normalisation that follows the data: inputs scaled to unit RMS, outputs in units of the
    // targets' RMS, from the current training batch. A scale is replaced when it is unset or off by
    // more than 2x, and the first / last layer are rescaled with it so that the network computes
    // the same function in physical units (the Adam state restarts).
    int adapt_scales(uint32_t B, uint32_t offset, bool div) {
        std::vector<float> x((size_t)B * kMlpIn), t((size_t)B * kMlpOut);
        DF_CUDA(cudaMemcpyAsync(x.data(), tx, x.size() * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(t.data(), tt, t.size() * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        auto rms = [&](const std::vector<float>& v, int stride, int c, double mul) {
            double acc = 0.0;
            for (uint32_t k = 0; k < B; ++k) {
                const double e = (double)v[(size_t)k * stride + c] * mul;
                acc += e * e;
            }
            return std::sqrt(acc / (double)B);
        };
        MlpScales ns = h_scales;
        bool changed = false;
        for (int i = 0; i < 5; ++i) {
            const double r = rms(x, kMlpIn, i, 1.0);
            if (!(r > 1e-30) || !std::isfinite(r)) continue;
            const double ratio = (1.0 / r) / (double)h_scales.in_scale[i];
            if (!scales_set || ratio > 2.0 || ratio < 0.5) {
                ns.in_scale[i] = (float)(1.0 / r);
                changed = true;
            }
        }
        for (int o = 0; o < kMlpOut; ++o) {
            const double r = rms(t, kMlpOut, o, (double)h_scales.out_scale[o]);  // raw target RMS
            if (!(r > 1e-30) || !std::isfinite(r)) continue;
            const double ratio = r / (double)h_scales.out_scale[o];
            if (!scales_set || ratio > 2.0 || ratio < 0.5) {
                ns.out_scale[o] = (float)r;
                changed = true;
            }
        }
        scales_set = true;
        {  // loss of predicting zero on this batch, in the units the network trains in (new scales)
            double z = 0.0;
            for (uint32_t k = 0; k < B; ++k)
                for (int o = 0; o < kMlpOut; ++o) {
                    const double e = (double)t[(size_t)k * kMlpOut + o] * (double)h_scales.out_scale[o] /
                                     (double)ns.out_scale[o];
                    z += e * e;
                }
            zero_loss = z / (double)B;
        }
        if (!changed) return DFSPH_OK;
        std::vector<float> prm(kMlpParams);
        DF_CUDA(cudaMemcpyAsync(prm.data(), mlp.params, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        for (int j = 0; j < kMlpHidden; ++j)
            for (int i = 0; i < kMlpIn; ++i)
                if (ns.in_scale[i] != 0.0f)
                    prm[kW1 + j * kMlpIn + i] *= h_scales.in_scale[i] / ns.in_scale[i];
        for (int o = 0; o < kMlpOut; ++o) {
            const float f = h_scales.out_scale[o] / ns.out_scale[o];
            for (int j = 0; j < kMlpHidden; ++j) prm[kW3 + o * kMlpHidden + j] *= f;
            prm[kB3 + o] *= f;
        }
        DF_CUDA(cudaMemcpyAsync(mlp.params, prm.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaMemsetAsync(mlp.adam_m, 0, kMlpParams * sizeof(float), stream));
        DF_CUDA(cudaMemsetAsync(mlp.adam_v, 0, kMlpParams * sizeof(float), stream));
        adam_t = 0;
        h_scales = ns;
        DF_TRY(upload_scales());  // synchronises: prm goes out of scope
        launch_gather_training<Real>(ds, n, B, offset, div, tx, tt, stream);  // targets / new scale
        launches += 1;
        return DFSPH_OK;
    }

    // One online training round at the end of a step: a batch of this step's (features, needed
    // coefficients) pairs, train_iters Adam steps, then the BF16 inference copies.
    int train_online(bool div) {
        uint32_t B = std::min<uint32_t>(std::min<uint32_t>(train_batch, kMaxTrainBatch), n);
        if (!B) return DFSPH_OK;
        const uint32_t offset = (uint32_t)((lsteps * 2654435761ull) % n);
        launch_gather_training<Real>(ds, n, B, offset, div, tx, tt, stream);
        launches += 1;
        DF_TRY(adapt_scales(B, offset, div));
        if (!h_loss) DF_CUDA(cudaMallocHost((void**)&h_loss, sizeof(double)));
        const bool evaluated = mlp_ready && train_iters > 0;
        for (int it = 0; it < train_iters; ++it) {
            launch_mlp_train_step(mlp, tx, tt, B, 1, (float)lr, 0.9f, 0.999f, 1e-8f, ++adam_t, stream);
            // the first step's loss is the current network's, before it has seen this batch
            if (it == 0) DF_CUDA(cudaMemcpyAsync(h_loss, mlp.loss, sizeof(double), cudaMemcpyDeviceToHost, stream));
        }
        launch_mlp_pack(mlp, stream);
        launches += 1 + 2ull * (uint64_t)train_iters;
        DF_CUDA(cudaStreamSynchronize(stream));
        if (evaluated) {
            heldout_loss = *h_loss;
            net_useful = zero_loss > 0.0 && heldout_loss < useful_ratio * zero_loss;
        }
        mlp_ready = true;
        step_trained = true;
        ++trainings;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int stage_batch(const float* x, const float* t, uint32_t B) {
        DF_CHECK(B > 0 && B <= kMaxTrainBatch, DFSPH_E_INVALID, "batch must be in [1, 65536]");
        DF_CHECK(x, DFSPH_E_INVALID, "null inputs");
        DF_TRY(ensure_mlp());
        DF_CUDA(cudaMemcpyAsync(tx, x, (size_t)B * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (t) DF_CUDA(cudaMemcpyAsync(tt, t, (size_t)B * kMlpOut * sizeof(float), cudaMemcpyHostToDevice, stream));
        return DFSPH_OK;
    }

    int mlp_get_params(float* out, size_t count) {
        DF_CHECK(out && count >= (size_t)kMlpParams, DFSPH_E_INVALID, "output needs DFSPH_MLP_PARAMS floats");
        DF_TRY(ensure_mlp());
        DF_CUDA(cudaMemcpyAsync(out, mlp.params, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        return DFSPH_OK;
    }

    int mlp_set_params(const float* in, size_t count) {
        DF_CHECK(in && count >= (size_t)kMlpParams, DFSPH_E_INVALID, "input needs DFSPH_MLP_PARAMS floats");
        DF_TRY(ensure_mlp());
        DF_CUDA(cudaMemcpyAsync(mlp.params, in, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaMemsetAsync(mlp.adam_m, 0, kMlpParams * sizeof(float), stream));
        DF_CUDA(cudaMemsetAsync(mlp.adam_v, 0, kMlpParams * sizeof(float), stream));
        launch_mlp_pack(mlp, stream);
        launches += 1;
        DF_CUDA(cudaStreamSynchronize(stream));
        adam_t = 0;
        mlp_ready = true;
        net_useful = true;  // a network given by the caller is used as given
        return DFSPH_OK;
    }

    int mlp_get_scales(float* in_scale, float* out_scale) {
        DF_CHECK(in_scale && out_scale, DFSPH_E_INVALID, "null output");
        DF_TRY(ensure_mlp());
        std::memcpy(in_scale, h_scales.in_scale, sizeof(h_scales.in_scale));
        std::memcpy(out_scale, h_scales.out_scale, sizeof(h_scales.out_scale));
        return DFSPH_OK;
    }

    int mlp_set_scales(const float* in_scale, const float* out_scale) {
        DF_CHECK(in_scale && out_scale, DFSPH_E_INVALID, "null input");
        DF_TRY(ensure_mlp());
        for (int o = 0; o < kMlpOut; ++o)
            DF_CHECK(std::isfinite(out_scale[o]) && out_scale[o] != 0.0f, DFSPH_E_INVALID,
                     "output scales must be finite and non-zero");
        std::memcpy(h_scales.in_scale, in_scale, sizeof(h_scales.in_scale));
        std::memcpy(h_scales.out_scale, out_scale, sizeof(h_scales.out_scale));
        DF_TRY(upload_scales());
        scales_set = true;
        return DFSPH_OK;
    }

    int mlp_forward_host(const float* x, uint32_t B, float* y) {
        DF_CHECK(y, DFSPH_E_INVALID, "null output");
        DF_TRY(stage_batch(x, nullptr, B));
        launch_mlp_forward(mlp, tx, B, tt, status, stream);
        launches += 1;
        DF_CUDA(cudaMemcpyAsync(y, tt, (size_t)B * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int mlp_gradient_host(const float* x, const float* t, uint32_t B, float* grad, double* loss) {
        DF_CHECK(t, DFSPH_E_INVALID, "null targets");
        DF_TRY(stage_batch(x, t, B));
        launch_mlp_train_step(mlp, tx, tt, B, 0, 0.0f, 0.9f, 0.999f, 1e-8f, 1, stream);
        launches += 2;
        if (grad)
            DF_CUDA(cudaMemcpyAsync(grad, mlp.grad, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, stream));
        double l = 0.0;
        DF_CUDA(cudaMemcpyAsync(&l, mlp.loss, sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        if (loss) *loss = l;
        return DFSPH_OK;
    }

    int mlp_train_host(const float* x, const float* t, uint32_t B, int iters, double rate, double* loss) {
        DF_CHECK(t, DFSPH_E_INVALID, "null targets");
        DF_CHECK(iters > 0 && rate > 0 && std::isfinite(rate), DFSPH_E_INVALID, "iters and rate must be > 0");
        DF_TRY(stage_batch(x, t, B));
        for (int it = 0; it < iters; ++it)
            launch_mlp_train_step(mlp, tx, tt, B, 1, (float)rate, 0.9f, 0.999f, 1e-8f, ++adam_t, stream);
        launch_mlp_pack(mlp, stream);
        launches += 1 + 2ull * (uint64_t)iters;
        double l = 0.0;
        DF_CUDA(cudaMemcpyAsync(&l, mlp.loss, sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        if (loss) *loss = l;
        mlp_ready = true;
        net_useful = true;  // trained by the caller on its own data: used as given
        return DFSPH_OK;
    }

    // ------------------------------------------------------------------------------------------
    int download(int field, int dtype, void* out, size_t n_elems, int order) {
        DF_CHECK(out, DFSPH_E_INVALID, "null output buffer");
        DF_CHECK(order == DFSPH_ORDER_ID || order == DFSPH_ORDER_SORTED, DFSPH_E_INVALID, "unknown order");
        const Real* src = nullptr;
        int sstride = 1, comps = 1;
        uint32_t count = n;
        const uint32_t* idmap = (order == DFSPH_ORDER_ID) ? id[cur] : nullptr;
        switch (field) {
            case DFSPH_F_POSITION: src = (const Real*)pos[cur]; sstride = 4; comps = 3; break;
            case DFSPH_F_VELOCITY: src = (const Real*)vel[cur]; sstride = 4; comps = 3; break;
            case DFSPH_F_MASS: src = (const Real*)pos[cur] + 3; sstride = 4; comps = 1; break;
            case DFSPH_F_DENSITY: src = density; break;
            case DFSPH_F_FACTOR: src = factor; break;
            case DFSPH_F_DENSITY_ADV: src = densityAdv; break;
            case DFSPH_F_KAPPA: src = kappa[cur]; break;
            case DFSPH_F_KAPPA_V: src = kappaV[cur]; break;
            case DFSPH_F_ACCELERATION: src = (const Real*)acc; sstride = 4; comps = 3; break;
            case DFSPH_F_BOUNDARY_PSI:
                src = (const Real*)bpos[0] + 3; sstride = 4; comps = 1; count = nb;
                idmap = (order == DFSPH_ORDER_ID) ? bid : nullptr;
                break;
            case DFSPH_F_BOUNDARY_POSITION:
                src = (const Real*)bpos[0]; sstride = 4; comps = 3; count = nb;
                idmap = (order == DFSPH_ORDER_ID) ? bid : nullptr;
                break;
            case DFSPH_F_BOUNDARY_VELOCITY:
                src = (const Real*)bvel[0]; sstride = 4; comps = 3; count = nb;
                idmap = (order == DFSPH_ORDER_ID) ? bid : nullptr;
                break;
            case DFSPH_F_BOUNDARY_FORCE:
                DF_CHECK(bforce, DFSPH_E_STATE, "boundary forces are off (set_param boundary_forces 1)");
                launch_force_from_fx<Real>(bforce_fx, nb, bforce, stream);
                launches += 1;
                src = bforce; sstride = 4; comps = 3; count = nb;
                idmap = (order == DFSPH_ORDER_ID) ? bid : nullptr;
                break;
            case DFSPH_F_FEATURES: {
                DF_CHECK(features, DFSPH_E_STATE, "warm-start features exist only after a learned-mode step");
                DF_CHECK(dtype == DFSPH_DTYPE_F32, DFSPH_E_INVALID, "features download as f32");
                DF_CHECK(n_elems >= (size_t)n * kMlpFeatures, DFSPH_E_INVALID, "output buffer too small");
                if (!n) return DFSPH_OK;
                launch_pack_field<float, float>(features, kMlpIn, kMlpFeatures, idmap, n, (float*)dl, stream);
                launches += 1;
                DF_CUDA(cudaMemcpyAsync(out, dl, (size_t)n * kMlpFeatures * sizeof(float), cudaMemcpyDeviceToHost,
                                        stream));
                DF_CUDA(cudaStreamSynchronize(stream));
                return DFSPH_OK;
            }
            case DFSPH_F_ID:
            case DFSPH_F_NEIGHBOR_COUNTS: {
                DF_CHECK(dtype == DFSPH_DTYPE_U32, DFSPH_E_INVALID, "id and neighbour counts download as u32");
                const int c = field == DFSPH_F_ID ? 1 : 2;
                DF_CHECK(n_elems >= (size_t)n * c, DFSPH_E_INVALID, "output buffer too small");
                if (field == DFSPH_F_ID) launch_pack_u32(id[cur], 1, idmap, n, (uint32_t*)dl, stream);
                else launch_unpack_counts(counts, idmap, n, (uint32_t*)dl, stream);
                launches += 1;
                DF_CUDA(cudaMemcpyAsync(out, dl, (size_t)n * c * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
                DF_CUDA(cudaStreamSynchronize(stream));
                return DFSPH_OK;
            }
            default: DF_CHECK(false, DFSPH_E_INVALID, "unknown field");
        }
        DF_CHECK(dtype == DFSPH_DTYPE_F32 || dtype == DFSPH_DTYPE_F64, DFSPH_E_INVALID, "float fields need f32/f64");
        DF_CHECK(n_elems >= (size_t)count * comps, DFSPH_E_INVALID, "output buffer too small");
        if (!count) return DFSPH_OK;
        if (dtype == DFSPH_DTYPE_F32) launch_pack_field<Real, float>(src, sstride, comps, idmap, count, (float*)dl, stream);
        else launch_pack_field<Real, double>(src, sstride, comps, idmap, count, (double*)dl, stream);
        launches += 1;
        const size_t bytes = (size_t)count * comps * (dtype == DFSPH_DTYPE_F32 ? 4 : 8);
        DF_CUDA(cudaMemcpyAsync(out, dl, bytes, cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        if (field == DFSPH_F_DENSITY) {  // the device keeps rho - rho0
            if (dtype == DFSPH_DTYPE_F32)
                for (uint32_t i = 0; i < count; ++i) ((float*)out)[i] = (float)(sc.density0 + ((float*)out)[i]);
            else
                for (uint32_t i = 0; i < count; ++i) ((double*)out)[i] = sc.density0 + ((double*)out)[i];
        }
        return DFSPH_OK;
    }

    // ---- binary checkpoint: the complete solver state, for exact resume ---------------------------
    // Layout: magic, version, sizeof(Real), counts, the scene block, dt history, grid, then the
    // fluid arrays in their current (cell-sorted) order, the boundary arrays in sorted order with
    // their upload indices, and the learned warm-start state when the mode is on. Restoring the
    // internal order (not just the particles) is what makes a resumed run bit-identical.
    static constexpr char kCkptMagic[8] = {'D', 'F', 'S', 'P', 'H', 'C', 'K', '1'};

    template <class T> int dev_to_file(std::ofstream& f, const T* d, size_t count) {
        std::vector<T> h(count);
        if (count) {
            DF_CUDA(cudaMemcpyAsync(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
        }
        f.write(reinterpret_cast<const char*>(h.data()), (std::streamsize)(count * sizeof(T)));
        return DFSPH_OK;
    }
    template <class T> int file_to_dev(std::ifstream& f, T* d, size_t count) {
        std::vector<T> h(count);
        f.read(reinterpret_cast<char*>(h.data()), (std::streamsize)(count * sizeof(T)));
        DF_CHECK((bool)f, DFSPH_E_INVALID, "truncated checkpoint");
        if (count) {
            DF_CUDA(cudaMemcpyAsync(d, h.data(), count * sizeof(T), cudaMemcpyHostToDevice, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
        }
        return DFSPH_OK;
    }
    template <class T> static void put(std::ofstream& f, const T& v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }
    template <class T> static bool get(std::ifstream& f, T& v) { return (bool)f.read(reinterpret_cast<char*>(&v), sizeof(T)); }

    // DFSPHCData::readDynamicData (DFSPH_c_arrays_structure.cpp:1120-1150): positions and velocities
    // in id order with one wait (both packed, both copies queued, then one synchronisation).
    int read_dynamic_data(float* xyz, float* vxyz) {
        DF_CHECK(xyz || vxyz, DFSPH_E_INVALID, "null outputs");
        if (!n) return DFSPH_OK;
        float* px = (float*)dl;
        float* pv = px + 3 * (size_t)n;
        if (xyz) launch_pack_field<Real, float>((const Real*)pos[cur], 4, 3, id[cur], n, px, stream);
        if (vxyz) launch_pack_field<Real, float>((const Real*)vel[cur], 4, 3, id[cur], n, pv, stream);
        if (xyz) DF_CUDA(cudaMemcpyAsync(xyz, px, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, stream));
        if (vxyz) DF_CUDA(cudaMemcpyAsync(vxyz, pv, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        launches += (xyz ? 1 : 0) + (vxyz ? 1 : 0);
        return DFSPH_OK;
    }

    // Force and torque of the fluid on boundary bodies (readDynamicObjectsData + the rigid-body
    // solver's sum over the body's particles): bodies are ranges of the boundary upload order.
    double* wrench_buf = nullptr;  // 6 Bc doubles (positions, forces in upload order) + bodies
    size_t wrench_cap = 0;
    int body_wrench(uint32_t nbod, const uint32_t* first, const uint32_t* count, const double* centers,
                    double* out) {
        DF_CHECK(bforce, DFSPH_E_STATE, "boundary forces are off (set_param boundary_forces 1)");
        DF_CHECK(nbod == 0 || (first && count && centers && out), DFSPH_E_INVALID, "null body arrays");
        for (uint32_t b = 0; b < nbod; ++b)
            DF_CHECK((uint64_t)first[b] + count[b] <= nb, DFSPH_E_INVALID, "body range beyond the boundary particles");
        if (!nbod) return DFSPH_OK;
        const size_t need = 6 * (size_t)Bc + (size_t)nbod * (2 + 3 + 6);
        if (need > wrench_cap) {
            if (wrench_buf) cudaFree(wrench_buf);
            wrench_buf = nullptr;
            DF_TRY(dalloc(&wrench_buf, need));
            wrench_cap = need;
        }
        double* xp = wrench_buf;
        double* fp = wrench_buf + 3 * (size_t)Bc;
        uint32_t* dfirst = (uint32_t*)(wrench_buf + 6 * (size_t)Bc);
        uint32_t* dcount = dfirst + nbod;
        double* dcent = wrench_buf + 6 * (size_t)Bc + nbod;  // 2 nbod uint32 = nbod doubles
        double* dout = dcent + 3 * (size_t)nbod;
        if (nb) {
            launch_pack_field<Real, double>((const Real*)bpos[0], 4, 3, bid, nb, xp, stream);
            launch_force_from_fx<Real>(bforce_fx, nb, bforce, stream);
            launch_pack_field<Real, double>(bforce, 4, 3, bid, nb, fp, stream);
        }
        DF_CUDA(cudaMemcpyAsync(dfirst, first, nbod * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaMemcpyAsync(dcount, count, nbod * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        DF_CUDA(cudaMemcpyAsync(dcent, centers, 3 * nbod * sizeof(double), cudaMemcpyHostToDevice, stream));
        launch_body_wrench(xp, fp, dfirst, dcount, dcent, nbod, dout, stream);
        DF_CUDA(cudaMemcpyAsync(out, dout, 6 * nbod * sizeof(double), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        DF_CUDA(cudaGetLastError());
        launches += nb ? 3 : 1;
        return DFSPH_OK;
    }

    // The fluid as a partio particle file (partioExport, Demos/StaticBoundaryDemo/main.cpp:485-496).
    int export_bgeo(const char* path) {
        DF_CHECK(path, DFSPH_E_INVALID, "null path");
        std::vector<float> x((size_t)n * 3), v((size_t)n * 3);
        if (n) {
            DF_TRY(download(DFSPH_F_POSITION, DFSPH_DTYPE_F32, x.data(), x.size(), DFSPH_ORDER_ID));
            DF_TRY(download(DFSPH_F_VELOCITY, DFSPH_DTYPE_F32, v.data(), v.size(), DFSPH_ORDER_ID));
        }
        std::string err;
        DF_CHECK(bgeo_write(path, n, x.data(), v.data(), (float)sc.particle_radius, err), DFSPH_E_INVALID, err);
        return DFSPH_OK;
    }

    int save_checkpoint(const char* path) {
        DF_CHECK(path, DFSPH_E_INVALID, "null path");
        DF_CHECK(grid_ready, DFSPH_E_STATE, "nothing to checkpoint");
        DF_TRY(bin_boundary_now());  // the file keeps the boundary in its sorted order
        DF_TRY(pull_dt());
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        DF_CHECK(f.is_open(), DFSPH_E_INVALID, std::string("cannot open ") + path);
        f.write(kCkptMagic, 8);
        put(f, (int32_t)4);
        put(f, (int32_t)sizeof(Real));
        put(f, n);
        put(f, nb);
        put(f, sc);
        for (double v : {h, h_future, h_past, inv_h, inv_h_future, h_ratio, h_ratio2, time_step}) put(f, v);
        for (int a = 0; a < 3; ++a) put(f, (int32_t)off[a]);
        for (int a = 0; a < 3; ++a) put(f, (int32_t)dim[a]);
        put(f, (int32_t)(boundary_moving ? 1 : 0));
        put(f, (int32_t)(learned ? 1 : 0));
        DF_TRY(dev_to_file(f, pos[cur], n));
        DF_TRY(dev_to_file(f, vel[cur], n));
        DF_TRY(dev_to_file(f, kappa[cur], n));
        DF_TRY(dev_to_file(f, kappaV[cur], n));
        DF_TRY(dev_to_file(f, id[cur], n));
        DF_TRY(dev_to_file(f, bpos[0], nb));
        DF_TRY(dev_to_file(f, bvel[0], nb));
        DF_TRY(dev_to_file(f, bid, nb));
        if (learned) {
            DF_TRY(dev_to_file(f, kappaT[cur], n));
            DF_TRY(dev_to_file(f, kappaVT[cur], n));
            DF_TRY(dev_to_file(f, mlp.params, (size_t)kMlpParams));
            DF_TRY(dev_to_file(f, mlp.adam_m, (size_t)kMlpParams));
            DF_TRY(dev_to_file(f, mlp.adam_v, (size_t)kMlpParams));
            put(f, h_scales);
            for (int32_t v : {adam_t, (int32_t)mlp_ready, (int32_t)scales_set, (int32_t)probe, train_interval,
                              train_start, train_iters, (int32_t)train_batch})
                put(f, v);
            for (double v : {lr, damping}) put(f, v);
            for (uint64_t v : {lsteps, trainings, kept_v, kept_p, solves_v, solves_p}) put(f, v);
            put(f, mlp_seed);
            // cost gate (version 2): its schedule, and the iterations counted so far in its phase
            uint32_t it = 0, itv = 0;
            DF_TRY(gate_sums(it, itv));
            for (int32_t v : {(int32_t)gate, gate_period, gate_window, gate_recheck, gate_phase, gate_left, gate_len})
                put(f, v);
            for (uint32_t v : {it - gate_it0, itv - gate_itv0}) put(f, v);
            for (double v : {gate_margin, gate_last_excess}) put(f, v);
            for (uint64_t v : {gate_learned_steps, gate_plain_steps}) put(f, v);
            // version 3: whether the network's correction is in use, and the losses that decided it
            put(f, (int32_t)(net_useful ? 1 : 0));
            put(f, (int32_t)(last_lp ? 1 : 0));
            for (double v : {useful_ratio, zero_loss, heldout_loss}) put(f, v);
        }
        put(f, inflow_mass);  // version 4
        DF_CHECK(f.good(), DFSPH_E_INVALID, std::string("write failed: ") + path);
        return DFSPH_OK;
    }

    int load_checkpoint(const char* path) {
        DF_CHECK(path, DFSPH_E_INVALID, "null path");
        std::ifstream f(path, std::ios::binary);
        DF_CHECK(f.is_open(), DFSPH_E_INVALID, std::string("cannot open ") + path);
        char magic[8];
        f.read(magic, 8);
        DF_CHECK(f && std::memcmp(magic, kCkptMagic, 8) == 0, DFSPH_E_INVALID, "not a DFSPH checkpoint");
        int32_t version = 0, rbytes = 0;
        uint32_t cn = 0, cnb = 0;
        dfsph_scene csc{};
        DF_CHECK(get(f, version) && version >= 1 && version <= 4 && get(f, rbytes) && get(f, cn) && get(f, cnb) &&
                     get(f, csc),
                 DFSPH_E_INVALID, "bad checkpoint header");
        DF_CHECK(rbytes == (int32_t)sizeof(Real), DFSPH_E_INVALID, "checkpoint precision differs from the context's");
        DF_CHECK(cn <= Nc && cnb <= Bc, DFSPH_E_INVALID, "checkpoint exceeds the context's capacities");
        DF_CHECK(csc.neighbor_capacity == sc.neighbor_capacity, DFSPH_E_INVALID, "neighbor_capacity differs");
        double dt[8];
        for (double& v : dt) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
        int32_t g[6], moving = 0, was_learned = 0;
        for (int32_t& v : g) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
        DF_CHECK(get(f, moving) && get(f, was_learned), DFSPH_E_INVALID, "truncated checkpoint");
        // scene parameters of the run; this context keeps its own capacities, device and graph mode
        csc.fluid_capacity = sc.fluid_capacity;
        csc.boundary_capacity = sc.boundary_capacity;
        csc.device = sc.device;
        csc.use_graphs = sc.use_graphs;
        sc = csc;
        for (int a = 0; a < 3; ++a) {
            off[a] = g[a];
            dim[a] = g[3 + a];
            DF_CHECK(dim[a] > 0 && dim[a] <= 1024, DFSPH_E_INVALID, "bad grid in checkpoint");
        }
        DF_TRY(alloc_grid());
        grid_ready = true;
        invalidate_graphs();
        n = cn;
        nb = cnb;
        cur = 0;
        DF_TRY(file_to_dev(f, pos[0], n));
        DF_TRY(file_to_dev(f, vel[0], n));
        DF_TRY(file_to_dev(f, kappa[0], n));
        DF_TRY(file_to_dev(f, kappaV[0], n));
        DF_TRY(file_to_dev(f, id[0], n));
        DF_TRY(file_to_dev(f, bpos[1], nb));  // sorted order; re-sorting keeps it and rebuilds the table
        DF_TRY(file_to_dev(f, bvel[1], nb));
        std::vector<uint32_t> saved_bid(nb);
        f.read(reinterpret_cast<char*>(saved_bid.data()), (std::streamsize)(nb * sizeof(uint32_t)));
        DF_CHECK((bool)f, DFSPH_E_INVALID, "truncated checkpoint");
        if (nb) {
            DF_TRY(sort_boundary(false));
            DF_CUDA(cudaMemcpyAsync(bid, saved_bid.data(), nb * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }
        boundary_moving = moving != 0;
        bin_rigid = bshifted = false;  // the next rigid motion re-bins
        for (int a = 0; a < 3; ++a) bin_p[a] = bshift_d[a] = 0.0;
        DF_CUDA(cudaMemsetAsync(counts, 0, (size_t)Nc * sizeof(uint32_t), stream));
        DF_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(uint32_t), stream));
        if (was_learned) {
            learned = false;
            DF_TRY(enable_learned(true));
            DF_TRY(file_to_dev(f, kappaT[0], n));
            DF_TRY(file_to_dev(f, kappaVT[0], n));
            DF_TRY(file_to_dev(f, mlp.params, (size_t)kMlpParams));
            DF_TRY(file_to_dev(f, mlp.adam_m, (size_t)kMlpParams));
            DF_TRY(file_to_dev(f, mlp.adam_v, (size_t)kMlpParams));
            int32_t iv[8];
            double dv[2];
            uint64_t uv[6];
            DF_CHECK(get(f, h_scales), DFSPH_E_INVALID, "truncated checkpoint");
            for (int32_t& v : iv) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
            for (double& v : dv) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
            for (uint64_t& v : uv) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
            DF_CHECK(get(f, mlp_seed), DFSPH_E_INVALID, "truncated checkpoint");
            adam_t = iv[0];
            mlp_ready = iv[1] != 0;
            scales_set = iv[2] != 0;
            probe = iv[3] != 0;
            train_interval = iv[4];
            train_start = iv[5];
            train_iters = iv[6];
            train_batch = (uint32_t)iv[7];
            lr = dv[0];
            damping = dv[1];
            lsteps = uv[0]; trainings = uv[1]; kept_v = uv[2]; kept_p = uv[3]; solves_v = uv[4]; solves_p = uv[5];
            if (version >= 2) {
                int32_t gi[7];
                uint32_t part[2];
                double gd[2];
                uint64_t gu[2];
                for (int32_t& v : gi) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
                for (uint32_t& v : part) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
                for (double& v : gd) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
                for (uint64_t& v : gu) DF_CHECK(get(f, v), DFSPH_E_INVALID, "truncated checkpoint");
                gate = gi[0] != 0;
                gate_period = gi[1];
                gate_window = gi[2];
                gate_recheck = gi[3];
                gate_phase = gi[4];
                gate_left = gi[5];
                gate_len = gi[6];
                gate_margin = gd[0];
                gate_last_excess = gd[1];
                gate_learned_steps = gu[0];
                gate_plain_steps = gu[1];
                uint32_t it = 0, itv = 0;  // this context's counters: keep the phase's partial sums
                DF_TRY(gate_sums(it, itv));
                gate_it0 = it - part[0];
                gate_itv0 = itv - part[1];
            }
            if (version >= 3) {
                int32_t used = 0, prev = 0;
                DF_CHECK(get(f, used) && get(f, prev) && get(f, useful_ratio) && get(f, zero_loss) &&
                             get(f, heldout_loss),
                         DFSPH_E_INVALID, "truncated checkpoint");
                net_useful = used != 0;
                last_lp = prev != 0;
            } else {
                net_useful = mlp_ready;  // earlier files: the network was used whenever trained
                last_lp = false;
            }
            DF_TRY(upload_scales());
            launch_mlp_pack(mlp, stream);
            launches += 1;
        } else if (learned) {
            DF_TRY(enable_learned(false));
        }
        if (version >= 4) {
            DF_CHECK(get(f, inflow_mass), DFSPH_E_INVALID, "truncated checkpoint");
        } else {  // earlier files: the default mass
            const double d = 2.0 * sc.particle_radius;
            inflow_mass = (float)(0.8 * d * d * d * sc.density0);
        }
        h = dt[0]; h_future = dt[1]; h_past = dt[2]; inv_h = dt[3]; inv_h_future = dt[4];
        h_ratio = dt[5]; h_ratio2 = dt[6]; time_step = dt[7];
        use_graphs = sc.use_graphs != 0;
        push_dt();
        DF_TRY(sync_state());
        DF_CUDA(cudaStreamSynchronize(stream));
        return DFSPH_OK;
    }

    // ---- snapshots (reference text format, see dfsph_c.h) -----------------------------------------
    static std::string join(const char* dir, const char* name) {
        std::string d(dir);
        if (!d.empty() && d.back() != '/') d += '/';
        return d + name;
    }

    int write_set(const std::string& path, bool boundary) {
        const uint32_t count = boundary ? nb : n;
        std::vector<float> x((size_t)count * 3), v((size_t)count * 3), m(count);
        if (count) {
            DF_TRY(download(boundary ? DFSPH_F_BOUNDARY_POSITION : DFSPH_F_POSITION, DFSPH_DTYPE_F32, x.data(),
                            x.size(), DFSPH_ORDER_ID));
            DF_TRY(download(boundary ? DFSPH_F_BOUNDARY_VELOCITY : DFSPH_F_VELOCITY, DFSPH_DTYPE_F32, v.data(),
                            v.size(), DFSPH_ORDER_ID));
            DF_TRY(download(boundary ? DFSPH_F_BOUNDARY_PSI : DFSPH_F_MASS, DFSPH_DTYPE_F32, m.data(), m.size(),
                            DFSPH_ORDER_ID));
        }
        std::ofstream f(path, std::ios::trunc);
        DF_CHECK(f.is_open(), DFSPH_E_INVALID, "cannot open " + path + " for writing");
        f << std::setprecision(9);
        f << count << (boundary ? " 0 0 0" : " 1 1 0") << "\n";
        for (uint32_t i = 0; i < count; ++i)
            f << m[i] << " " << x[3 * i] << " " << x[3 * i + 1] << " " << x[3 * i + 2] << " " << v[3 * i] << " "
              << v[3 * i + 1] << " " << v[3 * i + 2] << " \n";
        DF_CHECK(f.good(), DFSPH_E_INVALID, "write failed: " + path);
        return DFSPH_OK;
    }

    // Reads a particle file (UnifiedParticleSet::load_from_file); a dynamic-body line is skipped.
    int read_set(const std::string& path, std::vector<float>& m, std::vector<float>& x, std::vector<float>& v) {
        std::ifstream f(path);
        DF_CHECK(f.is_open(), DFSPH_E_INVALID, "cannot open " + path);
        long long count = -1;
        int has_factor = 0, vel_impacted = 0, dynamic = 0;
        f >> count >> has_factor >> vel_impacted >> dynamic;
        DF_CHECK(f.good() && count >= 0 && count <= (long long)UINT32_MAX, DFSPH_E_INVALID, "bad header in " + path);
        if (dynamic) {  // position, velocity, quaternion (v, s), angular velocity of the rigid body
            double skip;
            for (int k = 0; k < 13; ++k) f >> skip;
        }
        m.resize((size_t)count);
        x.resize((size_t)count * 3);
        v.resize((size_t)count * 3);
        for (long long i = 0; i < count; ++i) {
            f >> m[i] >> x[3 * i] >> x[3 * i + 1] >> x[3 * i + 2] >> v[3 * i] >> v[3 * i + 1] >> v[3 * i + 2];
            DF_CHECK(!f.fail(), DFSPH_E_INVALID, "truncated particle file " + path);
        }
        return DFSPH_OK;
    }

    int save_snapshot(const char* dir, int what) {
        DF_CHECK(dir, DFSPH_E_INVALID, "null directory");
        DF_TRY(pull_dt());
        if (what & DFSPH_SNAP_FLUID) {
            DF_TRY(write_set(join(dir, "fluid_file.txt"), false));
            std::ofstream g(join(dir, "general_data.txt"), std::ios::trunc);
            DF_CHECK(g.is_open(), DFSPH_E_INVALID, "cannot write general_data.txt");
            g << std::setprecision(17) << h;
        }
        if (what & DFSPH_SNAP_BOUNDARY) DF_TRY(write_set(join(dir, "boundaries_file.txt"), true));
        return DFSPH_OK;
    }

    int load_snapshot(const char* dir, int what, bool load_velocities) {
        DF_CHECK(dir, DFSPH_E_INVALID, "null directory");
        std::vector<float> m, x, v;
        if (what & DFSPH_SNAP_BOUNDARY) {
            DF_TRY(read_set(join(dir, "boundaries_file.txt"), m, x, v));
            DF_CHECK(x.size() / 3 <= Bc, DFSPH_E_INVALID, "boundary file exceeds boundary_capacity");
            DF_TRY(set_boundary(x.data(), nullptr, (uint32_t)(x.size() / 3)));  // psi recomputed
            if (load_velocities && !x.empty()) {
                bool any = false;
                for (float e : v) any = any || e != 0.0f;
                if (any) DF_TRY(move_boundary(x.data(), v.data()));
            }
        }
        if (what & DFSPH_SNAP_FLUID) {
            DF_TRY(read_set(join(dir, "fluid_file.txt"), m, x, v));
            DF_CHECK(x.size() / 3 <= Nc, DFSPH_E_INVALID, "fluid file exceeds fluid_capacity");
            std::ifstream g(join(dir, "general_data.txt"));
            double hs = 0.0;
            DF_CHECK(g.is_open() && (g >> hs) && hs > 0 && std::isfinite(hs), DFSPH_E_INVALID,
                     "general_data.txt missing or without a positive time step");
            DF_TRY(upload_fluid(x.data(), load_velocities ? v.data() : nullptr, m.data(), (uint32_t)(x.size() / 3)));
            // updateTimeStep(h) + onSimulationStepEnd() twice: h = h_future = h_past = stored step
            time_step = hs;
            reset_dt();
            DF_TRY(sync_state());
        }
        return DFSPH_OK;
    }

    int get_neighbors(uint32_t* cnt_out, uint32_t* lists_out, uint32_t row) {
        DF_CHECK(cnt_out && lists_out, DFSPH_E_INVALID, "null output");
        DF_CHECK(row >= cap, DFSPH_E_INVALID, "row length smaller than neighbor_capacity");
        if (!n) return DFSPH_OK;
        std::vector<uint32_t> c(n), t((size_t)cap * stride), ids(n), bids(std::max<uint32_t>(nb, 1));
        DF_CUDA(cudaMemcpyAsync(c.data(), counts, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(t.data(), nbr, t.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(ids.data(), id[cur], n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        if (nb) DF_CUDA(cudaMemcpyAsync(bids.data(), bid, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t me = ids[i];
            const uint32_t nf = c[i] & 0xFFFFu, nbc = c[i] >> 16;
            cnt_out[2 * (size_t)me] = nf;
            cnt_out[2 * (size_t)me + 1] = nbc;
            for (uint32_t k = 0; k < nf + nbc && k < cap; ++k) {
                const uint32_t j = t[(size_t)k * stride + i];
                lists_out[(size_t)me * row + k] = (k < nf) ? ids[j] : bids[j];
            }
        }
        return DFSPH_OK;
    }

    int set_param(const std::string& k, double v) {
        bool dt_changed = false;
        if (k == "viscosity") sc.viscosity = v;
        else if (k == "density0") sc.density0 = v;
        else if (k == "max_error") sc.max_error = v;
        else if (k == "max_error_v") sc.max_error_v = v;
        else if (k == "max_iterations") sc.max_iterations = (int32_t)v;
        else if (k == "max_iterations_v") sc.max_iterations_v = (int32_t)v;
        else if (k == "enable_divergence_solver") sc.enable_divergence_solver = (int32_t)v;
        else if (k == "cfl_method") sc.cfl_method = (int32_t)v;
        else if (k == "cfl_factor") sc.cfl_factor = v;
        else if (k == "cfl_max_time_step") sc.cfl_max_time_step = v;
        else if (k == "cfl_min_time_step") sc.cfl_min_time_step = v;
        else if (k == "time_step") {
            DF_CHECK(v > 0, DFSPH_E_INVALID, "time_step must be > 0");
            DF_TRY(pull_dt());
            time_step = v;
            dt_changed = true;
        }
        else if (k == "gravitation_x") sc.gravitation[0] = v;
        else if (k == "gravitation_y") sc.gravitation[1] = v;
        else if (k == "gravitation_z") sc.gravitation[2] = v;
        else if (k == "use_graphs") { use_graphs = v != 0; }
        else if (k == "h") { DF_TRY(pull_dt()); h = v; dt_changed = true; }
        else if (k == "h_future") { DF_TRY(pull_dt()); h_future = v; dt_changed = true; }
        else if (k == "h_past") { DF_TRY(pull_dt()); h_past = v; dt_changed = true; }
        else if (k == "inv_h") { DF_TRY(pull_dt()); inv_h = v; dt_changed = true; }
        else if (k == "iterations_sum") {  // clears both loops' iteration counters
            if (gate) {  // the gate's start counts move with the counters (its partial sums stay)
                uint32_t it = 0, itv = 0;
                DF_TRY(gate_sums(it, itv));
                gate_it0 -= it;
                gate_itv0 -= itv;
            }
            DF_CUDA(cudaMemsetAsync(&ctl[0].iter_sum, 0, sizeof(uint32_t), stream));
            DF_CUDA(cudaMemsetAsync(&ctl[1].iter_sum, 0, sizeof(uint32_t), stream));
        }
        else if (k == "timing") timing = v != 0;
        else if (k == "learned_warm_start") return enable_learned(v != 0);
        else if (k == "warm_start_probe") probe = v != 0;
        else if (k == "learned_base_only") base_only = v != 0;
        else if (k == "network_useful_ratio") {
            DF_CHECK(v >= 0, DFSPH_E_INVALID, "network_useful_ratio must be >= 0");
            useful_ratio = v;
        }
        else if (k == "checked_corrupt_neighbor") {
#ifdef DFSPH_CHECKED
            DF_CHECK(v >= 1 && v <= 64 && n + (uint32_t)v <= Nc, DFSPH_E_INVALID,
                     "checked_corrupt_neighbor must be in [1, 64] and stay inside fluid_capacity");
            corrupt_neighbor = (uint32_t)v;
#else
            DF_CHECK(false, DFSPH_E_INVALID, "checked_corrupt_neighbor exists only in the checked build");
#endif
        }
        else if (k == "sort_withhold_tile") sort_withheld_tile = v < 0 ? kNoWithheldTile : (uint32_t)v;
        else if (k == "remove_escaped") remove_escaped = v != 0;
        else if (k == "inflow_mass") {
            DF_CHECK(v > 0 && std::isfinite(v), DFSPH_E_INVALID, "inflow_mass must be positive");
            inflow_mass = (float)v;
        }
        else if (k == "boundary_forces") {
            if (v != 0 && !bforce) {
                DF_TRY(dalloc(&bforce, (size_t)Bc * 4));
                DF_TRY(dalloc(&bforce_fx, (size_t)Bc * 3));
                DF_CUDA(cudaMemsetAsync(bforce, 0, (size_t)Bc * 4 * sizeof(Real), stream));
                DF_CUDA(cudaMemsetAsync(bforce_fx, 0, (size_t)Bc * 3 * sizeof(unsigned long long), stream));
            }
            boundary_forces = v != 0;
            invalidate_graphs();  // the loop graphs read the DevState block; rebuilt for clarity
        }
        else if (k == "warm_start_damping") {
            DF_CHECK(v > 0 && v <= 1, DFSPH_E_INVALID, "warm_start_damping must be in (0, 1]");
            damping = v;
        }
        else if (k == "learned_gate") {
            gate = v != 0;
            gate_phase = kGateLearned;  // the schedule starts with a probe window
            gate_left = 0;
        }
        else if (k == "gate_period") { DF_CHECK(v >= 1, DFSPH_E_INVALID, "gate_period must be >= 1"); gate_period = (int)v; }
        else if (k == "gate_window") { DF_CHECK(v >= 1, DFSPH_E_INVALID, "gate_window must be >= 1"); gate_window = (int)v; }
        else if (k == "gate_recheck") { DF_CHECK(v >= 1, DFSPH_E_INVALID, "gate_recheck must be >= 1"); gate_recheck = (int)v; }
        else if (k == "gate_margin") { DF_CHECK(v >= 0, DFSPH_E_INVALID, "gate_margin must be >= 0"); gate_margin = v; }
        else if (k == "train_interval") { DF_CHECK(v >= 0, DFSPH_E_INVALID, "train_interval must be >= 0"); train_interval = (int)v; }
        else if (k == "train_start") { DF_CHECK(v >= 0, DFSPH_E_INVALID, "train_start must be >= 0"); train_start = (int)v; }
        else if (k == "train_iters") { DF_CHECK(v >= 0, DFSPH_E_INVALID, "train_iters must be >= 0"); train_iters = (int)v; }
        else if (k == "train_batch") {
            DF_CHECK(v >= 1 && v <= kMaxTrainBatch, DFSPH_E_INVALID, "train_batch must be in [1, 65536]");
            train_batch = (uint32_t)v;
        }
        else if (k == "learning_rate") { DF_CHECK(v > 0, DFSPH_E_INVALID, "learning_rate must be > 0"); lr = v; }
        else if (k == "mlp_seed") {
            DF_CHECK(v >= 0 && v < 4294967296.0, DFSPH_E_INVALID, "mlp_seed must fit 32 bits");
            if (!mlp.params) {
                mlp_seed = (uint32_t)v;
                return DFSPH_OK;
            }
            return mlp_reset((uint32_t)v);
        }
        else DF_CHECK(false, DFSPH_E_INVALID, "unknown parameter key: " + k);
        if (dt_changed) push_dt();
        return sync_state();
    }

    int get_param(const std::string& k, double* v) {
        DF_CHECK(v, DFSPH_E_INVALID, "null output");
        if (k == "h" || k == "h_future" || k == "h_past" || k == "inv_h" || k == "h_ratio_to_past" ||
            k == "h_ratio_to_past2")
            DF_TRY(pull_dt());
        if (k == "iterations_sum" || k == "iterations_v_sum") {
            LoopCtl c[2];
            DF_CUDA(cudaMemcpyAsync(c, ctl, 2 * sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            *v = k == "iterations_sum" ? c[1].iter_sum : c[0].iter_sum;
            return DFSPH_OK;
        }
        if (k == "viscosity") *v = sc.viscosity;
        else if (k == "density0") *v = sc.density0;
        else if (k == "max_error") *v = sc.max_error;
        else if (k == "max_error_v") *v = sc.max_error_v;
        else if (k == "max_iterations") *v = sc.max_iterations;
        else if (k == "max_iterations_v") *v = sc.max_iterations_v;
        else if (k == "enable_divergence_solver") *v = sc.enable_divergence_solver;
        else if (k == "cfl_method") *v = sc.cfl_method;
        else if (k == "cfl_factor") *v = sc.cfl_factor;
        else if (k == "cfl_max_time_step") *v = sc.cfl_max_time_step;
        else if (k == "cfl_min_time_step") *v = sc.cfl_min_time_step;
        else if (k == "time_step") *v = time_step;
        else if (k == "use_graphs") *v = use_graphs ? 1 : 0;
        else if (k == "h") *v = h;
        else if (k == "h_future") *v = h_future;
        else if (k == "h_past") *v = h_past;
        else if (k == "inv_h") *v = inv_h;
        else if (k == "h_ratio_to_past") *v = h_ratio;
        else if (k == "h_ratio_to_past2") *v = h_ratio2;
        else if (k == "timing") *v = timing ? 1 : 0;
        else if (k == "num_boundary") *v = nb;
        else if (k == "grid_dim_x") *v = dim[0];
        else if (k == "grid_dim_y") *v = dim[1];
        else if (k == "grid_dim_z") *v = dim[2];
        else if (k == "grid_offset_x") *v = off[0];
        else if (k == "grid_offset_y") *v = off[1];
        else if (k == "grid_offset_z") *v = off[2];
        else if (k == "sort_passes") *v = key_passes;
        else if (k == "iterations") *v = last_iters;
        else if (k == "iterations_v") *v = last_iters_v;
        else if (k == "learned_warm_start") *v = learned ? 1 : 0;
        else if (k == "warm_start_probe") *v = probe ? 1 : 0;
        else if (k == "learned_base_only") *v = base_only ? 1 : 0;
        else if (k == "network_useful_ratio") *v = useful_ratio;
        else if (k == "network_used") *v = net_useful ? 1 : 0;
        else if (k == "mlp_heldout_ratio") *v = zero_loss > 0 ? heldout_loss / zero_loss : -1.0;
        else if (k == "checked_build") {
#ifdef DFSPH_CHECKED
            *v = 1;
#else
            *v = 0;
#endif
        }
        else if (k == "boundary_forces") *v = boundary_forces ? 1 : 0;
        else if (k == "remove_escaped") *v = remove_escaped ? 1 : 0;
        else if (k == "boundary_shift_active") *v = bshifted ? 1 : 0;
        else if (k == "inflow_mass") *v = new_particle_mass();
        else if (k == "escaped_removed") *v = (double)escaped_removed;
        else if (k == "warm_start_damping") *v = damping;
        else if (k == "learned_gate") *v = gate ? 1 : 0;
        else if (k == "gate_period") *v = gate_period;
        else if (k == "gate_window") *v = gate_window;
        else if (k == "gate_recheck") *v = gate_recheck;
        else if (k == "gate_margin") *v = gate_margin;
        else if (k == "gate_learned_steps") *v = (double)gate_learned_steps;
        else if (k == "gate_plain_steps") *v = (double)gate_plain_steps;
        else if (k == "gate_last_excess") *v = gate_last_excess;
        else if (k == "train_interval") *v = train_interval;
        else if (k == "train_start") *v = train_start;
        else if (k == "train_iters") *v = train_iters;
        else if (k == "train_batch") *v = train_batch;
        else if (k == "learning_rate") *v = lr;
        else if (k == "mlp_seed") *v = mlp_seed;
        else if (k == "mlp_ready") *v = mlp_ready ? 1 : 0;
        else if (k == "mlp_trainings") *v = (double)trainings;
        else if (k == "mlp_adam_steps") *v = adam_t;
        else if (k == "learned_kept_v") *v = (double)kept_v;
        else if (k == "learned_kept_p") *v = (double)kept_p;
        else if (k == "learned_solves_v") *v = (double)solves_v;
        else if (k == "learned_solves_p") *v = (double)solves_p;
        else if (k == "mlp_loss") {
            double l = 0.0;
            if (mlp.loss) {
                DF_CUDA(cudaMemcpyAsync(&l, mlp.loss, sizeof(double), cudaMemcpyDeviceToHost, stream));
                DF_CUDA(cudaStreamSynchronize(stream));
            }
            *v = l;
        }
        else DF_CHECK(false, DFSPH_E_INVALID, "unknown parameter key: " + k);
        return DFSPH_OK;
    }

    void launch_kernel(int k) {
        switch (k) {
            case DFSPH_K_NEIGHBOR_BUILD: launch_build_neighbors<Real>(ds, n, ftab, btab, stream, bshifted); break;
            case DFSPH_K_DENSITY_ALPHA: launch_density_alpha<Real>(ds, n, false, false, stream); break;
            case DFSPH_K_DIVERGENCE_JACOBI: launch_divergence_jacobi<Real>(ds, n, 0, false, stream); break;
            case DFSPH_K_DIVERGENCE_RESIDUAL:
                launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream);
                break;
            case DFSPH_K_VISCOSITY: launch_viscosity<Real>(ds, n, false, stream); break;
            case DFSPH_K_PRESSURE_WARM_JACOBI:
                launch_pressure_warm_jacobi<Real>(ds, n, false, nullptr, nullptr, stream);
                break;
            case DFSPH_K_PRESSURE_RESIDUAL:
                launch_pressure_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream);
                break;
            case DFSPH_K_PRESSURE_JACOBI: launch_pressure_jacobi<Real>(ds, n, 0, false, stream); break;
            case DFSPH_K_UPDATE_POS: launch_update_pos<Real>(ds, n, stream); break;
            default: break;
        }
        launches += 1;
    }

    int time_kernel(int k, int reps, double* ms) {
        DF_CHECK(ms, DFSPH_E_INVALID, "null output");
        DF_CHECK(k >= 0 && k < DFSPH_K_COUNT && reps > 0, DFSPH_E_INVALID, "bad kernel id or reps");
        DF_CHECK(n > 0, DFSPH_E_STATE, "no fluid");
        double total = 0.0;
        for (int r = 0; r < reps; ++r) {
            DF_CUDA(cudaEventRecord(ev0, stream));
            if (k == DFSPH_K_SORT_REORDER) {
                // keys -> radix sort -> reorder -> cell table: the first part of the neighbour search
                const StepParams<Real> p = params();
                launch_cell_keys<Real>(pos[cur], n, p, sb.keys_a, status, stream);
                uint32_t *skeys, *perm;
                radix_sort_pairs(sb, n, key_passes, true, stream, status, &launches, &skeys, &perm);
                const int nx = 1 - cur;
                launch_reorder_fluid<Real>(perm, n, pos[cur], vel[cur], kappa[cur], kappaV[cur], id[cur], pos[nx],
                                           vel[nx], kappa[nx], kappaV[nx], id[nx], stream);
                if (learned) {
                    launch_reorder_pair<Real>(perm, n, kappaT[cur], kappaVT[cur], kappaT[nx], kappaVT[nx], stream);
                    launches += 1;
                }
                DF_CUDA(cudaMemsetAsync(ftab, 0, cells * sizeof(uint2), stream));
                launch_cell_bounds(skeys, n, dim[0], dim[1], dim[2], ftab, stream);
                cur = nx;
                launches += 3;
                launch_set_state<Real>(ds, (hs.pos = pos[cur], hs.vel = vel[cur], hs.kappa = kappa[cur],
                                            hs.kappaV = kappaV[cur], hs.id = id[cur], hs.kappaT = kappaT[cur],
                                            hs.kappaVT = kappaVT[cur], hs), stream);
            } else {
                launch_kernel(k);
            }
            DF_CUDA(cudaEventRecord(ev1, stream));
            DF_CUDA(cudaEventSynchronize(ev1));
            float t = 0.0f;
            DF_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
            total += t;
        }
        DF_CUDA(cudaGetLastError());
        *ms = total / reps;
        return DFSPH_OK;
    }

    int get_status(uint32_t* out, int clear) {
        DF_CUDA(cudaMemcpyAsync(h_status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
        uint32_t st = h_status[0];
        if (out) *out = st;
        if (clear) DF_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(uint32_t), stream));
        return DFSPH_OK;
    }
};

}  // namespace dfsph

struct dfsph_ctx {
    std::string err;
    int device = 0;
    std::unique_ptr<dfsph::Solver<float>> f32;
    std::unique_ptr<dfsph::Solver<double>> f64;
};

#define DFSPH_DISPATCH(ctx, call)                                                              \
    do {                                                                                       \
        if (!(ctx)) return DFSPH_E_INVALID;                                                    \
        if (cudaSetDevice((ctx)->device) != cudaSuccess) {                                     \
            (ctx)->err = "cudaSetDevice failed";                                               \
            return DFSPH_E_CUDA;                                                               \
        }                                                                                      \
        const int pre = (ctx)->f32 ? (ctx)->f32->enter() : (ctx)->f64->enter();                \
        if (pre != DFSPH_OK) return pre;                                                       \
        return (ctx)->f32 ? (ctx)->f32->call : (ctx)->f64->call;                               \
    } while (0)
// The step applies velocities pending from dfsph_update_fluid inside its binning; a rigid boundary
// motion touches neither the fluid nor the upload staging, so the pending copy keeps overlapping.
#define DFSPH_DISPATCH_STEP(ctx, call)                                                         \
    do {                                                                                       \
        if (!(ctx)) return DFSPH_E_INVALID;                                                    \
        if (cudaSetDevice((ctx)->device) != cudaSuccess) {                                     \
            (ctx)->err = "cudaSetDevice failed";                                               \
            return DFSPH_E_CUDA;                                                               \
        }                                                                                      \
        return (ctx)->f32 ? (ctx)->f32->call : (ctx)->f64->call;                               \
    } while (0)

namespace {
template <class S> int solve_div(S* s, uint32_t max_iter, double max_error, int32_t* iters) {
    int r = s->divergence_solve((int)max_iter, max_error);
    if (r != DFSPH_OK) return r;
    if (iters) {
        r = s->collect(true, (int)max_iter, s->sc.max_iterations);
        if (r != DFSPH_OK) return r;
        *iters = s->last_iters_v;
    }
    return DFSPH_OK;
}
template <class S> int solve_pres(S* s, uint32_t max_iter, double max_error, int32_t* iters) {
    int r = s->pressure_solve((int)max_iter, max_error, false);
    if (r != DFSPH_OK) return r;
    if (iters) {
        r = s->collect(false, s->sc.max_iterations_v, (int)max_iter);
        if (r != DFSPH_OK) return r;
        *iters = s->last_iters;
    }
    return DFSPH_OK;
}
}  // namespace

extern "C" {

int dfsph_scene_defaults(dfsph_scene* s) {
    if (!s) return DFSPH_E_INVALID;
    std::memset(s, 0, sizeof(*s));
    s->particle_radius = 0.025;
    s->density0 = 1000.0;
    s->viscosity = 0.01;
    s->gravitation[0] = 0.0;
    s->gravitation[1] = -9.81;
    s->gravitation[2] = 0.0;
    s->time_step = 0.001;
    s->max_iterations = 100;
    s->max_error = 0.01;
    s->max_iterations_v = 100;
    s->max_error_v = 0.1;
    s->enable_divergence_solver = 1;
    s->cfl_method = 0;
    s->cfl_factor = 0.5;
    s->cfl_max_time_step = 0.01;
    s->cfl_min_time_step = 0.0001;
    s->fluid_capacity = 1u << 16;
    s->boundary_capacity = 1u << 16;
    s->neighbor_capacity = 96;
    s->precision = 32;
    s->device = 0;
    s->use_graphs = 1;
    return DFSPH_OK;
}

int dfsph_create(const dfsph_scene* scene, dfsph_ctx** out) {
    if (!scene || !out) {
        dfsph::g_create_error = "null argument";
        return DFSPH_E_INVALID;
    }
    *out = nullptr;
    if (scene->precision != 32 && scene->precision != 64) {
        dfsph::g_create_error = "precision must be 32 or 64";
        return DFSPH_E_INVALID;
    }
    auto* ctx = new dfsph_ctx();
    ctx->device = scene->device;
    int r;
    if (scene->precision == 32) {
        ctx->f32 = std::make_unique<dfsph::Solver<float>>(ctx->err);
        r = ctx->f32->init(*scene);
    } else {
        ctx->f64 = std::make_unique<dfsph::Solver<double>>(ctx->err);
        r = ctx->f64->init(*scene);
    }
    if (r != DFSPH_OK) {
        dfsph::g_create_error = ctx->err;
        delete ctx;
        return r;
    }
    *out = ctx;
    return DFSPH_OK;
}

int dfsph_destroy(dfsph_ctx* ctx) {
    if (!ctx) return DFSPH_OK;
    cudaSetDevice(ctx->device);
    delete ctx;
    return DFSPH_OK;
}

const char* dfsph_last_error(const dfsph_ctx* ctx) {
    return ctx ? ctx->err.c_str() : dfsph::g_create_error.c_str();
}

int dfsph_set_boundary(dfsph_ctx* ctx, const float* xyz, const float* psi, uint32_t n) {
    DFSPH_DISPATCH(ctx, set_boundary(xyz, psi, n));
}
int dfsph_move_boundary(dfsph_ctx* ctx, const float* xyz, const float* vxyz) {
    DFSPH_DISPATCH(ctx, move_boundary(xyz, vxyz));
}
int dfsph_move_boundary_rigid(dfsph_ctx* ctx, uint32_t first, uint32_t count, const double* q, const double* position,
                              const double* velocity, const double* angular_velocity) {
    DFSPH_DISPATCH_STEP(ctx, move_boundary_rigid(first, count, q, position, velocity, angular_velocity));
}
int dfsph_upload_fluid(dfsph_ctx* ctx, const float* xyz, const float* vxyz, const float* mass, uint32_t n) {
    DFSPH_DISPATCH(ctx, upload_fluid(xyz, vxyz, mass, n));
}
int dfsph_update_fluid(dfsph_ctx* ctx, const float* xyz, const float* vxyz) {
    DFSPH_DISPATCH(ctx, update_fluid(xyz, vxyz));
}
int dfsph_download(dfsph_ctx* ctx, int field, int dtype, void* out, size_t n_elems, int order) {
    DFSPH_DISPATCH(ctx, download(field, dtype, out, n_elems, order));
}
int dfsph_get_neighbors(dfsph_ctx* ctx, uint32_t* counts, uint32_t* lists, uint32_t cap) {
    DFSPH_DISPATCH(ctx, get_neighbors(counts, lists, cap));
}
int dfsph_step(dfsph_ctx* ctx, dfsph_step_stats* stats) { DFSPH_DISPATCH_STEP(ctx, step(stats)); }
int dfsph_neighbors_search(dfsph_ctx* ctx, int sort) {
    (void)sort;
    DFSPH_DISPATCH(ctx, neighbors_search());
}


int dfsph_divergence_solve(dfsph_ctx* ctx, uint32_t max_iter, double max_error, int32_t* iters) {
    if (!ctx) return DFSPH_E_INVALID;
    cudaSetDevice(ctx->device);
    return ctx->f32 ? solve_div(ctx->f32.get(), max_iter, max_error, iters)
                    : solve_div(ctx->f64.get(), max_iter, max_error, iters);
}
int dfsph_external_forces(dfsph_ctx* ctx) {
    if (!ctx) return DFSPH_E_INVALID;
    cudaSetDevice(ctx->device);
    return ctx->f32 ? ctx->f32->external_forces(ctx->f32->sc.cfl_method != 0)
                    : ctx->f64->external_forces(ctx->f64->sc.cfl_method != 0);
}
int dfsph_update_time_step(dfsph_ctx* ctx, double h_future) { DFSPH_DISPATCH(ctx, update_time_step(h_future)); }
int dfsph_cfl(dfsph_ctx* ctx, double min_dt, double cfl_factor, double max_dt) {
    DFSPH_DISPATCH(ctx, cfl(min_dt, cfl_factor, max_dt));
}
int dfsph_update_vel(dfsph_ctx* ctx) { DFSPH_DISPATCH(ctx, update_vel()); }
int dfsph_pressure_solve(dfsph_ctx* ctx, uint32_t max_iter, double max_error, int32_t* iters) {
    if (!ctx) return DFSPH_E_INVALID;
    cudaSetDevice(ctx->device);
    return ctx->f32 ? solve_pres(ctx->f32.get(), max_iter, max_error, iters)
                    : solve_pres(ctx->f64.get(), max_iter, max_error, iters);
}
int dfsph_update_pos(dfsph_ctx* ctx) { DFSPH_DISPATCH(ctx, update_pos()); }
int dfsph_on_step_end(dfsph_ctx* ctx) { DFSPH_DISPATCH(ctx, on_step_end()); }
int dfsph_set_param(dfsph_ctx* ctx, const char* key, double value) {
    if (!key) return DFSPH_E_INVALID;
    DFSPH_DISPATCH(ctx, set_param(std::string(key), value));
}
int dfsph_get_param(dfsph_ctx* ctx, const char* key, double* value) {
    if (!key) return DFSPH_E_INVALID;
    DFSPH_DISPATCH(ctx, get_param(std::string(key), value));
}
int dfsph_status(dfsph_ctx* ctx, uint32_t* status, int clear) { DFSPH_DISPATCH(ctx, get_status(status, clear)); }
int dfsph_num_fluid(dfsph_ctx* ctx, uint32_t* n) {
    if (!ctx || !n) return DFSPH_E_INVALID;
    *n = ctx->f32 ? ctx->f32->n : ctx->f64->n;
    return DFSPH_OK;
}
int dfsph_synchronize(dfsph_ctx* ctx) { DFSPH_DISPATCH(ctx, synchronize_all()); }
int dfsph_get_stream(dfsph_ctx* ctx, void** stream) {
    if (!ctx || !stream) return DFSPH_E_INVALID;
    *stream = (void*)(ctx->f32 ? ctx->f32->stream : ctx->f64->stream);
    return DFSPH_OK;
}
int dfsph_time_kernel(dfsph_ctx* ctx, int kernel, int reps, double* ms_per_launch) {
    DFSPH_DISPATCH(ctx, time_kernel(kernel, reps, ms_per_launch));
}
int dfsph_save_snapshot(dfsph_ctx* ctx, const char* dir, int what) { DFSPH_DISPATCH(ctx, save_snapshot(dir, what)); }
int dfsph_checkpoint_save(dfsph_ctx* ctx, const char* path) { DFSPH_DISPATCH(ctx, save_checkpoint(path)); }
int dfsph_export_bgeo(dfsph_ctx* ctx, const char* path) { DFSPH_DISPATCH(ctx, export_bgeo(path)); }
int dfsph_read_dynamic_data(dfsph_ctx* ctx, float* xyz, float* vxyz) {
    DFSPH_DISPATCH(ctx, read_dynamic_data(xyz, vxyz));
}
int dfsph_body_wrench(dfsph_ctx* ctx, uint32_t n_bodies, const uint32_t* first, const uint32_t* count,
                      const double* centers, double* force_torque) {
    DFSPH_DISPATCH(ctx, body_wrench(n_bodies, first, count, centers, force_torque));
}
int dfsph_check_particles_positions(dfsph_ctx* ctx, int mode, uint32_t* count) {
    DFSPH_DISPATCH(ctx, check_particles_positions(mode, count));
}
int dfsph_open_boundary_init(dfsph_ctx* ctx, const dfsph_surface* boundary, const dfsph_surface* interior,
                             const dfsph_surface* fluid_surface, const float* sample_xyz, uint32_t n_samples,
                             uint32_t* n_kept) {
    DFSPH_DISPATCH(ctx, open_boundary_init(boundary, interior, fluid_surface, sample_xyz, n_samples, n_kept));
}
int dfsph_open_boundary_apply(dfsph_ctx* ctx, double allowed_distance, double allowed_density, int use_inflow,
                              int use_outflow, uint32_t* added, uint32_t* removed) {
    DFSPH_DISPATCH(ctx, open_boundary_apply(allowed_distance, allowed_density, use_inflow != 0, use_outflow != 0,
                                            added, removed));
}
int dfsph_open_boundary_shift(dfsph_ctx* ctx, const float* delta) { DFSPH_DISPATCH(ctx, open_boundary_shift(delta)); }
int dfsph_set_surface_mesh(dfsph_ctx* ctx, uint32_t mesh_id, const float* vertices, uint32_t n_vertices,
                           const uint32_t* triangles, uint32_t n_triangles) {
    DFSPH_DISPATCH(ctx, set_surface_mesh(mesh_id, vertices, n_vertices, triangles, n_triangles));
}
int dfsph_dynamic_window_init(dfsph_ctx* ctx, const double* lo, const double* hi, uint32_t wall_first,
                              uint32_t wall_count, const float* rest_xyz, uint32_t n_rest) {
    DFSPH_DISPATCH(ctx, dynamic_window_init(lo, hi, wall_first, wall_count, rest_xyz, n_rest));
}
int dfsph_dynamic_window_shift(dfsph_ctx* ctx, const double* displacement, double allowed_distance,
                               double allowed_density, uint32_t* added, uint32_t* removed) {
    DFSPH_DISPATCH(ctx, dynamic_window_shift(displacement, allowed_distance, allowed_density, added, removed));
}
int dfsph_dynamic_window_stabilize(dfsph_ctx* ctx, uint32_t iterations, double time_step, double damping,
                                   int tagged_only) {
    DFSPH_DISPATCH(ctx, dynamic_window_stabilize(iterations, time_step, damping, tagged_only));
}
int dfsph_fluid_level(dfsph_ctx* ctx, double* level) { DFSPH_DISPATCH(ctx, fluid_level(level)); }
int dfsph_fluid_level_control(dfsph_ctx* ctx, double target, uint32_t* removed, uint32_t* added) {
    DFSPH_DISPATCH(ctx, fluid_level_control(target, removed, added));
}
int dfsph_dynamic_window_displacement(dfsph_ctx* ctx, double* displacement) {
    DFSPH_DISPATCH(ctx, dynamic_window_state(displacement));
}
int dfsph_open_boundary_samples(dfsph_ctx* ctx, float* xyz, uint32_t capacity, uint32_t* count) {
    DFSPH_DISPATCH(ctx, open_boundary_samples(xyz, capacity, count));
}
int dfsph_bgeo_write(const char* path, const float* xyz, const float* vxyz, uint64_t count, float radius) {
    std::string err;
    if (!path) err = "dfsph_bgeo_write: null path";
    else if (dfsph::bgeo_write(path, count, xyz, vxyz, radius, err)) return DFSPH_OK;
    dfsph::set_global_error(err);
    return DFSPH_E_INVALID;
}
int dfsph_bgeo_read(const char* path, float* xyz, float* vxyz, uint64_t capacity, uint64_t* count, int* has_velocity) {
    std::string err;
    std::vector<float> x, v;
    bool hv = false;
    if (!path || !count) {
        dfsph::set_global_error("dfsph_bgeo_read: null path or count");
        return DFSPH_E_INVALID;
    }
    if (!dfsph::bgeo_read(path, x, v, hv, err)) {
        dfsph::set_global_error(err);
        return DFSPH_E_INVALID;
    }
    const uint64_t m = x.size() / 3;
    *count = m;
    if (has_velocity) *has_velocity = hv ? 1 : 0;
    if (!xyz) return DFSPH_OK;
    if (capacity < m) {
        dfsph::set_global_error("dfsph_bgeo_read: " + std::to_string(m) + " particles exceed the capacity " +
                                std::to_string(capacity));
        return DFSPH_E_INVALID;
    }
    std::memcpy(xyz, x.data(), x.size() * sizeof(float));
    if (vxyz) std::memcpy(vxyz, v.data(), v.size() * sizeof(float));
    return DFSPH_OK;
}
int dfsph_checkpoint_load(dfsph_ctx* ctx, const char* path) { DFSPH_DISPATCH(ctx, load_checkpoint(path)); }
int dfsph_load_snapshot(dfsph_ctx* ctx, const char* dir, int what, int load_velocities) {
    DFSPH_DISPATCH(ctx, load_snapshot(dir, what, load_velocities != 0));
}
int dfsph_mlp_get_params(dfsph_ctx* ctx, float* params, size_t n) { DFSPH_DISPATCH(ctx, mlp_get_params(params, n)); }
int dfsph_mlp_set_params(dfsph_ctx* ctx, const float* params, size_t n) {
    DFSPH_DISPATCH(ctx, mlp_set_params(params, n));
}
int dfsph_mlp_get_scales(dfsph_ctx* ctx, float* in_scale, float* out_scale) {
    DFSPH_DISPATCH(ctx, mlp_get_scales(in_scale, out_scale));
}
int dfsph_mlp_set_scales(dfsph_ctx* ctx, const float* in_scale, const float* out_scale) {
    DFSPH_DISPATCH(ctx, mlp_set_scales(in_scale, out_scale));
}
int dfsph_mlp_forward(dfsph_ctx* ctx, const float* x, uint32_t n, float* y) {
    DFSPH_DISPATCH(ctx, mlp_forward_host(x, n, y));
}
int dfsph_mlp_gradient(dfsph_ctx* ctx, const float* x, const float* t, uint32_t n, float* grad, double* loss) {
    DFSPH_DISPATCH(ctx, mlp_gradient_host(x, t, n, grad, loss));
}
int dfsph_mlp_train(dfsph_ctx* ctx, const float* x, const float* t, uint32_t n, int32_t iters, double learning_rate,
                    double* loss) {
    DFSPH_DISPATCH(ctx, mlp_train_host(x, t, n, iters, learning_rate, loss));
}
int dfsph_mlp_reset(dfsph_ctx* ctx, uint32_t seed) {
    if (!ctx) return DFSPH_E_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->f32) {
        const int r = ctx->f32->ensure_mlp();
        return r != DFSPH_OK ? r : ctx->f32->mlp_reset(seed);
    }
    const int r = ctx->f64->ensure_mlp();
    return r != DFSPH_OK ? r : ctx->f64->mlp_reset(seed);
}
int dfsph_launch_count(dfsph_ctx* ctx, uint64_t* launches) {
    if (!ctx || !launches) return DFSPH_E_INVALID;
    *launches = ctx->f32 ? ctx->f32->launches : ctx->f64->launches;
    return DFSPH_OK;
}

}  // extern "C"
