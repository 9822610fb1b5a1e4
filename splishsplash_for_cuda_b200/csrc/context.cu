// context.cu — the solver context behind the C ABI (include/dfsph_c.h).
//
// Solver<Real> owns every device buffer of one fluid set and one static/moving boundary set (what
// SPH::DFSPHCData + UnifiedParticleSet + NeighborsSearchDataSet own in the reference,
// DFSPH_c_arrays_structure.h:36-496) and drives the time step of DFSPHCUDA::step()
// (DFSPH_CUDA.cpp:82-794) on one private stream. Nothing here is a global or a function-local
// static, so several contexts may coexist (the reference keeps statics in cuda_neighborsSearch
// and cuda_CFL, DFSPH_core_cuda.cu:2653-2663, :3333-3348, and is one instance per process).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dfsph_state.cuh"
#include "io.cuh"
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
    uint32_t Nc = 0, Bc = 0, cap = 0, stride = 0;
    uint32_t n = 0, nb = 0;
    int cur = 0;
    bool grid_ready = false;
    bool boundary_moving = false;
    int key_passes = 4;
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

    // dt history (DFSPHCData h, h_future, h_past, h_ratio_to_past(2), invH, invH_future)
    double h = 0, h_future = 0, h_past = 0, inv_h = 0, inv_h_future = 0, h_ratio = 1, h_ratio2 = 1;
    double time_step = 0;
    bool use_graphs = true;
    cudaGraphExec_t g_loop[2] = {nullptr, nullptr};  // [0] divergence, [1] pressure
    uint32_t g_loop_n[2] = {0, 0};
    bool vel_updated = false;  // dfsph_update_vel ran since the last external-force pass

    int last_iters = 0, last_iters_v = 0;
    double last_err = 0, last_err_v = 0;

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
        const uint32_t nmax = std::max(Nc, Bc);
        DF_TRY(dalloc(&sb.keys_a, nmax));
        DF_TRY(dalloc(&sb.keys_b, nmax));
        DF_TRY(dalloc(&sb.vals_a, nmax));
        DF_TRY(dalloc(&sb.vals_b, nmax));
        DF_TRY(dalloc(&sb.workspace, radix_sort_workspace_words(nmax, 4)));
        DF_TRY(dalloc(&partials, grid_for(nmax) + 1));
        DF_TRY(dalloc(&cfl_partials, grid_for(nmax) + 1));
        DF_TRY(dalloc(&ctl, 3));
        DF_TRY(dalloc(&status, 4));
        DF_TRY(dalloc(&stage, (size_t)nmax * 7));
        DF_CUDA(cudaMalloc(&dl, (size_t)nmax * 3 * sizeof(double)));
        DF_CUDA(cudaMalloc((void**)&ds, sizeof(DevState<Real>)));
        DF_CUDA(cudaMallocHost((void**)&h_ctl, 3 * sizeof(LoopCtl)));
        DF_CUDA(cudaMallocHost((void**)&h_status, 4 * sizeof(uint32_t)));
        DF_CUDA(cudaMemsetAsync(ctl, 0, 3 * sizeof(LoopCtl), stream));
        DF_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(uint32_t), stream));
        DF_CUDA(cudaMemsetAsync(counts, 0, Nc * sizeof(uint32_t), stream));
        DF_CUDA(cudaEventCreate(&ev0));
        DF_CUDA(cudaEventCreate(&ev1));
        time_step = s.time_step;
        use_graphs = s.use_graphs != 0;
        reset_dt();
        return sync_state();
    }

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        for (int k = 0; k < 2; ++k)
            if (g_loop[k]) cudaGraphExecDestroy(g_loop[k]);
        auto f = [](void* p) {
            if (p) cudaFree(p);
        };
        for (int b = 0; b < 2; ++b) {
            f(pos[b]); f(vel[b]); f(kappa[b]); f(kappaV[b]); f(id[b]); f(bpos[b]); f(bvel[b]);
        }
        f(density); f(factor); f(densityAdv); f(kcoef); f(acc); f(counts); f(nbr); f(bid);
        f(sb.keys_a); f(sb.keys_b); f(sb.vals_a); f(sb.vals_b); f(sb.workspace);
        f(partials); f(cfl_partials); f(ctl); f(status); f(stage); f(dl); f(ds); f(ftab); f(btab);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (h_status) cudaFreeHost(h_status);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    void reset_dt() {
        h = h_future = h_past = time_step;
        inv_h = inv_h_future = 1.0 / time_step;
        h_ratio = h_ratio2 = 1.0;
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
        hs.features = nullptr;
        hs.predicted = nullptr;
        launch_set_state<Real>(ds, hs, stream);
        launches += 1;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // Cell grid from a bounding box, following DFSPHCData::initGridOffset
    // (DFSPH_c_arrays_structure.cpp:1050-1098): offset = -(floor(min / H) - 5).
    int set_grid(const float mn[3], const float mx[3]) {
        const float H = (float)(4.0 * sc.particle_radius);
        int maxdim = 1;
        for (int a = 0; a < 3; ++a) {
            DF_CHECK(std::isfinite(mn[a]) && std::isfinite(mx[a]) && mx[a] >= mn[a], DFSPH_E_INVALID,
                     "invalid grid bounding box");
            const int fmin = (int)std::floor(mn[a] / H);
            const int fmax = (int)std::floor(mx[a] / H);
            off[a] = -(fmin - 5);
            dim[a] = fmax + off[a] + 6;
            DF_CHECK(dim[a] <= 1024, DFSPH_E_INVALID,
                     "domain too large: more than 1024 cells of size 4r along one axis");
            maxdim = std::max(maxdim, dim[a]);
        }
        int bits = 1;
        while ((1 << bits) < maxdim) ++bits;
        key_passes = std::min(4, (3 * bits + 1 + 7) / 8);
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
            if (psi)
                DF_CUDA(cudaMemcpyAsync(stage + (size_t)count * 3, psi, (size_t)count * sizeof(float),
                                        cudaMemcpyHostToDevice, stream));
            launch_unpack_boundary<Real>(stage, psi ? stage + (size_t)count * 3 : nullptr, count, bpos[1], bvel[1],
                                         stream);
            launches += 1;
            DF_TRY(sort_boundary(psi == nullptr));
        }
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
        if (vxyz) DF_CUDA(cudaMemcpyAsync(sv, vxyz, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
        launch_update_fluid<Real>(sx, vxyz ? sv : nullptr, n, id[cur], pos[cur], vel[cur], stream);
        launches += 1;
        return DFSPH_OK;
    }

    // ------------------------------------------------------------------------------------------
    // cuda_neighborsSearch: keys -> stable radix sort -> reorder (double buffer) -> cell table ->
    // neighbour lists. The particle order is always refreshed (the reference's sort flag is kept in
    // the signature; unsorted searching is not offered).
    int neighbors_search() {
        DF_CHECK(grid_ready, DFSPH_E_STATE, "no grid: set a boundary or upload fluid first");
        if (!n) return DFSPH_OK;
        const StepParams<Real> p = params();
        launch_cell_keys<Real>(pos[cur], n, p, sb.keys_a, status, stream);
        uint32_t *skeys, *perm;
        radix_sort_pairs(sb, n, key_passes, true, stream, status, &launches, &skeys, &perm);
        const int nx = 1 - cur;
        launch_reorder_fluid<Real>(perm, n, pos[cur], vel[cur], kappa[cur], kappaV[cur], id[cur], pos[nx], vel[nx],
                                   kappa[nx], kappaV[nx], id[nx], stream);
        cur = nx;
        DF_CUDA(cudaMemsetAsync(ftab, 0, cells * sizeof(uint2), stream));
        launch_cell_bounds(skeys, n, dim[0], dim[1], dim[2], ftab, stream);
        DF_TRY(sync_state());
        launch_build_neighbors<Real>(ds, n, ftab, btab, stream);
        launches += 4;
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    int invalidate_graphs() {
        for (int k = 0; k < 2; ++k) {
            if (g_loop[k]) cudaGraphExecDestroy(g_loop[k]);
            g_loop[k] = nullptr;
            g_loop_n[k] = 0;
        }
        return DFSPH_OK;
    }

    // A while-loop graph: body = Jacobi pass + residual pass whose last block sets the condition.
    int build_loop_graph(int kind) {
        cudaGraph_t g = nullptr;
        DF_CUDA(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle handle;
        DF_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        DF_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        DF_CUDA(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        if (kind == 0) {
            launch_divergence_jacobi<Real>(ds, n, handle, true, stream);
            launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, handle, true, stream);
        } else {
            launch_pressure_jacobi<Real>(ds, n, handle, true, stream);
            launch_pressure_residual<Real>(ds, n, false, 0.0, 0, 0, handle, true, stream);
        }
        cudaGraph_t captured = nullptr;
        DF_CUDA(cudaStreamEndCapture(stream, &captured));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        DF_CUDA(e);
        g_loop[kind] = exec;
        g_loop_n[kind] = n;
        return DFSPH_OK;
    }

    // Runs the iterations of one solver loop after its init pass. Graph mode: one graph launch,
    // no host round trip. Host mode: one small readback per iteration (what the reference does).
    int run_loop(int kind, int max_iter) {
        if (max_iter <= 0) return DFSPH_OK;
        if (use_graphs) {
            if (!g_loop[kind] || g_loop_n[kind] != n) DF_TRY(build_loop_graph(kind));
            DF_CUDA(cudaGraphLaunch(g_loop[kind], stream));
            launches += 1;
            return DFSPH_OK;
        }
        uint32_t cont = 1;
        while (cont) {
            if (kind == 0) {
                launch_divergence_jacobi<Real>(ds, n, 0, false, stream);
                launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream);
            } else {
                launch_pressure_jacobi<Real>(ds, n, 0, false, stream);
                launch_pressure_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream);
            }
            launches += 2;
            DF_CUDA(cudaMemcpyAsync(h_ctl + kind, ctl + kind, sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            cont = h_ctl[kind].cont;
        }
        return DFSPH_OK;
    }

    // cuda_divergenceSolve (DFSPH_core_cuda.cu:785-861).
    int divergence_solve(int max_iter, double max_error) {
        if (!n) return DFSPH_OK;
        DF_CUDA(cudaMemsetAsync(&ctl[0].ticket, 0, sizeof(uint32_t), stream));
        launch_density_alpha<Real>(ds, n, true, stream);
        launch_divergence_warm_jacobi<Real>(ds, n, stream);
        const double eta = max_error * 0.01 * sc.density0 / h;
        launch_divergence_residual<Real>(ds, n, true, eta, kMinItersV, max_iter, 0, false, stream);
        launches += 3;
        DF_TRY(run_loop(0, max_iter));
        DF_CUDA(cudaGetLastError());
        return DFSPH_OK;
    }

    // cuda_pressureSolve (DFSPH_core_cuda.cu:1338-1419); with fused_vel the velocity update of
    // cuda_update_vel is applied inside the warm-start pass.
    int pressure_solve(int max_iter, double max_error, bool fused_vel) {
        if (!n) return DFSPH_OK;
        DF_CUDA(cudaMemsetAsync(&ctl[1].ticket, 0, sizeof(uint32_t), stream));
        launch_pressure_warm_jacobi<Real>(ds, n, fused_vel, stream);
        const double eta = max_error * 0.01 * sc.density0;
        launch_pressure_residual<Real>(ds, n, true, eta, kMinItersP, max_iter, 0, false, stream);
        launches += 2;
        DF_TRY(run_loop(1, max_iter));
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

    int update_time_step(double hf) {
        DF_CHECK(hf > 0 && std::isfinite(hf), DFSPH_E_INVALID, "time step must be finite and > 0");
        h_future = hf;
        inv_h_future = 1.0 / hf;
        h_ratio = h / hf;
        h_ratio2 = (h * h) / (hf * hf);
        return sync_state();
    }

    // cuda_CFL (DFSPH_core_cuda.cu:3321-3394): dt = cfl * 0.4 * 2r / sqrt(max |v + a h|^2), clamped.
    int cfl(double min_dt, double factor_, double max_dt) {
        double vmax = 0.0;
        if (n) {
            launch_cfl_reduce<Real>(ds, grid_for(n), stream);
            launches += 1;
            DF_CUDA(cudaMemcpyAsync(h_ctl + 2, ctl + 2, sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
            DF_CUDA(cudaStreamSynchronize(stream));
            vmax = h_ctl[2].sum;
        }
        double hn = factor_ * 0.4 * (2.0 * sc.particle_radius / std::sqrt(vmax));
        hn = std::min(hn, max_dt);
        hn = std::max(hn, min_dt);
        return update_time_step(hn);
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
        h_past = h;
        h = h_future;
        inv_h = inv_h_future;
        return sync_state();
    }

    // Reads the loop control blocks and the status word (one synchronisation).
    int collect(bool div_ran, int max_iter_v, int max_iter) {
        DF_CUDA(cudaMemcpyAsync(h_ctl, ctl, 2 * sizeof(LoopCtl), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaMemcpyAsync(h_status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        DF_CUDA(cudaStreamSynchronize(stream));
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

    int step(dfsph_step_stats* st) {
        DF_CHECK(grid_ready, DFSPH_E_STATE, "step before any boundary or fluid upload");
        if (timing) DF_CUDA(cudaEventRecord(ev0, stream));
        const double h_used = h;
        DF_TRY(neighbors_search());
        const bool div = sc.enable_divergence_solver != 0;
        if (div) {
            DF_TRY(divergence_solve(sc.max_iterations_v, sc.max_error_v));
        } else if (n) {
            launch_density_alpha<Real>(ds, n, false, stream);
            launches += 1;
        }
        const bool use_cfl = sc.cfl_method != 0;
        DF_TRY(external_forces(use_cfl));
        if (use_cfl) {
            DF_TRY(cfl(sc.cfl_min_time_step, sc.cfl_factor, sc.cfl_max_time_step));
        } else {
            DF_TRY(update_time_step(time_step));
        }
        DF_TRY(pressure_solve(sc.max_iterations, sc.max_error, true));
        DF_TRY(update_pos());
        const double h_next = h_future;
        DF_TRY(on_step_end());
        if (timing) DF_CUDA(cudaEventRecord(ev1, stream));
        DF_TRY(collect(div, sc.max_iterations_v, sc.max_iterations));
        if (st) {
            st->iterations = last_iters;
            st->iterations_v = last_iters_v;
            st->density_error = last_err;
            st->divergence_error = last_err_v;
            st->h = h_used;
            st->h_future = h_next;
            st->status = h_status[0];
            st->num_fluid = n;
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
        else if (k == "time_step") { DF_CHECK(v > 0, DFSPH_E_INVALID, "time_step must be > 0"); time_step = v; }
        else if (k == "gravitation_x") sc.gravitation[0] = v;
        else if (k == "gravitation_y") sc.gravitation[1] = v;
        else if (k == "gravitation_z") sc.gravitation[2] = v;
        else if (k == "use_graphs") { use_graphs = v != 0; }
        else if (k == "h") { h = v; dt_changed = true; }
        else if (k == "h_future") { h_future = v; dt_changed = true; }
        else if (k == "h_past") { h_past = v; dt_changed = true; }
        else if (k == "inv_h") { inv_h = v; dt_changed = true; }
        else if (k == "timing") timing = v != 0;
        else DF_CHECK(false, DFSPH_E_INVALID, "unknown parameter key: " + k);
        (void)dt_changed;
        return sync_state();
    }

    int get_param(const std::string& k, double* v) {
        DF_CHECK(v, DFSPH_E_INVALID, "null output");
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
        else DF_CHECK(false, DFSPH_E_INVALID, "unknown parameter key: " + k);
        return DFSPH_OK;
    }

    void launch_kernel(int k) {
        switch (k) {
            case DFSPH_K_NEIGHBOR_BUILD: launch_build_neighbors<Real>(ds, n, ftab, btab, stream); break;
            case DFSPH_K_DENSITY_ALPHA: launch_density_alpha<Real>(ds, n, false, stream); break;
            case DFSPH_K_DIVERGENCE_JACOBI: launch_divergence_jacobi<Real>(ds, n, 0, false, stream); break;
            case DFSPH_K_DIVERGENCE_RESIDUAL:
                launch_divergence_residual<Real>(ds, n, false, 0.0, 0, 0, 0, false, stream);
                break;
            case DFSPH_K_VISCOSITY: launch_viscosity<Real>(ds, n, false, stream); break;
            case DFSPH_K_PRESSURE_WARM_JACOBI: launch_pressure_warm_jacobi<Real>(ds, n, false, stream); break;
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
                DF_CUDA(cudaMemsetAsync(ftab, 0, cells * sizeof(uint2), stream));
                launch_cell_bounds(skeys, n, dim[0], dim[1], dim[2], ftab, stream);
                cur = nx;
                launches += 3;
                launch_set_state<Real>(ds, (hs.pos = pos[cur], hs.vel = vel[cur], hs.kappa = kappa[cur],
                                            hs.kappaV = kappaV[cur], hs.id = id[cur], hs), stream);
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
int dfsph_step(dfsph_ctx* ctx, dfsph_step_stats* stats) { DFSPH_DISPATCH(ctx, step(stats)); }
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
int dfsph_synchronize(dfsph_ctx* ctx) {
    if (!ctx) return DFSPH_E_INVALID;
    cudaSetDevice(ctx->device);
    const cudaError_t e = cudaStreamSynchronize(ctx->f32 ? ctx->f32->stream : ctx->f64->stream);
    if (e != cudaSuccess) {
        ctx->err = std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e);
        return DFSPH_E_CUDA;
    }
    return DFSPH_OK;
}
int dfsph_get_stream(dfsph_ctx* ctx, void** stream) {
    if (!ctx || !stream) return DFSPH_E_INVALID;
    *stream = (void*)(ctx->f32 ? ctx->f32->stream : ctx->f64->stream);
    return DFSPH_OK;
}
int dfsph_time_kernel(dfsph_ctx* ctx, int kernel, int reps, double* ms_per_launch) {
    DFSPH_DISPATCH(ctx, time_kernel(kernel, reps, ms_per_launch));
}
int dfsph_launch_count(dfsph_ctx* ctx, uint64_t* launches) {
    if (!ctx || !launches) return DFSPH_E_INVALID;
    *launches = ctx->f32 ? ctx->f32->launches : ctx->f64->launches;
    return DFSPH_OK;
}

}  // extern "C"
