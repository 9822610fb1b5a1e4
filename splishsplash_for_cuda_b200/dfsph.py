"""Host-side mirror of the reference solver interface for the DFSPH time step.

`DFSPHCUDA` has the public surface of SPH::DFSPHCUDA (SPlisHSPlasH/DFSPH/DFSPH_CUDA.h:26-154) and of
its base SPH::TimeStep (SPlisHSPlasH/TimeStep.h:79-103): step(), reset(), the iteration counters and
the max error / max iteration / CFL / divergence-solver setters, all backed by the sm_100a kernels
of libdfsph_b200.so through the C ABI. `DFSPHCData` exposes the state accessors the reference
callers use (fluid particle count, dynamic data readback, dt history).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .scene import Scene

_f32p = C.POINTER(C.c_float)


def _fptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(_f32p)


def scene_struct(scene: Scene, precision: int = 32, device: int = 0, use_graphs: bool = True,
                 neighbor_capacity: int = 96, fluid_capacity: int | None = None,
                 boundary_capacity: int | None = None, lib_path: str | None = None,
                 grid_box=None) -> _capi.DfsphScene:
    lib = _capi.load(lib_path)
    s = _capi.DfsphScene()
    _capi.check(lib, None, lib.dfsph_scene_defaults(C.byref(s)))
    cfg = scene.config
    s.particle_radius = cfg.particleRadius
    s.density0 = cfg.density0
    s.viscosity = cfg.viscosity
    for a in range(3):
        s.gravitation[a] = cfg.gravitation[a]
    s.time_step = cfg.timeStepSize
    s.max_iterations = cfg.maxIterations
    s.max_error = cfg.maxError
    s.max_iterations_v = cfg.maxIterationsV
    s.max_error_v = cfg.maxErrorV
    s.enable_divergence_solver = 1 if cfg.enableDivergenceSolver else 0
    s.cfl_method = cfg.cflMethod
    s.cfl_factor = cfg.cflFactor
    s.cfl_max_time_step = cfg.cflMaxTimeStepSize
    s.fluid_capacity = max(1, fluid_capacity if fluid_capacity is not None else scene.n_fluid)
    s.boundary_capacity = max(1, boundary_capacity if boundary_capacity is not None else scene.n_boundary)
    s.neighbor_capacity = neighbor_capacity
    s.precision = precision
    s.device = device
    s.use_graphs = 1 if use_graphs else 0
    if grid_box is not None:  # (min x, y, z, max x, y, z): the cell grid's domain (else the boundary's box)
        g = np.asarray(grid_box, np.float64).reshape(6)
        for a in range(3):
            s.grid_min[a] = g[a]
            s.grid_max[a] = g[3 + a]
    return s


class DFSPHData:
    """State accessors of one solver context (the parts of SPH::DFSPHCData callers read)."""

    def __init__(self, owner: "DFSPHCUDA"):
        self._o = owner

    def getFluidParticlesCount(self) -> int:
        n = C.c_uint32()
        self._o._call(self._o._lib.dfsph_num_fluid(self._o._ctx, C.byref(n)))
        return int(n.value)

    def readDynamicData(self, out_positions: np.ndarray | None = None, out_velocities: np.ndarray | None = None):
        """Positions and velocities (n, 3) float32 in particle-id order (DFSPHCData::readDynamicData),
        read with one wait; the outputs may be given (C-contiguous float32, e.g. pinned memory)."""
        n = self.getFluidParticlesCount()
        x = np.empty((n, 3), np.float32) if out_positions is None else out_positions
        v = np.empty((n, 3), np.float32) if out_velocities is None else out_velocities
        for a in (x, v):
            if a.dtype != np.float32 or not a.flags.c_contiguous or a.size != 3 * n:
                raise ValueError("outputs must be C-contiguous float32 arrays of n x 3")
        self._o._call(self._o._lib.dfsph_read_dynamic_data(self._o._ctx, x.ctypes.data, v.ctypes.data))
        return x, v

    @property
    def h(self) -> float:
        return self._o.get_param("h")

    @property
    def h_future(self) -> float:
        return self._o.get_param("h_future")

    @property
    def h_past(self) -> float:
        return self._o.get_param("h_past")

    def updateTimeStep(self, h_future: float) -> None:
        self._o._call(self._o._lib.dfsph_update_time_step(self._o._ctx, float(h_future)))

    def onSimulationStepEnd(self) -> None:
        self._o._call(self._o._lib.dfsph_on_step_end(self._o._ctx))


class DFSPHCUDA:
    """Drop-in for SPH::DFSPHCUDA over one scene (fluid + static box walls)."""

    def __init__(self, scene: Scene, precision: int | None = None, device: int = 0, use_graphs: bool = True,
                 neighbor_capacity: int = 96, boundary_psi: np.ndarray | None = None,
                 fluid_capacity: int | None = None, lib_path: str | None = None, grid_box=None):
        """precision None takes the scene's (Configuration "precision", default 32); the scene's
        "learnedWarmStart" block, when present, configures the learned warm start."""
        self._lib = _capi.load(lib_path)
        self.scene = scene
        if precision is None:
            precision = int(getattr(scene.config, "precision", 32) or 32)
        self.precision = precision
        self._struct = scene_struct(scene, precision, device, use_graphs, neighbor_capacity, fluid_capacity,
                                    lib_path=lib_path, grid_box=grid_box)
        ctx = C.c_void_p()
        code = self._lib.dfsph_create(C.byref(self._struct), C.byref(ctx))
        if code != _capi.DFSPH_OK:
            raise _capi.DfsphError(code, self._lib.dfsph_last_error(None).decode())
        self._ctx = ctx
        self._psi = None if boundary_psi is None else np.ascontiguousarray(boundary_psi, dtype=np.float32)
        self.m_iterations = 0
        self.m_iterationsV = 0
        self.last_stats = None
        self.m_data = DFSPHData(self)
        self.reset()
        lws = getattr(scene.config, "learnedWarmStart", None)
        if lws and lws.get("enabled", True):
            if "damping" in lws:
                self.set_param("warm_start_damping", float(lws["damping"]))
            self.set_learned_warm_start(True, probe=bool(lws.get("probe", True)),
                                        train_interval=lws.get("trainInterval"), train_iters=lws.get("trainIters"),
                                        train_batch=lws.get("trainBatch"), learning_rate=lws.get("learningRate"))

    # ---- lifetime ------------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.dfsph_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, code: int) -> None:
        _capi.check(self._lib, self._ctx, code)

    def reset(self) -> None:
        """DFSPHCUDA::reset (DFSPH_CUDA.cpp:796-817): reload boundary and fluid from the scene."""
        b = np.ascontiguousarray(self.scene.boundary, dtype=np.float32)
        self._call(self._lib.dfsph_set_boundary(self._ctx, _fptr(b), _fptr(self._psi), b.shape[0]))
        x = np.ascontiguousarray(self.scene.fluid, dtype=np.float32)
        v = None if self.scene.fluid_velocity is None else np.ascontiguousarray(self.scene.fluid_velocity,
                                                                                 dtype=np.float32)
        m = None if self.scene.fluid_mass is None else np.ascontiguousarray(self.scene.fluid_mass, dtype=np.float32)
        self._call(self._lib.dfsph_upload_fluid(self._ctx, _fptr(x), _fptr(v), _fptr(m), x.shape[0]))
        self.m_iterations = 0
        self.m_iterationsV = 0

    # ---- the time step ----------------------------------------------------------------------------
    def step(self) -> _capi.DfsphStepStats:
        st = _capi.DfsphStepStats()
        self._call(self._lib.dfsph_step(self._ctx, C.byref(st)))
        self.m_iterations = st.iterations
        self.m_iterationsV = st.iterations_v
        self.last_stats = st
        return st

    # piecewise host functions of DFSPH_core_cuda.h
    def step_async(self) -> None:
        """Enqueues one time step without waiting or reading anything back (dfsph_step with null
        stats); synchronize() waits, status() and get_param() read the results."""
        self._call(self._lib.dfsph_step(self._ctx, None))

    def neighbors_search(self) -> None:
        self._call(self._lib.dfsph_neighbors_search(self._ctx, 1))

    def divergence_solve(self, max_iter: int | None = None, max_error: float | None = None) -> int:
        it = C.c_int32()
        self._call(self._lib.dfsph_divergence_solve(
            self._ctx, self.getMaxIterationsV() if max_iter is None else max_iter,
            self.getMaxErrorV() if max_error is None else max_error, C.byref(it)))
        return int(it.value)

    def external_forces(self) -> None:
        self._call(self._lib.dfsph_external_forces(self._ctx))

    def update_time_step(self, h_future: float) -> None:
        self._call(self._lib.dfsph_update_time_step(self._ctx, h_future))

    def update_vel(self) -> None:
        self._call(self._lib.dfsph_update_vel(self._ctx))

    def pressure_solve(self, max_iter: int | None = None, max_error: float | None = None) -> int:
        it = C.c_int32()
        self._call(self._lib.dfsph_pressure_solve(
            self._ctx, self.getMaxIterations() if max_iter is None else max_iter,
            self.getMaxError() if max_error is None else max_error, C.byref(it)))
        return int(it.value)

    def update_pos(self) -> None:
        self._call(self._lib.dfsph_update_pos(self._ctx))

    def on_step_end(self) -> None:
        self._call(self._lib.dfsph_on_step_end(self._ctx))

    # ---- TimeStep accessors ------------------------------------------------------------------------
    def getIterationCount(self) -> int:
        return self.m_iterations

    def getIterationCountV(self) -> int:
        return self.m_iterationsV

    def get_param(self, key: str) -> float:
        v = C.c_double()
        self._call(self._lib.dfsph_get_param(self._ctx, key.encode(), C.byref(v)))
        return float(v.value)

    def set_param(self, key: str, value: float) -> None:
        self._call(self._lib.dfsph_set_param(self._ctx, key.encode(), float(value)))

    def getMaxError(self) -> float: return self.get_param("max_error")
    def setMaxError(self, v: float) -> None: self.set_param("max_error", v)
    def getMaxIterations(self) -> int: return int(self.get_param("max_iterations"))
    def setMaxIterations(self, v: int) -> None: self.set_param("max_iterations", v)
    def getMaxErrorV(self) -> float: return self.get_param("max_error_v")
    def setMaxErrorV(self, v: float) -> None: self.set_param("max_error_v", v)
    def getMaxIterationsV(self) -> int: return int(self.get_param("max_iterations_v"))
    def setMaxIterationsV(self, v: int) -> None: self.set_param("max_iterations_v", v)
    def getCflMethod(self) -> int: return int(self.get_param("cfl_method"))
    def setCflMethod(self, v: int) -> None: self.set_param("cfl_method", v)
    def getCflFactor(self) -> float: return self.get_param("cfl_factor")
    def setCflFactor(self, v: float) -> None: self.set_param("cfl_factor", v)
    def getCflMaxTimeStepSize(self) -> float: return self.get_param("cfl_max_time_step")
    def setCflMaxTimeStepSize(self, v: float) -> None: self.set_param("cfl_max_time_step", v)
    def getEnableDivergenceSolver(self) -> bool: return bool(self.get_param("enable_divergence_solver"))
    def setEnableDivergenceSolver(self, v: bool) -> None: self.set_param("enable_divergence_solver", 1 if v else 0)
    def getViscosity(self) -> float: return self.get_param("viscosity")
    def setViscosity(self, v: float) -> None: self.set_param("viscosity", v)

    # ---- state readback ----------------------------------------------------------------------------
    def num_fluid(self) -> int:
        return self.m_data.getFluidParticlesCount()

    def field(self, name: str, dtype=np.float32, order: int = _capi.ORDER_ID,
              out: np.ndarray | None = None) -> np.ndarray:
        """Downloads one field (shape (n,) or (n, comps)). `out`, when given, must be a C-contiguous
        array of the right size and dtype (e.g. pinned host memory) and is filled in place."""
        fid, comps = _capi.FIELDS[name]
        if out is None:
            n = int(self.get_param("num_boundary")) if name.startswith("boundary") else self.num_fluid()
            out = np.empty((n, comps) if comps > 1 else n, dtype=np.uint32 if name in ("id", "neighbor_counts")
                           else dtype)
        if not out.flags.c_contiguous:
            raise ValueError("out must be C-contiguous")
        if name in ("id", "neighbor_counts"):
            code = _capi.DTYPE_U32
            if out.dtype != np.uint32:
                raise ValueError("id and neighbor_counts download as uint32")
        else:
            code = _capi.DTYPE_F64 if out.dtype == np.float64 else _capi.DTYPE_F32
            if out.dtype not in (np.float32, np.float64):
                raise ValueError("float fields download as float32 or float64")
        self._call(self._lib.dfsph_download(self._ctx, fid, code, out.ctypes.data_as(C.c_void_p), out.size, order))
        return out

    def positions(self, dtype=np.float32) -> np.ndarray:
        return self.field("position", dtype)

    def velocities(self, dtype=np.float32) -> np.ndarray:
        return self.field("velocity", dtype)

    def neighbors(self, row: int | None = None):
        """(counts[N, 2], lists[N, row]) in particle-id space: fluid ids first, then boundary indices."""
        n = self.num_fluid()
        row = row or self._struct.neighbor_capacity
        counts = np.zeros((n, 2), dtype=np.uint32)
        lists = np.zeros((n, row), dtype=np.uint32)
        self._call(self._lib.dfsph_get_neighbors(self._ctx, counts.ctypes.data_as(_capi._U),
                                                 lists.ctypes.data_as(_capi._U), row))
        return counts, lists

    def status(self, clear: bool = False) -> int:
        s = C.c_uint32()
        self._call(self._lib.dfsph_status(self._ctx, C.byref(s), 1 if clear else 0))
        return int(s.value)

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._call(self._lib.dfsph_launch_count(self._ctx, C.byref(v)))
        return int(v.value)

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._call(self._lib.dfsph_get_stream(self._ctx, C.byref(p)))
        return int(p.value or 0)

    def time_kernel(self, name: str, reps: int = 5) -> float:
        """Mean device ms per launch of one kernel of the step (modifies the state)."""
        ms = C.c_double()
        self._call(self._lib.dfsph_time_kernel(self._ctx, _capi.KERNELS.index(name), reps, C.byref(ms)))
        return float(ms.value)

    def synchronize(self) -> None:
        self._call(self._lib.dfsph_synchronize(self._ctx))

    def update_fluid(self, positions: np.ndarray, velocities: np.ndarray | None = None) -> None:
        x = np.ascontiguousarray(positions, dtype=np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float32)
        self._call(self._lib.dfsph_update_fluid(self._ctx, _fptr(x), _fptr(v)))

    def body_wrench(self, first, count, centers) -> tuple[np.ndarray, np.ndarray]:
        """Force (k, 3) and torque (k, 3) of the fluid during the last step on k boundary bodies,
        body b being boundary particles first[b] .. first[b] + count[b] - 1 (upload order), torque
        about centers[b]. Needs set_param("boundary_forces", 1)."""
        f = np.ascontiguousarray(first, dtype=np.uint32).reshape(-1)
        c = np.ascontiguousarray(count, dtype=np.uint32).reshape(-1)
        ce = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        k = f.size
        if c.size != k or ce.shape[0] != k:
            raise ValueError("first, count and centers must describe the same bodies")
        out = np.zeros((k, 6), np.float64)
        self._call(self._lib.dfsph_body_wrench(self._ctx, k, f.ctypes.data, c.ctypes.data, ce.ctypes.data,
                                               out.ctypes.data))
        return out[:, :3].copy(), out[:, 3:].copy()

    def checkParticlesPositions(self, mode: int = 2) -> int:
        """DFSPHCData::checkParticlesPositions: the number of fluid particles outside the domain box;
        mode 2 also removes them (mode 0 only counts)."""
        c = C.c_uint32(0)
        self._call(self._lib.dfsph_check_particles_positions(self._ctx, int(mode), C.byref(c)))
        return c.value

    # ---- simple open boundary (OpenBoundariesSimpleInterface) ------------------------------------
    def init_open_boundary(self, boundary, interior, fluid_surface, samples: np.ndarray) -> int:
        """OpenBoundariesSimpleInterface::init: keeps the inflow samples outside `interior` and inside
        `fluid_surface` (surfaces from splishsplash_for_cuda_b200.open_boundary); returns their count."""
        x = np.ascontiguousarray(samples, dtype=np.float32).reshape(-1, 3)
        kept = C.c_uint32(0)
        self._call(self._lib.dfsph_open_boundary_init(self._ctx, C.byref(boundary), C.byref(interior),
                                                      C.byref(fluid_surface), _fptr(x), x.shape[0], C.byref(kept)))
        return kept.value

    def apply_open_boundary(self, allowed_distance: float | None = None, allowed_density: float = 700.0,
                            use_inflow: bool = True, use_outflow: bool = True) -> tuple[int, int]:
        """OpenBoundariesSimpleInterface::applyOpenBoundary between steps; the defaults are the
        reference driver's (DFSPH_CUDA.cpp:3903-3906: 1.75 r and 700). Returns (added, removed)."""
        if allowed_distance is None:
            allowed_distance = 1.75 * self.scene.config.particleRadius
        added, removed = C.c_uint32(0), C.c_uint32(0)
        self._call(self._lib.dfsph_open_boundary_apply(self._ctx, float(allowed_distance), float(allowed_density),
                                                       int(use_inflow), int(use_outflow), C.byref(added),
                                                       C.byref(removed)))
        return added.value, removed.value

    def open_boundary_samples(self) -> np.ndarray:
        """The kept inflow samples (n, 3), in sample order."""
        cnt = C.c_uint32(0)
        self._call(self._lib.dfsph_open_boundary_samples(self._ctx, None, 0, C.byref(cnt)))
        x = np.zeros((cnt.value, 3), np.float32)
        self._call(self._lib.dfsph_open_boundary_samples(self._ctx, _fptr(x), cnt.value, C.byref(cnt)))
        return x

    def set_surface_mesh(self, mesh_id: int, vertices, triangles) -> None:
        """Registers the triangle mesh mesh_id for open-boundary surfaces of type mesh
        (open_boundary.mesh): vertices (V, 3), triangles (T, 3) vertex indices."""
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        self._call(self._lib.dfsph_set_surface_mesh(self._ctx, int(mesh_id), v.ctypes.data_as(C.c_void_p), v.shape[0],
                                                    t.ctypes.data_as(C.c_void_p), t.shape[0]))

    def shift_open_boundary(self, delta) -> None:
        """Moves the open boundary's surfaces and samples (dynamic-window displacement)."""
        d = np.ascontiguousarray(delta, dtype=np.float32).reshape(3)
        self._call(self._lib.dfsph_open_boundary_shift(self._ctx, _fptr(d)))

    def move_boundary(self, positions: np.ndarray, velocities: np.ndarray | None = None) -> None:
        x = np.ascontiguousarray(positions, dtype=np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float32)
        self._call(self._lib.dfsph_move_boundary(self._ctx, _fptr(x), _fptr(v)))

    def move_boundary_rigid(self, first: int = 0, count: int | None = None, q=None, position=None, velocity=None,
                            angular_velocity=None) -> None:
        """Rigid motion of the boundary particles [first, first + count) on the device
        (update_dynamicObject_UnifiedParticleSet_cuda): x = R(q) x0 + position, v = angular_velocity x
        (x - position) + velocity, x0 the positions given to set_boundary; q = (w, x, y, z)."""
        if count is None:
            count = int(self.get_param("num_boundary")) - first
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in
                (q, position, velocity, angular_velocity)]
        ptrs = [None if a is None else a.ctypes.data_as(C.c_void_p) for a in arrs]
        self._call(self._lib.dfsph_move_boundary_rigid(self._ctx, int(first), int(count), *ptrs))

    # ---- dynamic window (DynamicWindowInterface, driven like DFSPHCUDA::applyDynamicWindow) ----------
    def init_dynamic_window(self, lo, hi, wall_first: int, wall_count: int, rest_positions) -> None:
        """The window box [lo, hi] walled by boundary particles [wall_first, wall_first + wall_count),
        and a fluid at rest tiling it (rest_positions (n, 3))."""
        lo_ = np.ascontiguousarray(lo, dtype=np.float64).reshape(3)
        hi_ = np.ascontiguousarray(hi, dtype=np.float64).reshape(3)
        x = np.ascontiguousarray(rest_positions, dtype=np.float32).reshape(-1, 3)
        self._call(self._lib.dfsph_dynamic_window_init(self._ctx, lo_.ctypes.data, hi_.ctypes.data, int(wall_first),
                                                       int(wall_count), x.ctypes.data, x.shape[0]))

    def shift_dynamic_window(self, displacement, allowed_distance: float, allowed_density: float) -> tuple:
        """Moves the window by displacement (between steps). Returns (added, removed)."""
        d = np.ascontiguousarray(displacement, dtype=np.float64).reshape(3)
        a, r = C.c_uint32(), C.c_uint32()
        self._call(self._lib.dfsph_dynamic_window_shift(self._ctx, d.ctypes.data, float(allowed_distance),
                                                        float(allowed_density), C.byref(a), C.byref(r)))
        return int(a.value), int(r.value)

    def stabilize_dynamic_window(self, iterations: int = 5, time_step: float = 0.003, damping: float = 1.0,
                                 tagged_only: bool = True) -> None:
        """DynamicWindowInterface::stabilizeFluid, method 0: after a shift, `iterations` steps of the
        fixed `time_step` with the warm starts cleared, the particles the shift added damped by
        `damping` before each position update and, with tagged_only, the others held in place."""
        self._call(self._lib.dfsph_dynamic_window_stabilize(self._ctx, int(iterations), float(time_step),
                                                            float(damping), 1 if tagged_only else 0))

    def fluid_level(self) -> float:
        """DFSPHCData::computeFluidLevel: the highest splash-free column height (-1: none)."""
        v = C.c_double()
        self._call(self._lib.dfsph_fluid_level(self._ctx, C.byref(v)))
        return v.value

    def fluid_level_control(self, target: float) -> tuple[int, int]:
        """DFSPHCData::handleFLuidLevelControl: removes the particles above target when the level is
        more than 5 cm above it, places new ones near the walls when it is more than 5 cm below;
        returns (removed, added)."""
        r, a = C.c_uint32(), C.c_uint32()
        self._call(self._lib.dfsph_fluid_level_control(self._ctx, float(target), C.byref(r), C.byref(a)))
        return r.value, a.value

    def dynamic_window_displacement(self) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self._call(self._lib.dfsph_dynamic_window_displacement(self._ctx, out.ctypes.data))
        return out

    # ---- snapshots (DFSPHCUDA::handleSimulationSave / handleSimulationLoad) ----------------------
    def save_snapshot(self, folder, fluid: bool = True, boundary: bool = True) -> None:
        """Writes fluid_file.txt, general_data.txt and boundaries_file.txt (reference text format)."""
        what = (_capi.SNAP_FLUID if fluid else 0) | (_capi.SNAP_BOUNDARY if boundary else 0)
        self._call(self._lib.dfsph_save_snapshot(self._ctx, str(folder).encode(), what))

    def load_snapshot(self, folder, fluid: bool = True, boundary: bool = True, load_velocities: bool = True) -> None:
        what = (_capi.SNAP_FLUID if fluid else 0) | (_capi.SNAP_BOUNDARY if boundary else 0)
        self._call(self._lib.dfsph_load_snapshot(self._ctx, str(folder).encode(), what, 1 if load_velocities else 0))

    def checkpoint_save(self, path) -> None:
        """Binary checkpoint of the complete state (exact resume)."""
        self._call(self._lib.dfsph_checkpoint_save(self._ctx, str(path).encode()))

    def checkpoint_load(self, path) -> None:
        self._call(self._lib.dfsph_checkpoint_load(self._ctx, str(path).encode()))

    def export_bgeo(self, path) -> None:
        """The fluid as a partio .bgeo file (positions, velocities, pscale, id), like the reference's
        partioExport (Demos/StaticBoundaryDemo/main.cpp:485-496)."""
        self._call(self._lib.dfsph_export_bgeo(self._ctx, str(path).encode()))

    # ---- learned warm start (no reference counterpart) ------------------------------------------
    def set_learned_warm_start(self, on: bool = True, probe: bool = True, train_interval: int | None = None,
                               train_iters: int | None = None, train_batch: int | None = None,
                               learning_rate: float | None = None, gate: bool | None = None,
                               gate_period: int | None = None, gate_window: int | None = None,
                               gate_margin: float | None = None, gate_recheck: int | None = None) -> None:
        """Switches the MLP warm start of both solvers on or off (step() only). With probe, each solve
        keeps the learned candidate only if its initial residual is not above the reference warm
        start's. The network trains online every `train_interval` steps. With gate, the learned passes
        run only while the plain warm start needs at least `gate_margin` iterations per step above the
        solves' minimum (measured on a plain probe window of `gate_window` steps after every
        `gate_period` learned steps, or over every `gate_recheck` steps while the gate keeps them
        off)."""
        for key, val in (("train_interval", train_interval), ("train_iters", train_iters),
                         ("train_batch", train_batch), ("learning_rate", learning_rate),
                         ("gate_period", gate_period), ("gate_window", gate_window), ("gate_margin", gate_margin),
                         ("gate_recheck", gate_recheck)):
            if val is not None:
                self.set_param(key, val)
        if gate is not None:
            self.set_param("learned_gate", 1 if gate else 0)
        self.set_param("warm_start_probe", 1 if probe else 0)
        self.set_param("learned_warm_start", 1 if on else 0)

    def mlp_params(self) -> np.ndarray:
        out = np.empty(_capi.MLP_PARAMS, dtype=np.float32)
        self._call(self._lib.dfsph_mlp_get_params(self._ctx, _fptr(out), out.size))
        return out

    def set_mlp_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32).ravel()
        self._call(self._lib.dfsph_mlp_set_params(self._ctx, _fptr(p), p.size))

    def mlp_scales(self) -> tuple[np.ndarray, np.ndarray]:
        a = np.empty(_capi.MLP_INPUTS, dtype=np.float32)
        b = np.empty(_capi.MLP_OUTPUTS, dtype=np.float32)
        self._call(self._lib.dfsph_mlp_get_scales(self._ctx, _fptr(a), _fptr(b)))
        return a, b

    def set_mlp_scales(self, in_scale: np.ndarray, out_scale: np.ndarray) -> None:
        a = np.ascontiguousarray(in_scale, dtype=np.float32)
        b = np.ascontiguousarray(out_scale, dtype=np.float32)
        if a.size != _capi.MLP_INPUTS or b.size != _capi.MLP_OUTPUTS:
            raise ValueError("scales need 8 input and 2 output entries")
        self._call(self._lib.dfsph_mlp_set_scales(self._ctx, _fptr(a), _fptr(b)))

    def mlp_forward(self, x: np.ndarray) -> np.ndarray:
        """Network outputs of samples x[n, 8] through the tensor-core inference path."""
        xs = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, _capi.MLP_INPUTS)
        y = np.empty((xs.shape[0], _capi.MLP_OUTPUTS), dtype=np.float32)
        self._call(self._lib.dfsph_mlp_forward(self._ctx, _fptr(xs), xs.shape[0], _fptr(y)))
        return y

    def mlp_gradient(self, x: np.ndarray, t: np.ndarray) -> tuple[np.ndarray, float]:
        xs = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, _capi.MLP_INPUTS)
        ts = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, _capi.MLP_OUTPUTS)
        if xs.shape[0] != ts.shape[0]:
            raise ValueError("inputs and targets differ in length")
        g = np.empty(_capi.MLP_PARAMS, dtype=np.float32)
        loss = C.c_double()
        self._call(self._lib.dfsph_mlp_gradient(self._ctx, _fptr(xs), _fptr(ts), xs.shape[0], _fptr(g),
                                                C.byref(loss)))
        return g, float(loss.value)

    def mlp_train(self, x: np.ndarray, t: np.ndarray, iters: int, learning_rate: float = 1e-3) -> float:
        xs = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, _capi.MLP_INPUTS)
        ts = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, _capi.MLP_OUTPUTS)
        if xs.shape[0] != ts.shape[0]:
            raise ValueError("inputs and targets differ in length")
        loss = C.c_double()
        self._call(self._lib.dfsph_mlp_train(self._ctx, _fptr(xs), _fptr(ts), xs.shape[0], int(iters),
                                             float(learning_rate), C.byref(loss)))
        return float(loss.value)

    def mlp_reset(self, seed: int = 1234567) -> None:
        self._call(self._lib.dfsph_mlp_reset(self._ctx, int(seed)))
