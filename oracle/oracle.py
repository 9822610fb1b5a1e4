"""ctypes wrapper of the CPU oracle (liboracle_dfsph.so). Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_dfsph.so"

FIELD_IDS = {"position": (0, 3), "velocity": (1, 3), "mass": (2, 1), "density": (3, 1), "factor": (4, 1),
             "density_adv": (5, 1), "kappa": (6, 1), "kappa_v": (7, 1), "acceleration": (8, 3),
             "boundary_psi": (10, 1), "boundary_position": (11, 3), "boundary_force": (14, 3),
             "kappa_needed": (20, 1), "kappa_v_needed": (21, 1)}


class OracleParams(C.Structure):
    _fields_ = [
        ("particle_radius", C.c_double),
        ("density0", C.c_double),
        ("viscosity", C.c_double),
        ("gravitation", C.c_double * 3),
        ("time_step", C.c_double),
        ("max_iterations", C.c_int32),
        ("max_error", C.c_double),
        ("max_iterations_v", C.c_int32),
        ("max_error_v", C.c_double),
        ("enable_divergence_solver", C.c_int32),
        ("cfl_method", C.c_int32),
        ("cfl_factor", C.c_double),
        ("cfl_max_time_step", C.c_double),
        ("cfl_min_time_step", C.c_double),
        ("neighbor_capacity", C.c_uint32),
        ("brute_force", C.c_int32),
    ]


class OracleSurface(C.Structure):
    """Same layout as the C ABI's dfsph_surface (restated)."""
    _fields_ = [
        ("type", C.c_int32),
        ("reversed", C.c_int32),
        ("origin", C.c_float * 3),
        ("normal", C.c_float * 3),
        ("center", C.c_float * 3),
        ("half_lengths", C.c_float * 3),
        ("radius", C.c_float),
        ("radius_internal", C.c_float),
        ("points", C.c_uint32),
        ("direction", C.c_float * 3),
    ]


def _surface(s) -> OracleSurface:
    return OracleSurface.from_buffer_copy(bytes(s))


def lib_path() -> Path:
    return LIB


def build(force: bool = False) -> Path:
    """Builds liboracle_dfsph.so with the Makefile beside this file."""
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "dfsph_oracle.cpp").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "liboracle_dfsph.so"], check=True, capture_output=True)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        vp, fp, dp, up = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint32)
        ip = C.POINTER(C.c_int32)
        sig = {
            "oracle_create": (vp, [C.c_int, C.POINTER(OracleParams)]),
            "oracle_destroy": (None, [vp]),
            "oracle_set_boundary": (C.c_int, [vp, fp, fp, C.c_uint32, dp]),
            "oracle_set_boundary_velocity": (C.c_int, [vp, fp, fp]),
            "oracle_set_fluid": (C.c_int, [vp, fp, fp, fp, C.c_uint32]),
            "oracle_update_fluid": (C.c_int, [vp, dp, dp]),
            "oracle_step": (C.c_int, [vp, ip, ip, dp, dp]),
            "oracle_neighbors": (C.c_int, [vp]),
            "oracle_divergence_solve": (C.c_int, [vp, C.c_int, C.c_double]),
            "oracle_density_alpha": (C.c_int, [vp, C.c_int]),
            "oracle_external_forces": (C.c_int, [vp]),
            "oracle_update_time_step": (C.c_int, [vp, C.c_double]),
            "oracle_update_vel": (C.c_int, [vp]),
            "oracle_pressure_solve": (C.c_int, [vp, C.c_int, C.c_double]),
            "oracle_update_pos": (C.c_int, [vp]),
            "oracle_on_step_end": (C.c_int, [vp]),
            "oracle_get": (C.c_int, [vp, C.c_int, dp]),
            "oracle_get_scalar": (C.c_int, [vp, C.c_char_p, dp]),
            "oracle_set_scalar": (C.c_int, [vp, C.c_char_p, C.c_double]),
            "oracle_get_neighbors": (C.c_int, [vp, up, up, C.c_uint32]),
            "oracle_kernel_values": (C.c_int, [C.c_double, dp, C.c_uint32, C.c_int, dp, dp]),
            "oracle_open_boundary_init": (C.c_int, [vp, C.POINTER(OracleSurface), C.POINTER(OracleSurface),
                                                    C.POINTER(OracleSurface), fp, C.c_uint32, up]),
            "oracle_open_boundary_apply": (C.c_int, [vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_uint32, up,
                                                     up]),
            "oracle_open_boundary_shift": (C.c_int, [vp, fp]),
            "oracle_remove_outside_box": (C.c_int, [vp, fp, fp, up]),
            "oracle_surface_eval": (C.c_int, [C.POINTER(OracleSurface), fp, C.c_uint32, C.c_void_p, fp]),
            "oracle_set_surface_mesh": (C.c_int, [C.c_uint32, fp, C.c_uint32, up, C.c_uint32]),
            "oracle_dynamic_window_stabilize": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_double, C.c_uint32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _f(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(C.POINTER(C.c_float))


class Oracle:
    """CPU restatement of the DFSPH step on one scene (fluid in original order)."""

    def __init__(self, scene, precision: int = 64, brute_force: bool = False, neighbor_capacity: int = 96,
                 boundary_psi=None, grid_box=None):
        self.lib = _load()
        cfg = scene.config
        p = OracleParams()
        p.particle_radius = cfg.particleRadius
        p.density0 = cfg.density0
        p.viscosity = cfg.viscosity
        for a in range(3):
            p.gravitation[a] = cfg.gravitation[a]
        p.time_step = cfg.timeStepSize
        p.max_iterations = cfg.maxIterations
        p.max_error = cfg.maxError
        p.max_iterations_v = cfg.maxIterationsV
        p.max_error_v = cfg.maxErrorV
        p.enable_divergence_solver = 1 if cfg.enableDivergenceSolver else 0
        p.cfl_method = cfg.cflMethod
        p.cfl_factor = cfg.cflFactor
        p.cfl_max_time_step = cfg.cflMaxTimeStepSize
        p.cfl_min_time_step = 0.0001
        p.neighbor_capacity = neighbor_capacity
        p.brute_force = 1 if brute_force else 0
        self.params = p
        self.h = self.lib.oracle_create(precision, C.byref(p))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.scene = scene
        b = np.ascontiguousarray(scene.boundary, dtype=np.float32)
        psi = None if boundary_psi is None else np.ascontiguousarray(boundary_psi, dtype=np.float32)
        self._keep = (b, psi)
        gb = None if grid_box is None else np.ascontiguousarray(np.asarray(grid_box, np.float64).reshape(6))
        self._keep = (b, psi, gb)
        if self.lib.oracle_set_boundary(self.h, _f(b), _f(psi), b.shape[0],
                                        None if gb is None else gb.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise RuntimeError("oracle_set_boundary failed")
        x = np.ascontiguousarray(scene.fluid, dtype=np.float32)
        v = None if scene.fluid_velocity is None else np.ascontiguousarray(scene.fluid_velocity, dtype=np.float32)
        self.n = x.shape[0]
        self.nb = b.shape[0]
        m = getattr(scene, "fluid_mass", None)
        self._keep_m = None if m is None else np.ascontiguousarray(m, dtype=np.float32)
        self.lib.oracle_set_fluid(self.h, _f(x), _f(v), _f(self._keep_m), self.n)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self):
        it, itv = C.c_int32(), C.c_int32()
        err, errv = C.c_double(), C.c_double()
        overflow = self.lib.oracle_step(self.h, C.byref(it), C.byref(itv), C.byref(err), C.byref(errv))
        self.n = int(self.scalar("n"))  # particles outside the domain box are removed at the step end
        return dict(iterations=it.value, iterations_v=itv.value, density_error=err.value,
                    divergence_error=errv.value, overflow=bool(overflow))

    def field(self, name: str) -> np.ndarray:
        fid, comps = FIELD_IDS[name]
        n = self.nb if name.startswith("boundary") else self.n
        out = np.empty(n * comps, dtype=np.float64)
        if self.lib.oracle_get(self.h, fid, out.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise KeyError(name)
        return out.reshape(n, comps) if comps > 1 else out

    def scalar(self, key: str) -> float:
        v = C.c_double()
        if self.lib.oracle_get_scalar(self.h, key.encode(), C.byref(v)) != 0:
            raise KeyError(key)
        return v.value

    def set_scalar(self, key: str, value: float) -> None:
        if self.lib.oracle_set_scalar(self.h, key.encode(), float(value)) != 0:
            raise KeyError(key)

    def neighbors(self, row: int = 96):
        self.lib.oracle_neighbors(self.h)
        return self.get_neighbors(row)

    def get_neighbors(self, row: int = 96):
        counts = np.zeros((self.n, 2), dtype=np.uint32)
        lists = np.zeros((self.n, row), dtype=np.uint32)
        self.lib.oracle_get_neighbors(self.h, counts.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      lists.ctypes.data_as(C.POINTER(C.c_uint32)), row)
        return counts, lists

    def set_positions(self, xyz: np.ndarray, vxyz: np.ndarray | None = None) -> None:
        x = np.ascontiguousarray(xyz, dtype=np.float64)
        v = None if vxyz is None else np.ascontiguousarray(vxyz, dtype=np.float64)
        self.lib.oracle_update_fluid(self.h, x.ctypes.data_as(C.POINTER(C.c_double)),
                                     None if v is None else v.ctypes.data_as(C.POINTER(C.c_double)))

    # piecewise phases
    def move_boundary(self, xyz: np.ndarray, vxyz: np.ndarray | None = None) -> None:
        """New boundary positions (and velocities) in upload order; psi is kept."""
        x = np.ascontiguousarray(xyz, dtype=np.float32)
        v = None if vxyz is None else np.ascontiguousarray(vxyz, dtype=np.float32)
        self._moved = (x, v)
        if self.lib.oracle_set_boundary_velocity(self.h, _f(x), _f(v)) != 0:
            raise RuntimeError("oracle_set_boundary_velocity failed")

    def divergence_solve(self, max_iter=None, max_error=None) -> int:
        c = self.scene.config
        return self.lib.oracle_divergence_solve(self.h, c.maxIterationsV if max_iter is None else max_iter,
                                                c.maxErrorV if max_error is None else max_error)

    def density_alpha(self, warm_v: bool = True):
        self.lib.oracle_density_alpha(self.h, 1 if warm_v else 0)

    def external_forces(self):
        self.lib.oracle_external_forces(self.h)

    def update_time_step(self, hf: float):
        self.lib.oracle_update_time_step(self.h, hf)

    def update_vel(self):
        self.lib.oracle_update_vel(self.h)

    def pressure_solve(self, max_iter=None, max_error=None) -> int:
        c = self.scene.config
        return self.lib.oracle_pressure_solve(self.h, c.maxIterations if max_iter is None else max_iter,
                                              c.maxError if max_error is None else max_error)

    def update_pos(self):
        self.lib.oracle_update_pos(self.h)

    def on_step_end(self):
        self.lib.oracle_on_step_end(self.h)

    # simple open boundary (surfaces: any ctypes structure with the dfsph_surface layout)
    def open_boundary_init(self, boundary, interior, fluid_surface, samples) -> int:
        x = np.ascontiguousarray(samples, dtype=np.float32).reshape(-1, 3)
        self._ob = (_surface(boundary), _surface(interior), _surface(fluid_surface))
        kept = C.c_uint32(0)
        self.lib.oracle_open_boundary_init(self.h, *[C.byref(q) for q in self._ob], _f(x), x.shape[0],
                                           C.byref(kept))
        return kept.value

    def open_boundary_apply(self, allowed_distance: float, allowed_density: float, use_inflow=True,
                            use_outflow=True, capacity: int = 2 ** 32 - 1):
        """Returns (added, removed, clipped)."""
        a, r = C.c_uint32(0), C.c_uint32(0)
        clipped = self.lib.oracle_open_boundary_apply(self.h, allowed_distance, allowed_density, int(use_inflow),
                                                      int(use_outflow), capacity, C.byref(a), C.byref(r))
        self.n = self.n + a.value - r.value
        return a.value, r.value, bool(clipped)

    def remove_outside_box(self, lo, hi) -> int:
        """Removes the fluid particles outside [lo, hi] (float32 bounds), keeping the others' order."""
        r = C.c_uint32()
        self.lib.oracle_remove_outside_box(self.h, _f(np.asarray(lo, np.float32).reshape(3)),
                                           _f(np.asarray(hi, np.float32).reshape(3)), C.byref(r))
        self.n = int(self.scalar("n"))
        return int(r.value)

    def dynamic_window_stabilize(self, iterations: int, time_step: float, damping: float, first: int) -> None:
        """The device's dfsph_dynamic_window_stabilize with the particles of ids >= first tagged."""
        self.lib.oracle_dynamic_window_stabilize(self.h, int(iterations), float(time_step), float(damping), int(first))

    def open_boundary_shift(self, delta) -> None:
        self.lib.oracle_open_boundary_shift(self.h, _f(np.asarray(delta, np.float32).reshape(3)))


def set_surface_mesh(mesh_id: int, vertices, triangles) -> None:
    """Registers the triangle mesh mesh_id for the oracle's type-3 surfaces (one table per process)."""
    lib = _load()
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    if lib.oracle_set_surface_mesh(int(mesh_id), _f(v), v.shape[0], t.ctypes.data_as(C.POINTER(C.c_uint32)),
                                   t.shape[0]) != 0:
        raise ValueError("invalid mesh")


def surface_eval(surface, points):
    """(inside (n,) bool, normal (n, 3) float32) of the oracle's BufferFluidSurface restatement."""
    lib = _load()
    p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    inside = np.zeros(p.shape[0], np.uint8)
    normal = np.zeros((p.shape[0], 3), np.float32)
    s = _surface(surface)
    lib.oracle_surface_eval(C.byref(s), _f(p), p.shape[0], inside.ctypes.data_as(C.c_void_p),
                            normal.ctypes.data_as(C.POINTER(C.c_float)))
    return inside.astype(bool), normal


def fluid_level(positions, particle_radius: float, grid_offset, grid_dims) -> float:
    """DFSPHCData::computeFluidLevel restated on the CPU (pure Python, small cases).

    find_splashless_column_max_height_kernel (SPlisHSPlasH/DFSPH/SPH_other_systems_cuda.cu:144-187):
    for every column (x, z) of the cell grid, the cells are read from the top (y = dims - 1) down; every
    particle of a cell is inserted into an ascending array of the three highest heights (initially
    -2); after a cell, the walk stops once more than two particles have been seen. The column's height
    is the middle entry when more than two were seen, else -2. find_fluid_height_cuda (:192-260): the
    level is the highest column height, starting from -1. Cells: floor(x / (4 r) + offset) in FP32.
    """
    x = np.asarray(positions, np.float32).reshape(-1, 3)
    H = np.float32(4.0 * particle_radius)
    off = np.asarray(grid_offset, np.float32).reshape(3)
    dims = [int(d) for d in grid_dims]
    cells: dict[tuple[int, int, int], list[float]] = {}
    for p in x:
        c = np.floor(p / H + off).astype(np.int64)
        if np.any(c < 0) or c[0] >= dims[0] or c[1] >= dims[1] or c[2] >= dims[2]:
            continue
        cells.setdefault((int(c[0]), int(c[1]), int(c[2])), []).append(float(p[1]))
    columns: dict[tuple[int, int], list[int]] = {}
    for (cx, cy, cz) in cells:
        columns.setdefault((cx, cz), []).append(cy)
    ranking = -1.0
    for (cx, cz), ys in columns.items():
        top = [-2.0, -2.0, -2.0]
        count = 0
        for cy in sorted(ys, reverse=True):
            for h in cells[(cx, cy, cz)]:
                count += 1
                sup = -1
                for k in range(3):
                    if h > top[k]:
                        sup = k
                if sup > -1:
                    for k in range(sup):
                        top[k] = top[k + 1]
                    top[sup] = h
            if count > 2:
                break
        col = top[1] if count > 2 else -2.0
        if ranking < col:
            ranking = col
    return ranking


def column_tops(positions, particle_radius: float, grid_offset, grid_dims) -> dict:
    """find_column_max_height_kernel (SPlisHSPlasH/DFSPH/SPH_other_systems_cuda.cu:292-318): per column
    (x, z) the highest particle of its top occupied cell, as float32."""
    x = np.asarray(positions, np.float32).reshape(-1, 3)
    H = np.float32(4.0 * particle_radius)
    off = np.asarray(grid_offset, np.float32).reshape(3)
    dims = [int(d) for d in grid_dims]
    best: dict[tuple[int, int], tuple[int, np.float32]] = {}
    for p in x:
        c = np.floor(p / H + off).astype(np.int64)
        if np.any(c < 0) or c[0] >= dims[0] or c[1] >= dims[1] or c[2] >= dims[2]:
            continue
        key = (int(c[0]), int(c[2]))
        cy, h = int(c[1]), np.float32(p[1])
        cur = best.get(key)
        if cur is None or cy > cur[0]:
            best[key] = (cy, max(np.float32(-2.0), h))
        elif cy == cur[0] and h > cur[1]:
            best[key] = (cy, h)
    return {k: v[1] for k, v in best.items()}


def fluid_level_raise(fluid_positions, boundary_positions, particle_radius: float, grid_offset, grid_dims,
                      target: float, level: float) -> np.ndarray:
    """The particles the raising branch of control_fluid_height_cuda places (float32, lattice order).

    SPlisHSPlasH/DFSPH/SPH_other_systems_cuda.cu: get_min_max_pos_kernel (:282-304) on the boundary
    in the reference's order (stable by the linear cell index x + 256 z + 65536 y; boundary_positions
    in upload order), the host's lattice size (:486-516), place_additional_particles_right_above_kernel
    (:321-408) with border_range = width / 3 (y 0), in its FP32 / FP64 operation order.
    """
    f32, f64 = np.float32, float
    b = np.asarray(boundary_positions, np.float32).reshape(-1, 3)
    H = f32(4.0 * particle_radius)
    off = np.asarray(grid_offset, np.float32).reshape(3)
    cells = np.floor(b / H + off).astype(np.int64)
    order = sorted(range(len(b)), key=lambda k: (cells[k][1], cells[k][2], cells[k][0]))
    mn = b[order[0]].copy()
    mx = b[order[-1]].copy()
    for k in range(min(10, len(b))):
        mn = np.minimum(mn, b[order[k]])
        mx = np.maximum(mx, b[order[len(b) - 1 - k]])
    r = f32(particle_radius)
    p = f32(r * f32(2))
    mn = (mn + f32(2) * r).astype(np.float32)
    mx = (mx - f32(2) * r).astype(np.float32)
    width = (mx - mn).astype(np.float32)
    host_x = f32(np.floor(width[0] / p) + f32(1))
    host_z = f32(np.floor(width[2] / p) + f32(1))
    layers = f32(np.floor((f32(target) - f32(level)) / p) + f32(1))
    want = int(f32(f32(host_x * layers) * host_z))
    cw_x = f32(np.floor(abs(width[0]) / p) + f32(1))
    cw_z = f32(np.floor(abs(width[2]) / p) + f32(1))
    border = np.array([width[0] / f32(3), 0, width[2] / f32(3)], np.float32)
    bordered = f32(border[0] * border[0]) + f32(border[2] * border[2]) > 0
    tops = column_tops(fluid_positions, particle_radius, grid_offset, grid_dims)
    out = []
    for i in range(want):
        row = int(f32(f32(i) / cw_x))
        lev = int(f32(f32(row) / cw_z))
        lx = f32(f32(f32(i) - f32(f32(row) * cw_x)) * p)
        ly = f32(f64(lev) * (f64(p) * 0.80))
        lz = f32(f32(f32(row) - f32(f32(lev) * cw_z)) * p)
        if lev & 1:
            lx = f32(lx + f32(p / f32(2)))
            lz = f32(lz + f32(p / f32(2)))
        tx, tz = f32(mn[0] + lx), f32(mn[2] + lz)
        if bordered and not (tx < f32(mn[0] + border[0]) or tz < f32(mn[2] + border[2]) or
                             tx > f32(mx[0] - border[0]) or tz > f32(mx[2] - border[2])):
            continue
        cx = int(np.floor(f32(f32(tx / H) + off[0])))
        cz = int(np.floor(f32(f32(tz / H) + off[2])))
        top = tops.get((cx, cz), f32(-2.0))
        y0 = f32(f64(f32(top + p)) + f64(p) / 4.0)
        out.append((f32(mn[0] + lx), f32(y0 + ly), f32(mn[2] + lz)))
    return np.array(out, np.float32).reshape(-1, 3)


def kernel_values(H: float, r: np.ndarray, precision: int = 32):
    lib = _load()
    r = np.ascontiguousarray(r, dtype=np.float64)
    w = np.empty_like(r)
    dw = np.empty_like(r)
    dp = C.POINTER(C.c_double)
    lib.oracle_kernel_values(H, r.ctypes.data_as(dp), r.size, precision, w.ctypes.data_as(dp), dw.ctypes.data_as(dp))
    return w, dw
