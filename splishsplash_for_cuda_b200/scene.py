"""Scenes for the DFSPH time step: the reference JSON scene format and seeded synthetic scenes.

The JSON reader follows the keys of the reference SceneLoader (Utilities/SceneLoader.cpp:39-320):
"Configuration" (timeStepSize, particleRadius, density0, viscosity, gravitation, cflMethod,
cflFactor, cflMaxTimeStepSize, maxIterations, maxError, maxIterationsV, maxErrorV,
enableDivergenceSolver), "FluidBlocks" (start/end boxes filled like DemoBase::createFluidBlocks,
Demos/Common/DemoBase.cpp:539-603), "FluidModels" (partio .bgeo particle files with translation,
rotationAxis/rotationAngle and scale) and "RigidBodies" (box walls, or samples from a .bgeo
"particleFile"). Wall bodies without a particle file are sampled as a single-layer
lattice of spacing 2r on the box surface instead of the Poisson-disk sampling of an OBJ mesh
(Demos/StaticBoundaryDemo/main.cpp:466-468); a body whose "geometryFile" names a unit box is the
box [translation - scale/2, translation + scale/2]. Extension keys (ignored by the reference):
"seed" and "jitter" (uniform jitter amplitude as a fraction of r).
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_LANES = 1024


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = x + np.uint64(0x9E3779B97F4A7C15)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _rotl(x: np.ndarray, k: int) -> np.ndarray:
    return (x << np.uint64(k)) | (x >> np.uint64(64 - k))


def xoshiro_uniform(n: int, seed: int) -> np.ndarray:
    """n doubles in [0, 1) from 1024 interleaved xoshiro256** streams (Blackman & Vigna); stream l
    is seeded by four splitmix64 steps from seed * 1024 + l, and value i comes from stream i % 1024.
    Vectorised over the streams, deterministic on every machine."""
    if n <= 0:
        return np.zeros(0, dtype=np.float64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & 0xFFFFFFFFFFFF) * np.uint64(_LANES) + np.arange(_LANES, dtype=np.uint64)
        st = []
        for _ in range(4):
            x = x + np.uint64(0x9E3779B97F4A7C15)
            st.append(_splitmix64(x))
        s0, s1, s2, s3 = st
        rounds = (n + _LANES - 1) // _LANES
        out = np.empty((rounds, _LANES), dtype=np.uint64)
        for r in range(rounds):
            out[r] = _rotl(s1 * np.uint64(5), 7) * np.uint64(9)
            t = s1 << np.uint64(17)
            s2 = s2 ^ s0
            s3 = s3 ^ s1
            s1 = s1 ^ s2
            s0 = s0 ^ s3
            s2 = s2 ^ t
            s3 = _rotl(s3, 45)
    return (out.ravel()[:n] >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _jitter(n: int, amplitude: float, seed: int) -> np.ndarray:
    """(n, 3) array of U(-amplitude, +amplitude) per coordinate."""
    if amplitude == 0.0 or n == 0:
        return np.zeros((n, 3), dtype=np.float64)
    u = xoshiro_uniform(3 * n, seed)
    return ((2.0 * u - 1.0) * amplitude).reshape(n, 3)


def fluid_block(box_min, box_max, radius: float) -> np.ndarray:
    """Dense-mode fluid block of DemoBase::createFluidBlocks: steps = round(extent / 2r) - 1 per axis,
    first particle at min + 2r, x outer, y middle, z inner loop order. Returns (n, 3) float64."""
    diam = 2.0 * radius
    mn = np.asarray(box_min, dtype=np.float64)
    mx = np.asarray(box_max, dtype=np.float64)
    steps = [int(round((mx[a] - mn[a]) / diam)) - 1 for a in range(3)]
    steps = [max(s, 0) for s in steps]
    start = mn + diam
    i, j, k = np.meshgrid(np.arange(steps[0]), np.arange(steps[1]), np.arange(steps[2]), indexing="ij")
    pts = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * diam + start
    return pts


def lattice_block(counts, radius: float, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
    """counts[0] x counts[1] x counts[2] lattice of spacing 2r whose first particle sits at origin + 2r
    (the fluid block [origin, origin + (counts + 1) 2r] of createFluidBlocks)."""
    diam = 2.0 * radius
    mn = np.asarray(origin, dtype=np.float64)
    mx = mn + (np.asarray(counts, dtype=np.float64) + 1.0) * diam
    return fluid_block(mn, mx, radius)


def box_wall(box_min, box_max, spacing: float) -> np.ndarray:
    """Single-layer surface lattice of an axis-aligned box: every lattice point of spacing `spacing`
    from box_min to box_max with at least one coordinate on a face. Returns (B, 3) float64."""
    mn = np.asarray(box_min, dtype=np.float64)
    mx = np.asarray(box_max, dtype=np.float64)
    cnt = [int(round((mx[a] - mn[a]) / spacing)) + 1 for a in range(3)]
    pts = []
    for a in range(3):
        b, c = [d for d in range(3) if d != a]
        for side in (0, cnt[a] - 1):
            # faces perpendicular to axis a; skip points already produced by earlier axes' faces
            ib = np.arange(cnt[b])
            ic = np.arange(cnt[c])
            if b < a:
                ib = ib[1:-1]
            if c < a:
                ic = ic[1:-1]
            gb, gc = np.meshgrid(ib, ic, indexing="ij")
            face = np.empty((gb.size, 3), dtype=np.float64)
            face[:, a] = side
            face[:, b] = gb.ravel()
            face[:, c] = gc.ravel()
            pts.append(face)
    idx = np.concatenate(pts, axis=0)
    return idx * spacing + mn


@dataclass
class Configuration:
    """The "Configuration" block of a reference scene (defaults of SPH::TimeStep, TimeStep.cpp:23-44)."""

    timeStepSize: float = 0.001
    particleRadius: float = 0.025
    density0: float = 1000.0
    viscosity: float = 0.01
    gravitation: tuple = (0.0, -9.81, 0.0)
    cflMethod: int = 0
    cflFactor: float = 0.5
    cflMaxTimeStepSize: float = 0.01
    maxIterations: int = 100
    maxError: float = 0.01
    maxIterationsV: int = 100
    maxErrorV: float = 0.1
    enableDivergenceSolver: bool = True
    simulationMethod: int = 6
    # extensions (keys the reference does not read): arithmetic precision of the solver (32 / 64) and
    # the learned warm start ({"enabled": true, "trainInterval": 50, "trainIters": 20,
    # "trainBatch": 4096, "learningRate": 1e-3, "damping": 0.95, "probe": true})
    precision: int = 32
    learnedWarmStart: dict | None = None


@dataclass
class Scene:
    config: Configuration
    fluid: np.ndarray  # (N, 3) float32
    boundary: np.ndarray  # (B, 3) float32
    fluid_velocity: np.ndarray | None = None
    name: str = "scene"
    box_min: tuple | None = None
    box_max: tuple | None = None
    meta: dict = field(default_factory=dict)
    fluid_mass: np.ndarray | None = None  # (N,) float32; None: FluidModel's default 0.8 rho0 (2r)^3

    @property
    def n_fluid(self) -> int:
        return int(self.fluid.shape[0])

    @property
    def n_boundary(self) -> int:
        return int(self.boundary.shape[0])


def _readvec(v, default):
    return tuple(float(x) for x in v) if v is not None else default


def _scene_relative(scene_path: Path, file: str) -> Path:
    f = Path(file)
    return f if f.is_absolute() else scene_path.parent / f


def load_scene(path: str | Path) -> Scene:
    """Reads a reference-format JSON scene."""
    path = Path(path)
    j = json.loads(path.read_text())
    c = j.get("Configuration", {})
    cfg = Configuration()
    for key in ("timeStepSize", "particleRadius", "density0", "viscosity", "cflFactor", "cflMaxTimeStepSize",
                "maxError", "maxErrorV"):
        if key in c:
            setattr(cfg, key, float(c[key]))
    for key in ("cflMethod", "maxIterations", "maxIterationsV", "simulationMethod"):
        if key in c:
            setattr(cfg, key, int(c[key]))
    if "enableDivergenceSolver" in c:
        cfg.enableDivergenceSolver = bool(c["enableDivergenceSolver"])
    if "precision" in c:
        cfg.precision = int(c["precision"])
        if cfg.precision not in (32, 64):
            raise ValueError("precision must be 32 or 64")
    lws = c.get("learnedWarmStart")
    if lws is not None:
        if not isinstance(lws, dict):
            raise ValueError("learnedWarmStart must be an object")
        unknown = set(lws) - {"enabled", "trainInterval", "trainIters", "trainBatch", "learningRate", "damping",
                              "probe"}
        if unknown:
            raise ValueError(f"unknown learnedWarmStart keys: {sorted(unknown)}")
        cfg.learnedWarmStart = dict(lws)
    cfg.gravitation = _readvec(c.get("gravitation"), cfg.gravitation)
    r = cfg.particleRadius
    seed = int(c.get("seed", 1))
    jitter = float(c.get("jitter", 0.0))
    fluid = []
    for fb in j.get("FluidBlocks", []):
        start = np.asarray(_readvec(fb.get("start"), (0.0, 0.0, 0.0)))
        end = np.asarray(_readvec(fb.get("end"), (1.0, 1.0, 1.0)))
        scale = np.asarray(_readvec(fb.get("scale"), (1.0, 1.0, 1.0)))
        trans = np.asarray(_readvec(fb.get("translation"), (0.0, 0.0, 0.0)))
        mn = np.minimum(start, end) * scale + trans
        mx = np.maximum(start, end) * scale + trans
        if int(fb.get("denseMode", 0)) != 0:
            raise ValueError("only denseMode 0 fluid blocks are supported")
        fluid.append(fluid_block(mn, mx, r))
    fluid_arr = np.concatenate(fluid, axis=0) if fluid else np.zeros((0, 3))
    fluid_arr = fluid_arr + _jitter(fluid_arr.shape[0], jitter * r, seed)
    # FluidModels: particle files appended after the blocks (DemoBase::initFluidData,
    # Demos/Common/DemoBase.cpp:514-534), x = R (s x) + t; velocities as stored.
    fluid_vel = [np.zeros_like(fluid_arr)]
    models = [fluid_arr]
    any_vel = False
    for fm in j.get("FluidModels", []):
        if "particleFile" not in fm:
            continue
        x, v = read_bgeo(_scene_relative(path, fm["particleFile"]))
        t, rot = _body_transform(fm)
        sc = float(fm.get("scale", 1.0))
        models.append((x.astype(np.float64) * sc) @ rot.T + t)
        fluid_vel.append(np.zeros_like(x, dtype=np.float64) if v is None else v.astype(np.float64))
        any_vel = any_vel or v is not None
    fluid_arr = np.concatenate(models, axis=0)
    walls = []
    bmin = bmax = None
    for rb in j.get("RigidBodies", []):
        scale = np.asarray(_readvec(rb.get("scale"), (1.0, 1.0, 1.0)))
        trans = np.asarray(_readvec(rb.get("translation"), (0.0, 0.0, 0.0)))
        if rb.get("particleFile"):
            # boundary samples from a file (Demos/StaticBoundaryDemo/main.cpp:416-420): x = R (s0 x) + t
            x, _ = read_bgeo(_scene_relative(path, rb["particleFile"]))
            t, rot = _body_transform(rb)
            pts = (x.astype(np.float64) * scale[0]) @ rot.T + t
            walls.append(pts)
            if pts.shape[0]:
                mn, mx = pts.min(axis=0), pts.max(axis=0)
                bmin = mn if bmin is None else np.minimum(bmin, mn)
                bmax = mx if bmax is None else np.maximum(bmax, mx)
            continue
        geo = str(rb.get("geometryFile", ""))
        if "box" not in geo.lower():
            raise ValueError(f"only box rigid bodies are supported, got {geo!r}")
        mn = trans - 0.5 * scale
        mx = trans + 0.5 * scale
        walls.append(box_wall(mn, mx, 2.0 * r))
        bmin = mn if bmin is None else np.minimum(bmin, mn)
        bmax = mx if bmax is None else np.maximum(bmax, mx)
    wall_arr = np.concatenate(walls, axis=0) if walls else np.zeros((0, 3))
    return Scene(
        config=cfg,
        fluid=fluid_arr.astype(np.float32),
        boundary=wall_arr.astype(np.float32),
        fluid_velocity=np.concatenate(fluid_vel, axis=0).astype(np.float32) if any_vel else None,
        name=path.stem,
        box_min=tuple(bmin) if bmin is not None else None,
        box_max=tuple(bmax) if bmax is not None else None,
    )


def load_scene_native(path: str | Path) -> tuple:
    """Reads a reference JSON scene with the library's own reader (dfsph_scene_load, the path C and
    C++ callers use). Returns (dfsph_scene struct, fluid (N, 3) float32, fluid velocity (N, 3) float32
    or None, boundary (B, 3) float32)."""
    import ctypes as C

    from . import _capi

    lib = _capi.load()
    sc = _capi.DfsphScene()
    h = C.c_void_p()
    _capi.check(lib, None, lib.dfsph_scene_load(str(path).encode(), C.byref(sc), C.byref(h)))
    try:
        n, nb, hv = C.c_uint32(), C.c_uint32(), C.c_int()
        _capi.check(lib, None, lib.dfsph_scene_file_counts(h, C.byref(n), C.byref(nb), C.byref(hv)))
        x = np.zeros((n.value, 3), np.float32)
        v = np.zeros((n.value, 3), np.float32)
        b = np.zeros((nb.value, 3), np.float32)
        _capi.check(lib, None, lib.dfsph_scene_file_fluid(h, x.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)))
        _capi.check(lib, None, lib.dfsph_scene_file_boundary(h, b.ctypes.data_as(C.c_void_p)))
    finally:
        lib.dfsph_scene_file_free(h)
    return sc, x, (v if hv.value else None), b


# Synthetic scenes of the five benchmark configurations. Every box dimension is twice the stated
# one because a lattice of spacing 2r with the stated particle counts does not fit the stated boxes
# (e.g. 30 x 2r = 1.5 m of fluid for a 1 m box); N, r, spacing, h = 4r, mass, dt and tolerances are
# kept as stated.
SYNTHETIC = {
    1: dict(name="dam_break_27k", counts=(30, 30, 30), radius=0.025, box=(2.0, 2.0, 2.0), seed=1,
            max_error=0.01, cfl_max=0.005),
    2: dict(name="dam_break_250k", counts=(63, 63, 63), radius=0.0125, box=(4.0, 2.0, 2.0), seed=2,
            max_error=0.01, cfl_max=0.005),
    3: dict(name="sloshing_1m", counts=(100, 100, 100), radius=0.01, box=(8.0, 4.0, 4.0), seed=3,
            max_error=0.01, cfl_max=0.005),
    4: dict(name="column_2m", counts=(100, 200, 100), radius=0.008, box=(6.0, 6.0, 6.0), seed=4,
            max_error=0.005, cfl_max=0.008),
    5: dict(name="wave_tank_4m", counts=(400, 100, 100), radius=0.01, box=(16.0, 4.0, 4.0), seed=5,
            max_error=0.01, cfl_max=0.005),
}


def synthetic_scene(config: int, jitter: float = 0.01, time_step: float | None = None, cfl: bool = False,
                    counts=None) -> Scene:
    """Seeded synthetic scene of benchmark configuration `config` (1..5). counts overrides the lattice
    size (same radius, box and seed) for reduced test cases."""
    spec = SYNTHETIC[config]
    r = spec["radius"]
    cnt = tuple(counts) if counts is not None else spec["counts"]
    fluid = lattice_block(cnt, r)
    fluid = fluid + _jitter(fluid.shape[0], jitter * r, spec["seed"])
    box = np.asarray(spec["box"], dtype=np.float64)
    walls = box_wall((0.0, 0.0, 0.0), box, 2.0 * r)
    cfg = Configuration(
        timeStepSize=time_step if time_step is not None else spec["cfl_max"],
        particleRadius=r,
        density0=1000.0,
        viscosity=0.01,
        gravitation=(0.0, -9.81, 0.0),
        cflMethod=1 if cfl else 0,
        cflFactor=0.4,
        cflMaxTimeStepSize=spec["cfl_max"],
        maxIterations=100,
        maxError=spec["max_error"],
        maxIterationsV=100,
        maxErrorV=0.1,
        enableDivergenceSolver=True,
    )
    return Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=walls.astype(np.float32),
                 name=spec["name"] if counts is None else f"{spec['name']}_{'x'.join(map(str, cnt))}",
                 box_min=(0.0, 0.0, 0.0), box_max=tuple(box), meta=dict(config=config, seed=spec["seed"]))


def sloshing_wall_motion(t: float, amplitude: float = 0.1, period: float = 2.0):
    """The sloshing tank's prescribed wall motion at simulated time t: a rigid translation along x,
    x(t) = amplitude sin(2 pi t / period). Returns (position, velocity) of the walls' frame, for
    DFSPHCUDA.move_boundary_rigid."""
    w = 2.0 * np.pi / period
    return (amplitude * np.sin(w * t), 0.0, 0.0), (amplitude * w * np.cos(w * t), 0.0, 0.0)


def column_scene(counts=(10, 80, 10), radius: float = 0.008, time_step: float = 0.004, max_error: float = 0.005,
                 jitter: float = 0.01, seed: int = 4, headroom: float = 1.25) -> Scene:
    """A tall resting water column in a tank that fits its footprint (the lid `headroom` times the
    column height up). The pressure grows with depth, so the pressure solve is stiff: from the
    reference warm start the Jacobi iteration needs tens of sweeps per step at a 0.005 % tolerance,
    which makes it the workload on which warm-start quality shows."""
    cnt = tuple(int(c) for c in counts)
    fluid = lattice_block(cnt, radius)
    fluid = fluid + _jitter(fluid.shape[0], jitter * radius, seed)
    d = 2.0 * radius
    box = np.array([(cnt[0] + 1) * d, (cnt[1] + 1) * d * headroom, (cnt[2] + 1) * d])
    box = np.round(box / d) * d
    walls = box_wall((0.0, 0.0, 0.0), box, d)
    cfg = Configuration(timeStepSize=time_step, particleRadius=radius, density0=1000.0, viscosity=0.01,
                        gravitation=(0.0, -9.81, 0.0), cflMethod=0, cflFactor=0.4, cflMaxTimeStepSize=time_step,
                        maxIterations=100, maxError=max_error, maxIterationsV=100, maxErrorV=0.1,
                        enableDivergenceSolver=True)
    return Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=walls.astype(np.float32),
                 name=f"column_{'x'.join(map(str, cnt))}", box_min=(0.0, 0.0, 0.0), box_max=tuple(box),
                 meta=dict(seed=seed))


def read_bgeo(path):
    """Reads a partio .bgeo particle file (Houdini BGEO v5, compressed or plain) through the library's
    reader: (positions (N, 3) float32, velocities (N, 3) float32 or None when the file has none),
    untransformed (PartioReaderWriter::readParticles, Utilities/PartioReaderWriter.cpp:8-66)."""
    import ctypes as C

    from . import _capi

    lib = _capi.load()
    n, hv = C.c_uint64(0), C.c_int(0)
    bp = str(path).encode()
    _capi.check(lib, None, lib.dfsph_bgeo_read(bp, None, None, 0, C.byref(n), C.byref(hv)))
    x = np.zeros((n.value, 3), np.float32)
    v = np.zeros((n.value, 3), np.float32)
    _capi.check(lib, None, lib.dfsph_bgeo_read(bp, x.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p),
                                               n.value, C.byref(n), C.byref(hv)))
    return x, (v if hv.value else None)


def write_bgeo(path, position, velocity=None, radius: float = 0.0) -> None:
    """Writes a gzip-compressed partio .bgeo file with the attributes of the reference's
    PartioReaderWriter::writeParticles (Utilities/PartioReaderWriter.cpp:189-231): position,
    velocity (when given), pscale (when radius != 0) and id."""
    import ctypes as C

    from . import _capi

    lib = _capi.load()
    x = np.ascontiguousarray(np.asarray(position, np.float32).reshape(-1, 3))
    v = None if velocity is None else np.ascontiguousarray(np.asarray(velocity, np.float32).reshape(-1, 3))
    if v is not None and v.shape != x.shape:
        raise ValueError("velocity must have the shape of position")
    _capi.check(lib, None, lib.dfsph_bgeo_write(str(path).encode(), x.ctypes.data_as(C.c_void_p),
                                                None if v is None else v.ctypes.data_as(C.c_void_p),
                                                x.shape[0], float(radius)))


def angle_axis_matrix(axis, angle: float) -> np.ndarray:
    """Rotation of `angle` radians about `axis` by the Rodrigues formula
    R = cos(a) I + (1 - cos(a)) u u^T + sin(a) [u]x, with u taken as given (the scene's
    rotationAxis, as Eigen's AngleAxis uses it in SceneLoader.cpp:228-233)."""
    u = np.asarray(axis, np.float64).reshape(3)
    c, s = np.cos(angle), np.sin(angle)
    cross = np.array([[0.0, -u[2], u[1]], [u[2], 0.0, -u[0]], [-u[1], u[0], 0.0]])
    return c * np.eye(3) + (1.0 - c) * np.outer(u, u) + s * cross


def _body_transform(obj: dict):
    t = np.asarray(_readvec(obj.get("translation"), (0.0, 0.0, 0.0)))
    if obj.get("rotationAxis") is not None and obj.get("rotationAngle") is not None:
        r = angle_axis_matrix(obj["rotationAxis"], float(obj["rotationAngle"]))
    else:
        r = np.eye(3)
    return t, r


def read_particle_file(path):
    """Reads a particle file of the reference's snapshot format (UnifiedParticleSet::load_from_file,
    DFSPH_c_arrays_structure.cpp:488-600): header "N has_factor velocity_impacted is_dynamic", for a
    dynamic body one line of 13 rigid-body values, then N lines "mass x y z vx vy vz". Returns
    (mass (N,), position (N, 3), velocity (N, 3), header flags (3,))."""
    tok = Path(path).read_text().split()
    n = int(tok[0])
    flags = tuple(int(t) for t in tok[1:4])
    k = 4 + (13 if flags[2] else 0)
    vals = np.asarray(tok[k:k + 7 * n], dtype=np.float64)
    if vals.size != 7 * n:
        raise ValueError(f"{path}: expected {n} particle lines")
    vals = vals.reshape(n, 7)
    return vals[:, 0].copy(), vals[:, 1:4].copy(), vals[:, 4:7].copy(), flags


def write_particle_file(path, mass, position, velocity=None, flags=(1, 1, 0)):
    """Writes a particle file of the reference's snapshot format (UnifiedParticleSet::write_to_file,
    DFSPH_c_arrays_structure.cpp:424-486), 9 significant digits."""
    m = np.asarray(mass, dtype=np.float64).reshape(-1)
    x = np.asarray(position, dtype=np.float64).reshape(-1, 3)
    v = np.zeros_like(x) if velocity is None else np.asarray(velocity, dtype=np.float64).reshape(-1, 3)
    lines = [f"{m.size} {flags[0]} {flags[1]} {flags[2]}"]
    lines += [" ".join(f"{e:.9g}" for e in (m[i], *x[i], *v[i])) + " " for i in range(m.size)]
    Path(path).write_text("\n".join(lines) + "\n")
