"""Surfaces of the simple open boundary (the reference's BufferFluidSurface shapes,
SPlisHSPlasH/DFSPH/BufferFluidSurface.cu:421-900) and the reference's built-in configurations
(OpenBoundariesSimple::init, OpenBoundariesSimple.cu:127-255).

The open boundary itself runs on the device (DFSPHCUDA.init_open_boundary / apply_open_boundary over
dfsph_open_boundary_init / _apply in include/dfsph_c.h).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from ._capi import (MAX_SURFACE_MESHES, SURFACE_CUBOID, SURFACE_CYLINDER, SURFACE_MESH, SURFACE_PLANE, SURFACE_SPHERE,
                    SURFACE_STAR, Surface)


def _v3(dst, v) -> None:
    a = np.asarray(v, dtype=np.float32).reshape(3)
    for k in range(3):
        dst[k] = float(a[k])


def plane(origin, normal, reversed: bool = False) -> Surface:
    """Half space (x - origin) . normal >= 0 (BufferFluidSurface::setPlane)."""
    s = Surface(type=SURFACE_PLANE, reversed=int(reversed))
    _v3(s.origin, origin)
    _v3(s.normal, normal)
    return s


def cuboid(center, half_lengths, reversed: bool = False) -> Surface:
    """|x - center| < half_lengths component-wise (setCuboid)."""
    s = Surface(type=SURFACE_CUBOID, reversed=int(reversed))
    _v3(s.center, center)
    _v3(s.half_lengths, half_lengths)
    return s


def cylinder(center, half_height: float, radius: float, reversed: bool = False) -> Surface:
    """Cylinder along y (setCylinder)."""
    s = Surface(type=SURFACE_CYLINDER, reversed=int(reversed), radius=float(np.float32(radius)))
    _v3(s.center, center)
    _v3(s.half_lengths, (0.0, half_height, 0.0))
    return s


def sphere(center, radius: float, reversed: bool = False) -> Surface:
    s = Surface(type=SURFACE_SPHERE, reversed=int(reversed), radius=float(np.float32(radius)))
    _v3(s.center, center)
    return s


def star(center, half_height: float, radius: float, radius_internal: float, points: int, direction,
         reversed: bool = False) -> Surface:
    """Infinite-prism star along y with `points` linear-sided points, the first along `direction`
    (setStar)."""
    if points < 1:
        raise ValueError("a star needs at least one point")
    s = Surface(type=SURFACE_STAR, reversed=int(reversed), radius=float(np.float32(radius)),
                radius_internal=float(np.float32(radius_internal)), points=int(points))
    _v3(s.center, center)
    _v3(s.half_lengths, (0.0, half_height, 0.0))
    _v3(s.direction, direction)
    return s


def mesh(mesh_id: int = 0, offset=(0.0, 0.0, 0.0), reversed: bool = False) -> Surface:
    """The closed triangle mesh registered under mesh_id (DFSPHCUDA.set_surface_mesh), translated by
    offset (MeshPerso with its offset): inside = an odd number of crossings of the fixed ray with its
    triangles."""
    if not 0 <= mesh_id < MAX_SURFACE_MESHES:
        raise ValueError(f"mesh id must be in [0, {MAX_SURFACE_MESHES})")
    s = Surface(type=SURFACE_MESH, reversed=int(reversed), points=int(mesh_id))
    _v3(s.center, offset)
    return s


def read_obj(path, lib_path=None) -> tuple[np.ndarray, np.ndarray]:
    """(vertices (V, 3) float32, triangles (T, 3) uint32) of a Wavefront OBJ file, read by the
    library's dfsph_read_obj (no GPU needed): faces split into fans, other records skipped."""
    import ctypes as C

    from . import _capi

    lib = _capi.load(lib_path)
    nv, nt = C.c_uint32(), C.c_uint32()
    p = str(path).encode()
    _capi.check(lib, None, lib.dfsph_read_obj(p, None, 0, C.byref(nv), None, 0, C.byref(nt)))
    v = np.zeros((nv.value, 3), np.float32)
    t = np.zeros((nt.value, 3), np.uint32)
    _capi.check(lib, None, lib.dfsph_read_obj(p, v.ctypes.data_as(C.c_void_p), nv.value, C.byref(nv),
                                              t.ctypes.data_as(C.c_void_p), nt.value, C.byref(nt)))
    return v, t


def box_mesh(lo, hi) -> tuple[np.ndarray, np.ndarray]:
    """(vertices, triangles) of the closed axis-aligned box [lo, hi]: 8 vertices, 12 triangles with
    outward normals."""
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    v = np.array([[lo[0] if i & 1 == 0 else hi[0], lo[1] if i & 2 == 0 else hi[1], lo[2] if i & 4 == 0 else hi[2]]
                  for i in range(8)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = np.array([tri for a, b, c, d in quads for tri in ((a, b, c), (a, c, d))], np.uint32)
    return v, t


def _f32(x) -> float:
    return float(np.float32(x))


def preset(config: int, particle_radius: float):
    """(boundary, interior, fluid_surface, inflow file name) of the reference's configuration
    `config`; the interior is the boundary shrunk by 3 r (5 r for the corridor), the fluid surface
    the plane y = 1 (inside below). Unknown configurations raise ValueError (the reference exits)."""
    r3 = _f32(np.float32(particle_radius) * np.float32(3))
    surf = plane((0.0, 1.0, 0.0), (0.0, -1.0, 0.0))
    cyl = {0: (1.5, "inflowPositionsSet_cylinder.txt"), 200: (2.5, "inflowPositionsSet_cylinder_r2_5m.txt"),
           210: (3.5, "inflowPositionsSet_cylinder_r3_5m.txt"), 220: (4.25, "inflowPositionsSet_cylinder_r4_25m.txt"),
           300: (5.0, "inflowPositionsSet_cylinder_r5m.txt")}
    if config in cyl:
        rad, name = cyl[config]
        return (cylinder((0, 0, 0), 10, rad), cylinder((0, 0, 0), 10, _f32(np.float32(rad) - np.float32(r3))),
                surf, name)
    sph = {100: (1.5, "inflowPositionsSet_sphere_1_5m.txt"), 500: (2.5, "inflowPositionsSet_sphere_2_5m.txt")}
    if config in sph:
        rad, name = sph[config]
        return (sphere((0, 1, 0), rad), sphere((0, 1, 0), _f32(np.float32(rad) - np.float32(r3))), surf, name)
    stars = {400: (3.5 / 2.0, 2.0 / 2.0, "inflowPositionsSet_star_re1_75_ri1.txt"),
             600: (3.5, 2.0, "inflowPositionsSet_star_re3_5_ri2.txt")}
    if config in stars:
        re, ri, name = stars[config]
        return (star((0, 0, 0), 10, re, ri, 5, (0, 0, 1)),
                star((0, 0, 0), 10, _f32(np.float32(re) - np.float32(r3)), _f32(np.float32(ri) - np.float32(r3)), 5,
                     (0, 0, 1)),
                surf, name)
    if config == 1001:
        r5 = np.float32(particle_radius) * np.float32(5)
        return (cuboid((0, 0, 0), (1, 10, 5)), cuboid((0, 0, -1), (1, 10, _f32(np.float32(1 + 5) - r5))), surf,
                "inflowPositionsSet_corridor.txt")
    raise ValueError(f"no open-boundary configuration {config}")


def read_inflow_samples(folder, name: str) -> np.ndarray:
    """Sample positions of an inflow file <folder>/inflowFolder/<name> (the reference's particle
    text format, UnifiedParticleSet::load_from_file)."""
    from .scene import read_particle_file

    _, x, _, _ = read_particle_file(Path(folder) / "inflowFolder" / name)
    return x.astype(np.float32)
