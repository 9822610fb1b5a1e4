"""Generates tests/golden/open_boundary/meshes.npz with the reference's own mesh inside test.

Run from the repository root after `make -C oracle/ref_harness` (which builds
oracle/_ref/libsurface_pin.so from SPlisHSPlasH/DFSPH/BufferFluidSurface.cu):

    python tests/golden/open_boundary/make_mesh_golden.py

Three closed meshes (an L-shaped prism, which is not convex; a box; an octahedron), each moved by two
offsets; per case seeded uniform points plus the points of a lattice whose planes pass through mesh
vertices and edges. `inside` is MeshPerso::isInside's answer (the box of the vertices and the origin,
the fixed ray, RayIntersectsTriangle) as pin_mesh_inside runs it.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[2]
sys.path.insert(0, str(ROOT))
from splishsplash_for_cuda_b200 import open_boundary as ob  # noqa: E402


def l_prism():
    """Prism over the L outline (0,0) (2,0) (2,1) (1,1) (1,2) (0,2) from z = 0 to 1, moved by 0.3."""
    outline = np.array([(0, 0), (2, 0), (2, 1), (1, 1), (1, 2), (0, 2)], np.float32)
    n = len(outline)
    v = np.concatenate([np.c_[outline, np.zeros(n)], np.c_[outline, np.ones(n)]]).astype(np.float32)
    tris = []
    for a, b, c in [(0, 1, 2), (0, 2, 3), (0, 3, 5), (3, 4, 5)]:
        tris += [(a, c, b), (a + n, b + n, c + n)]
    for i in range(n):
        j = (i + 1) % n
        tris += [(i, j, j + n), (i, j + n, i + n)]
    return v + np.float32(0.3), np.array(tris, np.uint32)


def octahedron():
    v = np.array([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)], np.float32) * 0.8 + 1.2
    t = np.array([(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)], np.uint32)
    return v.astype(np.float32), t


def meshes():
    return [l_prism(), ob.box_mesh((0.2, 0.1, 0.4), (1.7, 1.1, 0.9)), octahedron()]


def main():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libsurface_pin.so"))
    lib.pin_mesh_inside.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.c_uint32, C.c_void_p]
    rng = np.random.default_rng(777)
    out = {}
    g = (np.arange(0.0, 2.6, 0.15) + 0.1).astype(np.float32)
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    case = 0
    for m, (v, t) in enumerate(meshes()):
        for off in ((0.0, 0.0, 0.0), (0.05, -0.1, 0.2)):
            off = np.array(off, np.float32)
            p = np.concatenate([rng.uniform(-0.3, 2.7, size=(2000, 3)).astype(np.float32), grid])
            inside = np.zeros(p.shape[0], np.uint8)
            assert lib.pin_mesh_inside(v.ctypes.data, v.shape[0], t.ctypes.data, t.shape[0], off.ctypes.data,
                                       p.ctypes.data, p.shape[0], inside.ctypes.data) == 0
            out[f"v{case}"], out[f"t{case}"], out[f"off{case}"] = v, t, off
            out[f"p{case}"], out[f"in{case}"] = p, inside
            print(f"mesh {m} offset {off}: {int(inside.sum())} of {p.shape[0]} inside")
            case += 1
    out["cases"] = np.array(case)
    np.savez_compressed(HERE / "meshes.npz", **out)


if __name__ == "__main__":
    main()
