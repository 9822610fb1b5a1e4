"""Generates tests/golden/open_boundary/surfaces.npz with the reference's own BufferFluidSurface.

Run from the repository root after `make -C oracle/ref_harness` (which compiles
SPlisHSPlasH/DFSPH/BufferFluidSurface.cu as host code into oracle/_ref/libsurface_pin.so):

    python tests/golden/open_boundary/make_surface_golden.py

For each shape of the simple open boundary (plane, cuboid, cylinder, sphere, star; each also
reversed) it evaluates isinside() and getNormal() on seeded points, half of them within a few
particle radii of the surface, and stores points, the surface records and the results.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[2]
sys.path.insert(0, str(ROOT))
from splishsplash_for_cuda_b200 import open_boundary as ob  # noqa: E402


def shapes():
    out = [
        ob.plane((0.0, 1.0, 0.0), (0.0, -1.0, 0.0)),
        ob.plane((0.3, -0.2, 0.1), (0.3, 0.5, -0.8)),
        ob.cuboid((0.0, 0.0, 0.0), (1.0, 10.0, 5.0)),
        ob.cuboid((0.1, 0.2, -1.0), (0.9, 0.4, 0.97)),
        ob.cylinder((0.0, 0.0, 0.0), 10.0, 1.5),
        ob.cylinder((0.2, 0.5, -0.1), 0.6, 0.97),
        ob.sphere((0.0, 1.0, 0.0), 1.5),
        ob.sphere((0.3, -0.2, 0.4), 0.55),
        ob.star((0.0, 0.0, 0.0), 10.0, 1.75, 1.0, 5, (0.0, 0.0, 1.0)),
        ob.star((0.1, 0.0, -0.2), 0.8, 1.2, 0.6, 7, (0.6, 0.0, 0.8)),
        ob.star((0.0, 0.0, 0.0), 10.0, 3.5, 2.0, 3, (1.0, 0.0, 0.0)),
    ]
    rev = []
    for s in out:
        r = type(s).from_buffer_copy(bytes(s))
        r.reversed = 1
        rev.append(r)
    return out + rev


def main():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libsurface_pin.so"))
    lib.pin_surface_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(4242)
    recs, pts, ins, nrm = [], [], [], []
    for s in shapes():
        far = rng.uniform(-4.0, 4.0, size=(200, 3))
        # points near the outline: scaled copies of far points around the shape's center / origin
        c = np.array(s.origin if s.type == 0 else s.center, dtype=np.float64)
        d = rng.normal(size=(200, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        near = c + d * rng.uniform(0.0, 4.0, size=(200, 1))
        p = np.concatenate([far, near]).astype(np.float32)
        inside = np.zeros(p.shape[0], np.uint8)
        normal = np.zeros((p.shape[0], 3), np.float32)
        assert lib.pin_surface_eval(C.addressof(s), p.ctypes.data, p.shape[0], inside.ctypes.data,
                                    normal.ctypes.data) == 0
        recs.append(np.frombuffer(bytes(s), dtype=np.uint8))
        pts.append(p)
        ins.append(inside)
        nrm.append(normal)
    np.savez_compressed(HERE / "surfaces.npz", surfaces=np.stack(recs), points=np.stack(pts), inside=np.stack(ins),
                        normal=np.stack(nrm))
    print(len(recs), "surfaces,", pts[0].shape[0], "points each; inside fractions",
          [round(float(i.mean()), 3) for i in ins])


if __name__ == "__main__":
    main()
