"""Generates the .bgeo golden fixtures with the reference's own partio writer.

Run from the repository root after `make -C oracle/ref_harness` (which compiles the reference's
Utilities/PartioReaderWriter.cpp and its vendored partio into oracle/_ref/libpartio_pin.so):

    python tests/golden/bgeo/make_bgeo_golden.py

Writes, for each case, <case>.bgeo (written by PartioReaderWriter::writeParticles) and <case>.npz
(the inputs), and golden.json. It also reads the reference's sample files data/models/*.bgeo with
partio and with this library's reader and records that both agree (counts and a SHA-256 of the
positions), so the reader is pinned on files partio did not write in this run.
"""
import ctypes as C
import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[2]
sys.path.insert(0, str(ROOT))
from splishsplash_for_cuda_b200.scene import read_bgeo  # noqa: E402

# the reference checkout: REF_DIR, else a directory named "reference" beside this repository
REF_DIR = Path(os.environ.get("REF_DIR", str(ROOT.parent / "reference")))


def pin():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libpartio_pin.so"))
    lib.pin_partio_read.restype = C.c_long
    lib.pin_partio_read.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_long]
    lib.pin_partio_write.restype = None
    lib.pin_partio_write.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_void_p, C.c_float]
    return lib


def pin_read(lib, path, cap=1 << 22):
    x = np.zeros((cap, 3), np.float32)
    v = np.zeros((cap, 3), np.float32)
    n = lib.pin_partio_read(str(path).encode(), x.ctypes.data, v.ctypes.data, cap)
    if n < 0:
        raise RuntimeError(f"partio could not read {path} ({n})")
    return x[:n], v[:n]


CASES = {
    # name: (n, with velocity, radius)
    "fluid_vel_pscale": (300, True, 0.025),
    "boundary_positions": (1000, False, 0.0),
    "empty": (0, True, 0.01),
}


def main():
    lib = pin()
    rng = np.random.default_rng(20260)
    out = {"cases": {}, "reference_samples": {}}
    for name, (n, with_vel, radius) in CASES.items():
        x = (rng.uniform(-2.0, 2.0, size=(n, 3))).astype(np.float32)
        v = rng.normal(size=(n, 3)).astype(np.float32) if with_vel else None
        np.savez(HERE / f"{name}.npz", x=x, v=v if v is not None else np.zeros((0, 3), np.float32))
        lib.pin_partio_write(str(HERE / f"{name}.bgeo").encode(), n, x.ctypes.data,
                             v.ctypes.data if v is not None else None, radius)
        out["cases"][name] = {"n": n, "velocity": with_vel, "radius": radius}
    for f in sorted((REF_DIR / "data" / "models").glob("*.bgeo")):
        xp, vp = pin_read(lib, f)
        xo, vo = read_bgeo(f)
        vo = np.zeros_like(xo) if vo is None else vo
        assert np.array_equal(xp, xo) and np.array_equal(vp, vo), f
        out["reference_samples"][f.name] = {
            "n": int(xp.shape[0]),
            "positions_sha256": hashlib.sha256(xp.tobytes()).hexdigest(),
            "partio_and_library_agree": True,
        }
    (HERE / "golden.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
