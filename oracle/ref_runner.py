"""Runs the reference CPU solver harness (oracle/_ref/dfsph_ref) and the reference pin library
(oracle/_ref/libref_pins.so). Test infrastructure and CPU baseline only.

Both are built by oracle/ref_harness/Makefile from the reference's own sources; when they are
absent (no reference tree on this machine and nothing prebuilt) `available()` is False.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR_OUT = HERE / "_ref"
REF_BIN = REF_DIR_OUT / "dfsph_ref"
PINS_LIB = REF_DIR_OUT / "libref_pins.so"


def available() -> bool:
    return REF_BIN.exists() and PINS_LIB.exists()


def run_reference_full(scene, steps: int = 1, warmup: int = 0, time_budget: float | None = None,
                       threads: int | None = None, kernel: int = 0, mass: float | None = None) -> dict:
    """Runs TimeStepDFSPH on `scene` in a scratch directory. kernel: 0 analytic cubic (as the GPU
    path), 3 the reference default precomputed table. mass None keeps the reference default
    (FluidModel::initMasses: 0.8 rho0 (2r)^3). Returns timings, per-step iteration counts and the final
    fields in original particle order."""
    cfg = scene.config
    n, nb = scene.n_fluid, scene.n_boundary
    hdr = b"DFRF" + struct.pack("<i", 1)
    hdr += struct.pack("<10d", cfg.particleRadius, cfg.density0, cfg.viscosity, *cfg.gravitation, cfg.timeStepSize,
                       cfg.maxError, cfg.maxErrorV, -1.0 if mass is None else float(mass))
    hdr += struct.pack("<8i", cfg.maxIterations, cfg.maxIterationsV, 1 if cfg.enableDivergenceSolver else 0, kernel,
                       n, nb, warmup, steps)
    hdr += struct.pack("<d", 0.0 if time_budget is None else float(time_budget))
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or os.cpu_count() or 1)
    with tempfile.TemporaryDirectory(prefix="dfsph_ref_") as td:
        inp, outp = Path(td) / "in.bin", Path(td) / "out.bin"
        with open(inp, "wb") as f:
            f.write(hdr)
            f.write(np.ascontiguousarray(scene.fluid, dtype=np.float32).tobytes())
            f.write(np.ascontiguousarray(scene.boundary, dtype=np.float32).tobytes())
        subprocess.run([str(REF_BIN), str(inp), str(outp)], cwd=td, env=env, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        raw = outp.read_bytes()
    done = struct.unpack_from("<i", raw, 0)[0]
    ms = struct.unpack_from("<d", raw, 4)[0]
    off = 12
    its = np.frombuffer(raw, dtype=np.int32, count=done, offset=off)
    off += 4 * done
    itsv = np.frombuffer(raw, dtype=np.int32, count=done, offset=off)
    off += 4 * done
    arr = np.frombuffer(raw, dtype=np.float64, offset=off)
    x = arr[: 3 * n].reshape(n, 3)
    v = arr[3 * n: 6 * n].reshape(n, 3)
    rho = arr[6 * n: 7 * n]
    factor = arr[7 * n: 8 * n]
    psi = arr[8 * n: 8 * n + nb]
    return dict(steps=done, ms_per_step=ms, iterations=its.copy(), iterations_v=itsv.copy(), position=x.copy(),
                velocity=v.copy(), density=rho.copy(), factor=factor.copy(), boundary_psi=psi.copy())


def run_reference(ref_bin, scene, steps, warmup, time_budget, threads):
    """(ms_per_step, steps_timed) of the reference CPU solver on `scene` (bench's CPU baseline), with
    the reference's default kernel (the 10000-sample cubic table, DemoBase.cpp setKernel(3))."""
    r = run_reference_full(scene, steps=steps, warmup=warmup, time_budget=time_budget, threads=threads, kernel=3)
    return r["ms_per_step"], r["steps"]


_pins = None


def _pins_lib():
    global _pins
    if _pins is None:
        lib = C.CDLL(str(PINS_LIB))
        f, u, i = C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.POINTER(C.c_int)
        lib.ref_cubic_values.argtypes = [C.c_float, f, C.c_uint32, f, f]
        lib.ref_neighbor_lists.argtypes = [f, C.c_uint32, f, C.c_uint32, C.c_float, i, u, u, C.c_uint32]
        _pins = lib
    return _pins


def ref_cubic_values(H: float, r: np.ndarray):
    """W(r) and d/dx of W at (r, 0, 0) from the reference's FP32 CubicKernelPerso."""
    lib = _pins_lib()
    r = np.ascontiguousarray(r, dtype=np.float32)
    w = np.empty_like(r)
    g = np.empty_like(r)
    fp = C.POINTER(C.c_float)
    lib.ref_cubic_values(C.c_float(H), r.ctypes.data_as(fp), r.size, w.ctypes.data_as(fp), g.ctypes.data_as(fp))
    return w, g


def ref_neighbor_lists(fluid: np.ndarray, boundary: np.ndarray, H: float, offset, row: int = 128):
    """Neighbour lists through the reference's cell macros over its dense 256^3 table."""
    lib = _pins_lib()
    fl = np.ascontiguousarray(fluid, dtype=np.float32)
    bd = np.ascontiguousarray(boundary, dtype=np.float32)
    off = np.ascontiguousarray(offset, dtype=np.int32)
    n = fl.shape[0]
    counts = np.zeros((n, 2), dtype=np.uint32)
    lists = np.zeros((n, row), dtype=np.uint32)
    fp, up = C.POINTER(C.c_float), C.POINTER(C.c_uint32)
    rc = lib.ref_neighbor_lists(fl.ctypes.data_as(fp), n, bd.ctypes.data_as(fp), bd.shape[0], C.c_float(H),
                                off.ctypes.data_as(C.POINTER(C.c_int)), counts.ctypes.data_as(up),
                                lists.ctypes.data_as(up), row)
    if rc != 0:
        raise ValueError("scene outside the reference's 256^3 cell table")
    return counts, lists
