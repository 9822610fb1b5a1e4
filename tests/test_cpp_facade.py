"""The C++ facade (include/dfsph.hpp): tests/cpp/facade_demo.cpp is compiled against the library with
g++ and run. Without a GPU it must fail loudly (dfsph::Error, exit code 3); on a GPU its fused step()
and its piecewise cuda_* sequence must give the Python facade's state bit for bit."""
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.scene import synthetic_scene

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "splishsplash_for_cuda_b200"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")


def build_demo(tmp_path: Path) -> Path:
    _capi.load()  # the library must exist
    exe = tmp_path / "facade_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "facade_demo.cpp"), "-L", str(LIBDIR), "-ldfsph_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return exe


def write_scene(path: Path, scene, cfl: int = 0, precision: int = 32) -> None:
    c = scene.config
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", scene.n_fluid, scene.n_boundary))
        f.write(struct.pack("<10d", c.particleRadius, c.density0, c.viscosity, c.timeStepSize, c.maxError,
                            c.maxErrorV, cfl, precision, c.cflFactor, c.cflMaxTimeStepSize))
        f.write(np.ascontiguousarray(scene.fluid, np.float32).tobytes())
        f.write(np.ascontiguousarray(scene.boundary, np.float32).tobytes())


def read_out(path: Path):
    b = path.read_bytes()
    off, runs = 0, []
    for _ in range(2):
        (n,) = struct.unpack_from("<i", b, off)
        off += 4
        x = np.frombuffer(b, np.float32, 3 * n, off).reshape(n, 3)
        off += 12 * n
        v = np.frombuffer(b, np.float32, 3 * n, off).reshape(n, 3)
        off += 12 * n
        runs.append((x, v))
    its, itv = struct.unpack_from("<ii", b, off)
    return runs, its, itv


def test_facade_fails_loudly_without_gpu(tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    exe = build_demo(tmp_path)
    s = synthetic_scene(1, counts=(4, 4, 4))
    write_scene(tmp_path / "s.bin", s)
    r = subprocess.run([str(exe), str(tmp_path / "s.bin"), "1", str(tmp_path / "o.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 3 and "DFSPH error" in r.stderr
    assert not (tmp_path / "o.bin").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("cfl", [0, 1])
def test_facade_matches_python_facade(tmp_path, cuda_lib, cfl):
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    exe = build_demo(tmp_path)
    s = synthetic_scene(1, counts=(12, 12, 12), cfl=bool(cfl))
    write_scene(tmp_path / "s.bin", s, cfl=s.config.cflMethod)
    r = subprocess.run([str(exe), str(tmp_path / "s.bin"), "10", str(tmp_path / "o.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    (xf, vf), (xp, vp) = read_out(tmp_path / "o.bin")[0]
    its, itv = read_out(tmp_path / "o.bin")[1:]
    d = DFSPHCUDA(s)
    ti = tv = 0
    for _ in range(10):
        st = d.step()
        ti += st.iterations
        tv += st.iterations_v
    assert (its, itv) == (ti, tv)
    assert np.array_equal(xf, d.positions()) and np.array_equal(vf, d.velocities())
    assert np.array_equal(xp, xf) and np.array_equal(vp, vf)


def build_timestep_demo(tmp_path: Path) -> Path:
    _capi.load()
    exe = tmp_path / "timestep_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "timestep_demo.cpp"), "-L", str(LIBDIR), "-ldfsph_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return exe


def _scene_json(tmp_path: Path, cfl: int = 1) -> Path:
    import json

    r = 0.025
    scene = {"Configuration": {"particleRadius": r, "timeStepSize": 0.005, "cflMethod": cfl, "cflFactor": 0.4,
                               "cflMaxTimeStepSize": 0.005, "maxError": 0.01, "maxErrorV": 0.1, "jitter": 0.01,
                               "seed": 4},
             "FluidBlocks": [{"denseMode": 0, "start": [0.0, 0.0, 0.0], "end": [13 * 2 * r] * 3}],
             "RigidBodies": [{"geometryFile": "../models/UnitBox.obj", "translation": [0.5, 0.5, 0.5],
                              "scale": [1.0, 1.0, 1.0]}]}
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(scene))
    return p


def test_timestep_facade_reads_scene_without_python(tmp_path):
    """The C++ TimeStepDFSPH facade's scene reader (dfsph_scene_load) needs no GPU and no Python."""
    from splishsplash_for_cuda_b200.scene import load_scene

    exe = build_timestep_demo(tmp_path)
    p = _scene_json(tmp_path)
    r = subprocess.run([str(exe), "--load", str(p)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    s = load_scene(p)
    assert r.stdout.split() == ["fluid", str(s.n_fluid), "boundary", str(s.n_boundary), "radius", "0.025"]


@pytest.mark.gpu
def test_timestep_facade_from_json_matches_python_facade(tmp_path, cuda_lib):
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
    from splishsplash_for_cuda_b200.scene import load_scene

    exe = build_timestep_demo(tmp_path)
    p = _scene_json(tmp_path)
    r = subprocess.run([str(exe), str(p), "10", str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    b = (tmp_path / "o.bin").read_bytes()
    (n,) = struct.unpack_from("<i", b, 0)
    x = np.frombuffer(b, np.float32, 3 * n, 4).reshape(n, 3)
    v = np.frombuffer(b, np.float32, 3 * n, 4 + 12 * n).reshape(n, 3)
    its, itv = struct.unpack_from("<ii", b, 4 + 24 * n)
    d = DFSPHCUDA(load_scene(p))
    ti = tv = 0
    for _ in range(10):
        st = d.step()
        ti += st.iterations
        tv += st.iterations_v
    assert (its, itv) == (ti, tv)
    assert np.array_equal(x, d.positions()) and np.array_equal(v, d.velocities())


@pytest.mark.gpu
def test_host_operations(tmp_path, cuda_lib):
    """tests/cpp/host_ops_demo.cpp: the reference's host-side DFSPHCUDA operations through the facade
    (snapshot save and load, zeroFluidVelocities, updateTimeStepDuration, the fluid's impact on a
    dynamic body with reduction factors against dfsph_body_wrench, the fluid level and its control);
    the program checks itself."""
    _capi.load()
    exe = tmp_path / "host_ops_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "host_ops_demo.cpp"), "-L", str(LIBDIR), "-ldfsph_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    s = synthetic_scene(1, counts=(10, 10, 10))
    write_scene(tmp_path / "s.bin", s)
    folder = tmp_path / "snap"
    folder.mkdir()
    r = subprocess.run([str(exe), str(tmp_path / "s.bin"), str(folder) + "/"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (folder / "fluid_file.txt").exists() and (folder / "boundaries_file.txt").exists()
