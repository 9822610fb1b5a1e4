"""Partio .bgeo files: the library's reader and writer against files written by the reference's own
PartioReaderWriter (fixtures in tests/golden/bgeo/, made by make_bgeo_golden.py with the partio
library compiled from the reference's sources), byte-exact on the decompressed content; round trips
through that compiled partio when it is present (oracle/_ref/libpartio_pin.so); error handling; and
scenes whose fluid or boundary comes from .bgeo files. No GPU is needed."""
import ctypes as C
import gzip
import json
from pathlib import Path

import numpy as np
import pytest

from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.scene import angle_axis_matrix, load_scene, read_bgeo, write_bgeo

GOLD = Path(__file__).resolve().parent / "golden" / "bgeo"
PIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libpartio_pin.so"
CASES = json.loads((GOLD / "golden.json").read_text())["cases"]


def _inputs(name):
    z = np.load(GOLD / f"{name}.npz")
    c = CASES[name]
    return z["x"], (z["v"] if c["velocity"] else None), c["radius"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_reads_partio_files(name):
    x, v, _ = _inputs(name)
    xr, vr = read_bgeo(GOLD / f"{name}.bgeo")
    assert np.array_equal(xr, x)
    if v is None:
        assert vr is None
    else:
        assert np.array_equal(vr, v)


@pytest.mark.parametrize("name", sorted(CASES))
def test_writer_matches_partio_bytes(name, tmp_path):
    x, v, radius = _inputs(name)
    p = tmp_path / "out.bgeo"
    write_bgeo(p, x, v, radius)
    mine = gzip.decompress(p.read_bytes())
    ref = gzip.decompress((GOLD / f"{name}.bgeo").read_bytes())
    assert mine == ref


def test_plain_uncompressed_file_is_read(tmp_path):
    x, v, _ = _inputs("fluid_vel_pscale")
    plain = tmp_path / "plain.bgeo"
    plain.write_bytes(gzip.decompress((GOLD / "fluid_vel_pscale.bgeo").read_bytes()))
    xr, vr = read_bgeo(plain)
    assert np.array_equal(xr, x) and np.array_equal(vr, v)


def test_errors(tmp_path):
    with pytest.raises(_capi.DfsphError, match="cannot open"):
        read_bgeo(tmp_path / "missing.bgeo")
    bad = tmp_path / "bad.bgeo"
    bad.write_bytes(b"NotBgeo" + bytes(64))
    with pytest.raises(_capi.DfsphError, match="not a bgeo"):
        read_bgeo(bad)
    raw = gzip.decompress((GOLD / "fluid_vel_pscale.bgeo").read_bytes())
    cut = tmp_path / "cut.bgeo"
    cut.write_bytes(raw[:200])
    with pytest.raises(_capi.DfsphError, match="truncated"):
        read_bgeo(cut)
    lib = _capi.load()
    n = C.c_uint64(0)
    x = np.zeros((10, 3), np.float32)
    code = lib.dfsph_bgeo_read(str(GOLD / "fluid_vel_pscale.bgeo").encode(), x.ctypes.data_as(C.c_void_p), None,
                               10, C.byref(n), None)
    assert code == _capi.DFSPH_E_INVALID and n.value == 300
    assert b"capacity" in lib.dfsph_last_error(None)
    with pytest.raises(ValueError):
        write_bgeo(tmp_path / "x.bgeo", np.zeros((4, 3)), np.zeros((3, 3)))


@pytest.mark.skipif(not PIN.exists(), reason="partio compiled from the reference sources is not present")
@pytest.mark.parametrize("n,with_vel,radius", [(1, True, 0.5), (65536, False, 0.0), (65537, True, 0.01),
                                               (70001, False, 0.02)])
def test_round_trip_through_reference_partio(tmp_path, n, with_vel, radius):
    """65,536 points are the last that partio lists with 16-bit indices; above it, 32-bit."""
    lib = C.CDLL(str(PIN))
    lib.pin_partio_read.restype = C.c_long
    lib.pin_partio_read.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_long]
    lib.pin_partio_write.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_void_p, C.c_float]
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, 3)).astype(np.float32)
    v = rng.normal(size=(n, 3)).astype(np.float32) if with_vel else None
    ours, theirs = tmp_path / "ours.bgeo", tmp_path / "theirs.bgeo"
    write_bgeo(ours, x, v, radius)
    lib.pin_partio_write(str(theirs).encode(), n, x.ctypes.data, None if v is None else v.ctypes.data, radius)
    assert gzip.decompress(ours.read_bytes()) == gzip.decompress(theirs.read_bytes())
    xp = np.zeros((n, 3), np.float32)
    vp = np.zeros((n, 3), np.float32)
    assert lib.pin_partio_read(str(ours).encode(), xp.ctypes.data, vp.ctypes.data, n) == n
    assert np.array_equal(xp, x)
    assert np.array_equal(vp, v if v is not None else np.zeros_like(x))
    xr, vr = read_bgeo(theirs)
    assert np.array_equal(xr, x) and (vr is None if v is None else np.array_equal(vr, v))


def test_scene_with_particle_files(tmp_path):
    """FluidModels and RigidBodies particle files, placed by x = R (s x) + t (SceneLoader.cpp:212-242,
    160-200; DemoBase.cpp:514-534; StaticBoundaryDemo/main.cpp:416-420), appended after the fluid
    blocks; the fluid keeps the file's velocities."""
    rng = np.random.default_rng(7)
    xf = rng.uniform(0.0, 0.3, size=(50, 3)).astype(np.float32)
    vf = rng.normal(size=(50, 3)).astype(np.float32)
    xb = rng.uniform(-1.0, 1.0, size=(80, 3)).astype(np.float32)
    (tmp_path / "models").mkdir()
    write_bgeo(tmp_path / "models" / "drop.bgeo", xf, vf, 0.01)
    write_bgeo(tmp_path / "models" / "walls.bgeo", xb, None, 0.01)
    scene = {
        "Configuration": {"particleRadius": 0.025, "timeStepSize": 0.001},
        "FluidBlocks": [{"start": [0.0, 0.0, 0.0], "end": [0.3, 0.3, 0.3]}],
        "FluidModels": [{"particleFile": "models/drop.bgeo", "translation": [1.0, 2.0, 3.0],
                         "rotationAxis": [0.0, 1.0, 0.0], "rotationAngle": 0.5, "scale": 2.0}],
        "RigidBodies": [{"particleFile": "models/walls.bgeo", "geometryFile": "models/UnitBox.obj",
                         "translation": [0.5, 0.0, 0.0], "scale": [3.0, 3.0, 3.0]}],
    }
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(scene))
    s = load_scene(p)
    nb = s.n_fluid - 50
    assert nb > 0
    rot = angle_axis_matrix([0.0, 1.0, 0.0], 0.5)
    exp = ((xf.astype(np.float64) * 2.0) @ rot.T + np.array([1.0, 2.0, 3.0])).astype(np.float32)
    assert np.array_equal(s.fluid[nb:], exp)
    assert np.array_equal(s.fluid_velocity[nb:], vf)
    assert not s.fluid_velocity[:nb].any()
    expb = ((xb.astype(np.float64) * 3.0) + np.array([0.5, 0.0, 0.0])).astype(np.float32)
    assert np.array_equal(s.boundary, expb)


def test_angle_axis_matches_rotation():
    r = angle_axis_matrix([0.0, 0.0, 1.0], np.pi / 2)
    assert np.allclose(r @ np.array([1.0, 0.0, 0.0]), [0.0, 1.0, 0.0], atol=1e-15)
    u = np.array([1.0, 2.0, 2.0]) / 3.0
    r = angle_axis_matrix(u, 1.1)
    assert np.allclose(r @ r.T, np.eye(3), atol=1e-14) and np.isclose(np.linalg.det(r), 1.0)
    assert np.allclose(r @ u, u, atol=1e-15)
