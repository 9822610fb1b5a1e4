"""Scene generation and the reference JSON scene reader (Utilities/SceneLoader.cpp:39-320 keys):
synthetic benchmark configurations, a JSON scene equal to a synthetic one, and the extension keys."""
import json

import numpy as np
import pytest

from splishsplash_for_cuda_b200.scene import load_scene, synthetic_scene


@pytest.mark.parametrize("config,nf,nb", [(1, 27000, 9602), (2, 250047, 64002)])
def test_synthetic_counts(config, nf, nb):
    s = synthetic_scene(config)
    assert s.n_fluid == nf and s.n_boundary == nb
    assert s.fluid.dtype == np.float32 and np.isfinite(s.fluid).all()


def _dam_break_json(tmp_path, extra=None):
    r = 0.025
    conf = {"particleRadius": r, "timeStepSize": 0.005, "density0": 1000, "viscosity": 0.01, "cflMethod": 0,
            "maxIterations": 100, "maxError": 0.01, "maxIterationsV": 100, "maxErrorV": 0.1,
            "enableDivergenceSolver": True, "gravitation": [0, -9.81, 0], "jitter": 0.0}
    conf.update(extra or {})
    scene = {"Configuration": conf,
             "FluidBlocks": [{"denseMode": 0, "start": [0.0, 0.0, 0.0], "end": [31 * 2 * r] * 3}],
             "RigidBodies": [{"geometryFile": "../models/UnitBox.obj", "translation": [1.0, 1.0, 1.0],
                              "scale": [2.0, 2.0, 2.0], "isDynamic": False}]}
    p = tmp_path / "dam.json"
    p.write_text(json.dumps(scene))
    return p


def test_json_scene_equals_synthetic(tmp_path):
    s = load_scene(_dam_break_json(tmp_path))
    ref = synthetic_scene(1, jitter=0.0)
    assert np.array_equal(s.fluid, ref.fluid)
    assert np.array_equal(np.sort(s.boundary.view("f4,f4,f4"), axis=0), np.sort(ref.boundary.view("f4,f4,f4"), axis=0))
    assert s.config.particleRadius == 0.025 and s.config.maxError == 0.01 and s.config.cflMethod == 0
    assert s.config.precision == 32 and s.config.learnedWarmStart is None


def test_json_extension_keys(tmp_path):
    s = load_scene(_dam_break_json(tmp_path, {"precision": 64,
                                              "learnedWarmStart": {"enabled": True, "trainInterval": 25}}))
    assert s.config.precision == 64 and s.config.learnedWarmStart == {"enabled": True, "trainInterval": 25}
    with pytest.raises(ValueError):
        load_scene(_dam_break_json(tmp_path, {"precision": 16}))
    with pytest.raises(ValueError):
        load_scene(_dam_break_json(tmp_path, {"learnedWarmStart": {"epochs": 3}}))


def test_json_rejects_unsupported_geometry(tmp_path):
    p = _dam_break_json(tmp_path)
    j = json.loads(p.read_text())
    j["FluidBlocks"][0]["denseMode"] = 1
    p.write_text(json.dumps(j))
    with pytest.raises(ValueError):
        load_scene(p)


@pytest.mark.gpu
def test_json_extensions_configure_the_solver(cuda_lib, tmp_path):
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = load_scene(_dam_break_json(tmp_path, {"precision": 64, "learnedWarmStart": {"trainInterval": 25,
                                                                                     "damping": 0.9}}))
    d = DFSPHCUDA(s)
    assert d.precision == 64
    assert d.get_param("learned_warm_start") == 1 and d.get_param("train_interval") == 25
    assert d.get_param("warm_start_damping") == 0.9
    assert d.step().status == 0


# ---- the library's own JSON reader (dfsph_scene_load), for C and C++ callers -------------------------
def _check_native_equals_python(path, atol=0.0):
    from splishsplash_for_cuda_b200.scene import load_scene_native

    s = load_scene(path)
    sc, x, v, b = load_scene_native(path)
    assert x.shape == s.fluid.shape and b.shape == s.boundary.shape
    if atol == 0.0:
        assert np.array_equal(x, s.fluid) and np.array_equal(b, s.boundary)
    else:
        assert np.abs(x - s.fluid).max() <= atol and np.abs(b - s.boundary).max() <= atol
    if s.fluid_velocity is None:
        assert v is None
    else:
        assert np.array_equal(v, s.fluid_velocity)
    c = s.config
    assert (sc.particle_radius, sc.density0, sc.viscosity, tuple(sc.gravitation), sc.time_step) == \
        (c.particleRadius, c.density0, c.viscosity, tuple(c.gravitation), c.timeStepSize)
    assert (sc.max_iterations, sc.max_error, sc.max_iterations_v, sc.max_error_v) == \
        (c.maxIterations, c.maxError, c.maxIterationsV, c.maxErrorV)
    assert (sc.cfl_method, sc.cfl_factor, sc.cfl_max_time_step) == (c.cflMethod, c.cflFactor, c.cflMaxTimeStepSize)
    assert sc.enable_divergence_solver == (1 if c.enableDivergenceSolver else 0) and sc.precision == c.precision
    assert sc.fluid_capacity == max(1, s.n_fluid) and sc.boundary_capacity == max(1, s.n_boundary)
    return s


@pytest.mark.parametrize("extra", [{}, {"jitter": 0.01, "seed": 3}, {"cflMethod": 1, "precision": 64,
                                                                    "gravitation": [0.5, -9.0, 0.25]}])
def test_native_reader_equals_python_reader(tmp_path, extra):
    _check_native_equals_python(_dam_break_json(tmp_path, extra))


def test_native_reader_particle_files_and_rotation(tmp_path):
    """FluidModels and RigidBodies from .bgeo particle files, rotated and scaled (x = R (s x) + t)."""
    from splishsplash_for_cuda_b200.scene import write_bgeo

    rng = np.random.default_rng(5)
    xf = rng.uniform(0.2, 0.8, size=(500, 3)).astype(np.float32)
    vf = rng.uniform(-1, 1, size=(500, 3)).astype(np.float32)
    xb = rng.uniform(0.0, 1.0, size=(300, 3)).astype(np.float32)
    write_bgeo(tmp_path / "fluid.bgeo", xf, vf, 0.025)
    write_bgeo(tmp_path / "walls.bgeo", xb, None, 0.025)
    p = _dam_break_json(tmp_path, {"jitter": 0.02, "seed": 9})
    j = json.loads(p.read_text())
    j["FluidModels"] = [{"particleFile": "fluid.bgeo", "translation": [0.1, 0.2, 0.3], "scale": 1.5,
                         "rotationAxis": [0, 1, 0], "rotationAngle": 0.3}]
    j["RigidBodies"].append({"particleFile": "walls.bgeo", "translation": [0.0, -0.5, 0.0], "scale": [2.0, 2.0, 2.0],
                             "rotationAxis": [1, 0, 0], "rotationAngle": 1.1})
    p.write_text(json.dumps(j))
    s = _check_native_equals_python(p, atol=1e-6)
    assert s.n_fluid == 27000 + 500 and s.fluid_velocity is not None


@pytest.mark.parametrize("change,message", [
    (lambda j: j["FluidBlocks"][0].update(denseMode=1), b"denseMode"),
    (lambda j: j["Configuration"].update(precision=16), b"precision"),
    (lambda j: j["Configuration"].update(learnedWarmStart={"epochs": 3}), b"learnedWarmStart"),
    (lambda j: j["RigidBodies"][0].update(geometryFile="sphere.obj"), b"box"),
])
def test_native_reader_rejects_like_python(tmp_path, change, message):
    import ctypes as C

    from splishsplash_for_cuda_b200 import _capi

    p = _dam_break_json(tmp_path)
    j = json.loads(p.read_text())
    change(j)
    p.write_text(json.dumps(j))
    with pytest.raises(ValueError):
        load_scene(p)
    lib = _capi.load()
    h = C.c_void_p()
    assert lib.dfsph_scene_load(str(p).encode(), None, C.byref(h)) == _capi.DFSPH_E_INVALID
    assert message in lib.dfsph_last_error(None)
    p.write_text('{"Configuration": {"particleRadius": 0.025,}')
    assert lib.dfsph_scene_load(str(p).encode(), None, C.byref(h)) == _capi.DFSPH_E_INVALID


@pytest.mark.gpu
def test_create_from_scene_file_equals_python_facade(cuda_lib, tmp_path):
    """dfsph_create_from_scene_file (the C path: read, create, upload, learned block) steps exactly
    like the Python facade on the Python reader's scene."""
    import ctypes as C

    from splishsplash_for_cuda_b200 import _capi
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    p = _dam_break_json(tmp_path, {"jitter": 0.01, "seed": 2, "learnedWarmStart": {"trainInterval": 5}})
    ref = DFSPHCUDA(load_scene(p))
    lib = _capi.load()
    ctx = C.c_void_p()
    assert lib.dfsph_create_from_scene_file(str(p).encode(), C.byref(ctx)) == _capi.DFSPH_OK
    try:
        v = C.c_double()
        assert lib.dfsph_get_param(ctx, b"learned_warm_start", C.byref(v)) == 0 and v.value == 1
        assert lib.dfsph_get_param(ctx, b"train_interval", C.byref(v)) == 0 and v.value == 5
        st = _capi.DfsphStepStats()
        for _ in range(12):
            assert lib.dfsph_step(ctx, C.byref(st)) == 0
            sr = ref.step()
            assert (st.iterations, st.iterations_v) == (sr.iterations, sr.iterations_v)
        n = ref.num_fluid()
        x = np.empty((n, 3), np.float32)
        vv = np.empty((n, 3), np.float32)
        assert lib.dfsph_read_dynamic_data(ctx, x.ctypes.data, vv.ctypes.data) == 0
        assert np.array_equal(x, ref.positions()) and np.array_equal(vv, ref.velocities())
    finally:
        lib.dfsph_destroy(ctx)
