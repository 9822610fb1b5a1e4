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
