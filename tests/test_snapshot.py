"""Snapshot files in the reference's text format (DFSPHCUDA::handleSimulationSave / Load,
SPlisHSPlasH/DFSPH/DFSPH_CUDA.cpp:1885-1979; UnifiedParticleSet::write_to_file / load_from_file,
DFSPH_c_arrays_structure.cpp:424-600). The fixture under tests/golden/snapshot is written by hand in
that format (a 3-particle fluid; a 2-particle boundary with the dynamic-body line)."""
from pathlib import Path

import numpy as np
import pytest

from splishsplash_for_cuda_b200.scene import read_particle_file, synthetic_scene, write_particle_file

SNAP = Path(__file__).resolve().parent / "golden" / "snapshot"


def test_reads_reference_format_fixture():
    m, x, v, flags = read_particle_file(SNAP / "fluid_file.txt")
    assert flags == (1, 1, 0) and m.shape == (3,) and np.allclose(x[1], [0.15, 0.2, 0.3])
    assert np.allclose(v[2], [0.0, -0.49, 0.002])
    m, x, v, flags = read_particle_file(SNAP / "boundaries_file.txt")
    assert flags == (0, 0, 1) and np.allclose(m, [0.5, 0.5]) and np.allclose(x[1], [0.05, 0, 0])


def test_round_trip_is_exact_for_float32(tmp_path):
    s = synthetic_scene(1, counts=(5, 5, 5))
    rng = np.random.default_rng(0)
    v = rng.normal(size=s.fluid.shape).astype(np.float32)
    m = np.full(s.n_fluid, 0.0125, np.float32)
    write_particle_file(tmp_path / "f.txt", m, s.fluid, v)
    m2, x2, v2, flags = read_particle_file(tmp_path / "f.txt")
    assert flags == (1, 1, 0)
    assert np.array_equal(x2.astype(np.float32), s.fluid) and np.array_equal(v2.astype(np.float32), v)


@pytest.mark.gpu
def test_device_snapshot_save_load(cuda_lib, tmp_path):
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = synthetic_scene(1, counts=(12, 12, 12), cfl=True)
    a = DFSPHCUDA(s)
    for _ in range(10):
        a.step()
    a.save_snapshot(tmp_path)
    m, x, v, flags = read_particle_file(tmp_path / "fluid_file.txt")
    assert flags == (1, 1, 0)
    assert np.array_equal(x.astype(np.float32), a.positions()) and np.array_equal(v.astype(np.float32), a.velocities())
    assert np.array_equal(m.astype(np.float32), a.field("mass"))
    mb, xb, _, bflags = read_particle_file(tmp_path / "boundaries_file.txt")
    assert bflags == (0, 0, 0) and np.array_equal(xb.astype(np.float32), a.field("boundary_position"))
    h = float((tmp_path / "general_data.txt").read_text())
    assert h == a.get_param("h")
    b = DFSPHCUDA(s)
    b.load_snapshot(tmp_path)
    assert np.array_equal(b.positions(), a.positions()) and np.array_equal(b.velocities(), a.velocities())
    assert b.get_param("h") == h and b.get_param("h_future") == h and b.get_param("h_past") == h
    assert np.allclose(b.field("boundary_psi"), a.field("boundary_psi"), rtol=1e-6)
    st = b.step()
    assert st.status == 0


@pytest.mark.gpu
def test_export_bgeo(cuda_lib, tmp_path):
    """partioExport of the device state: positions, velocities, pscale = r and id, read back exactly;
    a scene built from the exported file starts from the same state."""
    import gzip
    import json

    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
    from splishsplash_for_cuda_b200.scene import load_scene, read_bgeo

    s = synthetic_scene(1, counts=(12, 12, 12), cfl=True)
    a = DFSPHCUDA(s)
    for _ in range(10):
        a.step()
    a.export_bgeo(tmp_path / "ParticleData1.bgeo")
    x, v = read_bgeo(tmp_path / "ParticleData1.bgeo")
    assert np.array_equal(x, a.positions()) and np.array_equal(v, a.velocities())
    raw = gzip.decompress((tmp_path / "ParticleData1.bgeo").read_bytes())
    assert b"pscale" in raw and b"velocity" in raw and int.from_bytes(raw[9:13], "big") == s.n_fluid
    scene = {"Configuration": {"particleRadius": s.config.particleRadius, "timeStepSize": s.config.timeStepSize},
             "FluidModels": [{"particleFile": "ParticleData1.bgeo"}]}
    (tmp_path / "scene.json").write_text(json.dumps(scene))
    ls = load_scene(tmp_path / "scene.json")
    assert np.array_equal(ls.fluid, a.positions()) and np.array_equal(ls.fluid_velocity, a.velocities())


@pytest.mark.gpu
def test_device_loads_reference_format_fixture(cuda_lib):
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = synthetic_scene(1, counts=(4, 4, 4))
    d = DFSPHCUDA(s)
    d.load_snapshot(SNAP, boundary=False)
    _, x, v, _ = read_particle_file(SNAP / "fluid_file.txt")
    assert d.num_fluid() == 3
    assert np.array_equal(d.positions(), x.astype(np.float32)) and np.array_equal(d.velocities(), v.astype(np.float32))
    assert d.get_param("h") == 0.00125


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "learned", "gated"])
def test_checkpoint_resume_bit_identical(cuda_lib, tmp_path, mode):
    """A run saved after 10 steps and resumed in a fresh context continues bit-identically (internal
    particle order, warm starts, dt history and, in the learned mode, the network and Adam state
    are part of the checkpoint; with the cost gate, its schedule and the iterations counted so far in
    its current phase, saved here in the middle of a phase)."""
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = synthetic_scene(1, counts=(14, 14, 14), cfl=True)
    a = DFSPHCUDA(s)
    gate = dict(gate=True, gate_period=4, gate_window=3, gate_recheck=5, gate_margin=0.0) if mode == "gated" else {}
    if mode != "plain":
        a.set_learned_warm_start(True, train_interval=4, train_batch=512, **gate)
    for _ in range(10):
        a.step()
    path = tmp_path / "run.ckpt"
    a.checkpoint_save(path)
    sa = [a.step() for _ in range(10)]
    b = DFSPHCUDA(s)
    b.set_param("inflow_mass", 1.0)  # replaced by the checkpoint's (format version 4)
    b.step()  # the resumed context's own counters differ from the saved run's
    b.checkpoint_load(path)
    assert b.get_param("inflow_mass") == a.get_param("inflow_mass")
    sb = [b.step() for _ in range(10)]
    if mode == "gated":
        for key in ("gate_learned_steps", "gate_plain_steps", "gate_last_excess"):
            assert a.get_param(key) == b.get_param(key), key
        assert 0 < a.get_param("gate_learned_steps") < 20
    assert [x.iterations for x in sa] == [x.iterations for x in sb]
    assert [x.h for x in sa] == [x.h for x in sb]
    assert np.array_equal(a.positions(), b.positions()) and np.array_equal(a.velocities(), b.velocities())
    if mode != "plain":
        assert np.array_equal(a.mlp_params(), b.mlp_params())


@pytest.mark.gpu
def test_gate_ignores_counter_reset(cuda_lib):
    """Clearing the user-visible iteration counters in the middle of a gate phase leaves the gate's
    decisions, and so the run, unchanged."""
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = synthetic_scene(1, counts=(14, 14, 14), cfl=True)
    runs = []
    for reset in (False, True):
        d = DFSPHCUDA(s)
        d.set_learned_warm_start(True, train_interval=4, train_batch=512, gate=True, gate_period=4, gate_window=3,
                                 gate_recheck=5, gate_margin=0.5)
        for k in range(24):
            d.step()
            if reset and k % 7 == 3:
                d.set_param("iterations_sum", 0)
        runs.append((d.get_param("gate_learned_steps"), d.get_param("gate_last_excess"), d.positions()))
    assert runs[0][:2] == runs[1][:2]
    assert np.array_equal(runs[0][2], runs[1][2])
