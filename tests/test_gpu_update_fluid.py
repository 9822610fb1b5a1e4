"""dfsph_update_fluid (DFSPHCData::loadDynamicData's role: new positions and velocities for the
fluid between steps, given in particle-id order). The positions are scattered on the solver's
stream at once; the velocities are copied on a second stream and applied inside the next step's
binning, or by whichever other call comes first. These tests check that the split is invisible:
every route to the next state gives the same bits."""
import numpy as np
import pytest

from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.scene import synthetic_scene

pytestmark = pytest.mark.gpu


def scene():
    return synthetic_scene(1, counts=(20, 20, 20), cfl=True)


def advanced(precision=32, steps=3):
    d = DFSPHCUDA(scene(), precision=precision)
    for _ in range(steps):
        d.step()
    return d


def new_state(d, seed=0):
    rng = np.random.default_rng(seed)
    x, v = d.m_data.readDynamicData()
    x2 = (x + rng.uniform(-1e-4, 1e-4, size=x.shape)).astype(np.float32)
    v2 = (0.5 * v + rng.normal(scale=0.05, size=v.shape)).astype(np.float32)
    return x2, v2


@pytest.mark.parametrize("precision", [32, 64])
def test_read_after_update_returns_the_new_state(cuda_lib, precision):
    d = advanced(precision)
    x2, v2 = new_state(d)
    d.update_fluid(x2, v2)
    x, v = d.m_data.readDynamicData()
    assert np.array_equal(x, x2) and np.array_equal(v, v2)
    d.update_fluid(x2, None)  # no velocities: zero
    assert np.array_equal(d.positions(), x2) and not d.velocities().any()


@pytest.mark.parametrize("precision", [32, 64])
def test_step_after_update_matches_every_route(cuda_lib, precision):
    """Velocities applied inside the step's binning (update, step), applied before the step by a
    read (update, read, step), by a synchronize, and overridden by a second update: same bits."""
    runs = []
    for route in ("step", "read", "sync", "twice"):
        d = advanced(precision)
        x2, v2 = new_state(d)
        if route == "twice":
            xa, va = new_state(d, seed=1)
            d.update_fluid(xa, va)
        d.update_fluid(x2, v2)
        if route == "read":
            d.m_data.readDynamicData()
        elif route == "sync":
            d.synchronize()
        st = d.step()
        d.step()
        runs.append((st.iterations, st.iterations_v, d.positions(), d.velocities()))
    for r in runs[1:]:
        assert r[0] == runs[0][0] and r[1] == runs[0][1]
        assert np.array_equal(r[2], runs[0][2]) and np.array_equal(r[3], runs[0][3])


def test_asynchronous_loop_matches_synchronous(cuda_lib):
    """The end-to-end pattern (update, asynchronous step, read) against update, step, read."""
    a, b = advanced(), advanced()
    for k in range(4):
        x2, v2 = new_state(a, seed=10 + k)
        a.update_fluid(x2, v2)
        a.step_async()
        xa, va = a.m_data.readDynamicData()
        b.update_fluid(x2, v2)
        b.step()
        xb, vb = b.m_data.readDynamicData()
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_update_with_unchanged_state_changes_nothing(cuda_lib):
    a, b = advanced(), advanced()
    x, v = a.m_data.readDynamicData()
    a.update_fluid(x, v)
    for _ in range(3):
        sa, sb = a.step(), b.step()
        assert sa.iterations == sb.iterations and sa.iterations_v == sb.iterations_v
    assert np.array_equal(a.positions(), b.positions()) and np.array_equal(a.velocities(), b.velocities())


def test_rigid_wall_motion_keeps_the_pending_velocities(cuda_lib):
    """A rigid boundary motion between the update and the step leaves the velocity copy in flight
    (it touches neither the fluid nor the upload staging): same bits as applying them first."""
    runs = []
    for flush_first in (False, True):
        d = advanced()
        nb = int(d.get_param("num_boundary"))
        x2, v2 = new_state(d)
        d.update_fluid(x2, v2)
        if flush_first:
            d.synchronize()
        d.move_boundary_rigid(0, nb, position=(0.002, 0.0, 0.0), velocity=(0.1, 0.0, 0.0))
        st = d.step()
        runs.append((st.iterations, st.iterations_v, d.positions(), d.velocities()))
    assert runs[0][:2] == runs[1][:2]
    assert np.array_equal(runs[0][2], runs[1][2]) and np.array_equal(runs[0][3], runs[1][3])
