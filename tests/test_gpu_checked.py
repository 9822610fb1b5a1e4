"""The checked build (libdfsph_b200_checked.so, compiled with -DDFSPH_CHECKED): every cell-table run
is range-checked while the lists are built, and every list entry and count after each neighbour
search, before any pass gathers through them; a value out of range raises DFSPH_ST_INDEX and is not
read (the run skipped, the particle's list emptied). It stands in for a memory checker on the small
parity cases: they must run with the bit clear and give exactly the unchecked build's bits (the
solver passes are the same code), and an index planted past the fluid count (inside the allocation,
so that no access could leave it even unchecked) must be reported."""
import numpy as np
import pytest

from oracle import Oracle
from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.scene import column_scene, synthetic_scene

pytestmark = pytest.mark.gpu
CHECKED = str(_capi.CHECKED_LIB_PATH)


def _moving_scene(counts=(14, 14, 14), seed=7, vmax=0.5):
    s = synthetic_scene(1, counts=counts)
    rng = np.random.default_rng(seed)
    s.fluid_velocity = rng.uniform(-vmax, vmax, size=s.fluid.shape).astype(np.float32)
    return s


@pytest.mark.parametrize("make,steps,learned", [(lambda: synthetic_scene(1, counts=(14, 14, 14), cfl=True), 10, False),
                                                (_moving_scene, 5, False),
                                                (lambda: column_scene(counts=(8, 20, 8), time_step=0.002), 30, True)])
def test_checked_build_runs_clean_and_bit_identical(make, steps, learned):
    s = make()
    a = DFSPHCUDA(s)
    b = DFSPHCUDA(s, lib_path=CHECKED)
    assert a.get_param("checked_build") == 0 and b.get_param("checked_build") == 1
    for d in (a, b):
        if learned:
            d.set_learned_warm_start(True, train_interval=10)
    for k in range(steps):
        sa, sb = a.step(), b.step()
        assert sb.status & _capi.ST_INDEX == 0, k
        assert (sa.iterations, sa.iterations_v, sa.status) == (sb.iterations, sb.iterations_v, sb.status), k
    for name in ("position", "velocity", "density", "kappa", "kappa_v"):
        assert np.array_equal(a.field(name), b.field(name)), name


def test_checked_build_matches_oracle_one_step():
    s = synthetic_scene(1, counts=(14, 14, 14), cfl=True)
    d = DFSPHCUDA(s, lib_path=CHECKED)
    o = Oracle(s, 64)
    st, ro = d.step(), o.step()
    assert st.status == 0 and st.iterations == ro["iterations"]
    v, vo = d.field("velocity", np.float64), o.field("velocity")
    assert np.max(np.linalg.norm(v - vo, axis=1) / np.linalg.norm(vo, axis=1)) < 1e-5


def test_checked_build_reports_planted_index():
    s = synthetic_scene(1, counts=(10, 10, 10))
    d = DFSPHCUDA(s, lib_path=CHECKED, fluid_capacity=s.n_fluid + 64)
    d.set_param("checked_corrupt_neighbor", 5)  # particle 0's first entry := n + 4
    st = d.step()
    assert st.status & _capi.ST_INDEX
    assert np.isfinite(d.positions()).all()
    d.status(clear=True)
    assert d.step().status & _capi.ST_INDEX == 0  # one search only
    u = DFSPHCUDA(s)
    with pytest.raises(_capi.DfsphError) as e:
        u.set_param("checked_corrupt_neighbor", 5)
    assert e.value.code == _capi.DFSPH_E_INVALID
