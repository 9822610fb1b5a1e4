"""Fluid level (DFSPHCData::computeFluidLevel / handleFLuidLevelControl, SPH_other_systems_cuda.cu:
144-547): the oracle's column rule on hand-built columns and its raising lattice (CPU), then the
device's level against the oracle on a settled tank, the removal of the particles above a lowered
target and the particles placed to raise it again, equal to the oracle's, called through the C ABI
(GPU)."""
import numpy as np
import pytest

from oracle.oracle import fluid_level, fluid_level_raise
from splishsplash_for_cuda_b200.scene import Configuration, Scene, box_wall, lattice_block

R = 0.025
H = 4 * R


def _col(cx, cz, heights):
    return [((cx + 0.5) * H, h, (cz + 0.5) * H) for h in heights]


def test_oracle_column_rule_skips_a_splash():
    # column (0, 0): a splash particle two cells above the surface, then one particle per cell below;
    # the walk stops after the third particle and keeps the middle of the three highest
    pts = _col(0, 0, [0.95, 0.35, 0.25, 0.15, 0.05])
    assert fluid_level(pts, R, (0, 0, 0), (4, 10, 4)) == pytest.approx(np.float32(0.35))


def test_oracle_column_rule_reads_whole_cells():
    # the top cell holds four particles: all of them are read before the walk stops
    pts = _col(1, 2, [0.31, 0.32, 0.33, 0.34, 0.05])
    assert fluid_level(pts, R, (0, 0, 0), (4, 10, 4)) == pytest.approx(np.float32(0.33))


def test_oracle_sparse_columns_and_highest_column():
    # a column of two particles counts -2; the level is the highest column's middle height
    pts = _col(0, 0, [0.9, 0.8]) + _col(2, 2, [0.45, 0.35, 0.25]) + _col(3, 1, [0.55, 0.45, 0.35, 0.25])
    assert fluid_level(pts, R, (0, 0, 0), (4, 10, 4)) == pytest.approx(np.float32(0.45))
    assert fluid_level(_col(0, 0, [0.9, 0.8]), R, (0, 0, 0), (4, 10, 4)) == -1.0
    assert fluid_level(np.zeros((0, 3)), R, (0, 0, 0), (4, 10, 4)) == -1.0


def test_oracle_ignores_particles_off_the_grid():
    pts = _col(0, 0, [0.35, 0.25, 0.15]) + _col(5, 0, [0.95, 0.85, 0.75])  # x cell 5 >= dims 4
    assert fluid_level(pts, R, (0, 0, 0), (4, 10, 4)) == pytest.approx(np.float32(0.25))


def test_oracle_raise_lattice():
    # a closed box of boundary particles, fluid up to y = 0.3: three layers of spacing 2r over the box
    # shrunk by 2r, only outside its central third in x or z, each lifted to its column's top + 2.5 r
    r = 0.025
    walls = box_wall(np.array([0.0, 0.0, 0.0]), np.array([0.6, 0.9, 0.4]), 2 * r).astype(np.float32)
    fluid = lattice_block((10, 6, 6), r).astype(np.float32)  # y up to 0.3
    off, dims = (2, 2, 2), (12, 14, 10)
    new = fluid_level_raise(fluid, walls, r, off, dims, target=0.4, level=0.3)
    assert len(new) > 0
    lo, hi = walls.min(0) + 2 * r, walls.max(0) - 2 * r
    w = hi - lo
    inner = ((new[:, 0] >= lo[0] + w[0] / 3) & (new[:, 0] <= hi[0] - w[0] / 3) &
             (new[:, 2] >= lo[2] + w[2] / 3) & (new[:, 2] <= hi[2] - w[2] / 3))
    assert not inner.any()
    # three layers 0.8 * 2r apart; odd layers shifted by r in x and z
    assert np.unique(np.round((new[:, 0] - lo[0]) / r, 3) % 2).size == 2
    # every point sits 2.5 r + a layer offset above its column's top (-2 where no fluid)
    over = fluid[:, 1].max() + 2.5 * r
    ys = np.unique(np.round(new[:, 1], 4))
    for y in ys:
        assert any(abs(y - (t + 2.5 * r + k * 0.8 * 2 * r)) < 1e-4 for t in (fluid[:, 1].max(), -2.0) for k in range(3)), y
    assert ys.max() <= over + 2 * 0.8 * 2 * r + 1e-4


def _tank():
    lo, hi = np.array([0.0, 0.0, 0.0]), np.array([0.6, 0.9, 0.4])
    walls = box_wall(lo, hi, 2 * R)
    fluid = lattice_block((10, 12, 6), R)  # up to y = 0.6
    cfg = Configuration(timeStepSize=0.003, particleRadius=R, cflMethod=0, maxError=0.01)
    return Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=walls.astype(np.float32), name="level")


def _device_level_inputs(d):
    off = [d.get_param(f"grid_offset_{a}") for a in "xyz"]
    dims = [int(d.get_param(f"grid_dim_{a}")) for a in "xyz"]
    return off, dims


@pytest.mark.gpu
def test_level_matches_oracle_and_control_removes_above_target():
    from splishsplash_for_cuda_b200 import _capi
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = _tank()
    d = DFSPHCUDA(s, fluid_capacity=s.n_fluid + 1000)
    levels = []
    for k in range(60):
        d.step()
        if k % 20 == 19:
            off, dims = _device_level_inputs(d)
            got = d.fluid_level()
            want = fluid_level(d.positions(), R, off, dims)
            assert got == want, k  # FP32 cells and heights on both sides: equal
            levels.append(got)
    level = levels[-1]
    assert 0.45 < level < 0.65
    n0 = d.num_fluid()
    # within 5 cm of the level: nothing changes
    assert d.fluid_level_control(level - 0.04) == (0, 0)
    assert d.fluid_level_control(level + 0.04) == (0, 0)
    assert d.num_fluid() == n0
    # lowered by 10 cm: every particle above the target (rounded to FP32) goes
    target = level - 0.1
    y = d.positions()[:, 1]
    above = int(np.count_nonzero(y > np.float32(target)))
    assert above > 0
    assert d.fluid_level_control(target) == (above, 0)
    assert d.num_fluid() == n0 - above
    assert d.positions()[:, 1].max() <= np.float32(target)
    bad = _capi.ST_NONFINITE | _capi.ST_NEIGHBOR_OVERFLOW | _capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_ESCAPED
    for _ in range(10):
        assert d.step().status & bad == 0
    low = d.fluid_level()
    assert low < level - 0.05
    # raised back to the first level: the oracle's lattice, appended in lattice order
    n1 = d.num_fluid()
    off, dims = _device_level_inputs(d)
    want = fluid_level_raise(d.positions(), d.field("boundary_position"), R, off, dims, level, low)
    assert len(want) > 0
    assert d.fluid_level_control(level) == (0, len(want))
    x = d.positions()
    assert len(x) == n1 + len(want)
    assert np.array_equal(x[n1:], want)
    assert np.array_equal(x[:n1], d.positions()[:n1])
    assert np.all(d.field("velocity")[n1:] == 0)
    for _ in range(10):
        assert d.step().status & bad == 0


@pytest.mark.gpu
def test_raise_stops_at_fluid_capacity():
    """Raising past fluid_capacity appends what fits, in lattice order, and sets
    DFSPH_ST_FLUID_CAPACITY; calls with a target <= 0 or within 5 cm change nothing."""
    from splishsplash_for_cuda_b200 import _capi
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    s = _tank()
    d = DFSPHCUDA(s, fluid_capacity=s.n_fluid + 10)
    d.step()
    level = d.fluid_level()
    assert d.fluid_level_control(0.0) == (0, 0)
    assert d.fluid_level_control(-1.0) == (0, 0)
    off, dims = _device_level_inputs(d)
    want = fluid_level_raise(d.positions(), d.field("boundary_position"), R, off, dims, level + 0.2, level)
    assert len(want) > 10
    d.status(clear=True)
    assert d.fluid_level_control(level + 0.2) == (0, 10)
    assert d.num_fluid() == s.n_fluid + 10
    assert np.array_equal(d.positions()[s.n_fluid:], want[:10])
    assert d.status() & _capi.ST_FLUID_CAPACITY
