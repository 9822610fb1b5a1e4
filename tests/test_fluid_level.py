"""Fluid level (DFSPHCData::computeFluidLevel / handleFLuidLevelControl, SPH_other_systems_cuda.cu:
144-260 and 414-470): the oracle's column rule on hand-built columns (CPU), then the device's level
against the oracle on a settled tank and the removal of the particles above a lowered target, called
through the C ABI (GPU)."""
import numpy as np
import pytest

from oracle.oracle import fluid_level
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
    d = DFSPHCUDA(s)
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
    # within 5 cm of the level, or above it: nothing changes
    assert d.fluid_level_control(level - 0.04) == 0
    assert d.fluid_level_control(level + 0.2) == 0
    assert d.num_fluid() == n0
    # lowered by 10 cm: every particle above the target (rounded to FP32) goes
    target = level - 0.1
    y = d.positions()[:, 1]
    above = int(np.count_nonzero(y > np.float32(target)))
    assert above > 0
    assert d.fluid_level_control(target) == above
    assert d.num_fluid() == n0 - above
    assert d.positions()[:, 1].max() <= np.float32(target)
    bad = _capi.ST_NONFINITE | _capi.ST_NEIGHBOR_OVERFLOW | _capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_ESCAPED
    for _ in range(10):
        assert d.step().status & bad == 0
    assert d.fluid_level() < level - 0.05
