"""The dynamic window (dfsph_dynamic_window_init / _shift), called through the C ABI, in lockstep with
the CPU oracle composed of the same three operations: the walls translated, the fluid outside the
moved box removed, and the rest samples of the newly covered region inserted by the open boundary's
inflow rule (oracle_open_boundary_init / _apply with the previous box as the interior). Same particle
counts added and removed at every shift, same iteration counts, positions within 2e-4 m (FP32 vs
FP64 over 16 steps with three shifts; measured 1.0e-4)."""
import numpy as np
import pytest

from oracle import Oracle
from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.open_boundary import cuboid, plane
from splishsplash_for_cuda_b200.scene import Configuration, Scene, box_wall, lattice_block

pytestmark = pytest.mark.gpu

R = 0.025


def _window_scene():
    lo, hi = np.array([0.0, 0.0, 0.0]), np.array([1.1, 0.8, 0.55])
    walls = box_wall(lo, hi, 2 * R)
    fluid = lattice_block((20, 8, 10), R)                      # x in [0.05, 1.0], up to y = 0.4
    rest = lattice_block((21, 8, 10), R)                       # tiles the window up to the same height
    cfg = Configuration(timeStepSize=0.004, particleRadius=R, cflMethod=0, maxError=0.01)
    s = Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=walls.astype(np.float32), name="window")
    grid = (lo[0] - 0.2, lo[1] - 0.2, lo[2] - 0.2, hi[0] + 1.0, hi[1] + 0.2, hi[2] + 0.2)
    return s, lo, hi, rest.astype(np.float32), grid


def _f32box(lo, hi, disp):
    return (lo + disp).astype(np.float32), (hi + disp).astype(np.float32)


def test_dynamic_window_lockstep_with_oracle():
    s, lo, hi, rest, grid = _window_scene()
    nb = s.n_boundary
    d = DFSPHCUDA(s, grid_box=grid, fluid_capacity=s.n_fluid + 4000)
    d.set_param("remove_escaped", 0)
    d.init_dynamic_window(lo, hi, 0, nb, rest)
    o = Oracle(s, 64, grid_box=grid)
    o.set_scalar("remove_escaped", 0)
    disp = np.zeros(3)
    samples = rest.copy()  # moved with the window as the device moves them (FP32 additions)
    walls0 = s.boundary.astype(np.float32)
    shift = np.array([0.1, 0.0, 0.0])
    totals = []
    for k in range(16):
        if k in (4, 9, 13):
            old_lo, old_hi = lo + disp, hi + disp
            disp = disp + shift
            added, removed = d.shift_dynamic_window(shift, 0.9 * 2 * R, 1100.0)
            # the oracle: walls, removal, then the inflow of the newly covered region
            walls = (walls0 + disp.astype(np.float32)).astype(np.float32)
            o.move_boundary(walls, np.zeros_like(walls))
            blo, bhi = _f32box(lo, hi, disp)
            r_o = o.remove_outside_box(blo, bhi)
            samples = (samples + np.float32(shift[0]) * np.array([1, 0, 0], np.float32)).astype(np.float32)
            prev = cuboid(0.5 * (old_lo + old_hi), 0.5 * (old_hi - old_lo))
            box = cuboid(0.5 * (lo + hi) + disp, 0.5 * (hi - lo))
            everything = plane((0.0, 3.0e38, 0.0), (0.0, -1.0, 0.0))
            o.open_boundary_init(box, prev, everything, samples)
            a_o, _, _ = o.open_boundary_apply(0.9 * 2 * R, 1100.0, use_inflow=True, use_outflow=False)
            assert (added, removed) == (a_o, r_o), k
            assert added > 0 and removed > 0
            totals.append((added, removed))
            assert np.allclose(d.dynamic_window_displacement(), disp)
        st, ro = d.step(), o.step()
        assert st.status & (_capi.ST_NONFINITE | _capi.ST_NEIGHBOR_OVERFLOW | _capi.ST_PRESSURE_NOT_CONVERGED) == 0, k
        assert st.num_fluid == o.n, k
        assert (st.iterations, st.iterations_v) == (ro["iterations"], ro["iterations_v"]), k
    x, xo = d.field("position", np.float64), o.field("position")
    assert np.abs(x - xo).max() <= 2e-4  # FP32 vs FP64 over 16 steps and three shifts (measured 1.0e-4)
    v, vo = d.field("velocity", np.float64), o.field("velocity")
    assert np.abs(v - vo).max() <= 1e-3 * max(1.0, np.abs(vo).max())
    bx = d.field("boundary_position", np.float64)
    assert np.array_equal(bx.astype(np.float32), (walls0 + disp.astype(np.float32)).astype(np.float32))


@pytest.mark.parametrize("tagged_only", [True, False])
def test_window_stabilisation_lockstep_with_oracle(tagged_only):
    """dfsph_dynamic_window_stabilize after a shift against the oracle's restatement: 4 steps of 3 ms
    with the added particles damped by 0.5; with tagged_only the other particles do not move (bit
    for bit) and only the added ones settle; afterwards the warm starts are clear, the dt history is
    back and the run continues in lockstep (positions within 2e-4 m, FP32 vs FP64)."""
    s, lo, hi, rest, grid = _window_scene()
    nb = s.n_boundary
    d = DFSPHCUDA(s, grid_box=grid, fluid_capacity=s.n_fluid + 4000)
    d.set_param("remove_escaped", 0)
    d.init_dynamic_window(lo, hi, 0, nb, rest)
    o = Oracle(s, 64, grid_box=grid)
    o.set_scalar("remove_escaped", 0)
    for _ in range(3):
        d.step()
        o.step()
    shift = np.array([0.1, 0.0, 0.0])
    added, removed = d.shift_dynamic_window(shift, 0.9 * 2 * R, 1100.0)
    walls = (s.boundary.astype(np.float32) + shift.astype(np.float32)).astype(np.float32)
    o.move_boundary(walls, np.zeros_like(walls))
    blo, bhi = _f32box(lo, hi, shift)
    r_o = o.remove_outside_box(blo, bhi)
    samples = (rest + np.float32(shift[0]) * np.array([1, 0, 0], np.float32)).astype(np.float32)
    prev = cuboid(0.5 * (lo + hi), 0.5 * (hi - lo))
    box = cuboid(0.5 * (lo + hi) + shift, 0.5 * (hi - lo))
    o.open_boundary_init(box, prev, plane((0.0, 3.0e38, 0.0), (0.0, -1.0, 0.0)), samples)
    a_o, _, _ = o.open_boundary_apply(0.9 * 2 * R, 1100.0, use_inflow=True, use_outflow=False)
    assert (added, removed) == (a_o, r_o) and added > 0
    n = d.num_fluid()
    first = n - added if tagged_only else 0
    h0 = d.get_param("h")
    x_before = d.positions()
    d.stabilize_dynamic_window(4, 0.003, 0.5, tagged_only)
    o.dynamic_window_stabilize(4, 0.003, 0.5, first)
    x_after = d.positions()
    if tagged_only:
        assert np.array_equal(x_after[:first], x_before[:first])
    assert not np.array_equal(x_after[n - added:], x_before[n - added:])
    assert d.get_param("h") == h0
    assert not d.field("kappa").any() and not d.field("kappa_v").any()
    xd, xo = d.field("position", np.float64), o.field("position")
    assert np.abs(xd - xo).max() <= 2e-4
    for k in range(4):
        st, ro = d.step(), o.step()
        assert (st.iterations, st.iterations_v) == (ro["iterations"], ro["iterations_v"]), k
    assert np.abs(d.field("position", np.float64) - o.field("position")).max() <= 2e-4


def test_dynamic_window_arguments_are_checked():
    s, lo, hi, rest, grid = _window_scene()
    d = DFSPHCUDA(s, grid_box=grid)
    with pytest.raises(_capi.DfsphError) as e:
        d.shift_dynamic_window((0.1, 0, 0), 0.05, 1100.0)
    assert e.value.code == _capi.DFSPH_E_STATE
    with pytest.raises(_capi.DfsphError):
        d.init_dynamic_window(hi, lo, 0, s.n_boundary, rest)
    with pytest.raises(_capi.DfsphError):
        d.init_dynamic_window(lo, hi, 0, s.n_boundary + 1, rest)
    d.init_dynamic_window(lo, hi, 0, s.n_boundary, rest)
    with pytest.raises(_capi.DfsphError):
        d.shift_dynamic_window((0.1, 0, 0), 0.0, 1100.0)
    for args in [(2, 0.0, 1.0), (2, 0.003, 1.5), (2, float("nan"), 1.0)]:
        with pytest.raises(_capi.DfsphError):
            d.stabilize_dynamic_window(*args)
