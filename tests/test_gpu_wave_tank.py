"""The wave-tank workload (splishsplash_for_cuda_b200/wave_tank.py) on a reduced tank: piston, absorbing
open boundary, floating box of density 500 and the dynamic window together, through the C ABI. Over
450 steps (dt at most 1 ms), the window checked at most every 30 steps at the piston's furthest
advance: no non-finite, escaped or non-converged state, no particle faster than 5 m/s (the piston
moves at most 0.9 m/s), the fluid count within 15 % of the initial one (a shift removes a 0.5 m slab,
a fifth of this short tank, that the piston's stroke has raised; the new slab is at rest), the window
shifts toward the box, the layer and the window exchange particles, and the box keeps floating near
the rest level (density 500: half submerged)."""
import numpy as np
import pytest

from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.wave_tank import WaveTank, wave_tank_scene

pytestmark = pytest.mark.gpu
BAD = (_capi.ST_NONFINITE | _capi.ST_ESCAPED | _capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_NEIGHBOR_OVERFLOW
       | _capi.ST_FLUID_CAPACITY)


def test_wave_tank_runs_clean():
    scene, layout = wave_tank_scene(counts=(120, 20, 20), box_offset=0.4)
    tank = WaveTank(scene, layout, window_every=30, open_boundary_every=5)
    y0 = tank.body.x[1]
    n0 = scene.n_fluid
    for _ in range(450):
        st = tank.step()
        assert st.status & BAD == 0, tank.steps
        if tank.steps % 10 == 0:
            speed = np.linalg.norm(tank.d.velocities(), axis=1)
            assert speed.max() < 5.0, (tank.steps, float(speed.max()))
            assert abs(tank.d.num_fluid() - n0) < 0.15 * n0, (tank.steps, tank.d.num_fluid())
    assert tank.shifts >= 1
    assert tank.added > 0 and tank.removed > 0
    assert abs(tank.body.x[1] - y0) < 0.1
    x = tank.d.positions()
    assert np.isfinite(x).all()
    disp = tank.d.dynamic_window_displacement()
    assert disp[0] == pytest.approx(0.5 * tank.shifts * np.sign(disp[0]))
