"""The wave-tank workload: a piston wavemaker, the simple open boundary as an absorbing layer at the
far end, a floating rigid box of density 500 kg/m^3 and a dynamic window that follows the box, all on
one device context.

The pieces are the reference's (OpenBoundariesSimple, DynamicWindow, dynamic rigid bodies driven by
DFSPHCUDA::step, SPlisHSPlasH/DFSPH/DFSPH_CUDA.cpp:82-794 and :3889-4139); the scene and the way they
are combined are this workload's own:

- the window box is [0.4, L] x [0, 4] x [0, W] in its own frame (L = 8.24 m, W = 2.04 m); the tank
  walls are sampled on [0, L] x [0, 4] x [0, W] with the face x = 0 replaced by the piston, whose rest
  place is x = 0.2 m and which moves rigidly as x = 0.2 + a sin(2 pi t / T) (a = 0.2 m, T = 1.5 s):
  it sweeps [0, 0.4], behind the window box;
- the fluid is the 400 x 100 x 100 lattice of spacing 2r (r = 0.01 m) in front of the piston, x from
  0.22 m, 2 m deep, filling the tank's width, with seeded jitter;
- the absorbing layer is the open boundary with the window box as its boundary, an interior that
  holds everything up to 0.3 m before the far wall (the piston's sweep and the space behind it
  included, so that no inflow sample lies where the piston moves) and the fluid's rest level
  (y = 2 m) as its surface: particles in the layer above the rest level leave, samples of the rest
  fluid refill it below (every `open_boundary_every` steps);
- the box (0.4 x 0.2 x 0.2 m, density 500) floats at the rest level at a seeded place ahead of the
  window's centre; it moves with the fluid's force and torque (rigid.RigidBody) and is placed on the
  device by a rigid motion of its boundary range;
- the window is checked at most once every `window_every` steps, at the first step where the piston
  stands at its furthest advance (sin(2 pi t / T) >= 0.99, the piston's face then within 2 mm of the
  window box's near face): it shifts 0.5 m toward the box when the box is more than 0.25 m from the
  window's centre along x; its walls, the piston's rest place, the open boundary and the rest samples
  move with it. Shifting at the furthest advance leaves no fluid behind the piston and no void in
  front of it (the window's removal takes the fluid of [lo, lo + 0.5 m) along x, where the piston
  moves to).
"""
from __future__ import annotations

import numpy as np

from .rigid import RigidBody
from .scene import Configuration, Scene, box_wall, lattice_block, _jitter

R = 0.01
L = 8.24
H_TANK = 4.0
W = 2.04
REST_LEVEL = 2.0
PISTON_REST = 0.2
PISTON_AMPLITUDE = 0.2
PISTON_PERIOD = 1.5
LAYER = 0.3
WINDOW_STEP = 0.5
# inflow rule of the open boundary and of the window's newly covered region: a sample becomes a fluid
# particle only with no fluid particle within 1.75 r and a density estimate of at most 700 kg/m^3 (the
# reference's values, DFSPH_CUDA.cpp:3903-3906), so a full region is not refilled
ALLOWED_DISTANCE = 1.75 * R
ALLOWED_DENSITY = 700.0


def wave_tank_scene(counts=(400, 100, 100), seed: int = 5, box_offset: float = 1.5):
    """(scene, layout) of the wave tank. counts scales the fluid lattice (x, y, z); the tank follows
    its extent. layout holds the boundary ranges, the window box, the grid box, the rest samples and
    the floating body."""
    d = 2.0 * R
    nx, ny, nz = counts
    length = PISTON_REST + (nx + 1) * d
    width = (nz + 1) * d
    level = ny * d
    tank_hi = np.array([length, max(2.0 * level, level + 0.5), width])
    walls = box_wall((0.0, 0.0, 0.0), tank_hi, d)
    cnt_y, cnt_z = int(round(tank_hi[1] / d)) + 1, int(round(width / d)) + 1
    piston = cnt_y * cnt_z  # box_wall puts the face x = 0 first
    walls[:piston, 0] += PISTON_REST
    lattice = lattice_block(counts, R, origin=(PISTON_REST, 0.0, 0.0))
    fluid = lattice + _jitter(lattice.shape[0], 0.01 * R, seed)
    rng = np.random.default_rng(seed)
    center = np.array([0.5 * (2 * PISTON_REST + length) + box_offset + rng.uniform(-0.1, 0.1), level,
                       0.5 * width + rng.uniform(-0.1, 0.1)])
    # the box's faces lie on lattice planes (its sizes are whole multiples of 2r), and it displaces
    # its volume: the fluid lattice keeps the planes 2r and more from its faces, as it sits at the
    # walls, so the fluid around the box starts at rest density
    center[0] = PISTON_REST + d * np.round((center[0] - PISTON_REST) / d)
    center[2] = d * np.round(center[2] / d)
    size = np.array([0.4, 0.2, 0.2])
    body = RigidBody.box(center, size, 500.0, d)
    bx, _ = body.particles()
    inside = np.all(np.abs(lattice - center) < 0.5 * size + 0.5 * d, axis=1)
    fluid = fluid[~inside]
    boundary = np.concatenate([walls, bx]).astype(np.float32)
    # dt at most 1 ms: at 5 ms the density solve, stopped by its average error after the minimum
    # iterations, carries only about half of a floating body's weight in a 2 m deep tank
    cfg = Configuration(timeStepSize=0.001, particleRadius=R, density0=1000.0, viscosity=0.01, cflMethod=1,
                        cflFactor=0.4, cflMaxTimeStepSize=0.001, maxIterations=100, maxError=0.01,
                        maxIterationsV=100, maxErrorV=0.1, enableDivergenceSolver=True)
    scene = Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=boundary, name="wave_tank_4m"
                  if tuple(counts) == (400, 100, 100) else f"wave_tank_{'x'.join(map(str, counts))}",
                  box_min=(0.0, 0.0, 0.0), box_max=tuple(tank_hi))
    layout = dict(
        piston=(0, piston), walls=(piston, walls.shape[0] - piston), body=(walls.shape[0], bx.shape[0]),
        window_lo=np.array([2 * PISTON_REST, 0.0, 0.0]), window_hi=tank_hi.copy(),
        # the cell grid covers the window's path: 12 shifts ahead, some room behind and above
        grid=(-0.5, -0.5, -0.5, tank_hi[0] + 12 * WINDOW_STEP + 0.5, tank_hi[1] + 0.5, tank_hi[2] + 0.5),
        rest=lattice.astype(np.float32), level=level, body_model=body, body_center0=center.copy())
    return scene, layout


class WaveTank:
    """Runs the wave tank on one device context: step() applies the piston's motion, the absorbing
    layer, the window and the floating body around each DFSPHCUDA step."""

    def __init__(self, scene: Scene, layout: dict, device: int = 0, learned: bool = True, window_every: int = 200,
                 open_boundary_every: int = 5):
        from . import open_boundary as ob
        from .dfsph import DFSPHCUDA

        self.scene, self.layout = scene, layout
        extra = int(0.1 * scene.n_fluid) + 1000
        self.d = DFSPHCUDA(scene, device=device, grid_box=layout["grid"], fluid_capacity=scene.n_fluid + extra)
        self.d.set_param("boundary_forces", 1)
        self.d.set_param("remove_escaped", 0)
        if learned:
            self.d.set_learned_warm_start(True, gate=True)
        lo, hi = layout["window_lo"], layout["window_hi"]
        self.d.init_dynamic_window(lo, hi, layout["walls"][0], layout["walls"][1], layout["rest"])
        self.window_every, self.open_boundary_every = window_every, open_boundary_every
        center = 0.5 * (lo + hi)
        half = 0.5 * (hi - lo)
        # interior: from 1 m behind the tank's near end to the layer, 1 m beyond the other faces
        ilo = np.array([-1.0, lo[1] - 1.0, lo[2] - 1.0])
        ihi = np.array([hi[0] - LAYER, hi[1] + 1.0, hi[2] + 1.0])
        rest = layout["rest"]
        self.d.init_open_boundary(ob.cuboid(center, half), ob.cuboid(0.5 * (ilo + ihi), 0.5 * (ihi - ilo)),
                                  ob.plane((0.0, layout["level"], 0.0), (0.0, -1.0, 0.0)), rest)
        self.body = layout["body_model"]
        self.c0 = layout["body_center0"]
        self.t = 0.0
        self.steps = 0
        self.shifts = 0
        self.window_x = 0.0
        self.last_check = 0
        self.added = self.removed = 0
        self.status = 0
        self.move_piston()

    def move_piston(self) -> None:
        first, count = self.layout["piston"]
        osc = PISTON_AMPLITUDE * np.sin(2 * np.pi * self.t / PISTON_PERIOD)
        vel = PISTON_AMPLITUDE * (2 * np.pi / PISTON_PERIOD) * np.cos(2 * np.pi * self.t / PISTON_PERIOD)
        self.d.move_boundary_rigid(first, count, None, (self.window_x + osc, 0.0, 0.0), (vel, 0.0, 0.0), None)

    def place_body(self) -> None:
        """The body's samples at x = R x0 + p with x0 their rest places (centre c0) and p = x_body - R c0;
        move_boundary_rigid gives them w x (x - p) + v, so v = v_body - w x (R c0) makes the field the
        body's own, v_body + w x (x - x_body)."""
        first, count = self.layout["body"]
        rot = self.body.rotation()
        arm = rot @ self.c0
        p = self.body.x - arm
        v = self.body.v - np.cross(self.body.w, arm)
        self.d.move_boundary_rigid(first, count, self.body.q, p, v, self.body.w)

    def maybe_shift(self) -> None:
        lo, hi = self.layout["window_lo"], self.layout["window_hi"]
        center = 0.5 * (lo[0] + hi[0]) + self.window_x
        gap = self.body.x[0] - center
        if abs(gap) <= 0.25:
            return
        step = np.sign(gap) * WINDOW_STEP
        a, r = self.d.shift_dynamic_window((step, 0.0, 0.0), ALLOWED_DISTANCE, ALLOWED_DENSITY)
        self.d.shift_open_boundary((step, 0.0, 0.0))
        self.window_x += step
        self.move_piston()  # with the walls, before the next step
        self.shifts += 1
        self.added += a
        self.removed += r

    def step(self):
        if self.steps and self.steps % self.open_boundary_every == 0:
            a, r = self.d.apply_open_boundary(ALLOWED_DISTANCE, ALLOWED_DENSITY)
            self.added += a
            self.removed += r
        if (self.steps - self.last_check >= self.window_every
                and np.sin(2 * np.pi * self.t / PISTON_PERIOD) >= 0.99):
            self.last_check = self.steps
            self.maybe_shift()
        st = self.d.step()
        self.status |= st.status
        first, count = self.layout["body"]
        f, tq = self.d.body_wrench([first], [count], [self.body.x])
        self.body.integrate(f[0], tq[0], st.h, self.scene.config.gravitation)
        self.t += st.h
        self.steps += 1
        self.move_piston()
        self.place_body()
        return st
