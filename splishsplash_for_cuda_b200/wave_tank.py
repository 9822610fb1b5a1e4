"""The wave-tank workload: a piston wavemaker, the simple open boundary as an absorbing layer at the
far end, a floating rigid box of density 500 kg/m^3 and a dynamic window that follows the box, all on
one device context.

The pieces are the reference's (OpenBoundariesSimple, DynamicWindow, dynamic rigid bodies driven by
DFSPHCUDA::step, SPlisHSPlasH/DFSPH/DFSPH_CUDA.cpp:82-794 and :3889-4139); the scene and the way they
are combined are this workload's own:

- the fluid is the 400 x 100 x 100 lattice of spacing s = 18.59 mm (about 0.8^(1/3) 2r, r = 0.01 m)
  with seeded jitter, 1.86 m deep, filling the tank's width, its rows g = 1.14 s from the walls: with
  the reference's particle mass 0.8 rho0 (2r)^3 it starts at rest density, next to the walls too (at
  spacing 2r the 2 m column would first fall by a fifth of its height);
- the tank is [0, L] x [0, H] x [0, W] (L = 7.66 m, H = 3.74 m, W = 1.90 m: the lattice's extent plus
  the two gaps, in whole multiples of 2r), its walls sampled every 2r, with the face x = 0 replaced by
  the piston (that face's inner samples), whose rest place is x = 0.2 m and which moves rigidly as
  x = 0.2 + a sin(2 pi t / T) (a = 0.2 m, T = 1.5 s), raised from rest over the first quarter period:
  it sweeps [0, 0.4]; psi of the walls and of the box come from each object's own samples, the
  piston's from its samples and the walls beside them;
- the window box is [0.4 + g, L] x [0, H] x [0, W] in its own frame, one wall gap in front of the
  piston's furthest advance;
- the absorbing layer is the open boundary with the window box as its boundary, an interior that
  holds everything up to 0.3 m before the far wall (the piston's sweep and the space behind it
  included, so that no inflow sample lies where the piston moves) and the fluid's rest level
  (half a spacing above the lattice's top row) as its surface: particles in the layer above the rest
  level leave, samples of the rest fluid (the lattice) refill it below (every `open_boundary_every`
  steps);
- the box (0.403 x 0.199 x 0.199 m, density 500, sampled about every 2r) floats half submerged at a
  seeded place ahead of the window's centre: it takes the place of whole lattice planes and keeps the
  wall gap to the fluid; it moves with the fluid's force and torque (rigid.RigidBody) and is placed on
  the device by a rigid motion of its boundary range;
- the window is checked at most once every `window_every` steps, at the first step where the piston
  stands at its furthest advance (sin(2 pi t / T) >= 0.99, the piston's face then within 2 mm of its
  furthest place): it shifts 0.5 m toward the box when the box is more than 0.25 m from the window's
  centre along x; its walls, the piston's rest place, the open boundary and the rest samples move
  with it. Shifting at the furthest advance leaves no fluid behind the piston and no void in front
  of it: the window's removal takes the fluid of [lo, lo + 0.5 m) along x, and the piston moves to
  at least the wall gap before the fluid that remains.
"""
from __future__ import annotations

import numpy as np

from .rigid import RigidBody
from .scene import Configuration, Scene, box_wall, _jitter

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
# lattice spacing of the fluid: with the reference's particle mass 0.8 rho0 (2r)^3 a cubic lattice of
# spacing 2r has 0.8 rho0 (the cubic spline's lattice sum times the spacing cubed is 1), so a 2 m
# column would first fall by a fifth of its height; at 18.59 mm (about 0.8^(1/3) 2r) the lattice's
# density is rho0 to within 1e-4
SPACING = 0.01859
# distance of the lattice from the walls (and of the box's faces from the fluid): a single layer of
# wall samples every 2r adds to the density of the fluid next to it; at 1.14 spacings the first row
# starts at rest density to within 0.2 % (at one spacing it would start 9 % compressed)
WALL_GAP = 1.14 * SPACING


def boundary_psi(x, radius: float, density0: float = 1000.0) -> np.ndarray:
    """Akinci psi of one boundary object: rho0 / sum_k W(x_b - x_k) over its own samples (the cubic
    spline of support 4r, self term included), in double precision."""
    from scipy.spatial import cKDTree

    x = np.asarray(x, np.float64)
    h = 4.0 * radius
    k = 8.0 / (np.pi * h ** 3)
    i, j = cKDTree(x).query_pairs(h, output_type="ndarray").T
    q = np.linalg.norm(x[i] - x[j], axis=1) / h
    w = np.where(q <= 0.5, k * (6.0 * q ** 3 - 6.0 * q ** 2 + 1.0), 2.0 * k * (1.0 - q) ** 3)
    total = np.full(len(x), k)  # W(0)
    np.add.at(total, i, w)
    np.add.at(total, j, w)
    return density0 / total


def _box_body(center, size, density: float, cells) -> RigidBody:
    """A solid box of the given density sampled on its surface by cells[a] + 1 points along each axis
    (spacing size[a] / cells[a], about 2r)."""
    size = np.asarray(size, np.float64)
    local = box_wall((0.0, 0.0, 0.0), cells, 1.0) * (size / np.asarray(cells, np.float64)) - 0.5 * size
    m = float(density * size.prod())
    a, b, c = size
    inertia = np.diag([m * (b * b + c * c) / 12.0, m * (a * a + c * c) / 12.0, m * (a * a + b * b) / 12.0])
    return RigidBody(mass=m, inertia_body=inertia, local=local, x=np.asarray(center, np.float64).copy())


def wave_tank_scene(counts=(400, 100, 100), seed: int = 5, box_offset: float = 1.5):
    """(scene, layout) of the wave tank. counts scales the fluid lattice (x, y, z); the tank follows
    its extent. layout holds the boundary ranges, the window box, the grid box, the rest samples and
    the floating body."""
    d = 2.0 * R
    s, g = SPACING, WALL_GAP
    nx, ny, nz = counts

    def whole(x):  # the walls are sampled every 2r: extents are whole multiples of 2r
        return d * np.ceil(x / d - 1e-9)

    length = whole(PISTON_REST + (nx - 1) * s + 2 * g)
    width = whole((nz - 1) * s + 2 * g)
    top = g + (ny - 1) * s  # the lattice's top row; its free surface sits about s / 2 higher
    tank_hi = np.array([length, whole(max(2.0 * top, top + 0.5)), width])
    box = box_wall((0.0, 0.0, 0.0), tank_hi, d)
    cnt_y, cnt_z = int(round(tank_hi[1] / d)) + 1, int(round(width / d)) + 1
    # box_wall puts the face x = 0 first (y-major); its inner points are the piston, its edge lines stay
    # with the walls (a piston row on the floor's or a side wall's line would double those samples)
    iy, iz = np.divmod(np.arange(cnt_y * cnt_z), cnt_z)
    inner = (iy > 0) & (iy < cnt_y - 1) & (iz > 0) & (iz < cnt_z - 1)
    piston_x = box[:cnt_y * cnt_z][inner] + np.array([PISTON_REST, 0.0, 0.0])
    walls = np.concatenate([box[:cnt_y * cnt_z][~inner], box[cnt_y * cnt_z:]])
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    origin = np.array([PISTON_REST + g, g, g])
    lattice = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1) * s + origin
    fluid = lattice + _jitter(lattice.shape[0], 0.01 * R, seed)
    rng = np.random.default_rng(seed)
    cx = 0.5 * (2 * PISTON_REST + length) + box_offset + rng.uniform(-0.1, 0.1)
    cz = 0.5 * width + 0.05 * width * rng.uniform(-1.0, 1.0)
    # the box takes the place of 23 x 6 x 12 lattice planes (x, the top six rows, z) and its faces
    # keep the wall gap to the planes that remain: 24 s - 2 g by 13 s - 2 g by 13 s - 2 g
    # (0.403 x 0.199 x 0.199 m); with its centre at the free surface it is half submerged (density 500)
    size = np.array([24.0, 13.0, 13.0]) * s - 2.0 * g
    # centre: on plane ix along x (planes ix - 11 ... ix + 11 go), midway between planes iz and iz + 1
    # along z (iz - 5 ... iz + 6 go), half a spacing above the top row along y
    ix = int(np.round((cx - origin[0]) / s))
    iz = int(np.round((cz - origin[2]) / s - 0.5))
    center = np.array([origin[0] + ix * s, top + 0.5 * s, origin[2] + (iz + 0.5) * s])
    body = _box_body(center, size, 500.0, (20, 10, 10))
    bx, _ = body.particles()
    inside = np.all(np.abs(lattice - center) < 0.5 * size + 0.5 * s, axis=1)
    fluid = fluid[~inside]
    boundary = np.concatenate([piston_x, walls, bx]).astype(np.float32)
    # Akinci psi per object (the reference keeps the static boundary and every dynamic body in separate
    # particle sets): the walls' and the box's from their own samples, so that a moving piston or box
    # leaves no weakened strip of wall where it stood at the start; the piston's from its samples
    # together with the walls' (its edges slide along the floor and the side walls, which look the
    # same at every x), so that its edge columns count the walls beside them as a corner does
    psi = np.concatenate([boundary_psi(np.concatenate([piston_x, walls]), R)[:len(piston_x)],
                          boundary_psi(walls, R), boundary_psi(bx, R)]).astype(np.float32)
    # dt at most 1 ms: at 5 ms the density solve, stopped by its average error after the minimum
    # iterations, carries only about half of a floating body's weight in a 2 m deep tank
    cfg = Configuration(timeStepSize=0.001, particleRadius=R, density0=1000.0, viscosity=0.01, cflMethod=1,
                        cflFactor=0.4, cflMaxTimeStepSize=0.001, maxIterations=100, maxError=0.01,
                        maxIterationsV=100, maxErrorV=0.1, enableDivergenceSolver=True)
    scene = Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=boundary, name="wave_tank_4m"
                  if tuple(counts) == (400, 100, 100) else f"wave_tank_{'x'.join(map(str, counts))}",
                  box_min=(0.0, 0.0, 0.0), box_max=tuple(tank_hi))
    layout = dict(
        piston=(0, len(piston_x)), walls=(len(piston_x), len(walls)), body=(len(piston_x) + len(walls), len(bx)),
        psi=psi,
        window_lo=np.array([PISTON_REST + PISTON_AMPLITUDE + g, 0.0, 0.0]), window_hi=tank_hi.copy(),
        # the cell grid covers the window's path: 12 shifts ahead, some room behind and above
        grid=(-0.5, -0.5, -0.5, tank_hi[0] + 12 * WINDOW_STEP + 0.5, tank_hi[1] + 0.5, tank_hi[2] + 0.5),
        rest=lattice.astype(np.float32), level=top + 0.5 * s, body_model=body, body_center0=center.copy())
    return scene, layout


def piston_motion(t: float) -> tuple[float, float]:
    """Displacement and velocity of the piston from its rest place: a sin(2 pi t / T) raised from rest
    by a smoothstep over the first quarter period (velocity and acceleration start at zero; full
    amplitude at the first furthest advance, t = T / 4)."""
    w = 2.0 * np.pi / PISTON_PERIOD
    u = min(t / (0.25 * PISTON_PERIOD), 1.0)
    ramp, dramp = u * u * (3.0 - 2.0 * u), (6.0 * u * (1.0 - u) / (0.25 * PISTON_PERIOD) if u < 1.0 else 0.0)
    return (PISTON_AMPLITUDE * ramp * np.sin(w * t),
            PISTON_AMPLITUDE * (dramp * np.sin(w * t) + ramp * w * np.cos(w * t)))


class WaveTank:
    """Runs the wave tank on one device context: step() applies the piston's motion, the absorbing
    layer, the window and the floating body around each DFSPHCUDA step."""

    def __init__(self, scene: Scene, layout: dict, device: int = 0, learned: bool = True, window_every: int = 200,
                 open_boundary_every: int = 5):
        from . import open_boundary as ob
        from .dfsph import DFSPHCUDA

        self.scene, self.layout = scene, layout
        extra = int(0.1 * scene.n_fluid) + 1000
        self.d = DFSPHCUDA(scene, device=device, grid_box=layout["grid"], fluid_capacity=scene.n_fluid + extra,
                           boundary_psi=layout["psi"])
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
        osc, vel = piston_motion(self.t)
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
