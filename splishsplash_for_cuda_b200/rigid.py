"""Two-way coupling of rigid bodies with the device time step.

The reference moves its dynamic bodies with an external rigid-body solver (the un-vendored PBD
library behind DynamicBoundaryDemo): each step it uploads the bodies' particle positions and
velocities (DFSPHCData::loadDynamicObjectsData, DFSPH_c_arrays_structure.cpp:1152-1175) and reads
back the per-particle fluid forces (readDynamicObjectsData, :1177-1193). The device side of that
exchange is dfsph_move_boundary + dfsph_body_wrench here; this module supplies the rigid-body
solver as a plain symplectic-Euler integrator of a body's centre of mass and orientation (our own,
as the reference's is not available): v += h (F / m + g), w += h I^-1 (tau - w x I w),
x += h v, q += h/2 (0, w) q (normalised), with I the world-frame inertia R I_body R^T.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def quat_to_matrix(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def quat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


@dataclass
class RigidBody:
    """A rigid body represented by `local` boundary samples (body frame, relative to the centre of
    mass) placed at x with orientation q."""
    mass: float
    inertia_body: np.ndarray  # (3, 3) about the centre of mass, body frame
    local: np.ndarray         # (k, 3) sample positions in the body frame
    x: np.ndarray             # centre of mass
    q: np.ndarray = field(default_factory=lambda: np.array([1.0, 0.0, 0.0, 0.0]))
    v: np.ndarray = field(default_factory=lambda: np.zeros(3))
    w: np.ndarray = field(default_factory=lambda: np.zeros(3))
    fixed: bool = False

    @staticmethod
    def box(center, size, density: float, spacing: float, fixed: bool = False) -> "RigidBody":
        """A solid box of the given density, sampled on its surface with a lattice of `spacing`."""
        from .scene import box_wall

        size = np.asarray(size, np.float64)
        half = 0.5 * size
        local = box_wall(-half, half, spacing)
        m = float(density * size.prod())
        a, b, c = size
        inertia = np.diag([m * (b * b + c * c) / 12.0, m * (a * a + c * c) / 12.0, m * (a * a + b * b) / 12.0])
        return RigidBody(mass=m, inertia_body=inertia, local=local, x=np.asarray(center, np.float64).copy(),
                         fixed=fixed)

    def rotation(self) -> np.ndarray:
        return quat_to_matrix(self.q)

    def particles(self) -> tuple[np.ndarray, np.ndarray]:
        """World positions and velocities v + w x r of the samples."""
        r = self.local @ self.rotation().T
        return self.x + r, self.v + np.cross(self.w, r)

    def integrate(self, force: np.ndarray, torque: np.ndarray, h: float, gravity) -> None:
        if self.fixed:
            return
        g = np.asarray(gravity, np.float64)
        self.v = self.v + h * (np.asarray(force, np.float64) / self.mass + g)
        rot = self.rotation()
        inertia = rot @ self.inertia_body @ rot.T
        rhs = np.asarray(torque, np.float64) - np.cross(self.w, inertia @ self.w)
        self.w = self.w + h * np.linalg.solve(inertia, rhs)
        self.x = self.x + h * self.v
        q = self.q + 0.5 * h * quat_mul(np.array([0.0, *self.w]), self.q)
        self.q = q / np.linalg.norm(q)


class RigidCoupling:
    """Static boundary + rigid bodies on one device context. The boundary given to the solver is
    the static samples followed by every body's samples (body b occupies a contiguous range)."""

    def __init__(self, static_boundary: np.ndarray, bodies: list[RigidBody]):
        self.static = np.asarray(static_boundary, np.float32).reshape(-1, 3)
        self.bodies = bodies
        first, counts = [], []
        k = self.static.shape[0]
        for b in bodies:
            first.append(k)
            counts.append(b.local.shape[0])
            k += b.local.shape[0]
        self.first = np.array(first, np.uint32)
        self.count = np.array(counts, np.uint32)
        self.n_boundary = k

    def boundary(self) -> tuple[np.ndarray, np.ndarray]:
        """All boundary positions and velocities (static ones at rest)."""
        xs = [self.static]
        vs = [np.zeros_like(self.static)]
        for b in self.bodies:
            x, v = b.particles()
            xs.append(x.astype(np.float32))
            vs.append(v.astype(np.float32))
        return np.concatenate(xs), np.concatenate(vs)

    def step(self, solver, gravity=None) -> tuple[np.ndarray, np.ndarray]:
        """One fluid step, then one rigid-body step with the fluid's force and torque on each body;
        the bodies' new samples are uploaded for the next step. Returns (forces, torques)."""
        st = solver.step()
        centers = np.array([b.x for b in self.bodies])
        f, t = solver.body_wrench(self.first, self.count, centers)
        g = solver.scene.config.gravitation if gravity is None else gravity
        for k, b in enumerate(self.bodies):
            b.integrate(f[k], t[k], st.h, g)
        x, v = self.boundary()
        solver.move_boundary(x, v)
        return f, t
