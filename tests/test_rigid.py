"""The host rigid-body integrator of splishsplash_for_cuda_b200.rigid (no GPU)."""
import numpy as np

from splishsplash_for_cuda_b200.rigid import RigidBody, RigidCoupling, quat_to_matrix


def test_box_mass_and_inertia():
    b = RigidBody.box((0, 0, 0), (0.2, 0.1, 0.4), 500.0, 0.02)
    m = 500.0 * 0.2 * 0.1 * 0.4
    assert np.isclose(b.mass, m)
    assert np.allclose(np.diag(b.inertia_body), [m * (0.01 + 0.16) / 12, m * (0.04 + 0.16) / 12,
                                                 m * (0.04 + 0.01) / 12])
    assert np.allclose(b.local.mean(0), 0.0, atol=1e-12)
    assert np.all(np.abs(b.local) <= np.array([0.1, 0.05, 0.2]) + 1e-12)


def test_free_fall_and_spin():
    b = RigidBody.box((0, 1, 0), (0.1, 0.1, 0.1), 500.0, 0.02)
    h, g = 1e-3, np.array([0.0, -9.81, 0.0])
    for _ in range(1000):
        b.integrate(np.zeros(3), np.zeros(3), h, g)
    # symplectic Euler: x_n = x_0 + g h^2 n (n + 1) / 2
    assert np.isclose(b.x[1], 1.0 - 9.81 * h * h * 1000 * 1001 / 2, rtol=1e-12)
    s = RigidBody.box((0, 0, 0), (0.1, 0.2, 0.3), 500.0, 0.02)
    s.w = np.array([0.0, 0.0, 2.0])  # spin about a principal axis: steady
    for _ in range(500):
        s.integrate(np.zeros(3), np.zeros(3), 1e-3, np.zeros(3))
    assert np.isclose(np.linalg.norm(s.q), 1.0) and np.allclose(s.w, [0, 0, 2.0])
    angle = 2 * np.arctan2(s.q[3], s.q[0])
    assert np.isclose(angle, 1.0, rtol=1e-6)
    r = quat_to_matrix(s.q)
    assert np.allclose(r @ r.T, np.eye(3), atol=1e-12)


def test_coupling_ranges_and_rigid_velocities():
    walls = np.random.default_rng(0).uniform(size=(50, 3)).astype(np.float32)
    a = RigidBody.box((0.5, 0.5, 0.5), (0.1, 0.1, 0.1), 500.0, 0.02)
    b = RigidBody.box((0.2, 0.5, 0.5), (0.06, 0.1, 0.1), 800.0, 0.02)
    b.v = np.array([1.0, 0.0, 0.0])
    b.w = np.array([0.0, 3.0, 0.0])
    c = RigidCoupling(walls, [a, b])
    assert list(c.first) == [50, 50 + a.local.shape[0]] and c.n_boundary == 50 + a.local.shape[0] + b.local.shape[0]
    x, v = c.boundary()
    assert np.array_equal(x[:50], walls) and not v[:50].any()
    sl = slice(int(c.first[1]), int(c.first[1] + c.count[1]))
    r = x[sl].astype(np.float64) - b.x
    assert np.allclose(v[sl], b.v + np.cross(b.w, r), atol=1e-6)
