"""Rigid bodies coupled with the device time step: the device-side force/torque sum against the host
sum of the per-particle forces, the buoyancy of a fixed half-submerged box, and a free box of half
the fluid's density floating at rest (rigid-body integrator in splishsplash_for_cuda_b200.rigid)."""
import numpy as np
import pytest

from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.rigid import RigidBody, RigidCoupling
from splishsplash_for_cuda_b200.scene import Configuration, Scene, box_wall, lattice_block, synthetic_scene
from tests._compare import neighbor_sets

pytestmark = pytest.mark.gpu
R = 0.01
TANK = np.array([0.6, 0.5, 0.6])


def tank_with_box(box_center, box_size, density, fixed, depth_cells=10, seed=3):
    cfg = Configuration()
    cfg.particleRadius = R
    cfg.timeStepSize = 0.001
    walls = box_wall((0.0, 0.0, 0.0), TANK, 2 * R)
    fluid = lattice_block((29, depth_cells, 29), R)  # up to y = (depth + 1) 2r
    body = RigidBody.box(box_center, box_size, density, 2 * R, fixed=fixed)
    lo = np.asarray(box_center) - 0.5 * np.asarray(box_size) - R
    hi = np.asarray(box_center) + 0.5 * np.asarray(box_size) + R
    inside = np.all((fluid > lo) & (fluid < hi), axis=1)
    fluid = fluid[~inside]
    rng = np.random.default_rng(seed)
    fluid = fluid + rng.uniform(-0.01 * R, 0.01 * R, size=fluid.shape)
    coupling = RigidCoupling(walls, [body])
    bx, _ = coupling.boundary()
    scene = Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=bx, name="tank_box")
    d = DFSPHCUDA(scene)
    d.set_param("boundary_forces", 1)
    return d, coupling, body


def test_body_wrench_matches_host_sum(cuda_lib):
    d, c, body = tank_with_box((0.3, 0.2, 0.3), (0.12, 0.12, 0.12), 500.0, fixed=True)
    for _ in range(20):
        d.step()
    centers = np.array([body.x])
    f, t = d.body_wrench(c.first, c.count, centers)
    fb = d.field("boundary_force", np.float64)
    xb = d.field("boundary_position", np.float64)
    sl = slice(int(c.first[0]), int(c.first[0] + c.count[0]))
    fh = fb[sl].sum(0)
    th = np.cross(xb[sl] - centers[0], fb[sl]).sum(0)
    assert np.abs(f[0] - fh).max() <= 1e-12 * np.abs(fh).max()
    assert np.abs(t[0] - th).max() <= 1e-12 * max(np.abs(th).max(), np.abs(fh).max() * 0.1)
    # walls + body: every particle in exactly one range when the static part is a body too
    f2, _ = d.body_wrench([0, c.first[0]], [c.first[0], c.count[0]], np.zeros((2, 3)))
    assert np.allclose(f2.sum(0), fb.sum(0), rtol=1e-12, atol=1e-12 * np.abs(fb).sum())


def test_fixed_half_submerged_box_buoyancy(cuda_lib):
    """Archimedes for a fixed box, half submerged in a settled layer: the fluid's vertical force lies
    between rho0 g V for the geometric box and for the box grown by r on every side (a single-layer
    boundary sampled every 2r keeps the fluid about r farther out than the box faces), and the
    vertical forces on walls and box together carry the fluid's weight (within 5 %). Averages over
    the last 100 of 400 steps."""
    size = np.array([0.12, 0.12, 0.12])
    d, c, body = tank_with_box((0.3, 0.2, 0.3), size, 500.0, fixed=True)
    fy, total = [], []
    for k in range(400):
        st = d.step()
        if k >= 300:
            f, _ = d.body_wrench([0, c.first[0]], [c.first[0], c.count[0]], np.array([body.x, body.x]))
            fy.append(f[1, 1])
            total.append(f[0, 1] + f[1, 1])
    x = d.positions().astype(np.float64)
    far = (np.abs(x[:, 0] - 0.3) > 0.15) | (np.abs(x[:, 2] - 0.3) > 0.15)
    surface = np.quantile(x[far, 1], 0.995) + R
    bottom = body.x[1] - 0.5 * size[1]
    lo = 1000.0 * 9.81 * size[0] * size[2] * (surface - bottom)
    hi = 1000.0 * 9.81 * (size[0] + 2 * R) * (size[2] + 2 * R) * (surface - bottom + R)
    assert st.status == 0
    assert 0.95 * lo <= np.mean(fy) <= 1.05 * hi, (np.mean(fy), lo, hi)
    weight = 9.81 * d.field("mass", np.float64).sum()
    # forces of the fluid on the boundary: downward in total, the fluid's weight
    assert abs(-np.mean(total) - weight) <= 0.05 * weight, (np.mean(total), weight)


def test_free_box_floats_at_rest(cuda_lib):
    """A flat box (stable upright; a cube of half the fluid's density would roll over) of density 500
    released with its bottom at the surface floats: after 1.2 s it is nearly at rest with the fluid's
    vertical force balancing its weight (within 10 %, averaged over the last 300 steps), partly
    submerged, and has not drifted sideways."""
    size = np.array([0.16, 0.06, 0.16])
    surface0 = (10 + 1) * 2 * R
    d, c, body = tank_with_box((0.3, surface0 + 0.5 * size[1], 0.3), size, 500.0, fixed=False)
    fy, ys = [], []
    for k in range(1500):
        f, _ = c.step(d)
        if k >= 1200:
            fy.append(f[0, 1])
            ys.append(body.x[1])
    x = d.positions().astype(np.float64)
    far = (np.abs(x[:, 0] - 0.3) > 0.15) | (np.abs(x[:, 2] - 0.3) > 0.15)
    surface = np.quantile(x[far, 1], 0.995) + R
    depth = surface - (np.mean(ys) - 0.5 * size[1])
    weight = body.mass * 9.81
    assert np.isfinite(body.x).all() and abs(body.x[0] - 0.3) < 0.05 and abs(body.x[2] - 0.3) < 0.05
    assert abs(np.mean(fy) - weight) <= 0.1 * weight, (np.mean(fy), weight)
    assert 0.2 * size[1] <= depth <= 0.8 * size[1], (depth, surface)
    assert np.linalg.norm(body.v) < 0.05 and np.linalg.norm(body.w) < 0.5


def test_whole_boundary_translation_keeps_neighbour_sets():
    """A translation of the whole boundary within half a cell of its binning is applied without
    re-binning (the neighbour search looks the boundary up at x_i minus the shift): against the same
    positions uploaded with dfsph_move_boundary (a full re-binning each step), the same neighbour
    sets, the same iteration counts and positions within 1e-5 m over ten steps; a larger translation
    re-bins; a checkpoint taken while shifted reloads to the same state."""
    import tempfile

    s = synthetic_scene(1, counts=(14, 14, 14))
    a, b = DFSPHCUDA(s), DFSPHCUDA(s)
    b0 = s.boundary.astype(np.float64)
    nb = b0.shape[0]
    H = 4 * s.config.particleRadius
    for k in range(10):
        p = np.array([0.3 * H * np.sin(0.7 * k), 0.0, -0.2 * H * np.sin(0.4 * k)])
        v = np.array([0.1, 0.0, -0.05])
        a.move_boundary_rigid(0, nb, None, p, v, None)
        assert a.get_param("boundary_shift_active") == (1.0 if np.any(p != 0.0) else 0.0)
        b.move_boundary((b0 + p).astype(np.float32), np.tile(v, (nb, 1)).astype(np.float32))
        assert np.abs(a.field("boundary_position", np.float64) - b.field("boundary_position", np.float64)).max() <= 1e-6
        a.neighbors_search()
        b.neighbors_search()
        ca, la = a.neighbors()
        cb, lb = b.neighbors()
        assert np.array_equal(ca, cb), k
        assert neighbor_sets(ca, la) == neighbor_sets(cb, lb), k
        sa, sb = a.step(), b.step()
        assert (sa.iterations, sa.iterations_v) == (sb.iterations, sb.iterations_v), k
    assert np.abs(a.positions(np.float64) - b.positions(np.float64)).max() <= 1e-5
    a.move_boundary_rigid(0, nb, None, np.array([0.6 * H, 0.0, 0.0]), None, None)
    assert a.get_param("boundary_shift_active") == 0.0
    a.move_boundary_rigid(0, nb, None, np.array([0.7 * H, 0.0, 0.0]), None, None)
    assert a.get_param("boundary_shift_active") == 1.0
    with tempfile.TemporaryDirectory() as tmp:
        a.checkpoint_save(f"{tmp}/c.bin")
        assert a.get_param("boundary_shift_active") == 0.0
        c = DFSPHCUDA(s)
        c.checkpoint_load(f"{tmp}/c.bin")
        sa, sc = a.step(), c.step()
        assert (sa.iterations, sa.iterations_v) == (sc.iterations, sc.iterations_v)
        assert np.array_equal(a.positions(), c.positions())
