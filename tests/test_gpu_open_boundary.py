"""Simple open boundary on the device against the oracle (and, for the shapes, against the reference's
own BufferFluidSurface through the committed fixtures).

Bars: kept samples, added and removed particles identical (positions bit-exact, ids in sample order,
survivors in their previous order); velocities of new particles within 1e-5 of the largest fluid
speed (kernel sums in another order); then the usual lockstep bar of 1e-4 over three steps (1e-10
for the FP64 build)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import Oracle
from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200 import open_boundary as ob
from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.scene import Configuration, Scene

from test_open_boundary import R, tank_samples, tank_scene, tank_surfaces

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "open_boundary" / "surfaces.npz"
MESH_GOLD = Path(__file__).resolve().parent / "golden" / "open_boundary" / "meshes.npz"


def check(name, a, b, tol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, name
    scale = max(np.abs(b).max(), 1e-12)
    err = np.abs(a - b).max() / scale
    assert err <= tol, (name, err)


def test_device_surfaces_match_reference(cuda_lib):
    """Samples kept by init = points outside the shape (interior) and inside an all-space plane, for
    every fixture shape: the device's isinside() against the reference's. Star shapes go through
    CUDA's acosf / cosf / sinf instead of the host's; they must agree too on these points."""
    z = np.load(GOLD)
    cfg = Configuration()
    cfg.particleRadius = 0.05
    corners = np.array([[x, y, z_] for x in (-4.5, 4.5) for y in (-4.5, 4.5) for z_ in (-4.5, 4.5)], np.float32)
    scene = Scene(config=cfg, fluid=np.zeros((1, 3), np.float32), boundary=corners)
    d = DFSPHCUDA(scene)
    everything = ob.plane((0.0, -100.0, 0.0), (0.0, 1.0, 0.0))
    mism = []
    for k in range(z["surfaces"].shape[0]):
        s = _capi.Surface.from_buffer_copy(z["surfaces"][k].tobytes())
        pts = z["points"][k]
        kept = d.init_open_boundary(everything, s, everything, pts)
        exp = pts[~z["inside"][k].astype(bool)]
        got = d.open_boundary_samples()
        assert kept == got.shape[0]
        if not (got.shape == exp.shape and np.array_equal(got, exp)):
            mism.append((k, int(s.type), got.shape[0], exp.shape[0]))
    assert not mism, mism


def test_device_mesh_surfaces_match_reference(cuda_lib):
    """Mesh surfaces (type 3) on the device: the samples kept outside each fixture mesh equal the
    reference's MeshPerso::isInside answers (fixture made from its own RayIntersectsTriangle)."""
    z = np.load(MESH_GOLD)
    cfg = Configuration()
    cfg.particleRadius = 0.05
    corners = np.array([[x, y, z_] for x in (-4.5, 4.5) for y in (-4.5, 4.5) for z_ in (-4.5, 4.5)], np.float32)
    d = DFSPHCUDA(Scene(config=cfg, fluid=np.zeros((1, 3), np.float32), boundary=corners))
    everything = ob.plane((0.0, -100.0, 0.0), (0.0, 1.0, 0.0))
    for k in range(int(z["cases"])):
        d.set_surface_mesh(k % _capi.MAX_SURFACE_MESHES, z[f"v{k}"], z[f"t{k}"])
        pts = z[f"p{k}"]
        d.init_open_boundary(everything, ob.mesh(k % _capi.MAX_SURFACE_MESHES, offset=z[f"off{k}"]), everything, pts)
        assert np.array_equal(d.open_boundary_samples(), pts[~z[f"in{k}"].astype(bool)]), k


def test_mesh_surfaces_in_the_open_boundary(cuda_lib):
    """The tank's open boundary with box meshes in place of its cuboids runs exactly as with the
    cuboids (kept samples, added / removed particles, the state after three steps); with a non-convex
    interior (an L-shaped prism) and a shift, the device matches the oracle."""
    s = tank_scene(vx=0.3)
    b, i, f = tank_surfaces()
    runs = []
    for meshes in (False, True):
        d = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
        d.step()
        if meshes:
            d.set_surface_mesh(0, *ob.box_mesh((0.0, 0.0, 0.0), (1.0, 1.0, 0.5)))
            d.set_surface_mesh(1, *ob.box_mesh((0.075, 0.075, 0.075), (0.925, 0.925, 0.425)))
            kept = d.init_open_boundary(ob.mesh(0), ob.mesh(1), f, tank_samples())
        else:
            kept = d.init_open_boundary(b, i, f, tank_samples())
        added = d.apply_open_boundary(1.75 * R, 700.0)
        for _ in range(3):
            d.step()
        runs.append((kept, added, d.open_boundary_samples(), d.positions(), d.velocities()))
    assert runs[0][0] == runs[1][0] and runs[0][1] == runs[1][1] and runs[0][1][0] > 0
    for a, c in zip(runs[0][2:], runs[1][2:]):
        assert np.array_equal(a, c)
    # non-convex interior: the tank without the L-shaped prism over x, y in [0.1, 0.9], z in [0.1, 0.4]
    outline = np.array([(0.1, 0.1), (0.9, 0.1), (0.9, 0.5), (0.5, 0.5), (0.5, 0.9), (0.1, 0.9)], np.float32)
    n = len(outline)
    v = np.concatenate([np.c_[outline, np.full(n, 0.1)], np.c_[outline, np.full(n, 0.4)]]).astype(np.float32)
    t = []
    for a_, b_, c_ in [(0, 1, 2), (0, 2, 3), (0, 3, 5), (3, 4, 5)]:
        t += [(a_, c_, b_), (a_ + n, b_ + n, c_ + n)]
    for k in range(n):
        j = (k + 1) % n
        t += [(k, j, j + n), (k, j + n, k + n)]
    t = np.array(t, np.uint32)
    from oracle.oracle import set_surface_mesh
    set_surface_mesh(2, v, t)
    d = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    d.set_surface_mesh(2, v, t)
    o = Oracle(s, 64)
    interior = ob.mesh(2)
    assert d.init_open_boundary(b, interior, f, tank_samples()) == o.open_boundary_init(b, interior, f, tank_samples())
    delta = np.array([0.02, 0.0, -0.01], np.float32)
    d.shift_open_boundary(delta)
    o.open_boundary_shift(delta)
    ad, rd = d.apply_open_boundary(1.75 * R, 700.0)
    ao, ro, _ = o.open_boundary_apply(1.75 * R, 700.0)
    assert (ad, rd) == (ao, ro) and ad > 0 and rd > 0
    assert np.array_equal(d.positions(), o.field("position").astype(np.float32))


@pytest.mark.parametrize("precision", [32, 64])
def test_inflow_outflow_lockstep_with_oracle(cuda_lib, precision):
    s = tank_scene(vx=0.3)
    d = DFSPHCUDA(s, precision=precision, fluid_capacity=2 * s.n_fluid)
    o = Oracle(s, 64)
    for _ in range(3):
        d.step()
        o.step()
    b, i, f = tank_surfaces()
    samples = tank_samples()
    assert d.init_open_boundary(b, i, f, samples) == o.open_boundary_init(b, i, f, samples) > 0
    n0 = d.num_fluid()
    ad, rd = d.apply_open_boundary(1.75 * R, 700.0)
    ao, ro, _ = o.open_boundary_apply(1.75 * R, 700.0)
    assert (ad, rd) == (ao, ro) and ad > 0 and rd > 0
    assert d.num_fluid() == n0 + ad - rd == o.n
    xd, xo = d.field("position", np.float64), o.field("position")
    assert np.abs(xd - xo).max() <= 1e-4 * np.abs(xo).max()  # the fluid moved for 3 steps
    # the new particles (the last ids among the survivors) sit exactly on their samples
    new = np.isin(xo.astype(np.float32), samples).all(1) & (np.arange(o.n) >= o.n - ad)
    assert new.sum() == ad and np.array_equal(xd[new].astype(np.float32), xo[new].astype(np.float32))
    vmax = np.abs(o.field("velocity")).max()
    assert np.abs(d.field("velocity", np.float64)[new] - o.field("velocity")[new]).max() <= 1e-5 * vmax
    assert np.all(d.field("kappa")[new] == 0) and np.all(d.field("kappa_v")[new] == 0)
    assert np.array_equal(d.field("mass", np.float64), o.field("mass"))
    ids = d.field("id", order=_capi.ORDER_SORTED)
    assert np.array_equal(np.sort(ids), np.arange(d.num_fluid()))
    for k in range(3):
        st = d.step()
        ro_ = o.step()
        assert st.iterations == ro_["iterations"] and st.iterations_v == ro_["iterations_v"], k
        assert st.status & (_capi.ST_ESCAPED | _capi.ST_NONFINITE) == 0
    for name in ["position", "velocity", "density"]:
        check(name, d.field(name, np.float64), o.field(name), 1e-4 if precision == 32 else 1e-10)


def test_inflow_velocity_against_boundary_normal(cuda_lib):
    """A cylindrical boundary: samples whose interpolated velocity points out of the cylinder
    (v . n < 0, n = center - x) stay empty."""
    s = tank_scene(vx=0.5)
    d = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    o = Oracle(s, 64)
    b = ob.cylinder((0.5, 0.5, 0.25), 10.0, 0.45)
    i = ob.cylinder((0.5, 0.5, 0.25), 10.0, 0.45 - 3 * R)
    f = ob.plane((0.0, 0.5, 0.0), (0.0, -1.0, 0.0))
    samples = tank_samples()
    assert d.init_open_boundary(b, i, f, samples) == o.open_boundary_init(b, i, f, samples) > 0
    ad, rd = d.apply_open_boundary(1.75 * R, 700.0, use_outflow=False)
    ao, ro, _ = o.open_boundary_apply(1.75 * R, 700.0, True, False)
    assert (ad, rd) == (ao, ro) and rd == 0 and ad > 0
    n0 = s.n_fluid
    xd, xo = d.field("position"), o.field("position").astype(np.float32)
    assert np.array_equal(xd, xo)
    vd, vo = d.field("velocity", np.float64)[n0:], o.field("velocity")[n0:]
    assert np.abs(vd - vo).max() <= 1e-5 * 0.5
    # samples at the fluid front that point outward were refused: some front sample has v . n < 0
    a2 = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    a2.init_open_boundary(b, i, f, samples)
    ad2, _ = a2.apply_open_boundary(1.75 * R, 1e9, use_outflow=False)
    assert ad2 >= ad


def test_learned_mode_matches_plain_through_open_boundary(cuda_lib):
    s = tank_scene(vx=0.3)
    b, i, f = tank_surfaces()
    runs = []
    for learned in (False, True):
        d = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
        if learned:
            d.set_learned_warm_start(True, train_interval=0)
        d.step()
        d.init_open_boundary(b, i, f, tank_samples())
        d.apply_open_boundary()
        for _ in range(3):
            d.step()
        runs.append((d.positions(), d.velocities()))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


def test_inflow_mass_follows_the_fluid(cuda_lib):
    """With masses given at upload, the particles the inflow adds get the first uploaded particle's
    mass (the reference gives them fluid->mass[0]), on the device as in the oracle; "inflow_mass"
    reads and overrides it."""
    s = tank_scene(vx=0.3)
    m0 = np.float32(1000.0 * (2 * R) ** 3)
    s.fluid_mass = np.full(s.n_fluid, m0, np.float32)
    b, i, f = tank_surfaces()
    d = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    o = Oracle(s, 64)
    assert d.get_param("inflow_mass") == pytest.approx(float(m0), rel=1e-7)
    d.init_open_boundary(b, i, f, tank_samples())
    o.open_boundary_init(b, i, f, tank_samples())
    ad, rd = d.apply_open_boundary(1.75 * R, 700.0)
    ao, ro, _ = o.open_boundary_apply(1.75 * R, 700.0)
    assert (ad, rd) == (ao, ro) and ad > 0
    assert np.array_equal(d.field("mass", np.float64), o.field("mass"))
    assert np.all(d.field("mass") == m0)
    d.set_param("inflow_mass", 0.5 * float(m0))
    assert d.get_param("inflow_mass") == pytest.approx(0.5 * float(m0), rel=1e-7)


def test_capacity_cut_and_status(cuda_lib):
    s = tank_scene()
    d = DFSPHCUDA(s, fluid_capacity=s.n_fluid + 5)
    b, i, f = tank_surfaces()
    d.init_open_boundary(b, i, f, tank_samples())
    d.status(clear=True)
    ad, _ = d.apply_open_boundary(use_outflow=False)
    assert ad == 5 and d.num_fluid() == s.n_fluid + 5
    assert d.status() & _capi.ST_FLUID_CAPACITY
    o = Oracle(s, 64)
    o.open_boundary_init(b, i, f, tank_samples())
    ao, _, clipped = o.open_boundary_apply(1.75 * R, 700.0, True, False, capacity=s.n_fluid + 5)
    assert ao == 5 and clipped
    assert np.array_equal(d.positions(), o.field("position").astype(np.float32))
    st = d.step()
    assert st.status & _capi.ST_NONFINITE == 0


def test_shift_moves_surfaces_and_samples(cuda_lib):
    s = tank_scene(vx=0.3)
    b, i, f = tank_surfaces()
    delta = np.array([0.05, 0.0, 0.0], np.float32)
    a = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    a.init_open_boundary(b, i, f, tank_samples())
    a.shift_open_boundary(delta)
    moved = []
    for surf in (b, i, f):
        c = _capi.Surface.from_buffer_copy(bytes(surf))
        field = c.origin if c.type == _capi.SURFACE_PLANE else c.center
        for k in range(3):
            field[k] = float(np.float32(field[k]) + delta[k])
        moved.append(c)
    g = DFSPHCUDA(s, fluid_capacity=2 * s.n_fluid)
    g.init_open_boundary(*moved, tank_samples() + delta)
    assert np.array_equal(a.open_boundary_samples(), g.open_boundary_samples())
    assert a.apply_open_boundary() == g.apply_open_boundary()
    assert np.array_equal(a.positions(), g.positions())


def test_errors(cuda_lib):
    s = tank_scene()
    d = DFSPHCUDA(s)
    with pytest.raises(_capi.DfsphError) as e:
        d.apply_open_boundary()
    assert e.value.code == _capi.DFSPH_E_STATE
    b, i, f = tank_surfaces()
    bad = _capi.Surface.from_buffer_copy(bytes(b))
    bad.type = 3  # a mesh id with no mesh registered
    with pytest.raises(_capi.DfsphError) as e:
        d.init_open_boundary(bad, i, f, tank_samples())
    assert e.value.code == _capi.DFSPH_E_INVALID
    for args in [(_capi.MAX_SURFACE_MESHES, *ob.box_mesh((0, 0, 0), (1, 1, 1))),
                 (0, np.zeros((3, 3), np.float32), np.array([[0, 1, 3]], np.uint32)),
                 (0, np.zeros((3, 3), np.float32), np.zeros((0, 3), np.uint32))]:
        with pytest.raises(_capi.DfsphError) as e:
            d.set_surface_mesh(*args)
        assert e.value.code == _capi.DFSPH_E_INVALID
    d.init_open_boundary(b, i, f, tank_samples())
    with pytest.raises(_capi.DfsphError) as e:
        d.apply_open_boundary(allowed_distance=0.0)
    assert e.value.code == _capi.DFSPH_E_INVALID
    assert d.apply_open_boundary(allowed_distance=0.0, use_inflow=False)[0] == 0
