"""Simple open boundary on the CPU: the oracle's restatement of BufferFluidSurface against the
reference's own class (fixtures made by tests/golden/open_boundary/make_surface_golden.py from
SPlisHSPlasH/DFSPH/BufferFluidSurface.cu compiled as host code; the live pin when it is built), the
reference's configuration table, and the oracle's inflow / outflow against a brute-force numpy
restatement of OpenBoundariesSimple.cu:352-492 on a small tank. No GPU is needed."""
import ctypes as C
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import Oracle
from oracle.oracle import OracleSurface, set_surface_mesh, surface_eval
from splishsplash_for_cuda_b200 import open_boundary as ob
from splishsplash_for_cuda_b200.scene import Configuration, Scene, box_wall, lattice_block

GOLD = Path(__file__).resolve().parent / "golden" / "open_boundary" / "surfaces.npz"
MESH_GOLD = Path(__file__).resolve().parent / "golden" / "open_boundary" / "meshes.npz"
PIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libsurface_pin.so"


def test_oracle_surfaces_match_reference_fixture():
    z = np.load(GOLD)
    assert z["surfaces"].shape[0] == 22
    for k in range(z["surfaces"].shape[0]):
        s = OracleSurface.from_buffer_copy(z["surfaces"][k].tobytes())
        inside, normal = surface_eval(s, z["points"][k])
        assert np.array_equal(inside, z["inside"][k].astype(bool)), k
        assert np.array_equal(normal, z["normal"][k]), k


@pytest.mark.skipif(not PIN.exists(), reason="BufferFluidSurface compiled from the reference sources is not present")
def test_oracle_surfaces_match_reference_live():
    lib = C.CDLL(str(PIN))
    lib.pin_surface_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(99)
    for s in [ob.cylinder((0.1, 0.0, 0.2), 0.5, 0.8, reversed=True), ob.star((0, 0, 0), 1.0, 2.0, 0.7, 6, (1, 0, 0)),
              ob.cuboid((0, 0, 0), (0.5, 0.25, 2.0)), ob.plane((0, 0.3, 0), (0.1, 1.0, 0.2), reversed=True),
              ob.sphere((1, 1, 1), 0.3)]:
        p = rng.uniform(-2.5, 2.5, size=(5000, 3)).astype(np.float32)
        ins = np.zeros(p.shape[0], np.uint8)
        nrm = np.zeros((p.shape[0], 3), np.float32)
        assert lib.pin_surface_eval(C.addressof(s), p.ctypes.data, p.shape[0], ins.ctypes.data, nrm.ctypes.data) == 0
        oi, on = surface_eval(s, p)
        assert np.array_equal(oi, ins.astype(bool)) and np.array_equal(on, nrm)


def test_oracle_mesh_surfaces_match_reference_fixture():
    """Type-3 (mesh) surfaces: the oracle's isinside against MeshPerso::isInside run on the reference's
    own RayIntersectsTriangle (fixture: an L-shaped prism, a box and an octahedron, two offsets each,
    random points and lattice points on planes through vertices), bit for bit; reversed flips it."""
    z = np.load(MESH_GOLD)
    for k in range(int(z["cases"])):
        set_surface_mesh(3, z[f"v{k}"], z[f"t{k}"])
        inside, normal = surface_eval(ob.mesh(3, offset=z[f"off{k}"]), z[f"p{k}"])
        assert np.array_equal(inside, z[f"in{k}"].astype(bool)), k
        assert not normal.any()
        rev, _ = surface_eval(ob.mesh(3, offset=z[f"off{k}"], reversed=True), z[f"p{k}"])
        assert np.array_equal(rev, ~z[f"in{k}"].astype(bool)), k


@pytest.mark.skipif(not PIN.exists(), reason="BufferFluidSurface compiled from the reference sources is not present")
def test_oracle_mesh_surfaces_match_reference_live():
    lib = C.CDLL(str(PIN))
    lib.pin_mesh_inside.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.c_uint32, C.c_void_p]
    z = np.load(MESH_GOLD)
    rng = np.random.default_rng(31)
    for k in range(int(z["cases"])):
        v, t = z[f"v{k}"], z[f"t{k}"]
        off = rng.uniform(-0.3, 0.3, size=3).astype(np.float32)
        p = rng.uniform(-0.5, 3.0, size=(4000, 3)).astype(np.float32)
        ins = np.zeros(p.shape[0], np.uint8)
        assert lib.pin_mesh_inside(v.ctypes.data, v.shape[0], t.ctypes.data, t.shape[0], off.ctypes.data,
                                   p.ctypes.data, p.shape[0], ins.ctypes.data) == 0
        set_surface_mesh(4, v, t)
        got, _ = surface_eval(ob.mesh(4, offset=off), p)
        assert np.array_equal(got, ins.astype(bool)), k


def test_box_mesh_equals_cuboid():
    lo, hi = np.array([0.1, -0.2, 0.3]), np.array([0.9, 0.6, 1.4])
    set_surface_mesh(5, *ob.box_mesh(lo, hi))
    rng = np.random.default_rng(2)
    p = rng.uniform(-0.5, 2.0, size=(20000, 3)).astype(np.float32)
    c = 0.5 * (lo + hi)
    gap = np.min(np.abs(np.abs(p - c) - 0.5 * (hi - lo)), axis=1)
    p = p[gap > 1e-4]  # not on a face
    a, _ = surface_eval(ob.mesh(5), p)
    b, _ = surface_eval(ob.cuboid(c, 0.5 * (hi - lo)), p)
    assert np.array_equal(a, b) and a.sum() > 500


def test_read_obj(tmp_path):
    """The library's OBJ reader (no GPU): quads split into two triangles, negative and v/t/n
    references, other records skipped; bad references are errors."""
    from splishsplash_for_cuda_b200 import _capi

    f = tmp_path / "m.obj"
    f.write_text("# box face and a triangle\no thing\nv 0 0 0\nv 1 0 0\nvt 0 0\nv 1 1 0\nv 0 1 0\n"
                 "vn 0 0 1\nf 1/1/1 2/1/1 3/1/1 4/1/1\nv 0.5 0.5 1\nf -1 1//1 2\ns off\n")
    v, t = ob.read_obj(f)
    assert v.shape == (5, 3) and v.dtype == np.float32
    assert np.array_equal(v[4], np.float32([0.5, 0.5, 1.0]))
    assert t.tolist() == [[0, 1, 2], [0, 2, 3], [4, 0, 1]]
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nf 1 2 3\n")
    with pytest.raises(_capi.DfsphError):
        ob.read_obj(bad)
    v2, t2 = ob.read_obj(_write_box_obj(tmp_path / "box.obj"))
    a, b = ob.box_mesh((0, 0, 0), (1, 2, 3))
    assert np.array_equal(v2, a) and np.array_equal(t2, b)


REF_DIR = Path(os.environ.get("REF_DIR", str(Path(__file__).resolve().parents[2] / "reference")))
REF_MODELS = ["UnitBox.obj", "EmitterBox.obj", "EmitterCylinder.obj", "2mBox_rotated45.obj", "Dragon_50k.obj"]


@pytest.mark.skipif(not PIN.exists() or not (REF_DIR / "data" / "models").is_dir(),
                    reason="the reference's OBJ_Loader pin or its models are not present")
def test_read_obj_matches_reference_loader():
    """dfsph_read_obj against the reference's own OBJ_Loader (as MeshPerso::loadFromFile calls it) on
    the reference's models: the same triangles, vertex positions bit for bit, in the same order."""
    lib = C.CDLL(str(PIN))
    lib.pin_obj_triangles.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
    for name in REF_MODELS:
        path = REF_DIR / "data" / "models" / name
        n = C.c_uint32()
        assert lib.pin_obj_triangles(str(path).encode(), None, 0, C.byref(n)) == 0
        want = np.zeros((n.value, 9), np.float32)
        assert lib.pin_obj_triangles(str(path).encode(), want.ctypes.data, n.value, C.byref(n)) == 0
        v, t = ob.read_obj(path)
        assert np.array_equal(v[t].reshape(-1, 9), want), name


def _write_box_obj(path):
    v, t = ob.box_mesh((0, 0, 0), (1, 2, 3))
    lines = [f"v {x:.9g} {y:.9g} {z:.9g}" for x, y, z in v] + [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in t]
    path.write_text("\n".join(lines) + "\n")
    return path


def test_presets():
    r = 0.01
    b, i, s, name = ob.preset(0, r)
    assert name == "inflowPositionsSet_cylinder.txt" and b.type == 2 and b.radius == 1.5
    assert i.radius == np.float32(np.float32(1.5) - np.float32(3 * r))
    assert s.type == 0 and tuple(s.normal) == (0.0, -1.0, 0.0) and tuple(s.origin) == (0.0, 1.0, 0.0)
    b, i, _, _ = ob.preset(600, r)
    assert b.type == 5 and b.points == 5 and b.radius == 3.5 and b.radius_internal == 2.0
    b, i, _, name = ob.preset(1001, r)
    assert b.type == 1 and tuple(i.center) == (0.0, 0.0, -1.0) and name.endswith("corridor.txt")
    for c in (100, 200, 210, 220, 300, 400, 500):
        ob.preset(c, r)
    with pytest.raises(ValueError):
        ob.preset(7, r)


# ---- a small tank: fluid in one half, taller than the fluid surface ----------------------------
R = 0.025


def tank_scene(vx=0.0):
    cfg = Configuration()
    cfg.particleRadius = R
    cfg.timeStepSize = 0.002
    walls = box_wall((0.0, 0.0, 0.0), (1.0, 1.0, 0.5), 2 * R)
    fluid = lattice_block((9, 13, 9), R)  # x, z in [0.05, 0.45], y up to 0.65
    rng = np.random.default_rng(5)
    fluid = fluid + rng.uniform(-0.01 * R, 0.01 * R, size=fluid.shape)
    vel = np.zeros_like(fluid)
    vel[:, 0] = vx * np.where(fluid[:, 2] < 0.25, 1.0, -1.0)
    return Scene(config=cfg, fluid=fluid.astype(np.float32), boundary=walls.astype(np.float32),
                 fluid_velocity=vel.astype(np.float32), name="tank")


def tank_samples():
    """The rest lattice of the whole tank with a 1 % r jitter (samples of a fluid at rest: an exact
    lattice would put new particles at exactly H from each other, where the FP32 pair predicate of
    the FP32 build and of the FP64 oracle's rounded positions can disagree)."""
    x = lattice_block((19, 19, 9), R)
    rng = np.random.default_rng(11)
    return (x + rng.uniform(-0.01 * R, 0.01 * R, size=x.shape)).astype(np.float32)


def tank_surfaces():
    return (ob.cuboid((0.5, 0.5, 0.25), (0.5, 0.5, 0.25)), ob.cuboid((0.5, 0.5, 0.25), (0.425, 0.425, 0.175)),
            ob.plane((0.0, 0.5, 0.0), (0.0, -1.0, 0.0)))


def _W(r, H):
    q = r / H
    k = 8.0 / (np.pi * H ** 3)
    return np.where(q <= 0.5, k * (6 * q ** 3 - 6 * q ** 2 + 1), np.where(q <= 1.0, k * 2 * (1 - q) ** 3, 0.0))


def test_oracle_open_boundary_against_numpy():
    s = tank_scene(vx=0.3)
    o = Oracle(s, 64)
    b, i, f = tank_surfaces()
    samples = tank_samples()
    kept = o.open_boundary_init(b, i, f, samples)
    ins_i, _ = surface_eval(i, samples)
    ins_f, _ = surface_eval(f, samples)
    ks = samples[~ins_i & ins_f]
    assert kept == ks.shape[0] > 0
    # numpy restatement: brute force over the fluid (every particle within H matters; the reference's
    # 27-cell iteration adds only particles beyond H, whose kernel weight is zero and which are
    # farther than allowed_distance)
    x = s.fluid.astype(np.float64)
    v = s.fluid_velocity.astype(np.float64)
    xb = s.boundary.astype(np.float64)
    psi = o.field("boundary_psi")
    H = 4 * R
    m = np.float32(0.8 * (2 * R) ** 3 * 1000.0)
    allowed = 1.75 * R
    exp_x, exp_v = [], []
    _, nrm = surface_eval(b, ks)
    for q, nq in zip(ks.astype(np.float64), nrm):
        d = np.linalg.norm(x - q, axis=1)
        if d.size and d.min() <= np.float32(allowed):
            continue
        w = _W(d, H) * m
        wb = _W(np.linalg.norm(xb - q, axis=1), H) * psi
        rho = _W(0.0, H) * m + w.sum() + wb.sum()
        ws = w.sum() + wb.sum()
        vq = (w[:, None] * v).sum(0) / ws if ws > 0 else np.zeros(3)
        if rho > 700.0 or float(np.dot(vq.astype(np.float32), nq)) < 0:
            continue
        exp_x.append(q)
        exp_v.append(vq)
    added, removed, clipped = o.open_boundary_apply(allowed, 700.0, True, False)
    assert not clipped and added == len(exp_x) > 0 and removed == 0
    xo, vo = o.field("position"), o.field("velocity")
    assert np.array_equal(xo[:s.n_fluid], x) and np.array_equal(xo[s.n_fluid:], np.array(exp_x))
    assert np.abs(vo[s.n_fluid:] - np.array(exp_v)).max() <= 1e-6 * max(1.0, np.abs(exp_v).max())
    assert np.all(o.field("kappa")[s.n_fluid:] == 0)
    # outflow: particles outside the interior and above the fluid surface, order kept
    xo = o.field("position")
    ii, _ = surface_eval(i, xo)
    ff, _ = surface_eval(f, xo)
    keep = ii | ff
    assert (~keep).sum() > 0
    a2, r2, _ = o.open_boundary_apply(allowed, 700.0, False, True)
    assert a2 == 0 and r2 == int((~keep).sum())
    assert np.array_equal(o.field("position"), xo[keep])
    # the fluid still steps
    o.step()
    assert np.isfinite(o.field("position")).all()
