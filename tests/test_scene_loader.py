"""Scene files: the library's TOML loader (arp_scene_file_load) against the
oracle restatement (oracle/scene_oracle.py) and hand-computed cases.

The loader replaces Config::parse (examples/test_mods/config.rs:298-474) and
the seeding in FluidSim::new (src/soft_body/mod.rs:70-86 calling
MaterialRegion::gen_particles, material_region/mod.rs:56-156).  Seeding is
integer and float32 work done on the host, so every record must agree bit for
bit.  These tests call no CUDA function.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

from arphys import FluidSim, scenes
from arphys.abi import ArpError
from oracle import scene_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = sorted(glob.glob(os.path.join(HERE, "golden", "scenes", "*.toml")))
# The reference's own example scenes, read as data from the directory named by
# ARP_REFERENCE_EXAMPLES (the reference's `examples/`); the tests that use them
# skip when it is unset or holds no scenes.
_EXAMPLES_DIR = os.environ.get("ARP_REFERENCE_EXAMPLES", "")
REFERENCE_EXAMPLES = sorted(glob.glob(os.path.join(_EXAMPLES_DIR, "*.toml"))) if _EXAMPLES_DIR else []

f32 = np.float32


def _write(tmp_path, text, name="scene.toml"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def assert_same_scene(lib_scene, orc):
    for key, recs in (("particles", lib_scene.particles), ("boundary", lib_scene.boundary)):
        o = orc[key]
        assert len(recs) == len(o["pos"]), key
        np.testing.assert_array_equal(recs["pos"], o["pos"], err_msg=key)
        np.testing.assert_array_equal(recs["vel"], o["vel"], err_msg=key)
        np.testing.assert_array_equal(recs["den"], o["den"], err_msg=key)
        np.testing.assert_array_equal(recs["mat"], o["mat"], err_msg=key)
    assert len(lib_scene.materials) == len(orc["materials"])
    for got, want in zip(lib_scene.materials, orc["materials"]):
        for field in scene_oracle.MATERIAL_FIELDS:
            assert got[field] == want[field], (field, got[field], want[field])
    m = len(orc["materials"])
    for i in range(m):
        for j in range(m):
            want = orc["interactions"][i][j]
            assert bool(lib_scene.interaction_given[i, j]) == (want is not None), (i, j)
            if want is not None:
                got = lib_scene.interactions[i, j]
                for field in ("potential", "strength", "radius", "friction", "dampening"):
                    assert got[field] == want[field], (i, j, field)
    assert f32(lib_scene.h) == orc["h"]
    assert f32(lib_scene.dt) == orc["dt"]
    assert f32(lib_scene.gravity) == orc["gravity"]
    assert f32(lib_scene.alpha) == orc["alpha"]
    assert lib_scene.subticks == orc["subticks"]
    assert lib_scene.name == orc["name"]
    np.testing.assert_array_equal(np.array(lib_scene.bounds_min, f32), orc["bounds_min"])
    np.testing.assert_array_equal(np.array(lib_scene.bounds_dim, f32), orc["bounds_dim"])
    clicks = lib_scene.meta["on_click"]
    assert len(clicks) == len(orc["on_click"])
    for got, want in zip(clicks, orc["on_click"]):
        assert got["relative"] == want["relative"]
        np.testing.assert_array_equal(got["particles"]["pos"], want["pos"])
        np.testing.assert_array_equal(got["particles"]["vel"], want["vel"])
        np.testing.assert_array_equal(got["particles"]["den"], want["den"])
        assert np.all(got["particles"]["mat"] == 0)
        for field in scene_oracle.MATERIAL_FIELDS:
            assert got["material"][field] == want["material"][field], field


@pytest.mark.parametrize("path", SCENES, ids=[os.path.basename(p) for p in SCENES])
def test_committed_scene_matches_the_oracle(path):
    assert_same_scene(scenes.load_toml(path), scene_oracle.load(path))


def _uses_stl(path):
    return "model" in str(scene_oracle.tomllib.load(open(path, "rb")))


@pytest.mark.skipif(not REFERENCE_EXAMPLES, reason="the reference's example scenes are not mounted")
@pytest.mark.parametrize("path", REFERENCE_EXAMPLES, ids=[os.path.basename(p) for p in REFERENCE_EXAMPLES])
def test_reference_example_scene_matches_the_oracle(path, monkeypatch):
    """Scene files name STL models relative to the reference's root, which is
    where its demo runs from.  The oracle walks every face for every lattice
    site, which takes minutes for the STL scenes: those run only with
    ARP_SLOW_TESTS=1."""
    if _uses_stl(path) and not os.environ.get("ARP_SLOW_TESTS"):
        pytest.skip("STL scene: set ARP_SLOW_TESTS=1")
    monkeypatch.chdir(os.path.dirname(os.path.dirname(path)))
    try:
        orc = scene_oracle.load(path)
    except (scene_oracle.SceneError, OSError) as err:  # a model file the reference does not ship
        with pytest.raises(ArpError) as e:
            scenes.load_toml(path)
        assert e.value.code == 8 and "STL" in str(e.value), err
        return
    assert_same_scene(scenes.load_toml(path), orc)


@pytest.mark.skipif(not REFERENCE_EXAMPLES, reason="the reference's example scenes are not mounted")
def test_seeded_fixtures_are_the_loaders_output(monkeypatch):
    """tests/golden/scenes_seeded holds what the loader seeds from the
    reference's shipped scenes (the GPU tests step them where the reference
    tree is absent); each fixture is the loader's output bit for bit."""
    from helpers import load_seeded_scene
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "golden", "scenes_seeded", "*.npz")))
    assert len(names) == 22
    monkeypatch.chdir(os.path.dirname(os.path.abspath(_EXAMPLES_DIR)))
    for name in names:
        fresh = scenes.load_toml(os.path.join(_EXAMPLES_DIR, name + ".toml"))
        fix = load_seeded_scene(name)
        for key in ("particles", "boundary", "materials", "interactions"):
            assert getattr(fresh, key).tobytes() == getattr(fix, key).tobytes(), (name, key)
        assert (fresh.h, fresh.dt, fresh.integrator, fresh.subticks) == (fix.h, fix.dt, fix.integrator, fix.subticks)


def _write_stl(path, tris, ascii=False):
    """Triangles (F x 3 x 3) with outward normals from the winding."""
    tris = np.asarray(tris, np.float32)
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0]).astype(np.float32)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    if ascii:
        with open(path, "w") as f:
            f.write("solid test\n")
            for k in range(len(tris)):
                f.write("facet normal %r %r %r\n outer loop\n" % tuple(float(x) for x in n[k]))
                for v in tris[k]:
                    f.write("  vertex %r %r %r\n" % tuple(float(x) for x in v))
                f.write(" endloop\nendfacet\n")
            f.write("endsolid test\n")
        return
    rec = np.zeros(len(tris), np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]))
    rec["n"], rec["v"] = n, tris
    with open(path, "wb") as f:
        f.write(b"binary test mesh".ljust(80, b" "))
        f.write(np.uint32(len(tris)).tobytes())
        f.write(rec.tobytes())


def _octahedron():
    c = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    faces = []
    for sx in (0, 1):
        for sy in (2, 3):
            for sz in (4, 5):
                a, b, d = c[sx], c[sy], c[sz]
                tri = [a, b, d]
                if np.dot(np.cross(np.subtract(b, a), np.subtract(d, a)), np.add(np.add(a, b), d)) < 0:
                    tri = [a, d, b]
                faces.append(tri)
    return faces


def test_stl_regions_match_the_oracle(tmp_path):
    """A closed mesh region (mesh.rs:26-77: parity of the faces above the
    point) and a shell of given thickness around a surface (mesh.rs:79-138),
    each scaled and translated by the region transform, from binary and ASCII
    STL files."""
    _write_stl(tmp_path / "oct.stl", _octahedron())
    _write_stl(tmp_path / "oct_ascii.stl", _octahedron(), ascii=True)
    path = _write(tmp_path, f"""
kernel_radius = 0.02
integrator = "rk4"
min = [-0.5, -0.5, -0.5]
dim = [1.0, 1.0, 1.0]
[objects.solid]
  density = 100.0
  region = {{model = "{tmp_path / 'oct.stl'}", scale = 0.15, translation = [0.1, 0.0, 0.0]}}
[objects.ascii]
  density = 50.0
  region = {{model = "{tmp_path / 'oct_ascii.stl'}", scale = [0.1, 0.05, 0.1], translation = [-0.2, 0.2, 0.0]}}
[boundaries.shell]
  region = {{model = "{tmp_path / 'oct.stl'}", border = 0.03, scale = 0.3}}
""")
    sc = scenes.load_toml(path)
    assert_same_scene(sc, scene_oracle.load(path))
    # mesh.rs:48-52 counts a face as above the point when any of its vertices
    # is, not its surface: for the octahedron every point over the upper half
    # of the diamond |x| + |y| <= r crosses one upper face and, below z = 0,
    # also one lower face, so the region is the prism 0 < z <= r over it
    solid = sc.particles[sc.particles["mat"] == 2]
    q = solid["pos"][:, :3] - np.array([0.1, 0.0, 0.0], np.float32)
    eps = 1e-5
    assert len(solid) > 100
    assert np.all(np.abs(q[:, 0]) + np.abs(q[:, 1]) <= 0.15 + eps)
    assert np.all(q[:, 2] > -eps) and np.all(q[:, 2] <= 0.15 + eps)
    assert np.any(np.abs(q).sum(axis=1) > 0.15 + 0.02)  # beyond the octahedron itself
    shell = sc.boundary["pos"][:, :3] / 0.3
    r1 = np.abs(shell).sum(axis=1)
    assert len(shell) > 100 and np.all(np.abs(r1 - 1.0) < 0.5)


def test_missing_stl_file_is_a_parse_error(tmp_path):
    path = _write(tmp_path, "[objects.a]\n  region = {model = \"absent.stl\"}\n")
    with pytest.raises(ArpError) as e:
        scenes.load_toml(path)
    assert e.value.code == 8 and "STL" in str(e.value)


def test_lattice_known_answer(tmp_path):
    """A 0.2 x 0.1 box at pitch 0.1 (packing 1, h 0.1): rows alternate the
    x offset h/2 and advance y by h/sqrt(2); a row stops after the step that
    leaves the box; the mass divides the box's mass by every lattice site."""
    path = _write(tmp_path, """
kernel_radius = 0.1
integrator = "euler"
min = [0.0, 0.0]
dim = [1.0, 1.0]
[objects.a]
  packing = 1.0
  density = 1000.0
  region = {min = [0.0, 0.0], dim = [0.2, 0.1]}
""")
    sc = scenes.load_toml(path)
    h = f32(0.1)
    dy = f32(h / np.sqrt(f32(2.0)))
    want = [(0.0, 0.0), (h, 0.0), (f32(h + h), 0.0), (f32(h / f32(2)), dy),
            (f32(f32(h / f32(2)) + h), dy)]
    np.testing.assert_array_equal(sc.particles["pos"][:, :2], np.array(want, f32))
    assert np.all(sc.particles["pos"][:, 2:] == 0)
    assert sc.materials["mass"][0] == f32(1000.0 * (float(f32(0.2)) * float(f32(0.1))) / 5)
    assert np.all(sc.particles["den"] == 1000.0)
    assert sc.integrator == "euler"


def test_rotation_keeps_the_reference_matrix(tmp_path):
    """config.rs:158-163 builds the rotation with u[1]*u[2]*(1-c) - u[1]*s in
    column 1, row 0, where Rodrigues' formula has u[0]*u[1]*(1-c) - u[2]*s.
    About the z axis the "rotation" by theta is therefore the shear
    (x, y) -> (c x, s x + c y), and the loader keeps it: the seeded particles
    are the lattice sites whose preimage under that map lies in the box."""
    path = _write(tmp_path, """
kernel_radius = 0.02
integrator = "rk4"
[objects.bar]
  region = {min = [0.0, 0.0], dim = [0.3, 0.1], rotation = 30.0}
""")
    p = scenes.load_toml(path).particles["pos"].astype(np.float64)
    assert len(p) > 50
    c, s = np.cos(np.radians(30.0)), np.sin(np.radians(30.0))
    x = p[:, 0] / c
    y = (p[:, 1] - s * x) / c
    eps = 1e-5
    assert x.min() >= -eps and x.max() <= 0.3 + eps
    assert y.min() >= -eps and y.max() <= 0.1 + eps
    # a true rotation by 30 degrees would not hold these sites
    xr, yr = c * p[:, 0] + s * p[:, 1], -s * p[:, 0] + c * p[:, 1]
    assert (yr < -eps).any() or (yr > 0.1 + eps).any() or (xr > 0.3 + eps).any()


def test_object_order_state_inference_and_interaction_lookup(tmp_path):
    path = _write(tmp_path, """
kernel_radius = 0.05
artificial_viscocity = 2.0
integrator = "rk2"
[objects.zeta]
  speed_of_sound = 10.0
  density = 3.0
  region = {min = [0.0, 0.0], dim = [0.1, 0.1]}
[objects.alpha]
  speed_of_sound = 10.0
  start_density = 1.0
  region = {min = [0.2, 0.2], dim = [0.1, 0.1]}
  zeta = {contact_strength = 5.0}
[objects.mid]
  region = {min = [0.4, 0.4], dim = [0.1, 0.1]}
[boundaries.floor]
  friction = 0.25
  region = {min = [-0.5, -0.5], dim = [1.0, 0.1]}
  mid = {potential = "zero", contact_factor = 3.0}
""")
    sc = scenes.load_toml(path)
    m = sc.materials
    # boundaries first, then objects, each in key order: floor, alpha, mid, zeta
    assert list(m["immobile"]) == [1, 0, 0, 0]
    assert m["visc"][0] == f32(0.25) and m["start_den"][0] == 1 and m["target_den"][0] == 1
    assert list(m["state_eq"]) == [0, 2, 0, 3]  # ideal gas needs a start/target density key
    assert m["bulk_visc"][3] == f32(f32(2.0) * f32(0.05)) * f32(10.0)
    assert m["target_den"][3] == 3.0 and m["start_den"][3] == 3.0
    g, it = sc.interaction_given, sc.interactions
    assert g[1, 3] and g[3, 1] and it[3, 1]["strength"] == 5.0  # found under (alpha, zeta)
    assert it[1, 3]["radius"] == f32(2.0 * float(f32(0.05))) and it[1, 3]["potential"] == 2
    assert g[0, 2] and g[2, 0] and it[2, 0]["potential"] == 0
    assert it[0, 2]["radius"] == f32(3.0 * float(f32(0.05)))
    assert not g[0, 1] and not g[1, 1]
    assert set(np.unique(sc.boundary["mat"])) == {0}
    assert set(np.unique(sc.particles["mat"])) == {1, 2, 3}


def test_defaults_scene_loads_with_the_verlet_default():
    path = os.path.join(HERE, "golden", "scenes", "defaults.toml")
    sc = scenes.load_toml(path)
    assert sc.name == "Fluid Test" and sc.integrator == "verlet"  # config.rs:451
    assert f32(sc.h) == f32(1.0 / 64.0) and f32(sc.dt) == f32(0.01)
    assert sc.bounds_min[:2] == (-1.0, -1.0) and sc.bounds_dim[:2] == (2.0, 2.0)


@pytest.mark.parametrize("text,code,needle", [
    ("kernel_radius = = 1\n", 8, "line 1"),
    ("integrator = \"leapfrog\"\n[objects.a]\n  region = {min = [0.0, 0.0], dim = [0.1, 0.1]}\n", 8, "integrator"),
    ("[objects.a]\n  state = \"plasma\"\n  region = {min = [0.0, 0.0], dim = [0.1, 0.1]}\n", 8, "plasma"),
    ("[objects.a]\n  density = 1.0\n", 8, "region"),
    ("[[objects]]\nname = \"a\"\n", 6, "arrays of tables"),
    ("[objects.a]\n  packing = 0.0\n  region = {min = [0.0, 0.0], dim = [0.1, 0.1]}\n", 8, "spacing"),
])
def test_scene_file_errors(tmp_path, text, code, needle):
    path = _write(tmp_path, text)
    with pytest.raises(ArpError) as e:
        scenes.load_toml(path)
    assert e.value.code == code and needle in str(e.value)


def test_missing_scene_file_is_an_io_error(tmp_path):
    with pytest.raises(ArpError) as e:
        scenes.load_toml(str(tmp_path / "absent.toml"))
    assert e.value.code == 9


def test_scene_file_handle_calls_reject_null(lib):
    assert lib.arp_scene_file_load(None, None) == 1
    assert lib.arp_scene_file_scene(None, None) == 1
    assert lib.arp_scene_file_name(None, None) == 1
    assert lib.arp_scene_file_on_click_count(None, None) == 1
    assert lib.arp_scene_file_on_click(None, 0, None, None, None, None) == 1
    assert lib.arp_scene_file_free(None) == 0


def test_on_click_objects_are_seeded_but_not_in_the_scene():
    """config.rs:426-446 keeps "on_click" objects out of the scene and its
    interaction table; they are seeded as FluidSim::add_particles would seed
    them (material id 0, velocity field about their own bound)."""
    sc = scenes.load_toml(os.path.join(HERE, "golden", "scenes", "csg_2d.toml"))
    clicks = sc.meta["on_click"]
    assert len(clicks) == 1 and clicks[0]["relative"]
    assert len(sc.materials) == 6  # 2 boundaries + 4 objects; "spawn" is not among them
    c = clicks[0]["particles"]
    assert len(c) > 50 and np.all(c["mat"] == 0) and np.all(c["den"] == 1000.0)
    assert np.all(np.hypot(c["pos"][:, 0], c["pos"][:, 1]) <= 0.05 + 1e-6)
