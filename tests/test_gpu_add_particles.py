"""FluidSim.add_particles (src/soft_body/mod.rs:180-206 with
Particles::add_particles, src/soft_body/particle_state/particles.rs:547-631)
on the GPU against the oracle's restatement of the same call.

After an addition the handle must hold the reference's material table,
interaction table, particle order and solid numbering, and later steps must
agree with the oracle within the 1e-5 norm-wise relative bound of the other
parity tests.
"""
import os

import numpy as np
import pytest

from arphys import FluidSim, scenes
from arphys.abi import ArpError, MATERIAL_DTYPE
from oracle.oracle import Oracle
from helpers import rel_err, gpu_state

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-5


def check_states(sim, o, name):
    g, r = gpu_state(sim), o.state()
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r[key])
        print(f"{name} {key}: gpu-vs-oracle32 {e:.2e}")
        assert e < TOL, (key, e)


def check_tables(sim, o):
    gm, om = sim.materials(), o.materials()
    assert gm.tobytes() == om.tobytes()
    gi = sim.interactions()
    oi = o.interactions()
    for f, k in (("potential", 0), ("strength", 1), ("radius", 2), ("dampening", 3), ("friction", 4)):
        np.testing.assert_array_equal(gi[f].astype(np.float64), oi[:, :, k], err_msg=f)
    p = sim.particles()
    r = o.state()
    np.testing.assert_array_equal(p["mat"], r["mat"])
    np.testing.assert_array_equal(p["solid_id"], r["solid_id"])


def test_on_click_object_added_mid_run_matches_the_oracle():
    path = os.path.join(HERE, "golden", "scenes", "csg_2d.toml")
    sc = scenes.load_toml(path)
    click = sc.meta["on_click"][0]
    sim = FluidSim.from_toml(path)
    sim.init()
    o = Oracle(sc, 32)
    for _ in range(3):
        sim.update()
        o.update()
    offset = np.array([0.1, -0.05, 0.0, 0.0], np.float32)
    added = sim.add_particles(click["particles"], click["material"], offset)
    assert added == o.add_particles(click["particles"], click["material"], offset)
    assert added  # the spawn object's material equals none of the scene's
    assert sim.n == sc.n + len(click["particles"])
    check_tables(sim, o)
    np.testing.assert_array_equal(sim.particles()["pos"][sc.n:], o.state()["pos"][sc.n:].astype(np.float32))
    # the same object again reuses the material appended the first time
    assert not sim.add_particles(click["particles"], click["material"], -offset)
    assert not o.add_particles(click["particles"], click["material"], -offset)
    check_tables(sim, o)
    assert sim.time() == pytest.approx(o.time, rel=1e-6)
    for _ in range(5):
        sim.update()
        o.update()
    check_states(sim, o, "csg_2d + on_click")


def _solid_block(origin, n, spacing, mat):
    pts = [(origin[0] + i * spacing, origin[1] + j * spacing) for j in range(n) for i in range(n)]
    p = np.zeros(len(pts), dtype=scenes.PARTICLE_DTYPE)
    p["pos"][:, :2] = np.array(pts, np.float32)
    p["den"] = mat["start_den"]
    p["solid_id"] = 0xFFFFFFFF
    return p


def test_solids_added_to_a_scene_without_solids_are_numbered_from_one():
    """A scene created without solids keeps a placeholder solid entry 0
    (particles.rs:502), so the added solids take ids 1.. and every added solid
    material is new, even when equal to an earlier one (particles.rs:550-556)."""
    sc = scenes.dam_break_2d(nx=24, ny=24, box=(0.64, 0.32))
    sim = FluidSim(sc)
    sim.init()
    o = Oracle(sc, 32)
    sim.step(2)
    o.step(2)
    h = sc.h
    mass = np.float32(500.0) * np.float32(0.6 * h) ** 2
    m = np.zeros((), dtype=MATERIAL_DTYPE)
    m["start_den"] = m["target_den"] = 500.0
    m["mass"] = mass
    m["normal_stiffness"] = -2e4
    m["shear_stiffness"] = -1e4
    m["strain_order"] = 2
    block = _solid_block((0.45, 0.12), 4, 0.6 * h, m)
    for k in range(2):
        blk = block.copy()
        blk["pos"][:, 0] += k * 0.06
        assert sim.add_particles(blk, m) and o.add_particles(blk, m)
    check_tables(sim, o)
    sid = sim.particles()["solid_id"]
    np.testing.assert_array_equal(sid[sc.n:], np.arange(1, 33, dtype=np.uint32))
    assert sim.ns == 32
    for _ in range(6):
        sim.step(1)
        o.step(1)
    check_states(sim, o, "dam break + 2 solid blocks")


def test_equal_fluid_material_is_reused_and_errors_are_reported():
    sc = scenes.dam_break_2d(nx=16, ny=16, box=(0.64, 0.32))
    sim = FluidSim(sc)
    with pytest.raises(ArpError):  # before init the reference has no state to add to
        sim.add_particles(sc.particles[:4], sc.materials[1])
    sim.init()
    fluid = int(sc.particles["mat"][0])
    drop = sc.particles[:8].copy()
    assert not sim.add_particles(drop, sc.materials[fluid], np.array([0.0, 0.1, 0.0, 0.0], np.float32))
    assert np.all(sim.particles()["mat"][-8:] == fluid)
    assert not sim.add_particles(drop[:0], sc.materials[fluid])  # nothing added
    assert sim.n == sc.n + 8
    boundary_mat = int(sc.boundary["mat"][0])
    with pytest.raises(ArpError) as e:
        sim.add_particles(drop, sc.materials[boundary_mat])
    assert e.value.code == 6
    batch = FluidSim.batch([sc, sc])
    batch.init()
    with pytest.raises(ArpError) as e:
        batch.add_particles(drop, sc.materials[fluid])
    assert e.value.code == 6
