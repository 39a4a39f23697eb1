"""GPU parity: the CUDA library, driven through the C ABI, against the CPU
oracle on the same seeded inputs.

Neighbor grids are compared bit for bit (cell of every particle, members of
every cell in ascending id, neighbor counts within h).  States are compared
per quantity with the norm-wise relative error max|gpu - oracle| / max|oracle|;
the bound is 1e-5 after 100 steps (the benchmark's stated FP32 tolerance),
and each quantity's error against the FP64 oracle is printed beside it.
"""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle.oracle import Oracle
from helpers import rel_err, gpu_state, oracle_csr

pytestmark = pytest.mark.gpu

TOL = 1e-5


def make(scene):
    sim = FluidSim(scene)
    sim.init()
    return sim


def small_2d():
    return scenes.dam_break_2d(nx=32, ny=32, box=(0.64, 0.32))


def small_3d():
    return scenes.small_fluid_bar_3d()


@pytest.mark.parametrize("factory", [small_2d, small_3d])
def test_neighbor_grid_bit_exact(factory):
    sc = factory()
    sim = make(sc)
    o = Oracle(sc)
    b = o.buckets()
    sub, nc = sim.grid()
    np.testing.assert_array_equal(sub[:3], o.sub[:3])
    assert nc == o.ncells
    g = sim.neighbors()
    start, members, bstart, bmembers = oracle_csr(b, sc.n, o.ncells)
    np.testing.assert_array_equal(g["cell_of"], b["pos_index"])
    np.testing.assert_array_equal(g["cell_start"], start)
    np.testing.assert_array_equal(g["members"], members)
    np.testing.assert_array_equal(g["nbr_count"], b["nbr_count"])
    gbs, gbm = sim.boundary_cells()
    np.testing.assert_array_equal(gbs, bstart)
    np.testing.assert_array_equal(gbm, bmembers)


@pytest.mark.parametrize("factory", [small_2d, small_3d])
def test_single_euler_step_matches_oracle(factory):
    """One Euler step exposes the derivative record k = (y1 - y0) / dt."""
    sc = factory()
    sc.integrator = "euler"
    sim = make(sc)
    o = Oracle(sc)
    sim.step(1)
    o.step(1)
    g, r = gpu_state(sim), o.state()
    p0 = sc.particles
    for key, y0 in (("den", p0["den"]), ("pos", p0["pos"]), ("vel", p0["vel"])):
        kg = g[key] - y0
        ko = r[key] - y0
        e = rel_err(kg, ko)
        print(f"{sc.name} {key} derivative rel err {e:.2e}")
        assert e < 1e-4, key


def run_pair(sc, steps):
    sim = make(sc)
    o32, o64 = Oracle(sc, 32), Oracle(sc, 64)
    sim.step(steps)
    o32.step(steps)
    o64.step(steps)
    return gpu_state(sim), o32.state(), o64.state(), sim


def check_states(name, g, r, r64):
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r[key])
        e64 = rel_err(g[key], r64[key])
        e_or = rel_err(r[key], r64[key])
        print(f"{name} {key}: gpu-vs-oracle32 {e:.2e}  gpu-vs-fp64 {e64:.2e}  oracle32-vs-fp64 {e_or:.2e}")
        assert e < TOL, (key, e)


def test_dam_break_small_rk4_100_steps():
    sc = small_2d()
    g, r, r64, _ = run_pair(sc, 100)
    check_states("dam_break_32x32", g, r, r64)


def test_fluid_bar_small_rk2_100_steps():
    sc = small_3d()
    g, r, r64, sim = run_pair(sc, 100)
    check_states("fluid_bar_small", g, r, r64)


def test_dam_break_full_size_rk4_100_steps():
    """The 2D dam break at its benchmark size (128x128 fluid, 2340 boundary)."""
    sc = scenes.dam_break_2d()
    g, r, r64, _ = run_pair(sc, 100)
    check_states("dam_break_128x128", g, r, r64)


def test_runs_are_deterministic():
    sc = small_3d()
    a, b = make(sc), make(sc)
    a.step(20)
    b.step(20)
    pa, pb = a.particles(), b.particles()
    assert pa.tobytes() == pb.tobytes()


def test_accessors_mirror_the_reference_interface():
    sc = small_3d()
    sim = make(sc)
    o = Oracle(sc)
    assert sim.num_materials() == len(sc.materials)
    assert sim.kernel_radius() == np.float32(sc.h)
    assert sim.ns == o.ns and sim.n == sc.n and sim.nb == sc.nb
    sim.update()
    assert abs(sim.time() - np.float32(sc.dt)) == 0
    solids = sim.solids()
    assert (solids["part_id"] == np.nonzero(sim.particles()["solid_id"] != 0xFFFFFFFF)[0]).all()
    it = sim.interactions()
    # default_between: fluid (Tait) vs bar (zero EOS) gets the linear contact
    assert it[2, 3]["potential"] == 2 and it[2, 3]["strength"] == 10000.0
    assert abs(it[2, 3]["radius"] - np.float32(sc.h) * 2) == 0
    assert it[2, 2]["potential"] == 0


def test_profile_and_launch_counters():
    sc = small_2d()
    sim = make(sc)
    sim.profile_enable(True)
    before = sim.launch_count()
    sim.step(3)
    prof = sim.profile_read()
    assert prof["steps"] == 3
    assert prof["stages"] == 12  # RK4
    assert prof["fluid_launches"] == 36  # per stage: the fused fluid kernel and its two overflow kernels
    assert prof["fluid_ms"] > 0 and prof["neighbor_ms"] > 0
    assert sim.launch_count() - before == prof["launches"]
    st = sim.stats()
    assert st["nonfinite_positions"] == 0 and st["max_cell_occupancy"] > 0
    # sampled: events on one step in every 3
    sim.profile_enable(True, every=3)
    sim.step(7)
    prof = sim.profile_read()
    assert prof["steps"] == 3 and prof["stages"] == 12  # steps 1, 4 and 7 of the 7
    assert prof["fluid_ms"] > 0
    sim.profile_enable(False)


def test_state_round_trip_and_validation():
    sc = small_3d()
    sim = make(sc)
    sim.step(2)
    p = sim.particles()
    sim.set_particles(p)
    q = sim.particles()
    assert p.tobytes() == q.tobytes()
    bad = p.copy()
    bad["mat"][5] = (bad["mat"][5] + 1) % len(sc.materials)
    with pytest.raises(Exception) as e:
        sim.set_particles(bad)
    assert "material" in str(e.value)
    bad = p.copy()
    bad["pos"][3, 3] = 1.0
    with pytest.raises(Exception):
        sim.set_particles(bad)
