"""Velocity Verlet (the reference's default integrator,
examples/test_mods/config.rs:451; selected at examples/test.rs:167) on the GPU
against the oracle's kick-drift-kick restatement: synthetic fluid and
fluid + solid scenes, and the reference's own Verlet scenes as seeded by the
scene loader (fixtures under tests/golden/scenes_seeded).  State within 1e-5
norm-wise relative error of the float oracle after the stated steps; the
error against the double oracle is printed beside it."""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle.oracle import Oracle
from helpers import compare_with_oracle as compare, load_seeded_scene, rel_err

pytestmark = pytest.mark.gpu


def test_verlet_dam_break_matches_oracle():
    sc = scenes.dam_break_2d(nx=48, ny=48, box=(0.96, 0.64), integrator="verlet")
    compare(sc, 100)


def test_verlet_fluid_and_solid_match_oracle():
    sc = scenes.small_fluid_bar_3d(integrator="verlet")
    compare(sc, 60)


def test_verlet_graph_replay_matches_plain_steps():
    sc = scenes.small_fluid_bar_3d(integrator="verlet")
    a = FluidSim(sc)
    a.init()
    a.step(7)
    b = FluidSim(sc)
    b.init()
    b.set_graph(True)
    b.step(7)
    assert a.particles().tobytes() == b.particles().tobytes()
    assert a.time() == b.time()


def test_verlet_restarts_from_a_new_state():
    """After set_particles the first step evaluates the forces at the new
    state again, as the oracle does after its state is replaced."""
    sc = scenes.dam_break_2d(nx=16, ny=16, box=(0.32, 0.32), integrator="verlet")
    sim = FluidSim(sc)
    sim.init()
    sim.step(5)
    p = sim.particles().copy()
    p["vel"][:, 0] += np.float32(0.05)
    sim.set_particles(p)
    sim.step(5)
    o = Oracle(sc, 32)
    o.step(5)
    s = o.state()
    o.set_state(den=s["den"], pos=s["pos"], vel=s["vel"] + np.array([0.05, 0, 0, 0]))
    o.step(5)
    r = o.state()
    for key in ("den", "pos", "vel"):
        assert rel_err(sim.particles()[key], r[key]) < 1e-5, key


@pytest.mark.parametrize("name,steps", [("cloth", 40), ("solid_test_3D", 60), ("spinning_ball", 60),
                                        ("container_buckling", 40)])
def test_reference_verlet_scenes_match_oracle(name, steps):
    """The reference's own Verlet scenes are stiff solids (cloth, elastic balls,
    a buckling container) at small time steps: the float oracle itself is
    ~1e-4 from the double oracle in velocity after these steps (with RK2 as
    with Verlet), so the GPU is held to the float oracle's distance from the
    double one."""
    sc = load_seeded_scene(name)
    assert sc.integrator == "verlet"
    compare(sc, steps, fp32_floor=True)


def test_verlet_bar_gradients_match_fp64_finite_differences():
    """Reverse mode of the Verlet step: the closing kick, the force
    evaluation at the drifted state, the kick-drift, and the force evaluation
    at y_0 the tape starts with, against FP64 central differences.  Verlet
    drifts solids at v where the Runge-Kutta tableaus move them at 2v (the
    reference's summed derivative records), so the same bar strains less and
    its stiffness gradient is about a fifth of the RK2 one: the bar starts
    from twice the velocity spread and runs 200 steps to lift that gradient
    clear of the float32 position resolution."""
    from test_gpu_adjoint import fd_check, report
    sc = scenes.cantilever_bar(n=(4, 16, 4), v_sigma=0.2, target_offset=(0.002, -0.02, 0.001), integrator="verlet")
    rng = np.random.default_rng(77)
    ds = [rng.normal(size=sc.n) for _ in range(8)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(16)]
    L, res = fd_check(sc, 200, 20, ("tip", sc.meta["tip"], sc.meta["target"]), ds, dv)
    assert report(res, 1e-4) == 0


def test_verlet_fluid_gradients_match_fp64_finite_differences():
    from test_gpu_adjoint import fd_check, report
    sc = scenes.dam_break_2d(nx=12, ny=12, box=(0.32, 0.24), integrator="verlet")
    rng = np.random.default_rng(78)
    sc.particles["vel"][:, :2] = rng.normal(0.0, 0.2, size=(sc.n, 2)).astype(np.float32)
    target = (sc.particles["pos"][:, :3] + rng.normal(0.0, 0.002, size=(sc.n, 3))).astype(np.float64)
    target[:, 2] = 0.0
    dv = []
    for _ in range(16):
        d = rng.normal(size=(sc.n, 3))
        d[:, 2] = 0.0
        dv.append(d)
    L, res = fd_check(sc, 20, 5, ("points", target), [], dv)
    assert report(res, 1e-4) == 0
