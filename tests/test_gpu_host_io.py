"""The asynchronous host exchange (arp_sim_set_particles_async,
arp_sim_get_particles_async, arp_sim_synchronize) against the synchronous
calls: the same inputs, one step each, give the same records bit for bit,
with graph replay and without, and for velocity Verlet, whose force record a
new state invalidates; record checks are reported by the next synchronize."""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from arphys.abi import ArpError

pytestmark = pytest.mark.gpu


def inputs(sc, count):
    """`count` distinct caller-order states: the scene's, with velocities
    scaled by seeded factors."""
    rng = np.random.default_rng(61)
    out = []
    for k in range(count):
        p = sc.particles.copy()
        p["vel"][:, :3] *= np.float32(1.0 + 0.1 * k)
        p["pos"][:, :3] += rng.uniform(-1e-4, 1e-4, size=(len(p), 3)).astype(np.float32)
        out.append(p)
    return out


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("integrator", ["rk2", "verlet"])
def test_async_exchange_matches_synchronous_calls(graph, integrator):
    sc = scenes.small_fluid_bar_3d(integrator=integrator)
    ins = inputs(sc, 6)
    a = FluidSim(sc)
    a.init()
    a.set_graph(graph)
    ref = []
    for p in ins:
        a.set_particles(p)
        a.step(1)
        ref.append(a.particles())
    b = FluidSim(sc)
    b.init()
    b.set_graph(graph)
    outs = [np.zeros(sc.n, dtype=ins[0].dtype) for _ in ins]
    for p, o in zip(ins, outs):
        b.set_particles_async(p)
        b.step(1)
        b.particles_async(o)
    b.synchronize()
    for k, (r, o) in enumerate(zip(ref, outs)):
        assert r.tobytes() == o.tobytes(), k
    # the synchronous calls see the state the asynchronous ones left
    assert b.particles().tobytes() == ref[-1].tobytes()


def test_async_set_reports_a_changed_material_at_synchronize():
    sc = scenes.small_fluid_bar_3d()
    sim = FluidSim(sc)
    sim.init()
    good = sim.particles()
    bad = good.copy()
    bad["mat"][0] = (int(bad["mat"][0]) + 1) % len(sc.materials)
    sim.set_particles_async(bad)
    sim.step(1)
    with pytest.raises(ArpError) as e:
        sim.synchronize()
    assert e.value.code == 1
    sim.synchronize()  # the report is cleared
    sim.set_particles_async(good)
    sim.step(1)
    out = np.zeros_like(good)
    sim.particles_async(out)
    sim.synchronize()
    ref = FluidSim(sc)
    ref.init()
    ref.set_particles(good)
    ref.step(1)
    assert out.tobytes() == ref.particles().tobytes()


def test_async_exchange_follows_added_particles():
    """The staging slots grow with the particle count: after add_particles
    the asynchronous calls move the new count of records, matching the
    synchronous calls on a twin handle."""
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes", "csg_2d.toml")
    sc = scenes.load_toml(path)
    click = sc.meta["on_click"][0]
    offset = np.array([0.1, -0.05, 0.0, 0.0], np.float32)
    a, b = FluidSim.from_toml(path), FluidSim.from_toml(path)
    a.init()
    b.init()
    p0 = a.particles()
    out = np.zeros_like(p0)
    b.set_particles_async(p0)
    b.step(1)
    b.particles_async(out)
    b.synchronize()
    a.set_particles(p0)
    a.step(1)
    assert a.particles().tobytes() == out.tobytes()
    a.add_particles(click["particles"], click["material"], offset)
    b.add_particles(click["particles"], click["material"], offset)
    p1 = a.particles()
    assert len(p1) > len(p0)
    out1 = np.zeros_like(p1)
    b.set_particles_async(p1)
    b.step(2)
    b.particles_async(out1)
    b.synchronize()
    a.set_particles(p1)
    a.step(2)
    assert a.particles().tobytes() == out1.tobytes()
