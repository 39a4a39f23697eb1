"""Scene files end to end: FluidSim.from_toml (arp_sim_create_from_toml) on
the GPU against the oracle stepping the same seeded scene.

The committed scenes cover every region form, a plastic solid, an ideal gas,
a constant-pressure fluid and non-default contact potentials; the states
after `update` calls must agree within the 1e-5 norm-wise relative bound of
the other parity tests.
"""
import os

import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle.oracle import Oracle
from helpers import rel_err, gpu_state

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-5


@pytest.mark.parametrize("name,updates", [("csg_2d.toml", 10), ("transforms_3d.toml", 10)])
def test_scene_file_steps_match_the_oracle(name, updates):
    path = os.path.join(HERE, "golden", "scenes", name)
    sc = scenes.load_toml(path)
    sim = FluidSim.from_toml(path)
    assert (sim.n, sim.nb) == (sc.n, sc.nb)
    np.testing.assert_array_equal(sim.particles()["pos"], sc.particles["pos"])
    sim.init()
    o = Oracle(sc, 32)
    for _ in range(updates):
        sim.update()
        o.update()
    assert sim.time() == pytest.approx(o.time, rel=1e-6)
    g, r = gpu_state(sim), o.state()
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r[key])
        print(f"{name} {key}: gpu-vs-oracle32 {e:.2e}")
        assert e < TOL, (key, e)
