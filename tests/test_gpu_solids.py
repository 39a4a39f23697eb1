"""GPU parity of the solid paths against the CPU oracle: self-contact,
Johnson-Cook plastic flow, Seth-Hill strain orders 0 (log series), 1
(Denman-Beavers square root) and 2, and 2D solids.  Each case starts from a
deformed state set through the C ABI (and the same state in the oracle)."""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from arphys.abi import PARTICLE_DTYPE
from oracle.oracle import Oracle
from helpers import rel_err, gpu_state

pytestmark = pytest.mark.gpu


def solid_block_scene(n=(6, 6, 6), spacing=0.01, dim=3, lam=-2e5, mu=-1e5, order=2, plastic=None, damp=(0.0, 0.0),
                      integrator="midpoint", dt=1e-5):
    s = spacing
    counts = n[:dim]
    ref = scenes.lattice(tuple(0.2 + 0.5 * s for _ in range(dim)), counts, s)
    mats = np.array([scenes.elastic_solid(1000.0, lam, mu, mass=1000.0 * s ** dim, strain_order=order,
                                          normal_damp=damp[0], shear_damp=damp[1], plastic=plastic)])
    p = scenes.particles(ref, 0, 1000.0)
    box = tuple([1.0] * dim + [0.0] * (4 - dim))
    return scenes.Scene(particles=p, boundary=np.zeros(0, PARTICLE_DTYPE), materials=mats,
                        bounds_min=(0.0, 0.0, 0.0, 0.0), bounds_dim=box, h=2 * s, integrator=integrator, dt=dt,
                        gravity=9.81, name=f"block{dim}d_order{order}")


def deform(p, dim, rng, stretch=1.03, shear=0.02, noise=2e-4):
    q = p.copy()
    x = q["pos"][:, :dim].astype(np.float64)
    c = x.mean(axis=0)
    y = c + (x - c) * stretch
    y[:, 0] += shear * (x[:, 1] - c[1])
    y += rng.uniform(-noise, noise, size=y.shape)
    q["pos"][:, :dim] = y
    return q


def run_both(sc, state, steps):
    sim = FluidSim(sc)
    sim.init()
    sim.set_particles(state)
    o32, o64 = Oracle(sc, 32), Oracle(sc, 64)
    for o in (o32, o64):
        o.set_state(den=state["den"], pos=state["pos"], vel=state["vel"])
    sim.step(steps)
    o32.step(steps)
    o64.step(steps)
    return sim, gpu_state(sim), o32.state(), o64.state()


def compare(name, g, r, r64, tol):
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r[key])
        print(f"{name} {key}: gpu-vs-oracle32 {e:.2e}  gpu-vs-fp64 {rel_err(g[key], r64[key]):.2e}  "
              f"oracle32-vs-fp64 {rel_err(r[key], r64[key]):.2e}")
        assert e < tol, (key, e)


@pytest.mark.parametrize("order", [2, 0, 1])
@pytest.mark.parametrize("dim", [2, 3])
def test_strain_orders_match_oracle(order, dim):
    n = (10, 8, 1) if dim == 2 else (6, 6, 6)
    sc = solid_block_scene(n=n, dim=dim, order=order, damp=(-50.0, -20.0))
    rng = np.random.default_rng(10 + order + dim)
    state = deform(sc.particles, dim, rng)
    _, g, r, r64 = run_both(sc, state, 20)
    compare(f"order{order}_{dim}d", g, r, r64, 2e-5)


def test_plastic_flow_matches_oracle():
    """metal_bar.toml-like material driven past its yield strength."""
    plastic = dict(yield_strength=5e5, work_hardening=1e5, work_hardening_exp=2.0, relaxation_time=1e3)
    sc = solid_block_scene(n=(12, 4, 1), dim=2, lam=-1e7, mu=-1e8, plastic=plastic, damp=(-500.0, -100.0),
                           dt=1e-7)
    rng = np.random.default_rng(7)
    state = deform(sc.particles, 2, rng, stretch=1.05, shear=0.05)
    sim, g, r, r64 = run_both(sc, state, 20)
    compare("plastic_2d", g, r, r64, 2e-5)
    pg = sim.solids()["stress"].astype(np.float64)
    o = Oracle(sc, 32)
    o.set_state(den=state["den"], pos=state["pos"], vel=state["vel"])
    o.step(20)
    po = o.state()["plastic"]
    assert np.abs(po).max() > 0, "the scene must actually yield"
    e = rel_err(pg, po)
    print(f"plastic strain rel err {e:.2e}")
    assert e < 1e-4


def test_self_contact_matches_oracle():
    """Two blocks of one material whose reference positions are far apart
    but whose current positions touch: the self-contact term is active."""
    s = 0.01
    # lattices sit half a spacing off the cell faces: the contact and
    # hourglass terms depend on which cells a particle is in, so a particle on
    # a face would make the result hinge on the last bit of its coordinate
    a = scenes.lattice((0.205, 0.205, 0.205), (4, 4, 4), s)
    b = scenes.lattice((0.205 + 20 * 2 * s, 0.205, 0.205), (4, 4, 4), s)
    mats = np.array([scenes.elastic_solid(1000.0, -2e5, -1e5, mass=1000.0 * s ** 3)])
    p = scenes.particles(np.concatenate([a, b]), 0, 1000.0)
    sc = scenes.Scene(particles=p, boundary=np.zeros(0, PARTICLE_DTYPE), materials=mats,
                      bounds_min=(0.0, 0.0, 0.0, 0.0), bounds_dim=(1.0, 1.0, 1.0, 0.0), h=2 * s,
                      integrator="midpoint", dt=1e-4, gravity=0.0, name="self_contact")
    state = p.copy()
    state["pos"][64:, 0] -= 20 * 2 * s - 4 * s - 0.5 * 2 * s  # block b now h/2 to the right of block a
    sim, g, r, r64 = run_both(sc, state, 20)
    moved = np.abs(r["vel"][:, 0]).max()
    assert moved > 1e-4, "contact must push the blocks"
    compare("self_contact", g, r, r64, 2e-5)
