"""Reverse mode (arp_tape_*) against central finite differences of the FP64
oracle.

The gradient of a loss after N steps with respect to the per-solid stiffness
and the initial velocities, taken by the GPU's hand-written stage adjoints
with checkpoints, must match (L(p + e d) - L(p - e d)) / 2e computed with the
double-precision oracle along seeded random directions d.  The FP32 forward
differs from the FP64 one by ~1e-6 relative, which bounds the agreement; the
bound used here is written in each test.
"""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def state_grad(n, gpos):
    g = np.zeros((n, 8), np.float32)
    g[:, :3] = gpos
    return g


def oracle_loss(sc, steps, stiff=None, vel=None, loss=None):
    sc2 = scenes.Scene(**{**sc.__dict__, "particles": sc.particles.copy()})
    if vel is not None:
        sc2.particles["vel"][:, :3] = vel
    o = Oracle(sc2, 64)
    if stiff is not None:
        o.set_solid_stiffness(stiff)
    o.step(steps)
    return loss(o.state()["pos"])


def fd_check(sc, steps, every, loss, directions_stiff, directions_vel, eps_rel=1e-4):
    stiff = sc.meta.get("stiffness")
    sim = FluidSim(sc)
    sim.init()
    if stiff is not None:
        sim.set_solid_stiffness(stiff)
    sim.tape_begin(every)
    sim.step(steps)
    before = sim.particles().copy()
    L, gx = loss(sim.particles()["pos"], True)
    g0, gs = sim.backward(state_grad(sc.n, gx))
    after = sim.particles()
    assert before.tobytes() == after.tobytes()  # the forward state is put back
    out = []
    v0 = sc.particles["vel"][:, :3].astype(np.float64)
    for d in directions_stiff:
        adj = float(np.sum(gs.astype(np.float64) * stiff.astype(np.float64) * d[:, None]))
        e = eps_rel
        lp = oracle_loss(sc, steps, stiff=stiff.astype(np.float64) * (1 + e * d[:, None]), loss=loss)
        lm = oracle_loss(sc, steps, stiff=stiff.astype(np.float64) * (1 - e * d[:, None]), loss=loss)
        out.append(("stiffness", adj, (lp - lm) / (2 * e)))
    for d in directions_vel:
        adj = float(np.sum(g0[:, 4:7].astype(np.float64) * d))
        e = eps_rel
        lp = oracle_loss(sc, steps, stiff=None if stiff is None else stiff.astype(np.float64), vel=v0 + e * d,
                         loss=loss)
        lm = oracle_loss(sc, steps, stiff=None if stiff is None else stiff.astype(np.float64), vel=v0 - e * d,
                         loss=loss)
        out.append(("velocity", adj, (lp - lm) / (2 * e)))
    sim.tape_end()
    return L, out


def test_cantilever_bar_gradients_match_fp64_finite_differences():
    sc = scenes.cantilever_bar(n=(4, 16, 4), v_sigma=0.2, target_offset=(0.002, -0.02, 0.001))
    tip, target = sc.meta["tip"], sc.meta["target"]

    def loss(pos, want_grad=False):
        L, g = scenes.tip_loss(pos, tip, target)
        return (L, g) if want_grad else L

    rng = np.random.default_rng(44)
    ds = [rng.normal(size=sc.n) for _ in range(3)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(3)]
    L, res = fd_check(sc, 200, 20, loss, ds, dv)
    for kind, adj, fd in res:
        err = abs(adj - fd) / max(abs(fd), 1e-30)
        print(f"{kind}: adjoint {adj:.6e} fd64 {fd:.6e} rel err {err:.2e}")
        assert err < 2e-3, (kind, adj, fd)


def test_fluid_gradients_match_fp64_finite_differences():
    sc = scenes.dam_break_2d(nx=12, ny=12, box=(0.32, 0.24), integrator="midpoint")
    rng = np.random.default_rng(7)
    sc.particles["vel"][:, :2] = rng.normal(0.0, 0.2, size=(sc.n, 2)).astype(np.float32)
    target = (sc.particles["pos"][:, :3] + rng.normal(0.0, 0.002, size=(sc.n, 3))).astype(np.float64)
    target[:, 2] = 0.0

    def loss(pos, want_grad=False):
        d = pos[:, :3].astype(np.float64) - target
        L = float(np.sum(d * d))
        return (L, 2.0 * d) if want_grad else L

    dv = []
    for _ in range(3):
        d = rng.normal(size=(sc.n, 3))
        d[:, 2] = 0.0
        dv.append(d)
    L, res = fd_check(sc, 20, 5, loss, [], dv)
    for kind, adj, fd in res:
        err = abs(adj - fd) / max(abs(fd), 1e-30)
        print(f"{kind}: adjoint {adj:.6e} fd64 {fd:.6e} rel err {err:.2e}")
        assert err < 2e-3, (kind, adj, fd)


def test_tape_refuses_plastic_materials_and_backward_without_tape():
    sc = scenes.cantilever_bar(n=(4, 8, 4))
    sc.materials["plastic"][1] = 1
    sc.materials["yield_strength"][1] = 1.0
    sim = FluidSim(sc)
    sim.init()
    with pytest.raises(Exception) as e:
        sim.tape_begin(4)
    assert e.value.code == 6
    sc = scenes.cantilever_bar(n=(4, 8, 4))
    sim = FluidSim(sc)
    sim.init()
    with pytest.raises(Exception) as e:
        sim.backward(np.zeros((sim.n, 8), np.float32))
    assert e.value.code == 1


def test_batched_gradients_equal_per_scene_gradients():
    """One backward pass over a batch of Rayleigh-Taylor scenes gives each
    scene the gradient its own handle gives."""
    scs = scenes.rayleigh_taylor_batch(count=3, n_min=400, n_max=900, seed=11)
    rng = np.random.default_rng(3)
    for sc in scs:
        sc.particles["vel"][:, :2] = rng.normal(0.0, 0.1, size=(sc.n, 2)).astype(np.float32)
    grads = []
    for sc in scs:
        sim = FluidSim(sc)
        sim.init()
        sim.tape_begin(5)
        sim.step(15)
        _, gx = scenes.separation(sim.particles()["pos"], sc.meta["heavy"])
        g0, _ = sim.backward(state_grad(sc.n, gx))
        grads.append(g0)
    batch = FluidSim.batch(scs)
    batch.init()
    batch.tape_begin(5)
    batch.step(15)
    pos = batch.particles()["pos"]
    off = np.cumsum([0] + [sc.n for sc in scs])
    gx = np.concatenate([scenes.separation(pos[off[k]:off[k + 1]], sc.meta["heavy"])[1]
                         for k, sc in enumerate(scs)])
    gb, _ = batch.backward(state_grad(int(off[-1]), gx))
    for k, g in enumerate(grads):
        part = gb[off[k]:off[k + 1]]
        err = np.abs(part - g).max() / np.abs(g).max()
        print(f"scene {k}: batch vs single max rel diff {err:.2e}")
        assert err < 1e-5
