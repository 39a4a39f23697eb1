"""Reverse mode (arp_tape_*) against central finite differences of the FP64
oracle.

The gradient of a loss after N steps with respect to the per-solid stiffness
and the initial velocities, taken by the GPU's hand-written stage adjoints
with checkpoints, must match (L(p + e d) - L(p - e d)) / 2e computed with the
double-precision oracle along seeded random directions d.  The FP32 forward
differs from the FP64 one by ~1e-6 relative, which bounds the agreement; the
bound used here is written in each test.
"""
import os

import numpy as np
import pytest

from arphys import FluidSim, scenes
from helpers import oracle_losses

pytestmark = pytest.mark.gpu


def state_grad(n, gpos):
    g = np.zeros((n, 8), np.float32)
    g[:, :3] = gpos
    return g


def gpu_gradients(sc, steps, every, loss, start=None):
    """Loss, dL/d(initial state) (n x 8) and dL/d(per-solid stiffness) (ns x 2)
    from the GPU tape."""
    stiff = sc.meta.get("stiffness")
    sim = FluidSim(sc)
    sim.init()
    if start is not None:
        sim.set_particles(start)
    if stiff is not None:
        sim.set_solid_stiffness(stiff)
    sim.tape_begin(every)
    sim.step(steps)
    before = sim.particles().copy()
    pos = sim.particles()["pos"][:, :3].astype(np.float64)
    gx = np.zeros((sc.n, 3))
    if loss[0] == "tip":
        d = pos[loss[1]].mean(axis=0) - np.asarray(loss[2], np.float64)
        L = float(d @ d)
        gx[loss[1]] = 2.0 * d / len(loss[1])
    else:
        d = pos - loss[1]
        L = float(np.sum(d * d))
        gx = 2.0 * d
    g0, gs = sim.backward(state_grad(sc.n, gx))
    after = sim.particles()
    assert before.tobytes() == after.tobytes()  # the forward state is put back
    sim.tape_end()
    return L, g0, gs


def retimed(sc, toward):
    """The scene with its float32 time step moved by one ulp: every product
    with dt, and so every rounding of the float32 trajectory, changes, while
    the problem itself moves by 6e-8 relative.  The spread between the GPU
    gradients of the two problems measures the FP32 noise of the gradient."""
    dt = np.nextafter(np.float32(sc.dt), np.float32(toward))
    return scenes.Scene(**{**sc.__dict__, "dt": float(dt)})


def fd_check(sc, steps, every, loss, directions_stiff, directions_vel, eps_rel=1e-4, eps_vel=1e-4, start=None):
    """The GPU gradient along each direction, the same for the problem with
    its time step one float32 ulp either way (the FP32 noise of the gradient
    itself), and the FP64 oracle's central difference (L(p + e d) - L(p - e d)) / 2e along the same
    direction.  `loss` is ("tip", ids, target) or ("points", targets); `start`
    (particle records) replaces the scene's initial state after creation,
    keeping the scene's positions as the solids' reference configuration."""
    stiff = sc.meta.get("stiffness")
    L, g0, gs = gpu_gradients(sc, steps, every, loss, start)
    spread = [gpu_gradients(retimed(sc, t), steps, every, loss, start)[1:] for t in (np.inf, -np.inf)]
    p0 = sc.particles if start is None else start
    v0 = p0["vel"][:, :3].astype(np.float64)
    x0 = None if start is None else start["pos"].astype(np.float64)
    s64 = None if stiff is None else stiff.astype(np.float64)
    tasks, adj, nudged = [], [], []
    for d in directions_stiff:
        a0 = float(np.sum(gs.astype(np.float64) * s64 * d[:, None]))
        adj.append(("stiffness", a0))
        nudged.append([a0 - float(np.sum(g[1].astype(np.float64) * s64 * d[:, None])) for g in spread])
        tasks += [(sc, steps, s64 * (1 + eps_rel * d[:, None]), v0, loss, x0),
                  (sc, steps, s64 * (1 - eps_rel * d[:, None]), v0, loss, x0)]
    for d in directions_vel:
        a0 = float(np.sum(g0[:, 4:7].astype(np.float64) * d))
        adj.append(("velocity", a0))
        nudged.append([a0 - float(np.sum(g[0][:, 4:7].astype(np.float64) * d)) for g in spread])
        tasks += [(sc, steps, s64, v0 + eps_vel * d, loss, x0), (sc, steps, s64, v0 - eps_vel * d, loss, x0)]
    ls = oracle_losses(tasks)
    out = []
    for q, (kind, a) in enumerate(adj):
        e = eps_rel if kind == "stiffness" else eps_vel
        out.append((kind, a, (ls[2 * q] - ls[2 * q + 1]) / (2 * e), nudged[q]))
    return L, out


def report(res, tol):
    """Per direction: the relative error |adj - fd| / |fd| against FP64 finite
    differences, and whether it is within `tol` or else within the FP32 noise
    of the gradient itself.  The noise is measured: the time step moved by
    one float32 ulp either way rounds every step of the float32 trajectory
    differently while leaving the problem the same to 6e-8; with sigma the RMS
    of the two gradients' differences from this one over all directions of a
    kind divided by sqrt 2 (each difference holds two independent roundings),
    a direction passes within 4 sigma.  The forward runs in float32, as the
    reference's shaders do: where a derivative is small against the
    gradient's size (random directions cancel) or is carried by small strains
    (float positions of order 1 m resolve them to ~1e-7), that noise exceeds
    tol of the derivative.  Returns the number of directions meeting neither
    bound."""
    bad = 0
    for kind in ("stiffness", "velocity"):
        rows = [(a, f, sp) for k, a, f, sp in res if k == kind]
        if not rows:
            continue
        sigma = float(np.sqrt(np.mean([x * x for _, _, sp in rows for x in sp]) / 2.0))
        errs = [abs(a - f) / max(abs(f), 1e-300) for a, f, _ in rows]
        mags = [abs(f) for _, f, _ in rows]
        within = sum(1 for e in errs if e < tol)
        noise_ok = sum(1 for (a, f, _), e in zip(rows, errs) if e >= tol and abs(a - f) <= 4.0 * sigma)
        fails = len(rows) - within - noise_ok
        na = np.array([a for a, _, _ in rows])
        nf = np.array([f for _, f, _ in rows])
        print(f"{kind}: {len(rows)} directions, |fd| {min(mags):.3e} .. {max(mags):.3e}, rel err median "
              f"{np.median(errs):.2e} max {max(errs):.2e}, norm-wise {np.linalg.norm(na - nf) / np.linalg.norm(nf):.2e}; "
              f"FP32 noise sigma {sigma:.2e}; {within} within {tol:.0e}, {noise_ok} within 4 sigma, {fails} neither")
        for (a, f, _), e in zip(rows, errs):
            if e >= tol:
                print(f"  adjoint {a:.6e} fd64 {f:.6e} rel err {e:.2e} |adj - fd| {abs(a - f):.2e} "
                      f"= {abs(a - f) / sigma:.1f} sigma")
        bad += fails
    return bad


def test_cantilever_bar_gradients_match_fp64_finite_differences():
    """The differentiation workload's bar at reduced size (4 x 32 x 4 sites,
    clamped base, lognormal E, gravity, RK2, checkpoints every 20) from a seeded
    random initial velocity field: the gradients of the tip-centroid loss with
    respect to the per-particle stiffness and the initial velocities along 32
    seeded directions each agree with FP64 central differences within 1e-4."""
    sc = scenes.cantilever_bar(n=(4, 32, 4), v_sigma=0.05, target_offset=(0.002, -0.02, 0.001))
    rng = np.random.default_rng(44)
    ds = [rng.normal(size=sc.n) for _ in range(32)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(32)]
    L, res = fd_check(sc, 200, 20, ("tip", sc.meta["tip"], sc.meta["target"]), ds, dv)
    assert report(res, 1e-4) == 0


def test_fluid_gradients_match_fp64_finite_differences():
    sc = scenes.dam_break_2d(nx=12, ny=12, box=(0.32, 0.24), integrator="midpoint")
    rng = np.random.default_rng(7)
    sc.particles["vel"][:, :2] = rng.normal(0.0, 0.2, size=(sc.n, 2)).astype(np.float32)
    target = (sc.particles["pos"][:, :3] + rng.normal(0.0, 0.002, size=(sc.n, 3))).astype(np.float64)
    target[:, 2] = 0.0
    dv = []
    for _ in range(32):
        d = rng.normal(size=(sc.n, 3))
        d[:, 2] = 0.0
        dv.append(d)
    L, res = fd_check(sc, 20, 5, ("points", target), [], dv)
    assert report(res, 1e-4) == 0


def sliding_block(friction=0.1, vx=0.5):
    """A 2D fluid block sliding along the floor of the dam-break box, away from
    the walls, with a friction coefficient on the wall material (the
    interaction of default_between carries the materials' visc sum,
    interaction.rs:42-50).  Its tangential velocity against the floor stays
    far from zero, where Coulomb friction switches direction and the loss
    would not be differentiable."""
    sc = scenes.dam_break_2d(nx=12, ny=6, box=(0.64, 0.24), integrator="midpoint")
    sc.materials["visc"][0] = friction
    sc.particles["pos"][:, 0] += np.float32(0.2)
    rng = np.random.default_rng(9)
    sc.particles["vel"][:, 0] = np.float32(vx) + rng.normal(0.0, 0.05, size=sc.n).astype(np.float32)
    sc.particles["vel"][:, 1] = rng.normal(0.0, 0.05, size=sc.n).astype(np.float32)
    return sc, rng


def test_friction_scene_matches_the_oracle():
    from helpers import rel_err
    from oracle.oracle import Oracle
    sc, _ = sliding_block(friction=5.0, vx=1.0)
    sim = FluidSim(sc)
    sim.init()
    sim.step(20)
    o = Oracle(sc, 32)
    o.step(20)
    g, r = sim.particles(), o.state()
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r[key])
        print(f"sliding block {key}: {e:.2e}")
        assert e < 1e-5, key


def test_friction_gradients_match_fp64_finite_differences():
    """The friction term of fluid.rs:192-199 differentiated with the rest of
    the fluid pair terms.  Friction moves this loss's derivatives by ~0.6 %,
    so besides the whole gradient the friction part alone (the gradient with
    friction minus the one without) is checked against the same difference
    of FP64 finite differences."""
    res = {}
    for mu in (5.0, 0.0):
        sc, rng = sliding_block(friction=mu, vx=1.0)
        target = (sc.particles["pos"][:, :3] + rng.normal(0.0, 0.002, size=(sc.n, 3))).astype(np.float64)
        target[:, 2] = 0.0
        dv = []
        for _ in range(16):
            d = rng.normal(size=(sc.n, 3))
            d[:, 2] = 0.0
            dv.append(d)
        L, res[mu] = fd_check(sc, 20, 5, ("points", target), [], dv)
    bad = report(res[5.0], 1e-4)
    sig = [float(np.sqrt(np.mean([x * x for r in res[m] for x in r[3]]) / 2.0)) for m in (5.0, 0.0)]
    for (_, a1, f1, _), (_, a0, f0, _) in zip(res[5.0], res[0.0]):
        da, df = a1 - a0, f1 - f0
        err = abs(da - df) / abs(df)
        print(f"friction part: adjoint {da:.6e} fd64 {df:.6e} rel err {err:.2e}")
        assert err < 1e-2 or abs(da - df) <= 4.0 * (sig[0] + sig[1])
    assert bad == 0


@pytest.mark.parametrize("order", [0, 1, -2, 3])
def test_strain_order_gradients_match_fp64_finite_differences(order):
    """Seth-Hill strains other than Green-Lagrange (solid.rs:105-204): the
    5-term log series (order 0), the Denman-Beavers square root (odd orders,
    differentiated through the Sylvester equation of the square root) and
    inverses (negative orders), with their strain rates."""
    sc = scenes.cantilever_bar(n=(4, 16, 4), v_sigma=0.1, target_offset=(0.002, -0.02, 0.001))
    sc.materials["strain_order"][1] = order
    rng = np.random.default_rng(60 + order)
    ds = [rng.normal(size=sc.n) for _ in range(8)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(8)]
    L, res = fd_check(sc, 100, 20, ("tip", sc.meta["tip"], sc.meta["target"]), ds, dv)
    assert report(res, 1e-4) == 0


def test_plastic_flow_gradients_match_fp64_finite_differences():
    """The bar of the differentiation workload, plastic: yield strength 100,
    relaxation time 1e4 (solid.rs:499-517), so the random initial velocities
    drive every particle past the yield surface and the plastic strain grows to
    ~3e-3.  The plastic strain enters the stress and its own rate, both
    differentiated, with the plastic strain's adjoint carried across stages,
    steps and checkpoints."""
    sc = scenes.cantilever_bar(n=(4, 16, 4), v_sigma=0.1, target_offset=(0.002, -0.02, 0.001))
    sc.materials["plastic"][1] = 1
    sc.materials["yield_strength"][1] = 100.0
    sc.materials["relaxation_time"][1] = 1e4
    sc.materials["work_hardening"][1] = 0.0
    sc.materials["work_hardening_exp"][1] = 2.0
    rng = np.random.default_rng(70)
    ds = [rng.normal(size=sc.n) for _ in range(16)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(16)]
    L, res = fd_check(sc, 100, 20, ("tip", sc.meta["tip"], sc.meta["target"]), ds, dv)
    assert report(res, 1e-4) == 0


def test_backward_without_tape_is_refused():
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


@pytest.mark.slow
@pytest.mark.skipif(not os.environ.get("ARP_SLOW_TESTS"), reason="full-size FP64 differences: set ARP_SLOW_TESTS=1")
def test_differentiation_workload_full_size_gradients_match_fp64_finite_differences():
    """The differentiation workload at its full size (16 x 16 x 256 bar, 65,024
    elastic particles, seeded initial velocities) over 20 RK2 steps (a
    reduced-step horizon: each FP64 oracle run of the full 400 steps takes
    minutes on one core), 4 seeded directions each for the per-particle
    stiffness and the initial velocities, within 1e-4."""
    sc = scenes.cantilever_bar(v_sigma=0.05)
    rng = np.random.default_rng(404)
    ds = [rng.normal(size=sc.n) for _ in range(4)]
    dv = [rng.normal(size=(sc.n, 3)) for _ in range(4)]
    L, res = fd_check(sc, 20, 20, ("tip", sc.meta["tip"], sc.meta["target"]), ds, dv)
    assert report(res, 1e-4) == 0
