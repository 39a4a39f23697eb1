"""CPU tests of the oracle (the CPU restatement of the reference shaders).

The reference ships no golden vectors, so the oracle is pinned by analytic
known-answer tests: kernel normalisation and gradient, the correction matrix
identity on a lattice, the sign of the elastic force on a stretched bar,
momentum balance of the pair terms, brute-force neighbor sets, and exact
integration of free fall by the Runge-Kutta tableaus, the order of
accuracy of every integrator on a smooth two-particle collision, and the
symmetries of the step (translation, Galilean boost, rotation) on a scene of
fluid, an elastic block and a wall.
"""
import numpy as np
import pytest

from arphys import scenes
from arphys.abi import INVALID, PARTICLE_DTYPE, MATERIAL_DTYPE
from oracle.oracle import Oracle, poly6, norm_const_f32


@pytest.mark.parametrize("dim", [2, 3])
def test_poly6_integrates_to_one(dim):
    h = 0.02
    m = 80 if dim == 3 else 400
    ax = (np.arange(m) + 0.5) / m * 2 * h - h
    grids = np.meshgrid(*([ax] * dim), indexing="ij")
    r = np.zeros((ax.size ** dim, 4))
    for a in range(dim):
        r[:, a] = grids[a].reshape(-1)
    w, _, _ = poly6(dim, h, r)
    cell = (2 * h / m) ** dim
    assert abs(w.sum() * cell - 1.0) < 2e-3


def test_poly6_gradient_matches_finite_difference():
    h = 0.02
    rng = np.random.default_rng(0)
    r = np.zeros((50, 4))
    r[:, :3] = rng.uniform(-0.6 * h, 0.6 * h, size=(50, 3))
    _, gw, _ = poly6(3, h, r)
    eps = 1e-7
    for a in range(3):
        rp, rm = r.copy(), r.copy()
        rp[:, a] += eps
        rm[:, a] -= eps
        fd = (poly6(3, h, rp)[0] - poly6(3, h, rm)[0]) / (2 * eps)
        np.testing.assert_allclose(gw[:, a], fd, rtol=1e-5, atol=1e-3 * np.abs(gw).max())


def test_norm_const_matches_closed_form():
    # poly6: 4/(pi h^8) in 2D, 315/(64 pi h^9) in 3D
    h = 0.02
    assert abs(norm_const_f32(2, h) / (4 / (np.pi * h ** 8)) - 1) < 1e-6
    assert abs(norm_const_f32(3, h) / (315 / (64 * np.pi * h ** 9)) - 1) < 1e-6


def test_deformation_gradient_is_identity_in_reference_configuration():
    sc, _ = scenes.stretched_bar(n=(8, 6, 6))
    o = Oracle(sc, precision=64)
    st = o.strains()
    F = st[:, 1].reshape(-1, 4, 4)  # column-major per solid
    for i in range(len(F)):
        np.testing.assert_allclose(F[i][:3, :3], np.eye(3), atol=1e-9)


@pytest.mark.parametrize("sign", [-1.0, 1.0])
def test_stretched_bar_force_sign(sign):
    """With the reference's convention (r = X_j - X_i, negative-definite L),
    negative stiffness is restoring and positive stiffness is not."""
    sc, stretched = scenes.stretched_bar(n=(20, 4, 4), lam=sign * 1e5, mu=sign * 1e5)
    o = Oracle(sc, precision=64)
    pos = o.state()["pos"]
    pos[:, :3] = stretched
    o.set_state(pos=pos)
    acc = o.derivative()["vel"][:, 0]
    x = stretched[:, 0]
    right = x > x.max() - 1e-9
    left = x < x.min() + 1e-9
    restoring = acc[right].mean() < 0 and acc[left].mean() > 0
    assert restoring == (sign < 0)


def test_fluid_pair_terms_conserve_momentum():
    """sum_i rho_i (dv_i/dt + g) = sum of antisymmetric pair terms = 0 for a
    fluid without boundary."""
    sc = scenes.dam_break_2d(nx=24, ny=24, box=(0.64, 0.64), alpha=0.5, visc=0.01)
    sc.boundary = sc.boundary[:0]
    rng = np.random.default_rng(3)
    o = Oracle(sc, precision=64)
    st = o.state()
    vel = st["vel"].copy()
    vel[:, :2] = rng.normal(size=(len(vel), 2)) * 0.1
    den = st["den"] * (1 + 0.01 * rng.normal(size=len(vel)))
    o.set_state(den=den, vel=vel)
    d = o.derivative()
    a = d["vel"][:, :2].copy()
    a[:, 1] += float(np.float32(sc.gravity))
    tot = (den[:, None] * a).sum(axis=0)
    scale = np.abs(den[:, None] * a).sum(axis=0)
    assert np.all(np.abs(tot) <= 1e-9 * scale)


def test_neighbor_buckets_match_brute_force():
    sc = scenes.dam_break_2d(nx=20, ny=24, box=(0.4, 0.4))
    o = Oracle(sc)
    b = o.buckets()
    pos = sc.particles["pos"][:, :2].astype(np.float32)
    bpos = sc.boundary["pos"][:, :2].astype(np.float32)
    h2 = np.float32(sc.h) * np.float32(sc.h)
    allpos = np.concatenate([pos, bpos])
    d = allpos[None, :, :] - pos[:, None, :]
    r2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(np.float32)
    brute = (h2 - r2 > 0).sum(axis=1)
    np.testing.assert_array_equal(b["nbr_count"], brute)
    assert np.all(b["pos_index"] != INVALID)
    # every particle is listed exactly once in the position sections
    cnt = b["counts"][:, 2].sum()
    assert cnt == sc.n


@pytest.mark.parametrize("integ", ["euler", "midpoint", "heun2", "ralston", "rk3", "heun3", "rk4", "rk_3_8", "verlet"])
def test_free_fall_is_integrated_exactly(integ):
    """An isolated particle feels only gravity; any consistent tableau
    integrates x(t) = x0 + v0 t - g t^2 / 2 exactly for order >= 2."""
    mats = np.array([scenes.liquid(1000.0, 20.0, 0.02, 0.0, mass=0.1)])
    p = np.zeros(1, dtype=PARTICLE_DTYPE)
    p["den"] = 1000.0
    p["mat"] = 0
    p["pos"][0, :2] = (0.5, 0.5)
    p["vel"][0, :2] = (0.3, 1.0)
    sc = scenes.Scene(particles=p, boundary=np.zeros(0, PARTICLE_DTYPE), materials=mats,
                      bounds_min=(0, 0, 0, 0), bounds_dim=(1, 1, 0, 0), h=0.02, integrator=integ, dt=1e-3,
                      gravity=9.81)
    o = Oracle(sc, precision=64)
    o.step(10)
    dt = float(np.float32(1e-3))
    t = 10 * dt
    assert abs(o.time - t) < 1e-8
    s = o.state()
    g = float(np.float32(9.81))
    if integ == "euler":
        y = 0.5 + 1.0 * t - g * dt * dt * 10 * 9 / 2  # sum of v_k dt
    else:
        y = 0.5 + 1.0 * t - g * t * t / 2
    assert abs(s["pos"][0, 1] - y) < 1e-9
    assert abs(s["vel"][0, 1] - (1.0 - g * t)) < 1e-9
    assert abs(s["pos"][0, 0] - (0.5 + 0.3 * t)) < 1e-9


def test_float_and_double_oracles_agree_over_steps():
    sc = scenes.dam_break_2d(nx=24, ny=24, box=(0.48, 0.48))
    a, b = Oracle(sc, 32), Oracle(sc, 64)
    a.step(20)
    b.step(20)
    sa, sb = a.state(), b.state()
    assert np.abs(sa["pos"] - sb["pos"]).max() < 1e-6
    assert np.abs(sa["den"] - sb["den"]).max() / 1000 < 1e-5


def test_literal_and_cutoff_evaluations_agree():
    sc = scenes.small_fluid_bar_3d()
    a, b = Oracle(sc, 32), Oracle(sc, 32, literal=True)
    a.step(2)
    b.step(2)
    sa, sb = a.state(), b.state()
    for k in ("pos", "vel", "den", "plastic"):
        np.testing.assert_array_equal(sa[k], sb[k])


def test_solid_scene_runs_and_stays_finite():
    sc = scenes.small_fluid_bar_3d()
    o = Oracle(sc)
    assert o.ns == sc.n_solids() > 1
    o.step(5)
    s = o.state()
    assert np.isfinite(s["pos"]).all() and np.isfinite(s["vel"]).all()


def test_batched_workload_layout():
    """The 256 batched scenes: total counts within 10% of their log-uniform
    targets in [2048, 65536], no two blocks within kernel range of one
    another (particles of one block closer than one spacing to another's, or
    different materials within h, start the step on overlapping bodies), and
    every body inside its scene's box."""
    from scipy.spatial import cKDTree
    scs = scenes.batched_scenes()
    assert len(scs) == 256
    for sc in scs:
        total = sc.n + len(sc.boundary)
        assert abs(total / sc.meta["n_target"] - 1.0) < 0.1, (sc.name, total, sc.meta["n_target"])
        p = sc.particles["pos"][:, :3].astype(np.float64)
        d, _ = cKDTree(p).query(p, k=2)
        assert d[:, 1].min() > 0.5 * 0.01, sc.name
        m = sc.particles["mat"]
        for a in np.unique(m):
            other = p[m != a]
            if len(other):
                dd, _ = cKDTree(other).query(p[m == a], k=1)
                assert dd.min() > sc.h, sc.name
        lo = np.asarray(sc.bounds_min[:3])
        assert (p > lo).all() and (p < lo + np.asarray(sc.bounds_dim[:3])).all(), sc.name


def test_batched_workload_sample_stays_in_its_box_for_200_steps():
    """The oracle runs the three smallest batched scenes with an elastic
    block for the workload's 200 RK2 steps: every state finite and inside
    the scene's box."""
    scs = scenes.batched_scenes()
    solid = [sc for sc in scs if (sc.materials["normal_stiffness"] != 0).any()]
    for sc in sorted(solid, key=lambda sc: sc.n)[:3]:
        o = Oracle(sc)
        o.step(200)
        p = o.state()["pos"][:, :3]
        lo = np.asarray(sc.bounds_min[:3])
        assert np.isfinite(p).all(), sc.name
        assert ((p > lo) & (p < lo + np.asarray(sc.bounds_dim[:3]))).all(), sc.name


def _pair_collision(integ, n, horizon=2.0 ** -6):
    """Two fluid particles 0.5 h apart moving towards each other (pressure,
    continuity, viscosity and artificial viscosity all active, every pair term
    smooth while they stay inside h), stepped to `horizon` in n steps of a time
    step that float32 represents exactly, in the FP64 oracle; returns the
    final positions, velocities and densities."""
    mats = np.array([scenes.liquid(1000.0, 20.0, 0.02, 0.0, mass=0.1)])
    p = np.zeros(2, dtype=PARTICLE_DTYPE)
    p["den"] = 1000.0
    p["pos"][0, :2] = (0.49, 0.5)
    p["pos"][1, :2] = (0.5, 0.503)
    p["vel"][0, :2] = (0.3, 0.1)
    p["vel"][1, :2] = (-0.2, -0.05)
    sc = scenes.Scene(particles=p, boundary=np.zeros(0, PARTICLE_DTYPE), materials=mats,
                      bounds_min=(0, 0, 0, 0), bounds_dim=(1, 1, 0, 0), h=0.02, integrator=integ,
                      dt=horizon / n, gravity=0.0)
    o = Oracle(sc, precision=64)
    o.step(n)
    assert o.time == horizon
    s = o.state()
    return np.concatenate([s["pos"][:, :2].ravel(), s["vel"][:, :2].ravel(), s["den"]])


@pytest.fixture(scope="module")
def collision_reference():
    return _pair_collision("rk4", 4096)


@pytest.mark.parametrize("integ,order", [("euler", 1), ("midpoint", 2), ("heun2", 2), ("ralston", 2),
                                         ("rk3", 3), ("heun3", 3), ("rk4", 4), ("rk_3_8", 4)])
def test_runge_kutta_tableaus_converge_at_their_order(integ, order, collision_reference):
    """Halving the time step divides the error of an order-p tableau by 2^p:
    the restated tableaus are the textbook ones (the reference's integrator
    crate is not vendored)."""
    errs = [np.abs(_pair_collision(integ, n) - collision_reference).max() for n in (16, 32, 64)]
    observed = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(abs(o - order) < 0.25 for o in observed), (errs, observed)


def test_velocity_verlet_converges_at_first_order_on_sph_states(collision_reference):
    """Velocity Verlet kicks density like velocity, so the force evaluation
    after the drift sees a half-updated density (and the density rate a
    half-kicked velocity): on an SPH state the scheme converges at first
    order, positions included, not at the second order it has for forces of
    position alone."""
    errs = [np.abs(_pair_collision("verlet", n) - collision_reference).max() for n in (128, 256, 512)]
    observed = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(abs(o - 1.0) < 0.2 for o in observed), (errs, observed)


_Q = 2.0 ** -20  # positions and velocities on this grid shift and rotate exactly in float32


def _fluid_block_wall(gravity=9.81, walls=True, seed=7):
    """2D: a 10 x 10 jittered fluid block (Tait, viscosity, artificial
    viscosity), a 6 x 6 elastic block moving into it, seeded velocities, and a
    three-row wall with Coulomb friction 5 under both (friction acts on the
    pairs of the wall with the fluid and the solid), every coordinate a
    multiple of 2^-20."""
    rng = np.random.default_rng(seed)
    s, h = 0.01, 0.02

    def q(a):
        return np.round(a / _Q) * _Q
    fluid = q(scenes.jitter(scenes.lattice((0.105, 0.035), (10, 10), s), 1e-3, rng))
    solid = q(scenes.jitter(scenes.lattice((0.225, 0.035), (6, 6), s), 1e-3, rng))
    fv = q(rng.normal(0, 0.3, size=fluid.shape))
    sv = q(rng.normal(0, 0.3, size=solid.shape))
    sv[:, 0] -= 0.5
    lam, mu = scenes.lame_from_young(1e5, 0.3)
    mats = np.array([scenes.immobile(5.0, mass=s * s), scenes.liquid(1000.0, 20.0, h, 0.1, visc=1e-3, mass=0.1),
                     scenes.elastic_solid(1000.0, lam, mu, mass=0.1)])
    p = np.concatenate([scenes.particles(fluid, 1, 1000.0, fv), scenes.particles(solid, 2, 1000.0, sv)])
    wall = q(scenes.lattice((0.005, 0.005), (40, 3), s)) if walls else np.zeros((0, 2))
    return scenes.Scene(particles=p, boundary=scenes.particles(wall, 0, 1.0), materials=mats,
                        bounds_min=(0, 0, 0, 0), bounds_dim=(0.4, 0.3, 0, 0), h=h, integrator="rk2", dt=1e-4,
                        gravity=gravity, alpha=0.1)


def _run64(sc, steps=20):
    o = Oracle(sc, precision=64)
    o.step(steps)
    return o.state()


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_step_is_invariant_under_translation():
    """Moving every particle and the box by the same vector moves the result
    by it: the pair terms see only differences, and the grid moves along."""
    a = _fluid_block_wall()
    b = _fluid_block_wall()
    d = np.array([0.5, 0.25])
    b.particles["pos"][:, :2] += d
    b.boundary["pos"][:, :2] += d
    b.bounds_min = (0.5, 0.25, 0.0, 0.0)
    sa, sb = _run64(a), _run64(b)
    assert _rel(sb["pos"][:, :2] - d, sa["pos"][:, :2]) < 1e-13
    assert _rel(sb["vel"], sa["vel"]) < 1e-13
    assert _rel(sb["den"], sa["den"]) < 1e-13


def test_step_is_galilean_invariant_with_solids_drifting_at_twice_their_velocity():
    """Adding one velocity u to every particle (no walls: they would not move
    with it) leaves densities and relative velocities unchanged.  Fluid
    particles end u t further on, elastic ones 2 u t: the fluid and the solid
    derivative records both carry dx/dt = v and the two are summed (the
    reference's shaders/mod.rs:79 with fluid.rs:247 and solid.rs:494)."""
    a = _fluid_block_wall(walls=False)
    b = _fluid_block_wall(walls=False)
    u = np.array([0.25, -0.125])
    b.particles["vel"][:, :2] += u
    sa, sb = _run64(a, 20), _run64(b, 20)
    t = 20 * float(np.float32(1e-4))
    solid = (b.particles["mat"] == 2)[:, None]
    shift = np.where(solid, 2.0, 1.0) * u * t
    assert _rel(sb["pos"][:, :2] - shift, sa["pos"][:, :2]) < 1e-13
    assert _rel(sb["vel"][:, :2] - u, sa["vel"][:, :2]) < 1e-13
    assert _rel(sb["den"], sa["den"]) < 1e-13


def test_step_is_invariant_under_a_quarter_turn():
    """Without gravity, turning every position and velocity (and the box) by
    90 degrees turns the result: the pair terms and the solid's strain and
    stress are isotropic."""
    def turn(v):
        return np.stack([-v[:, 1], v[:, 0]], axis=1)
    a = _fluid_block_wall(gravity=0.0)
    b = _fluid_block_wall(gravity=0.0)
    for arr in (b.particles, b.boundary):
        arr["pos"][:, :2] = turn(arr["pos"][:, :2].astype(np.float64))
        arr["vel"][:, :2] = turn(arr["vel"][:, :2].astype(np.float64))
    b.bounds_min = (-0.3, 0.0, 0.0, 0.0)
    b.bounds_dim = (0.3, 0.4, 0.0, 0.0)
    sa, sb = _run64(a), _run64(b)
    assert _rel(sb["pos"][:, :2], turn(sa["pos"][:, :2])) < 1e-13
    assert _rel(sb["vel"][:, :2], turn(sa["vel"][:, :2])) < 1e-13
    assert _rel(sb["den"], sa["den"]) < 1e-13
    moved = np.abs(sa["pos"][:, :2] - a.particles["pos"][:, :2]).max()
    assert moved > 1e-3  # the scene does move over the 20 steps


@pytest.mark.parametrize("order,plastic", [(2, False), (0, False), (1, False), (-2, False), (3, False),
                                           (2, True)])
def test_3d_step_commutes_with_a_cyclic_permutation_of_the_axes(order, plastic):
    """3D, without gravity: relabelling the axes (x, y, z) -> (z, x, y) for
    every position, velocity and the box relabels the result; the fluid pair
    terms, the solid's Seth-Hill strain of each order (log series,
    Denman-Beavers square root, inverse) and Johnson-Cook plastic flow are
    isotropic."""
    rng = np.random.default_rng(9)
    s, h = 0.01, 0.02

    def q(a):
        return np.round(a / _Q) * _Q
    fluid = q(scenes.jitter(scenes.lattice((0.105, 0.035, 0.105), (6, 6, 6), s), 1e-3, rng))
    solid = q(scenes.jitter(scenes.lattice((0.185, 0.035, 0.105), (4, 4, 4), s), 1e-3, rng))
    fv = q(rng.normal(0, 0.3, size=fluid.shape))
    sv = q(rng.normal(0, 0.3, size=solid.shape))
    sv[:, 0] -= 0.5
    lam, mu = scenes.lame_from_young(1e5, 0.3)
    mats = np.array([scenes.immobile(0.0, mass=s ** 3), scenes.liquid(1000.0, 20.0, h, 0.1, visc=1e-3, mass=1e-3),
                     scenes.elastic_solid(1000.0, lam, mu, mass=1e-3, strain_order=order,
                                          plastic=dict(yield_strength=1e3, work_hardening=1e2, work_hardening_exp=2.0,
                                                       relaxation_time=1e3) if plastic else None)])
    wall = q(scenes.lattice((0.005, 0.005, 0.005), (30, 2, 30), s))

    def make():
        p = np.concatenate([scenes.particles(fluid, 1, 1000.0, fv), scenes.particles(solid, 2, 1000.0, sv)])
        return scenes.Scene(particles=p, boundary=scenes.particles(wall, 0, 1.0), materials=mats,
                            bounds_min=(0, 0, 0, 0), bounds_dim=(0.3, 0.2, 0.3, 0), h=h, integrator="rk2",
                            dt=1e-4, gravity=0.0, alpha=0.1)

    def cyc(v):
        return np.stack([v[:, 2], v[:, 0], v[:, 1]], axis=1)
    a, b = make(), make()
    for arr in (b.particles, b.boundary):
        arr["pos"][:, :3] = cyc(arr["pos"][:, :3].astype(np.float64))
        arr["vel"][:, :3] = cyc(arr["vel"][:, :3].astype(np.float64))
    b.bounds_dim = (0.3, 0.3, 0.2, 0.0)
    sa, sb = _run64(a), _run64(b)
    assert _rel(sb["pos"][:, :3], cyc(sa["pos"][:, :3])) < 1e-13
    assert _rel(sb["vel"][:, :3], cyc(sa["vel"][:, :3])) < 1e-13
    assert _rel(sb["den"], sa["den"]) < 1e-13
    solids = a.particles["mat"] == 2
    assert np.abs(sa["vel"][solids, :3] - a.particles["vel"][solids, :3]).max() > 1e-3  # the solid is loaded
    if plastic:
        assert np.abs(sa["plastic"]).max() > 0  # and yields
