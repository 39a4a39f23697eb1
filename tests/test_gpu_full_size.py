"""Parity at the sizes the benchmark configurations name.

  * the 3D fluid + clamped bar at 1,048,576 particles (the benchmarked
    workload): neighbor grid bit-exact against the oracle's serial
    fill_buckets (neighbor_list.rs:37-143), state within 1e-5 of the float
    oracle after 3 RK2 steps, with the FP64 error printed;
  * the 256 batched scenes (2,048-65,536 particles each) stepped as one batch,
    against the oracle for 3 steps and finite and inside their boxes over
    the workload's 200 steps;
  * eight full-size Rayleigh-Taylor scenes (the first eight of the 64 of the
    batched differentiation workload, 8,192-131,072 particles each): forward
    parity, the batch's gradient equal to each scene's own, and FP64 finite
    differences on the smallest scene.
The oracle runs on all host cores; each test takes seconds to a minute.
"""
import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle.oracle import Oracle
from helpers import gpu_state, oracle_csr, oracle_losses, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5


def check(name, g, r32, r64):
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r32[key])
        e64 = rel_err(g[key], r64[key])
        print(f"{name} {key}: vs f32 oracle {e:.2e}, vs f64 oracle {e64:.2e}")
        assert e < TOL, (name, key, e)


@pytest.fixture(scope="module")
def bar_1m():
    return scenes.fluid_bar_3d()


def test_benchmark_scene_grid_is_bit_exact_at_1m(bar_1m):
    sc = bar_1m
    assert sc.n + sc.nb == 1_048_576
    sim = FluidSim(sc)
    sim.init()
    o = Oracle(sc)
    b = o.buckets()
    sub, nc = sim.grid()
    np.testing.assert_array_equal(sub[:3], o.sub[:3])
    assert nc == o.ncells
    assert int(b["counts"].sum(axis=1).max()) <= 128  # no bucket of the reference would drop a particle
    g = sim.neighbors()
    start, members, bstart, bmembers = oracle_csr(b, sc.n, o.ncells)
    np.testing.assert_array_equal(g["cell_of"], b["pos_index"])
    np.testing.assert_array_equal(g["cell_start"], start)
    np.testing.assert_array_equal(g["members"], members)
    np.testing.assert_array_equal(g["nbr_count"], b["nbr_count"])
    gbs, gbm = sim.boundary_cells()
    np.testing.assert_array_equal(gbs, bstart)
    np.testing.assert_array_equal(gbm, bmembers)
    print(f"1M grid: {nc} cells, {int(b['nbr_count'].sum())} neighbor pairs within h")


def test_benchmark_scene_state_after_3_rk2_steps(bar_1m):
    sc = bar_1m
    sim = FluidSim(sc)
    sim.init()
    sim.set_graph(True)  # as the benchmark steps it
    sim.step(3)
    o32, o64 = Oracle(sc, 32), Oracle(sc, 64)
    o32.step(3)
    o64.step(3)
    check("fluid_bar_3d_1M", gpu_state(sim), o32.state(), o64.state())


def test_batched_workload_all_256_scenes_match_the_oracle():
    scs = scenes.batched_scenes()
    assert len(scs) == 256
    batch = FluidSim.batch(scs)
    batch.init()
    batch.set_graph(True)
    batch.step(3)
    pb = batch.particles()
    worst = {k: 0.0 for k in ("den", "pos", "vel")}
    for k, sc in enumerate(scs):
        first, n = batch.scene_range(k)[:2]
        o = Oracle(sc)
        o.step(3)
        r = o.state()
        for key in worst:
            e = rel_err(pb[key][first:first + n], r[key])
            worst[key] = max(worst[key], e)
            assert e < TOL, (k, key, e)
    print("256 scenes, worst per quantity:", {k: f"{v:.2e}" for k, v in worst.items()})


def test_batched_workload_stays_finite_and_in_its_boxes_over_200_steps():
    """The batched workload over its 200 steps, as the benchmark times it
    (one batch, graph replay): every scene finite and inside its box, so the
    timed steps are the physics the workload describes."""
    scs = scenes.batched_scenes()
    batch = FluidSim.batch(scs)
    batch.init()
    batch.set_graph(True)
    batch.step(200)
    pb = batch.particles()
    bad = []
    for k, sc in enumerate(scs):
        first, n = batch.scene_range(k)[:2]
        p = pb["pos"][first:first + n, :3].astype(np.float64)
        lo = np.asarray(sc.bounds_min[:3], np.float64)
        hi = lo + np.asarray(sc.bounds_dim[:3], np.float64)
        if not (np.isfinite(p).all() and (p > lo).all() and (p < hi).all()):
            bad.append(k)
    assert not bad, bad


@pytest.fixture(scope="module")
def rt8():
    scs = scenes.rayleigh_taylor_batch(count=8)
    full = scenes.rayleigh_taylor_batch()
    for a, b in zip(scs, full[:8]):  # the first eight scenes of the 64
        assert a.particles.tobytes() == b.particles.tobytes()
    return scs


def test_eight_full_size_rayleigh_taylor_scenes_match_the_oracle(rt8):
    batch = FluidSim.batch(rt8)
    batch.init()
    batch.step(10)
    pb = batch.particles()
    for k, sc in enumerate(rt8):
        first, n = batch.scene_range(k)[:2]
        o32, o64 = Oracle(sc, 32), Oracle(sc, 64)
        o32.step(10)
        o64.step(10)
        check(f"rayleigh_taylor_{k} ({sc.n})", {key: pb[key][first:first + n] for key in ("den", "pos", "vel")},
              o32.state(), o64.state())


def _sep_grad(scs, pos, offsets):
    g = np.zeros((len(pos), 8), np.float32)
    for k, sc in enumerate(scs):
        _, gk = scenes.separation(pos[offsets[k]:offsets[k + 1]], sc.meta["heavy"])
        g[offsets[k]:offsets[k + 1], :3] = gk
    return g


def test_eight_full_size_scenes_batch_gradient_equals_single(rt8):
    steps, every = 10, 5
    offsets = np.cumsum([0] + [sc.n for sc in rt8])
    batch = FluidSim.batch(rt8)
    batch.init()
    batch.tape_begin(every)
    batch.step(steps)
    gb, _ = batch.backward(_sep_grad(rt8, batch.particles()["pos"], offsets))
    for k, sc in enumerate(rt8):
        sim = FluidSim(sc)
        sim.init()
        sim.tape_begin(every)
        sim.step(steps)
        g0, _ = sim.backward(_sep_grad([sc], sim.particles()["pos"], [0, sc.n]))
        part = gb[offsets[k]:offsets[k + 1]]
        err = np.abs(part - g0).max() / np.abs(g0).max()
        print(f"rayleigh_taylor_{k}: batch vs single {err:.2e}")
        assert err < 1e-5


def test_full_size_rayleigh_taylor_gradient_matches_fp64_finite_differences(rt8):
    """The smallest of the eight scenes, 10 RK2 steps, 8 seeded directions of
    the initial velocity field, against FP64 central differences of the
    heavy/light centroid separation, within 1e-4."""
    sc = min(rt8, key=lambda s: s.n)
    rng = np.random.default_rng(55)
    sc.particles["vel"][:, :2] = rng.normal(0.0, 0.05, size=(sc.n, 2)).astype(np.float32)
    steps = 10
    sim = FluidSim(sc)
    sim.init()
    sim.tape_begin(5)
    sim.step(steps)
    g0, _ = sim.backward(_sep_grad([sc], sim.particles()["pos"], [0, sc.n]))
    sim.tape_end()
    v0 = sc.particles["vel"][:, :3].astype(np.float64)
    heavy = np.zeros(sc.n, bool)
    heavy[sc.meta["heavy"]] = True
    tasks, adj, eps = [], [], 1e-4
    for _ in range(8):
        d = rng.normal(size=(sc.n, 3))
        d[:, 2] = 0.0
        adj.append(float(np.sum(g0[:, 4:7].astype(np.float64) * d)))
        tasks += [(sc, steps, None, v0 + eps * d, ("separation", heavy)),
                  (sc, steps, None, v0 - eps * d, ("separation", heavy))]
    ls = oracle_losses(tasks)
    for q, a in enumerate(adj):
        fd = (ls[2 * q] - ls[2 * q + 1]) / (2 * eps)
        err = abs(a - fd) / abs(fd)
        print(f"direction {q}: adjoint {a:.6e} fd64 {fd:.6e} rel err {err:.2e}")
        assert err < 1e-4
