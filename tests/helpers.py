"""Shared comparison helpers for the parity tests."""
import numpy as np


def rel_err(a, b, scale=None):
    """max |a - b| / max |b| (or / scale), the norm-wise relative error."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def gpu_state(sim):
    p = sim.particles()
    return dict(den=p["den"].astype(np.float64), pos=p["pos"].astype(np.float64), vel=p["vel"].astype(np.float64))


def oracle_csr(buckets, n, ncells):
    """Mobile section of the oracle's buckets as CSR (cell_start, members) with
    members ascending inside each cell, plus the boundary section."""
    counts = buckets["counts"].astype(np.int64)
    contents = buckets["contents"]
    col = np.arange(contents.shape[1])[None, :]

    def section(lo, cnt):
        mask = (col >= lo[:, None]) & (col < (lo + cnt)[:, None])
        cell = np.broadcast_to(np.arange(len(counts))[:, None], mask.shape)[mask]
        vals = contents[mask]
        order = np.lexsort((vals, cell))  # by cell, ascending id inside a cell
        start = np.zeros(ncells + 1, np.int64)
        start[1:] = np.cumsum(cnt)
        return start, vals[order].astype(np.uint32)

    start, members = section(counts[:, 0] + counts[:, 1], counts[:, 2])
    bstart, bmembers = section(np.zeros(len(counts), np.int64), counts[:, 0])
    return start, members, bstart, bmembers


def load_seeded_scene(name):
    """A seeded scene fixture of tests/golden/scenes_seeded (written by
    tests/golden/make_scene_fixtures.py from the reference's example files)."""
    import os
    from arphys import scenes
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes_seeded", name + ".npz"))
    h, dt, g, alpha = (float(x) for x in z["scalars"])
    return scenes.Scene(particles=z["particles"], boundary=z["boundary"], materials=z["materials"],
                        bounds_min=tuple(float(x) for x in z["bounds_min"]),
                        bounds_dim=tuple(float(x) for x in z["bounds_dim"]), h=h, integrator=str(z["integrator"]),
                        dt=dt, subticks=int(z["subticks"]), gravity=g, alpha=alpha, interactions=z["interactions"],
                        interaction_given=z["interaction_given"], name=str(z["name"]))


def _oracle_loss(task):
    """One FP64 oracle run for a finite difference: the scene stepped `steps`
    times from the given per-solid stiffness and initial velocity (set in
    double precision, so a small perturbation is not rounded to f32), and the
    loss of the final positions: ("tip", caller ids, target) for the squared
    distance of their centroid to the target, ("separation", heavy mask) for
    the heavy/light centroid separation, ("points", targets) for the summed
    squared distances to per-particle targets."""
    sc, steps, stiff, vel, loss = task[:5]
    pos0 = task[5] if len(task) > 5 else None  # a starting state other than the scene's
    from oracle.oracle import Oracle, lib
    lib().orc_set_threads(1)
    o = Oracle(sc, 64)
    if stiff is not None:
        o.set_solid_stiffness(np.ascontiguousarray(stiff, np.float64))
    if pos0 is not None:
        o.set_state(pos=np.ascontiguousarray(pos0, np.float64))
    if vel is not None:
        v = np.zeros((sc.n, 4))
        v[:, :3] = vel
        o.set_state(vel=v)
    o.step(steps)
    pos = o.state()["pos"][:, :3]
    if loss[0] == "tip":
        d = pos[loss[1]].mean(axis=0) - np.asarray(loss[2], np.float64)
        return float(d @ d)
    if loss[0] == "separation":  # heavy centroid height above the light one's
        heavy = loss[1]
        return float(pos[heavy, 1].mean() - pos[~heavy, 1].mean())
    d = pos - loss[1]
    return float(np.sum(d * d))


def oracle_losses(tasks, processes=None):
    """_oracle_loss over many tasks in a pool of spawned processes (spawned,
    not forked: the parent holds a CUDA context)."""
    import multiprocessing as mp
    import os
    procs = processes or max(1, min(32, os.cpu_count() or 1, len(tasks)))
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_oracle_loss, tasks, chunksize=1)


def compare_with_oracle(sc, steps, tol=1e-5, graph=False, fp32_floor=False):
    """GPU vs the float oracle within `tol`; with `fp32_floor`, a quantity may
    instead be as close to the double oracle as twice the float oracle's own
    distance from it (stiff solids, where float rounding alone moves the
    velocities by ~1e-4 relative within tens of steps)."""
    from arphys import FluidSim
    from oracle.oracle import Oracle
    sim = FluidSim(sc)
    sim.init()
    if graph:
        sim.set_graph(True)
    sim.step(steps)
    g = sim.particles()
    o32, o64 = Oracle(sc, 32), Oracle(sc, 64)
    o32.step(steps)
    o64.step(steps)
    r32, r64 = o32.state(), o64.state()
    assert abs(sim.time() - o32.time) < 1e-6
    for key in ("den", "pos", "vel"):
        e = rel_err(g[key], r32[key])
        e64 = rel_err(g[key], r64[key])
        e_or = rel_err(r32[key], r64[key])
        print(f"{sc.name} {key}: vs f32 oracle {e:.2e}, vs f64 oracle {e64:.2e} (f32 oracle vs f64 {e_or:.2e})")
        if fp32_floor:
            assert e < tol or e64 <= max(tol, 2.0 * e_or), (sc.name, key, e, e64, e_or)
        else:
            assert e < tol, (sc.name, key, e)
    return sim
