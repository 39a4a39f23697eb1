#!/usr/bin/env python
"""Benchmark of the SPH time step (particle-steps/s).

Workload (default): the 3D fluid + clamped elastic bar scene at 1,048,576
particles (96^3 Tait fluid, 32x128x32 bar with 2 clamped layers, 256x128
floor), RK2, dt = 1e-4, synthetic seeded inputs.  One "step" is one RK2
integrator step of the whole scene through the C ABI.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device-timed (CUDA events on the stream the library launches on,
L2 flushed between timed steps, max over ranks); `e2e` is the same metric
through the C ABI with host records copied in and out every step;
`roofline` covers the dominant kernel (fused fluid forces + stage update);
`cpu_baseline` is the CPU oracle (the restatement of the reference shaders)
on the host cores.  With N > 1 each rank runs an independent replica (the
plain step does not shard; scene-parallel replicas, weak scaling).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ar-physics_b200"))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 1M (vs HBM roofline); batched scenes/s; adjoint/fwd ratio"
UNIT = "particle-steps/s"
L2_FLUSH_BYTES = 256 << 20
PROFILE_EVERY = 10  # timed steps per step carrying the segment events


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the fluid kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    try:
        for line in open(p):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                out[parts[0]] = float(parts[2])
    except OSError:
        pass
    return out


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value, device):
    """The largest `value` over all ranks (the job's time is its slowest
    rank's); a no-op without a process group."""
    import torch
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, seconds):
    """Whole-job throughput: the units all ranks processed over the max time."""
    return units_per_rank * world / seconds


def make_scene(name):
    from arphys import scenes
    if name == "c1":
        return scenes.dam_break_2d()
    return scenes.fluid_bar_3d()


def config_of(sc, name):
    ns = sc.n_solids()
    return {
        "workload": ("fluid_bar_3d: 96^3 Tait fluid striking a 32x128x32 elastic bar (E=1e6, nu=0.3, 2 clamped "
                     "layers) on a 256x128 floor, h=2x spacing, RK2, dt=1e-4" if name == "c2" else
                     "dam_break_2d: 128x128 Tait fluid, 2340 boundary particles, h=2x spacing, RK4, dt=1e-4"),
        "particles": int(sc.n + sc.nb), "mobile": int(sc.n), "solids": ns, "boundary": int(sc.nb),
        "integrator": sc.integrator, "l2": "flushed between timed steps (256 MiB write)",
    }


def step_roofline(sc, stages, step_ms, peak):
    """Whole-step algorithmic bytes: per mobile particle 96 B per stage plus
    96 B for the grid build, per solid 196 B per stage (reference position,
    L, F written and read, plastic strain read and written), per boundary
    particle 16 B per stage."""
    ns = sc.n_solids()
    per_step = sc.n * (96.0 * stages + 96.0) + ns * 196.0 * stages + sc.nb * 16.0 * stages
    gbs = per_step / (step_ms / 1000.0) / 1e9
    return {"alg_bytes_per_step": per_step, "achieved": gbs, "unit": "GB/s", "frac": gbs / peak,
            "formula": "n*(96*S+96) + n_solid*196*S + n_boundary*16*S, S = stages per step"}


def candidate_count(sc):
    """Candidates the fluid kernel tests per stage: for each mobile particle,
    the mobile and boundary particles in its search rows (search cells halve
    the reference cells along x; rows of 5 search cells in x, 3 rows in y
    and, in 3D, in z), counted on the host from the initial positions."""
    sub = []
    for a in range(3):
        d = np.float32(sc.bounds_dim[a])
        sub.append(max(1, int(d / np.float32(sc.h))) if d > 0 else 1)
    sub[0] *= 2

    def cells(p):
        out = []
        for a in range(3):
            if sc.bounds_dim[a] > 0:
                t = np.clip((p[:, a] - sc.bounds_min[a]) / sc.bounds_dim[a], 0.0, 1.0)
                out.append(np.minimum((t * sub[a]).astype(np.int64), sub[a] - 1))
            else:
                out.append(np.zeros(len(p), np.int64))
        return out

    grid = np.zeros((sub[2] + 2, sub[1] + 2, sub[0] + 4), np.int64)  # padded by the reach
    mob = sc.particles["pos"].astype(np.float64)
    for p in (mob, sc.boundary["pos"].astype(np.float64)):
        cx, cy, cz = cells(p)
        np.add.at(grid, (cz + 1, cy + 1, cx + 2), 1)
    win = np.zeros((sub[2], sub[1], sub[0]), np.int64)
    for dz in range(3) if sc.dim == 3 else (1,):
        for dy in range(3):
            for dx in range(5):
                win += grid[dz:dz + sub[2], dy:dy + sub[1], dx:dx + sub[0]]
    cx, cy, cz = cells(mob)
    per = win[cz, cy, cx]
    return int(per.sum())


def load_issue():
    """Per-launch instruction figures of the fluid kernel from the committed ncu
    summary (profiles/ncu_issue.txt): warp instructions, issue-active %, long
    scoreboard stalls per issue, L1 hit %."""
    p = os.path.join(ROOT, "profiles", "ncu_issue.txt")
    out = {}
    try:
        for line in open(p):
            parts = line.split()
            if len(parts) >= 6 and not line.startswith("#"):
                out[parts[0]] = {"kernel": parts[1], "warp_instructions": float(parts[2]),
                                 "issue_active_pct": float(parts[3]), "long_scoreboard_per_issue": float(parts[4]),
                                 "l1_hit_pct": float(parts[5]), "source": "profiles/ncu_issue.txt"}
    except OSError:
        pass
    return out


def pair_rate(sc, stages, fluid_ms_per_step):
    """Fluid pair interactions per second: ordered pairs (i mobile, j mobile or
    boundary, j != i, |x_j - x_i| < h) in the initial state, counted with a
    k-d tree outside the timed region, times the stages of a step, over the
    fluid kernel's time per step."""
    from scipy.spatial import cKDTree
    d = sc.dim
    mob = sc.particles["pos"][:, :d].astype(np.float64)
    allp = np.concatenate([mob, sc.boundary["pos"][:, :d].astype(np.float64)])
    r = float(sc.h) * (1.0 - 1e-6)  # lattice pairs sit exactly at |r| = h, where W = 0
    pairs = int(cKDTree(mob).count_neighbors(cKDTree(allp), r)) - len(mob)
    cand = candidate_count(sc)
    return {"per_stage": pairs, "per_particle": pairs / max(sc.n, 1),
            "candidates_per_stage": cand, "candidates_per_particle": cand / max(sc.n, 1),
            "rate": pairs * stages / (fluid_ms_per_step / 1000.0), "unit": "pair-interactions/s"}


def oracle_sample(config, steps, warmup, max_seconds=60.0):
    """The CPU oracle (the float restatement of the reference's shaders) on
    all host cores: `warmup` untimed full-size steps (the first fills the
    boundary and reference buckets), then up to `steps` timed steps, one
    oracle step call each, stopping early after `max_seconds`.  Both the
    reference arm and the cpu_baseline leg run this, each in a process that
    has not loaded torch, so they time the same thing the same way."""
    from oracle import oracle as orc
    sc = make_scene(config)
    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    o = orc.Oracle(sc, 32)
    for _ in range(max(1, warmup)):
        o.step(1)
    t0 = time.perf_counter()
    done = 0
    while done < steps and time.perf_counter() - t0 < max_seconds:
        o.step(1)
        done += 1
    dt = time.perf_counter() - t0
    parts = sc.n + sc.nb
    return {"value": parts * done / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} full RK steps of the {parts}-particle scene after {max(1, warmup)} untimed "
                      f"step(s) (C++ oracle, float, OpenMP x{cores}); the reference's Rust/OpenGL path cannot "
                      f"run here", "seconds": dt, "steps": done}


def cpu_baseline(config, steps=20, warmup=1):
    """oracle_sample in a fresh interpreter (this process has loaded torch,
    whose OpenMP runtime would otherwise be the one the oracle runs on): 20
    full steps of the workload, about 13 s of host time on 16 cores."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--oracle-sample", config, str(steps),
                        str(warmup)], capture_output=True, text=True, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_batched(torch, stream, rank=0, world=1, steps_batch=200, rounds_loop=10, steps_variant=200):
    """256 independent scenes (2,048-65,536 particles each, own h, fluid
    blocks and elastic blocks): stepped as one batch (one set of launches per
    stage) and as a loop over 256 separate simulations, both on one GPU and
    both replaying each step from a CUDA graph.  The batch is timed over the
    configuration's 200 steps with the autotuner's launch shape; every
    persistent tile-queue shape of the fluid kernel is timed beside it over
    the same 200 steps from the same state.  With N ranks the scenes are
    sharded (scenes.partition_scenes, by particle count) and each rank steps
    its share; every time is the slowest rank's, and rates count all 256
    scenes."""
    from arphys import FluidSim, scenes
    everything = scenes.batched_scenes()
    mine = scenes.partition_scenes([sc.n + sc.nb for sc in everything], world)[rank]
    scs = [everything[k] for k in mine]
    parts_all = int(sum(sc.n + sc.nb for sc in everything))
    batch = FluidSim.batch(scs)
    batch.init()
    batch.set_stream(stream.cuda_stream)
    batch.set_graph(True)
    init = batch.particles().copy()
    batch.step(4)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.set_particles(init)
    e0.record(stream)
    batch.step(steps_batch)
    e1.record(stream)
    torch.cuda.synchronize()
    t_batch = max_over_ranks(e0.elapsed_time(e1) / 1000.0, "cuda")
    variant = batch.fluid_variant()
    # the persistent (scene, cell-tile) work-queue shapes, same state, same steps each
    shapes = {}
    for v in range(FluidSim.fluid_variant_count()):
        batch.set_fluid_variant(v)
        vi = batch.fluid_variant()
        if not vi["persistent"]:
            continue
        batch.set_particles(init)
        batch.step(2)  # captures this shape's step graphs
        batch.set_particles(init)
        e0.record(stream)
        batch.step(steps_variant)
        e1.record(stream)
        torch.cuda.synchronize()
        shapes[str(v)] = dict(vi, ms_per_step=max_over_ranks(e0.elapsed_time(e1), "cuda") / steps_variant)
    batch.set_fluid_variant(variant["variant"])
    best_pers = min(shapes, key=lambda k: shapes[k]["ms_per_step"]) if shapes else None
    # where a batch step goes: a few more steps, untimed, with the library's
    # per-segment events (graph replay off: the events sit between launches)
    batch.set_graph(False)
    batch.profile_enable(True)
    batch.step(4)
    torch.cuda.synchronize()
    prof = batch.profile_read()
    batch.profile_enable(False)
    segments = {k: prof[k] / max(prof["steps"], 1) for k in ("neighbor_ms", "solid_ms", "fluid_ms")}
    batch.close()
    sims = []
    for sc in scs:
        sim = FluidSim(sc)
        sim.init()
        sim.set_stream(stream.cuda_stream)
        sim.set_graph(True)
        sims.append(sim)
    for sim in sims:
        sim.step(2)  # captures each simulation's step graphs
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(rounds_loop):
        for sim in sims:
            sim.step(1)
    e1.record(stream)
    torch.cuda.synchronize()
    t_loop = max_over_ranks(e0.elapsed_time(e1) / 1000.0, "cuda")
    for sim in sims:
        sim.close()
    batched = len(everything) * steps_batch / t_batch
    loop = len(everything) * rounds_loop / t_loop
    return {"scenes": len(everything), "particles": parts_all, "integrator": "rk2", "steps": steps_batch,
            "sharding": f"scene-parallel x{world} (largest scene first to the least-loaded rank)",
            "scene_steps_per_s": batched, "particle_steps_per_s": parts_all * steps_batch / t_batch,
            "ms_per_step": t_batch * 1000.0 / steps_batch,
            "per_scene_loop_scene_steps_per_s": loop, "speedup_vs_per_scene_loop": batched / loop,
            "fluid_launch_shape": variant, "persistent_shapes": shapes, "best_persistent_shape": best_pers,
            "segments_ms_per_step": segments,
            "solids": int(sum(sc.n_solids() for sc in scs)),
            "note": ("no L2 flush: the batch's state (~%d MB) is larger than L2; both the batch and the "
                     "per-scene loop (%d rounds of one step per simulation) replay CUDA graphs"
                     % (parts_all * 32 * 4 // (1 << 20), rounds_loop))}


def _time_adjoint(torch, stream, sim, steps, every, loss_grad, stiff=None):
    """Plain forward, taped forward and backward of `steps` steps from the
    handle's current state (device time for the forwards, host wall clock
    around the backward call, which synchronizes)."""
    import time
    import numpy as np
    init = sim.particles().copy()
    # untimed warm-up of the whole reverse pass (first use of the tape's device memory)
    sim.tape_begin(every)
    sim.step(steps)
    sim.backward(np.zeros((sim.n, 8), np.float32))
    sim.tape_end()
    sim.set_particles(init)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1)
    # the forward as fast as the library runs it: each step replayed from a CUDA graph
    sim.set_particles(init)
    sim.set_graph(True)
    sim.step(2)  # captures the two step graphs
    sim.set_particles(init)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1)
    sim.set_graph(False)
    sim.set_particles(init)
    sim.tape_begin(every)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_tape = e0.elapsed_time(e1)
    grad = np.zeros((sim.n, 8), np.float32)
    L, gx = loss_grad(sim.particles()["pos"])
    grad[:, :3] = gx
    t_bwd = []
    for _ in range(2):  # two backward passes over the same tape
        t0 = time.perf_counter()
        g0, gs = sim.backward(grad)
        torch.cuda.synchronize()
        t_bwd.append((time.perf_counter() - t0) * 1000.0)
    sim.tape_end()
    t_mean = sum(t_bwd) / len(t_bwd)
    live = {}
    if stiff is not None:
        # dL/d(ln E) per particle: E scales both Lame parameters
        dlne = (gs.astype(np.float64) * stiff.astype(np.float64)).sum(axis=1)
        live = {"grad_lnE_norm": float(np.linalg.norm(dlne)),
                "grad_lnE_norm_over_loss": float(np.linalg.norm(dlne) / max(abs(L), 1e-300)),
                "grad_lnE_nonzero_particles": int(np.count_nonzero(np.abs(dlne) > 1e-6 * np.abs(dlne).max()))}
    return live | {"steps": steps, "checkpoint_every": every, "forward_ms": t_fwd, "forward_plain_launches_ms": t_plain,
            "forward_taped_ms": t_tape,
            "backward_ms": t_mean, "backward_ms_each": t_bwd, "adjoint_fwd_ratio": t_mean / t_fwd, "loss": L,
            "grad_v0_norm": float(np.linalg.norm(g0[:, 4:7])), "grad_stiffness_norm": float(np.linalg.norm(gs)),
            "fluid_launch_shape": sim.fluid_variant(),  # the autotuner's pick on the initial state
            "timing": "forwards: CUDA events on the library stream (forward_ms: steps replayed from CUDA graphs, "
                      "the ratio's denominator; taped: plain launches); backward: host wall clock around the call "
                      "(it synchronizes), including dL/dy upload and gradient download"}


def run_adjoint(torch, stream, bar_steps=400, rt_steps=300, only=None):
    """Reverse mode on the two differentiation workloads: the 16x16x256 bar
    (65,536 particles, per-particle E, 400 RK2 steps, checkpoints every 20;
    gradient of the tip-centroid loss w.r.t. per-particle stiffness and
    initial velocity) and 64 batched 2D Rayleigh-Taylor scenes (300 RK2 steps,
    gradient of the heavy/light centroid separation w.r.t. the initial
    velocities of all scenes, one backward pass for the batch)."""
    import numpy as np
    from arphys import FluidSim, scenes
    out = {}
    if only not in (None, "bar"):
        return out | run_adjoint_rt(torch, stream, rt_steps)
    sc = scenes.cantilever_bar(v_sigma=0.05)
    sim = FluidSim(sc)
    sim.init()
    sim.set_stream(stream.cuda_stream)
    sim.set_solid_stiffness(sc.meta["stiffness"])
    init = sim.particles().copy()
    sim.step(3)  # warm-up
    sim.set_particles(init)
    tip, target = sc.meta["tip"], sc.meta["target"]
    bar = _time_adjoint(torch, stream, sim, bar_steps, 20, lambda pos: scenes.tip_loss(pos, tip, target),
                        stiff=sc.meta["stiffness"])
    bar["workload"] = ("cantilever bar 16x16x256 (65,024 elastic + 512 clamped), per-particle E lognormal("
                       "ln 1e5, 0.3), nu 0.3, gravity, seeded initial velocities N(0, 0.05 m/s) per component, "
                       "RK2, dt 1e-4")
    if not bar["grad_lnE_norm_over_loss"] > 1e-6:
        # the elastic wave from the clamp crosses only ~0.46 m of the 2.54 m bar
        # in 400 steps, so the tip loss depends on E only through the motion
        # the initial velocity field starts near the tip; a zero gradient
        # means the workload is not the one meant
        raise RuntimeError(f"stiffness gradient of the bar workload is zero ({bar['grad_lnE_norm']:.3e})")
    sim.close()
    out["bar"] = bar
    if only == "bar":
        return out
    return out | run_adjoint_rt(torch, stream, rt_steps)


def run_adjoint_rt(torch, stream, steps):
    """The batched Rayleigh-Taylor part of run_adjoint."""
    import numpy as np
    from arphys import FluidSim, scenes
    scs = scenes.rayleigh_taylor_batch()
    batch = FluidSim.batch(scs)
    batch.init()
    batch.set_stream(stream.cuda_stream)
    init = batch.particles().copy()
    batch.step(3)  # warm-up
    batch.set_particles(init)
    offsets = np.cumsum([0] + [s.n for s in scs])

    def sep_grad(pos):
        g = np.zeros((len(pos), 3))
        tot = 0.0
        for k, s in enumerate(scs):
            L, gk = scenes.separation(pos[offsets[k]:offsets[k + 1]], s.meta["heavy"])
            g[offsets[k]:offsets[k + 1]] = gk
            tot += L
        return tot, g
    rt = _time_adjoint(torch, stream, batch, steps, 20, sep_grad)
    rt["workload"] = (f"{len(scs)} 2D Rayleigh-Taylor scenes, {int(offsets[-1])} particles (8,192-131,072 per "
                      "scene), heavy 1800 over light 1000, RK2, dt 1e-4; loss = sum of heavy/light centroid "
                      "separations")
    batch.close()
    return {"rayleigh_taylor_batch": rt}


def run_render(torch, sim, sc):
    """One 1920x1080 frame of the benchmark state (the demo's --record path),
    splat and lit, host wall clock around the call (frame read back to host)."""
    import time
    import numpy as np
    m = len(sc.materials)
    colors = np.tile(np.array([0.2, 0.4, 0.9, 1.0, 0.1, 0.1, 0.6, 1.0, 0.9, 0.9, 1.0, 1.0], np.float32), (m, 1))
    b, d = sc.bounds_min, sc.bounds_dim
    view = dict(angle=0.4, pos=(b[0] + 0.5 * d[0], -(b[1] + 0.5 * d[1])), scale=1.0)
    out = {"width": 1920, "height": 1080, "particles": int(sc.n + sc.nb)}
    for lit in (False, True):
        style = dict(render_h=sc.h, lighting=lit, colors=colors,
                     densities=sc.materials["start_den"].astype(np.float32))
        sim.render(1920, 1080, view, style)  # warm-up (buffers)
        t = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            img = sim.render(1920, 1080, view, style)
            t.append((time.perf_counter() - t0) * 1000.0)
        out["lit_ms" if lit else "splat_ms"] = min(t)
        out["lit_drawn_pixels" if lit else "splat_drawn_pixels"] = int(np.count_nonzero((img != 255).any(axis=2)))
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference's path cannot run here (Rust + OpenGL
    compute shaders, no GL stack), so the CPU restatement of its shaders is
    timed on the host cores, rank 0 only (oracle_sample, the same harness as
    the cpu_baseline leg)."""
    if rank != 0:
        return
    sc = make_scene(args.config)
    cb = oracle_sample(args.config, args.steps, args.warmup)
    v = cb["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": cb["steps"],
        "warmup": args.warmup, "ms_per_step": cb["seconds"] * 1000 / max(cb["steps"], 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": dict(config_of(sc, args.config), parallelism=f"replicas x{world}"),
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    from arphys import FluidSim

    torch.cuda.set_device(local_rank)
    dist = world > 1
    sc = make_scene(args.config)
    sim = FluidSim(sc)
    sim.init()
    if args.fluid_variant is not None:
        sim.set_fluid_variant(args.fluid_variant)
    # a dedicated stream: the library launches on it and the events below are
    # recorded on it (torch's default stream is the legacy NULL stream, which
    # the library's own non-blocking stream does not order against)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sim.set_stream(stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    sim.set_graph(True)  # each step replays a CUDA graph of its launches (captured in the warm-up)
    for _ in range(args.warmup):
        sim.step(1)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # the fluid kernel's launch times for the roofline: the library's CUDA
    # events around its segments on every PROFILE_EVERY-th timed step (an
    # event between two launches costs the step a few microseconds)
    sim.profile_enable(True, every=PROFILE_EVERY)
    sim.profile_read()
    l0 = sim.launch_count()
    clk = ClockSampler(local_rank)
    clk.start()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(1)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = sim.launch_count() - l0
    prof = sim.profile_read()
    sim.profile_enable(False)
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), "cuda")
    parts = sc.n + sc.nb
    value = aggregate_rate(parts * args.steps, world, total_ms / 1000.0)

    # end to end through the C ABI: host records in, one step (graph replay
    # stays on: setting particles keeps the step graphs), host records out,
    # the records living in page-locked host memory.  Pipelined: the
    # asynchronous exchange lets the copy of step i+1's input, step i and
    # the copy of step i-1's result overlap (two input states alternate, so
    # consecutive steps take different inputs); every step's input crosses
    # host->device and its result device->host inside the timed loop, which
    # ends with arp_sim_synchronize.  Serial: the synchronous calls, one step
    # at a time, as in the round trip set -> step -> get.
    from arphys import PARTICLE_DTYPE
    rec = PARTICLE_DTYPE.itemsize  # the reference's 48-byte Particle record

    def pinned_records():
        return torch.empty(sc.n * rec, dtype=torch.uint8).pin_memory().numpy().view(PARTICLE_DTYPE)
    host = pinned_records()
    sim.particles(out=host)
    serial_ms = []
    for i in range(max(3, min(args.steps, 20))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.set_particles(host)
        sim.step(1)
        sim.particles(out=host)
        serial_ms.append((time.perf_counter() - t0) * 1000)
    serial_step_ms = max_over_ranks(statistics.median(serial_ms), "cuda")
    ins = [pinned_records(), pinned_records()]
    outs = [pinned_records(), pinned_records()]
    sim.particles(out=ins[0])
    sim.step(1)
    sim.particles(out=ins[1])
    e2e_steps = max(args.steps, 20)
    for i in range(3):  # warm-up of the exchange (streams, staging slots)
        sim.set_particles_async(ins[i % 2])
        sim.step(1)
        sim.particles_async(outs[i % 2])
    sim.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        sim.set_particles_async(ins[i % 2])
        sim.step(1)
        sim.particles_async(outs[i % 2])
    sim.synchronize()
    e2e_step_ms = max_over_ranks((time.perf_counter() - t0) * 1000 / e2e_steps, "cuda")
    e2e = {"value": parts * world / (e2e_step_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": sc.n * rec, "d2h_bytes_per_step": sc.n * rec,
           "ms_per_step": e2e_step_ms, "steps": e2e_steps,
           "path": ("arp_sim_set_particles_async (host Particle records) + arp_sim_step(1) + "
                    "arp_sim_get_particles_async, arp_sim_synchronize after the last step; host wall clock"),
           "serial": {"value": parts * world / (serial_step_ms / 1000.0), "ms_per_step": serial_step_ms,
                      "path": "arp_sim_set_particles + arp_sim_step(1) + arp_sim_get_particles, median step"}}

    peak, peak_kind = load_peaks()
    fl = prof["stages"]
    fluid_ms = prof["fluid_ms"] / fl if fl else float("nan")  # per stage: tile kernel + overflow kernel
    alg_bytes = 96.0 * sc.n  # per stage: read y_s 32 B + read y0 32 B + write y_{s+1} 32 B per particle
    achieved = alg_bytes / (fluid_ms / 1000.0) / 1e9
    traffic = load_traffic().get(f"fluid_{args.config}")
    roofline = {"bound": "hbm", "kernel": "k_fluid (fused fluid forces + RK stage update)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                "avg_launch_ms": fluid_ms,
                "segments_ms_per_step": {k: prof[k] / max(prof["steps"], 1) for k in
                                         ("neighbor_ms", "solid_ms", "fluid_ms")}}
    stages = fl / max(prof["steps"], 1)
    roofline["step"] = step_roofline(sc, stages, total_ms / args.steps, peak)
    roofline["pairs"] = pair_rate(sc, stages, prof["fluid_ms"] / max(prof["steps"], 1))
    issue = load_issue().get(f"fluid_{args.config}_v{sim.fluid_variant()['variant']}")
    if issue:
        # the issue roofline: every warp instruction of a launch issued at one
        # per scheduler per cycle (148 SMs x 4 schedulers at the sampled clock)
        mhz = clocks.get("sm_mhz") or 1965.0
        t_issue = issue["warp_instructions"] / (148 * 4 * mhz * 1e6) * 1e3
        lanes = issue["warp_instructions"] * 32.0
        issue.update({"issue_bound_ms": t_issue, "issue_frac": t_issue / fluid_ms,
                      "lane_instructions_per_particle": lanes / sc.n,
                      "lane_instructions_per_candidate": lanes / max(roofline["pairs"]["candidates_per_stage"], 1),
                      "lane_instructions_per_pair": lanes / max(roofline["pairs"]["per_stage"], 1)})
        roofline["issue"] = issue
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": dict(config_of(sc, args.config), parallelism=f"replicas x{world}"),
        "e2e": e2e, "roofline": roofline, "clocks": clocks, "gpu_launches": launches,
    }
    line["fluid_launch_shape"] = sim.fluid_variant()
    # every rank takes part in the batched form (scene-parallel, collectives
    # for its max-over-ranks times) before rank 0 alone runs the rest
    if not args.no_batched:
        batched = run_batched(torch, stream, rank, world)
        if rank == 0:
            line["batched"] = batched
    if rank == 0 and not args.no_render:
        line["render"] = run_render(torch, sim, sc)
    if rank == 0 and not args.no_adjoint:
        line["adjoint"] = run_adjoint(torch, stream)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.config)
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-render", action="store_true")
    ap.add_argument("--fluid-variant", type=int, default=None, help="pin the fluid launch shape (profiling)")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched-scenes measurement and print its object (profiling)")
    ap.add_argument("--adjoint-only", choices=["bar", "rt", "both"], default=None,
                    help="run only the reverse-mode measurement and print its object (profiling)")
    ap.add_argument("--adjoint-steps", type=int, default=None,
                    help="steps of each reverse-mode workload (default: 400 for the bar, 300 for the batch)")
    ap.add_argument("--oracle-sample", nargs=3, metavar=("CONFIG", "STEPS", "WARMUP"), default=None,
                    help="time the CPU oracle alone and print its object (the cpu_baseline leg runs this)")
    args = ap.parse_args()
    if args.oracle_sample:
        c, k, w = args.oracle_sample
        print(json.dumps(oracle_sample(c, int(k), int(w))), flush=True)
        return
    if args.adjoint_only:
        import torch
        stream = torch.cuda.Stream()
        n = args.adjoint_steps
        print(json.dumps(run_adjoint(torch, stream, n or 400, n or 300,
                                     None if args.adjoint_only == "both" else args.adjoint_only)), flush=True)
        return
    if args.batched_only:
        import torch
        stream = torch.cuda.Stream()
        print(json.dumps(run_batched(torch, stream, steps_batch=args.steps)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
