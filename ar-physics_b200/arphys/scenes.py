"""Scene descriptions and seeded synthetic scene generators.

A `Scene` is everything `FluidSim::new` receives (src/soft_body/mod.rs:58-66)
after the reference's regions have been seeded into particles: mobile and
boundary particle records, the material table, an optional interaction table,
the AABB, kernel radius, integrator, time step, subticks and gravity.

Material constructors follow src/soft_body/material_region/material.rs:61-121
and the TOML mapping of examples/test_mods/config.rs:351-391 (bulk_visc =
alpha * h * c, state equation inferred from the keys given).  Masses follow
the reference's rule (material_region/mod.rs:144-149): start density times
the lattice cell volume.

The benchmark workloads are the five configurations the benchmark is quoted
on (2D dam break; 3D fluid + clamped elastic bar at 1,048,576 particles;
batched scenes; elastic bar for differentiation; batched Rayleigh-Taylor).
No dataset exists for them: every input is generated here from fixed seeds.
"""
from dataclasses import dataclass, field
import math

import numpy as np

from .abi import INTEGRATORS as INTEGRATOR_IDS
from .abi import (PARTICLE_DTYPE, MATERIAL_DTYPE, INTERACTION_DTYPE, INVALID, EOS_ZERO, EOS_TAIT,
                  EOS_IDEAL_GAS)


@dataclass
class Scene:
    particles: np.ndarray
    boundary: np.ndarray
    materials: np.ndarray
    bounds_min: tuple
    bounds_dim: tuple
    h: float
    integrator: str = "rk4"
    dt: float = 1e-4
    subticks: int = 1
    gravity: float = 9.81
    alpha: float = 0.0
    interactions: np.ndarray = None
    interaction_given: np.ndarray = None
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.particles)

    @property
    def nb(self):
        return len(self.boundary)

    @property
    def dim(self):
        return sum(1 for d in self.bounds_dim if d > 0)

    def n_solids(self):
        stiff = (self.materials["normal_stiffness"] != 0) | (self.materials["shear_stiffness"] != 0)
        return int(np.count_nonzero(stiff[self.particles["mat"]]))


def material(**kw):
    m = np.zeros((), dtype=MATERIAL_DTYPE)
    for k, v in kw.items():
        m[k] = v
    return m


def liquid(density, sound_speed, h, alpha, visc=0.0, mass=0.0, state=EOS_TAIT, target=None):
    """An `[objects]` fluid as config.rs:354-375 builds it (Tait unless told otherwise)."""
    return material(start_den=density, target_den=density if target is None else target,
                    sound_speed=sound_speed, visc=visc, bulk_visc=np.float32(alpha) * np.float32(h) *
                    np.float32(sound_speed), state_eq=state, mass=mass, strain_order=2)


def elastic_solid(density, lam, mu, mass, strain_order=2, normal_damp=0.0, shear_damp=0.0, plastic=None):
    m = material(start_den=density, target_den=density, state_eq=EOS_ZERO, mass=mass,
                 strain_order=strain_order, normal_stiffness=lam, shear_stiffness=mu,
                 normal_damp=normal_damp, shear_damp=shear_damp)
    if plastic:
        m["plastic"] = 1
        for k, v in plastic.items():
            m[k] = v
    return m


def immobile(friction, mass):
    """Material::new_immobile (material.rs:113-120); mass by the lattice rule."""
    return material(immobile=1, visc=friction, start_den=1.0, target_den=1.0, mass=mass)


def lame_from_young(E, nu):
    """Lame parameters of (E, nu), negated: the reference's force convention
    (solid.rs:366-368 with r = X_j - X_i and a negative-definite correction
    matrix) is restoring only for negative stiffness, which is why every solid
    scene it ships uses negative values (examples/metal_bar.toml:16-17)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return -lam, -mu


def particles(pos, mat, den, vel=None):
    n = len(pos)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["den"] = den
    p["mat"] = mat
    p["solid_id"] = INVALID
    p["pos"][:, :pos.shape[1]] = pos
    if vel is not None:
        p["vel"][:, :vel.shape[1]] = vel
    return p


def lattice(origin, counts, spacing):
    """Cubic lattice points origin + spacing * index, x fastest."""
    axes = [origin[a] + spacing * np.arange(counts[a], dtype=np.float64) for a in range(len(counts))]
    grids = np.meshgrid(*axes[::-1], indexing="ij")
    return np.stack([g.reshape(-1) for g in grids[::-1]], axis=1)


def jitter(pos, amp, rng):
    return pos + rng.uniform(-amp, amp, size=pos.shape)


def dam_break_2d(nx=128, ny=128, spacing=0.01, seed=1, steps=1000, integrator="rk4", dt=1e-4,
                 box=(2.56, 1.28), layers=3, c0=20.0, rho0=1000.0, alpha=0.1, visc=0.0):
    """2D dam break: nx x ny fluid lattice (spacing 0.01, jitter +-1e-4) at the
    left wall of a box, `layers` rows of static boundary particles outside the
    box walls, h = 2 x spacing, Tait (rho0, c0), artificial viscosity alpha."""
    rng = np.random.default_rng(seed)
    s = spacing
    h = 2.0 * s
    fluid = jitter(lattice((0.5 * s, 0.5 * s), (nx, ny), s), 1e-4, rng)
    bx, by = box
    mx, my = int(round(bx / s)), int(round(by / s))
    ring = lattice((-(layers - 0.5) * s, -(layers - 0.5) * s), (mx + 2 * layers, my + 2 * layers), s)
    inside = (ring[:, 0] > 0) & (ring[:, 0] < bx) & (ring[:, 1] > 0) & (ring[:, 1] < by)
    ring = ring[~inside]
    mats = np.array([
        immobile(0.0, mass=1.0 * s * s),
        liquid(rho0, c0, h, alpha, visc=visc, mass=rho0 * s * s),
    ])
    return Scene(
        particles=particles(fluid, 1, rho0), boundary=particles(ring, 0, 1.0), materials=mats,
        bounds_min=(0.0, 0.0, 0.0, 0.0), bounds_dim=(bx, by, 0.0, 0.0), h=h, integrator=integrator, dt=dt,
        subticks=1, gravity=9.81, alpha=alpha, name=f"dam_break_2d_{nx}x{ny}", meta={"steps": steps})


def fluid_bar_3d(fluid_n=(96, 96, 96), bar_n=(32, 128, 32), floor_n=(256, 128), spacing=0.01, seed=2,
                 clamp_layers=2, E=1e6, nu=0.3, c0=20.0, rho0=1000.0, alpha=0.1, integrator="rk2", dt=1e-4,
                 fluid_speed=2.0, box=(2.56, 1.28, 1.28), steps=500):
    """3D fluid block striking a vertical linear-elastic bar clamped at its
    base.  Default sizes: 96^3 fluid + 32x128x32 bar (2 clamped layers made
    immobile) + a 256x128 floor layer = 1,048,576 particles, h = 2 x spacing,
    Tait fluid, E = 1e6 / nu = 0.3 bar (strain order 2), RK2.

    The fluid starts 2.5 h from the bar moving towards it at `fluid_speed`.
    """
    rng = np.random.default_rng(seed)
    s = spacing
    h = 2.0 * s
    bx, by, bz = box
    fx, fy, fz = fluid_n
    ax, ay, az = bar_n
    # fluid block ends at 5/8 of the box; the bar (centred in z) starts 4
    # spacings after the last fluid column
    fluid_x0 = max(0.5 * s, 0.625 * bx - s * fx)
    bar_x0 = fluid_x0 + s * (fx + 4)
    zc = 0.5 * bz
    fluid = jitter(lattice((fluid_x0, 0.5 * s, zc - 0.5 * s * fz + 0.5 * s), (fx, fy, fz), s), 1e-4, rng)
    bar = lattice((bar_x0, 0.5 * s, zc - 0.5 * s * az + 0.5 * s), (ax, ay, az), s)
    clamped = bar[:, 1] < (clamp_layers * s)
    floor = lattice((0.5 * s, -0.5 * s, 0.5 * s), (floor_n[0], 1, floor_n[1]), s)
    lam, mu = lame_from_young(E, nu)
    mats = np.array([
        immobile(0.0, mass=1.0 * s ** 3),                         # 0 floor
        immobile(0.0, mass=1.0 * s ** 3),                         # 1 bar clamp
        liquid(rho0, c0, h, alpha, mass=rho0 * s ** 3),           # 2 water
        elastic_solid(rho0, lam, mu, mass=rho0 * s ** 3),         # 3 bar
    ])
    vel = np.zeros_like(fluid)
    vel[:, 0] = fluid_speed
    mobile = np.concatenate([particles(fluid, 2, rho0, vel), particles(bar[~clamped], 3, rho0)])
    bnd = np.concatenate([particles(floor, 0, 1.0), particles(bar[clamped], 1, 1.0)])
    return Scene(
        particles=mobile, boundary=bnd, materials=mats, bounds_min=(0.0, 0.0, 0.0, 0.0),
        bounds_dim=(bx, by, bz, 0.0), h=h, integrator=integrator, dt=dt, subticks=1, gravity=9.81, alpha=alpha,
        name=f"fluid_bar_3d_{len(mobile) + len(bnd)}", meta={"steps": steps, "E": E, "nu": nu})


def small_fluid_bar_3d(seed=5, integrator="rk2"):
    """A few-thousand-particle version of `fluid_bar_3d` for parity tests."""
    return fluid_bar_3d(fluid_n=(12, 12, 12), bar_n=(4, 16, 4), floor_n=(32, 16), spacing=0.01, seed=seed,
                        box=(0.32, 0.2, 0.16), integrator=integrator, fluid_speed=2.0)


def stretched_bar(n=(20, 4, 4), spacing=0.01, stretch=1.01, lam=-1e5, mu=-1e5, dim=3):
    """An elastic bar with positions stretched along x from its reference
    configuration (used to pin the sign of the elastic force)."""
    s = spacing
    h = 2.0 * s
    counts = n[:dim]
    ref = lattice(tuple(0.3 + 0.5 * s for _ in range(dim)), counts, s)
    mats = np.array([elastic_solid(1000.0, lam, mu, mass=1000.0 * s ** dim)])
    p = particles(ref, 0, 1000.0)
    box_dim = tuple([1.0] * dim + [0.0] * (4 - dim))
    sc = Scene(particles=p, boundary=np.zeros(0, dtype=PARTICLE_DTYPE), materials=mats,
               bounds_min=(0.0, 0.0, 0.0, 0.0), bounds_dim=box_dim, h=h, integrator="euler", dt=1e-5,
               gravity=0.0, name="stretched_bar")
    stretched = ref.copy()
    x0 = ref[:, 0].mean()
    stretched[:, 0] = x0 + (ref[:, 0] - x0) * stretch
    return sc, stretched


def batched_scenes(count=256, seed=3, spacing=0.01, n_min=2048, n_max=65536, integrator="midpoint", dt=1e-4,
                   c0=20.0, rho0=1000.0, alpha=0.1, steps=200, margin=4, gap=4, aspect=2.0):
    """Independent 3D scenes for the batched form: total particle counts
    (floor included) log-uniform in [n_min, n_max]; each scene a seeded mix
    of 1-3 Tait fluid blocks and 0-2 elastic blocks (E log-uniform in
    [1e4, 1e6], nu = 0.3, strain order 2 standing in for the Neo-Hookean
    model, which the reference does not have), with its own h drawn
    uniformly in [1.5, 2.5] x spacing, RK2.

    The blocks stand on a one-layer floor of boundary particles: columns of
    about `aspect` times their width, at least 3 sites on a side, laid out
    by shelf packing on the floor with `gap` spacings between blocks and
    `margin` spacings to the box's sides.  The gap exceeds the largest h, so
    no pair of particles from different blocks starts within kernel range,
    and no block overlaps another (particles placed on one another give the
    continuity equation diverging densities and the step non-finite
    states within a few hundred steps)."""
    rng = np.random.default_rng(seed)
    out = []
    s = spacing
    for k in range(count):
        n_target = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        h = float(rng.uniform(1.5, 2.5) * s)
        n_fluid = int(rng.integers(1, 4))
        n_solid = int(rng.integers(0, 3))
        split = rng.dirichlet(np.ones(n_fluid + n_solid))
        E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=n_solid))
        floor_n = 0
        for _ in range(4):  # the floor's size follows the layout, the layout the bodies' share
            body = max(n_target - floor_n, 64 * (n_fluid + n_solid))
            dims = []
            for share in split * body:
                w = max(3, int(round((share / aspect) ** (1.0 / 3.0))))
                dims.append((w, max(3, int(round(share / (w * w)))), w))
            row = int(np.ceil(np.sqrt(sum((d[0] + gap) ** 2 for d in dims))))
            place, x, z, depth_row, width = [], 0, 0, 0, 0
            for d in dims:
                if x and x + d[0] > row:
                    x, z, depth_row = 0, z + depth_row + gap, 0
                place.append((x, z))
                x += d[0] + gap
                width = max(width, x - gap)
                depth_row = max(depth_row, d[2])
            nx, nz = width + 2 * margin, z + depth_row + 2 * margin
            floor_n = nx * nz
        ny = max(d[1] for d in dims) + margin
        mats = [immobile(0.0, mass=1.0 * s ** 3), liquid(rho0, c0, h, alpha, mass=rho0 * s ** 3)]
        mobile = []
        for b, (d, (px, pz)) in enumerate(zip(dims, place)):
            pos = jitter(lattice(((margin + px + 0.5) * s, 0.5 * s, (margin + pz + 0.5) * s), d, s), 1e-4, rng)
            if b < n_fluid:
                mobile.append(particles(pos, 1, rho0))
            else:
                lam, mu = lame_from_young(float(E[b - n_fluid]), 0.3)
                mats.append(elastic_solid(rho0, lam, mu, mass=rho0 * s ** 3))
                mobile.append(particles(pos, len(mats) - 1, rho0))
        floor = lattice((0.5 * s, -0.5 * s, 0.5 * s), (nx, 1, nz), s)
        out.append(Scene(particles=np.concatenate(mobile), boundary=particles(floor, 0, 1.0), materials=np.array(mats),
                         bounds_min=(0.0, -s, 0.0, 0.0), bounds_dim=(nx * s, (ny + 1) * s, nz * s, 0.0), h=h,
                         integrator=integrator, dt=dt, gravity=9.81, alpha=alpha, name=f"batched_{k}",
                         meta={"steps": steps, "n_target": n_target}))
    return out


def partition_scenes(sizes, world):
    """Scene-parallel sharding of a batch over `world` ranks: each scene goes,
    largest first, to the rank with the least work so far (ties to the lower
    rank).  Scenes are independent, so ranks step their shares with no
    exchange.  Returns, per rank, the indices of its scenes in ascending
    order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    share = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        share[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(x) for x in share]


def load_toml(path):
    """A scene file in the reference's TOML schema (examples/test_mods/config.rs)
    parsed and seeded by the library (arp_scene_file_load), copied into a
    `Scene`.  Errors raise `ArpError`: ARP_ERR_IO, ARP_ERR_PARSE, or
    ARP_ERR_UNSUPPORTED for STL regions."""
    import ctypes
    from .abi import ArpScene, check, load_library
    L = load_library()
    f = ctypes.c_void_p()
    check(L.arp_scene_file_load(str(path).encode(), ctypes.byref(f)))
    try:
        sc = ArpScene()
        check(L.arp_scene_file_scene(f, ctypes.byref(sc)))
        name = ctypes.c_char_p()
        check(L.arp_scene_file_name(f, ctypes.byref(name)))

        def copy(addr, count, dtype):
            out = np.zeros(count, dtype=dtype)
            if count:
                ctypes.memmove(out.ctypes.data, addr, count * dtype.itemsize)
            return out

        m = sc.n_materials
        inv = {v: k for k, v in reversed(list(INTEGRATOR_IDS.items()))}
        from .abi import ArpView, ArpRenderStyle
        view, style = ArpView(), ArpRenderStyle()
        check(L.arp_scene_file_render_settings(f, ctypes.byref(view), ctypes.byref(style)))
        render = {"view": dict(angle=view.angle, pos=(view.pos[0], view.pos[1]), scale=view.scale),
                  "style": dict(render_h=style.render_h, lighting=bool(style.lighting),
                                light_pos=tuple(style.light_pos), light_color=tuple(style.light_color),
                                ambient=style.ambient, diffuse=style.diffuse, specular=style.specular,
                                colors=copy(style.colors, 12 * style.n_materials, np.dtype(np.float32)).reshape(-1, 12),
                                densities=copy(style.densities, style.n_materials, np.dtype(np.float32)))}
        count = ctypes.c_uint32()
        check(L.arp_scene_file_on_click_count(f, ctypes.byref(count)))
        on_click = []
        for i in range(count.value):
            pp, n, rel = ctypes.c_void_p(), ctypes.c_uint32(), ctypes.c_int()
            mat = np.zeros(1, dtype=MATERIAL_DTYPE)
            check(L.arp_scene_file_on_click(f, i, ctypes.byref(pp), ctypes.byref(n), mat.ctypes.data,
                                            ctypes.byref(rel)))
            on_click.append(dict(particles=copy(pp.value, n.value, PARTICLE_DTYPE), material=mat[0],
                                 relative=bool(rel.value)))
        return Scene(
            particles=copy(sc.particles, sc.n_particles, PARTICLE_DTYPE),
            boundary=copy(sc.boundary, sc.n_boundary, PARTICLE_DTYPE),
            materials=copy(sc.materials, m, MATERIAL_DTYPE),
            bounds_min=tuple(float(sc.bounds.min[i]) for i in range(4)),
            bounds_dim=tuple(float(sc.bounds.dim[i]) for i in range(4)),
            h=float(sc.kernel_radius), integrator=inv[sc.integrator], dt=float(sc.timestep),
            subticks=int(sc.subticks), gravity=float(sc.gravity), alpha=float(sc.artificial_viscocity),
            interactions=copy(sc.interactions, m * m, INTERACTION_DTYPE).reshape(m, m),
            interaction_given=copy(sc.interaction_given, m * m, np.dtype(np.uint8)).reshape(m, m),
            name=name.value.decode(), meta={"source": str(path), "on_click": on_click, "render": render})
    finally:
        L.arp_scene_file_free(f)


def cantilever_bar(n=(16, 256, 16), spacing=0.01, seed=4, E_median=1e5, E_sigma=0.3, nu=0.3, clamp_layers=2,
                   integrator="midpoint", dt=1e-4, v_sigma=0.0, gravity=9.81, target_offset=(0.002, -0.01, 0.002)):
    """The differentiation workload: an elastic bar of n[0] x n[1] x n[2] lattice
    sites (spacing 0.01, h = 2 x spacing), standing on its lowest `clamp_layers`
    layers, which are immobile, under gravity; per-particle Young's modulus
    lognormal(ln E_median, E_sigma), nu = 0.3, RK2 (midpoint).  The meta holds
    the per-solid (normal, shear) stiffness (negated Lame pair), the caller ids
    of the tip (top layer) and a seeded target for the tip centroid."""
    rng = np.random.default_rng(seed)
    s = spacing
    h = 2.0 * s
    nx, ny, nz = n
    origin = (0.1 + 0.5 * s, 0.05 + 0.5 * s, 0.1 + 0.5 * s)
    pos = lattice(origin, (nx, ny, nz), s)
    layer = np.rint((pos[:, 1] - origin[1]) / s).astype(int)
    clamp = layer < clamp_layers
    lam0, mu0 = lame_from_young(E_median, nu)
    mass = 1000.0 * s ** 3
    mats = np.array([immobile(0.0, mass=1.0 * s ** 3), elastic_solid(1000.0, lam0, mu0, mass=mass)])
    vel = np.zeros_like(pos)
    if v_sigma > 0:
        vel = rng.normal(0.0, v_sigma, size=pos.shape).astype(np.float32)
    p = particles(pos[~clamp], 1, 1000.0, vel[~clamp])
    b = particles(pos[clamp], 0, 1.0)
    E = np.exp(rng.normal(np.log(E_median), E_sigma, size=len(p))).astype(np.float64)
    lam, mu = lame_from_young(E, nu)
    stiff = np.stack([lam, mu], axis=1).astype(np.float32)
    tip = np.nonzero(layer[~clamp] == ny - 1)[0]
    target = p["pos"][tip, :3].mean(axis=0) + np.asarray(target_offset, np.float32)
    box_min = (0.0, 0.0, 0.0, 0.0)
    box_dim = (2 * origin[0] + nx * s, origin[1] + ny * s + 0.1, 2 * origin[2] + nz * s, 0.0)
    return Scene(particles=p, boundary=b, materials=mats, bounds_min=box_min, bounds_dim=box_dim, h=h,
                 integrator=integrator, dt=dt, subticks=1, gravity=gravity, alpha=0.0,
                 name=f"cantilever_bar_{nx}x{ny}x{nz}",
                 meta={"stiffness": stiff, "E": E, "nu": nu, "tip": tip, "target": target})


def tip_loss(pos, tip, target):
    """Squared distance of the tip centroid to the target and dL/dx (n x 3)."""
    c = pos[tip, :3].astype(np.float64).mean(axis=0)
    d = c - np.asarray(target, np.float64)
    grad = np.zeros((len(pos), 3))
    grad[tip] = 2.0 * d / len(tip)
    return float(d @ d), grad


def rayleigh_taylor_batch(count=64, seed=5, n_min=8192, n_max=131072, spacing=0.01, integrator="midpoint",
                          dt=1e-4, c0=20.0, alpha=0.1, layers=3):
    """The batched differentiation workload: `count` 2D Rayleigh-Taylor scenes,
    particle counts uniform in [n_min, n_max], each a heavy Tait fluid
    (rho0 = 1800) over a light one (rho0 = 1000) in a box twice as tall as
    wide, interface y0 + sum_m a_m cos(2 pi m x / L + phi_m) over modes 1..8
    with seeded amplitudes summing to 0.01 and seeded phases, `layers` rows of
    static boundary particles around the box, h = 2 x spacing, gravity 9.81."""
    rng = np.random.default_rng(seed)
    s = spacing
    h = 2.0 * s
    out = []
    for k in range(count):
        n_target = int(rng.integers(n_min, n_max + 1))
        nx = max(8, int(round(math.sqrt(n_target / 2.0))))
        ny = max(16, int(round(n_target / nx)))
        L, H = nx * s, ny * s
        pos = lattice((0.5 * s, 0.5 * s), (nx, ny), s)
        amps = rng.random(8)
        amps = 0.01 * amps / amps.sum()
        phases = rng.random(8) * 2.0 * math.pi
        modes = np.arange(1, 9)
        y_if = 0.5 * H + (amps[None, :] * np.cos(2.0 * math.pi * modes[None, :] * pos[:, :1] / L
                                                   + phases[None, :])).sum(axis=1)
        heavy = pos[:, 1] > y_if
        ring = lattice((-(layers - 0.5) * s, -(layers - 0.5) * s), (nx + 2 * layers, ny + 2 * layers), s)
        inside = (ring[:, 0] > 0) & (ring[:, 0] < L) & (ring[:, 1] > 0) & (ring[:, 1] < H)
        ring = ring[~inside]
        mats = np.array([
            immobile(0.0, mass=1.0 * s * s),
            liquid(1000.0, c0, h, alpha, mass=1000.0 * s * s),
            liquid(1800.0, c0, h, alpha, mass=1800.0 * s * s),
        ])
        mat = np.where(heavy, 2, 1)
        p = np.zeros(len(pos), dtype=PARTICLE_DTYPE)
        p["pos"][:, :2] = pos
        p["den"] = np.where(heavy, 1800.0, 1000.0)
        p["mat"] = mat
        p["solid_id"] = INVALID
        out.append(Scene(particles=p, boundary=particles(ring, 0, 1.0), materials=mats,
                         bounds_min=(0.0, 0.0, 0.0, 0.0), bounds_dim=(L, H, 0.0, 0.0), h=h, integrator=integrator,
                         dt=dt, subticks=1, gravity=9.81, alpha=alpha, name=f"rayleigh_taylor_{k}",
                         meta={"heavy": np.nonzero(heavy)[0], "height": H}))
    return out


def separation(pos, heavy):
    """Height of the heavy fluid's centroid above the light fluid's and its
    gradient dL/dx (n x 3).  It falls as the layers mix; the 5-95 % heavy-fraction
    height of a particle set is piecewise constant in the positions (its gradient
    is zero almost everywhere), so this centroid separation is the differentiable
    measure of mixing used for the gradient."""
    n = len(pos)
    mask = np.zeros(n, bool)
    mask[heavy] = True
    y = pos[:, 1].astype(np.float64)
    nh, nl = mask.sum(), n - mask.sum()
    L = float(y[mask].mean() - y[~mask].mean())
    grad = np.zeros((n, 3))
    grad[mask, 1] = 1.0 / nh
    grad[~mask, 1] = -1.0 / nl
    return L, grad
