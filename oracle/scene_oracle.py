"""CPU restatement of the reference's scene-file path -- TEST INFRASTRUCTURE ONLY.

Checks the library's TOML loader (arp_scene_file_load) record for record.  It
restates, in numpy float32/float64 arithmetic chosen operation by operation as
the Rust code chooses it:

  * examples/test_mods/config.rs:62-118   value helpers and their defaults
  * examples/test_mods/config.rs:120-252  region tables, CSG folds, transforms
  * examples/test_mods/config.rs:255-294  interaction tables
  * examples/test_mods/config.rs:298-474  Config::parse (materials, velocity
                                          fields, object order)
  * src/soft_body/material_region/region.rs:21-272  AABB, AABE, Transformed
                                          (Gauss-Jordan solve), Difference,
                                          Union, Intersection
  * src/soft_body/material_region/mod.rs:56-156  lattice seeding and the mass rule

The reference parses with the `toml` 0.5 crate, whose tables are ordered maps:
keys are visited in sorted order, which fixes the material numbering.  This
file parses with Python's tomllib and sorts explicitly.  cos/sin of the
rotation angle come from the C library's cosf/sinf, the functions Rust's f32
methods call on Linux.

Parity of this restatement is unpinned: the reference is Rust and no Rust
toolchain exists here, so its own loader cannot be run.  It is checked against
hand-computed cases in tests/test_scene_loader.py.
"""
import ctypes
import ctypes.util
import math
import tomllib

import numpy as np

f32 = np.float32
f64 = np.float64

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]

EOS = {"zero": 0, "constant": 1, "ideal_gas": 2, "tait": 3}
POTENTIALS = {"Zero": 0, "zero": 0, "Constant": 1, "constant": 1, "Linear": 2, "linear": 2, "Tait": 3,
              "tait": 3, "LennardJones": 4, "Lennard-Jones": 4, "Lennard Jones": 4, "lennard jones": 4,
              "lennard-jones": 4, "Hertz": 5, "hertz": 5}
INTEGRATORS = {"euler": 0, "rk1": 0, "midpoint": 1, "rk2": 1, "heun2": 2, "heun": 2, "ralston": 3, "rk3": 4,
               "heun3": 5, "rk4": 6, "rk_3_8": 7, "verlet": 8}


class SceneError(Exception):
    pass


def _num(v):
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise SceneError(f"expected a number, got {v!r}")
    return float(v)


def num_or(t, k, d):
    return _num(t[k]) if k in t else d


def to_vec4(arr):
    """config.rs:62-66: missing components are zero."""
    out = np.zeros(4, f32)
    for i, v in enumerate(arr[:4]):
        out[i] = f32(_num(v))
    return out


def vec4_or(t, k, d):
    return to_vec4(t[k]) if k in t else np.array(d, f32)


# ---- regions (region.rs) -------------------------------------------------------

class AABB:
    def __init__(self, mn, dim):
        self.min, self.dim = np.asarray(mn, f32), np.asarray(dim, f32)

    def bound(self):
        return self.min.copy(), self.dim.copy()

    def contains(self, P):
        ok = np.ones(len(P), bool)
        for i in range(4):
            ok &= ~((P[:, i] < self.min[i]) | ((P[:, i] - self.min[i]) > self.dim[i]))
        return ok


class AABE:
    def __init__(self, center, radii):
        self.center, self.radii = np.asarray(center, f32), np.asarray(radii, f32)

    def bound(self):
        return self.center - self.radii, f32(2.0) * self.radii

    def contains(self, P):
        lhs = np.zeros(len(P), f64)
        r = self.radii
        for i in range(4):
            d = (P[:, i] - self.center[i]).astype(f64)
            if f64(r[i]) > 0.0:
                coeff = f64(1.0)
                for j in range(4):
                    if r[j] > 0.0 and j != i:
                        coeff = coeff * f64(r[j])
                lhs = lhs + d * d * coeff * coeff
        rhs = f64(1.0)
        for i in range(4):
            if r[i] > 0.0:
                rhs = rhs * f64(r[i])
        return lhs <= rhs * rhs


class Transformed:
    """region.rs:125-217.  The elimination's branches test only the matrix, so
    its row operations are recorded once and replayed on all points."""

    def __init__(self, base, a, t):
        self.base, self.a, self.t = base, np.asarray(a, f32), np.asarray(t, f32)  # a[col][row]
        self.ops = self._eliminate()

    def bound(self):
        bmin, bdim = self.base.bound()
        mn, mx = self.t.copy(), self.t.copy()
        a = self.a
        for i in range(4):
            a_min = f32(0.0)
            for j in range(4):
                a_min = f32(a_min + a[j][i] * bmin[j])
            mn[i] = mn[i] + a_min
            mx[i] = mx[i] + a_min
            for j in range(4):
                mn[i] = mn[i] + np.fmin(a[j][i] * bdim[j], f32(0.0))
            for j in range(4):
                mx[i] = mx[i] + np.fmax(a[j][i] * bdim[j], f32(0.0))
        return mn, mx - mn

    def _eliminate(self):
        a = self.a.copy()
        ops = []
        i = j = 0
        while i < 4 and j < 4:
            if a[j][i] != 0.0:
                pivot = a[j][i]
                if pivot != 1.0:
                    fac = f32(f32(1.0) / pivot)
                    for k in range(j, 4):
                        a[k][i] = a[k][i] * fac
                    ops.append(("mul", i, fac))
                for k in range(4):
                    if k != i and a[j][k] != 0.0:
                        fac = -a[j][k]
                        for c in range(j, 4):
                            a[c][k] = a[c][k] + fac * a[c][i]
                        ops.append(("sum", i, fac, k))
                i += 1
                j += 1
            else:
                cont = False
                for k in range(i + 1, 4):
                    if a[j][k] != 0.0:
                        for c in range(j, 4):
                            a[c][i], a[c][k] = a[c][k], a[c][i]
                        ops.append(("swap", i, k))
                        cont = True
                if not cont:
                    j += 1
        return ops

    def contains(self, P):
        V = (P - self.t).astype(f32)
        for op in self.ops:
            if op[0] == "mul":
                V[:, op[1]] = V[:, op[1]] * op[2]
            elif op[0] == "sum":
                _, row, fac, dest = op
                V[:, dest] = V[:, dest] + fac * V[:, row]
            else:
                _, r1, r2 = op
                V[:, [r1, r2]] = V[:, [r2, r1]]
        return self.base.contains(V)


class Difference:
    def __init__(self, l, r):
        self.l, self.r = l, r

    def bound(self):
        return self.l.bound()

    def contains(self, P):
        return self.l.contains(P) & ~self.r.contains(P)


class Union(Difference):
    def bound(self):
        (lm, ld), (rm, rd) = self.l.bound(), self.r.bound()
        mn = np.fmin(lm, rm)
        return mn, np.fmax(lm + ld, rm + rd) - mn

    def contains(self, P):
        return self.l.contains(P) | self.r.contains(P)


class Intersection(Difference):
    def bound(self):
        (lm, ld), (rm, rd) = self.l.bound(), self.r.bound()
        mn = np.fmax(lm, rm)
        return mn, np.fmin(lm + ld, rm + rd) - mn

    def contains(self, P):
        return self.l.contains(P) & self.r.contains(P)


def aabb_border(mn, dim, b):  # region.rs:37-46
    c = mn + f32(0.5) * dim
    return Difference(AABB(mn, dim), AABB(np.fmin(mn + b, c), np.fmax(dim - f32(2.0) * b, f32(0.0))))


def aabe_border(center, radii, b):  # region.rs:54-63
    return Difference(AABE(center, radii), AABE(center, np.fmax(radii - b, f32(0.0))))


# ---- STL regions (examples/test_mods/mesh.rs) ----------------------------------

def read_stl(path):
    """Vertices (V x 3 f32, shared by exact value) and faces (F x 3 indices,
    F x 3 stored normals) of a binary or ASCII STL file, as stl_io 0.4 reads it."""
    data = open(path, "rb").read()
    tris = None
    if len(data) >= 84:
        count = int(np.frombuffer(data, np.uint32, 1, 80)[0])
        if len(data) == 84 + 50 * count:
            rec = np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")])
            arr = np.frombuffer(data, rec, count, 84)
            tris = (arr["n"].astype(f32), arr["v"].astype(f32))
    if tris is None:
        if not data.startswith(b"solid"):
            raise SceneError("not an STL file")
        toks = data.split()
        ns, vs = [], []
        for k, w in enumerate(toks):
            if w == b"normal":
                ns.append([float(x) for x in toks[k + 1:k + 4]])
            elif w == b"vertex":
                vs.append([float(x) for x in toks[k + 1:k + 4]])
        tris = (np.array(ns, f32).reshape(-1, 3), np.array(vs, f32).reshape(-1, 3, 3))
    normals, verts = tris
    flat = np.ascontiguousarray(verts.reshape(-1, 3))
    keys = flat.view(np.uint32)
    uniq, inv = np.unique(keys, axis=0, return_inverse=True)
    return uniq.view(f32).reshape(-1, 3), inv.reshape(-1, 3), normals


def _signum(x):
    return np.where(np.isnan(x), x, np.copysign(f32(1.0), x)).astype(f32)


def _mesh_bound(V):  # mesh.rs:12-24
    mn = np.zeros(4, f32)
    mx = np.zeros(4, f32)
    mn[:3] = V.min(axis=0)
    mx[:3] = V.max(axis=0)
    return mn, mx - mn


class Mesh:
    """mesh.rs:26-77: odd number of faces above the point whose xy triangle
    holds it."""

    def __init__(self, path):
        self.V, self.Fi, self.N = read_stl(path)

    def bound(self):
        return _mesh_bound(self.V)

    def contains(self, P):
        parity = np.zeros(len(P), np.int64)
        V, Fi = self.V, self.Fi
        step = max(1, 4_000_000 // max(len(P), 1))
        for c in range(0, len(Fi), step):
            v0, v1, v2 = V[Fi[c:c + step, 0]], V[Fi[c:c + step, 1]], V[Fi[c:c + step, 2]]
            pz = P[:, None, 2]
            above = (v0[None, :, 2] >= pz) | (v1[None, :, 2] >= pz) | (v2[None, :, 2] >= pz)
            s1x, s1y = v1[:, 0] - v0[:, 0], v1[:, 1] - v0[:, 1]
            s2x, s2y = v2[:, 0] - v0[:, 0], v2[:, 1] - v0[:, 1]
            dx = P[:, None, 0] - v0[None, :, 0]
            dy = P[:, None, 1] - v0[None, :, 1]
            a = s1x * s2y - s1y * s2x
            sg = _signum(a)
            sv = sg * (dx * s2y - dy * s2x)
            tv = sg * (s1x * dy - s1y * dx)
            a = np.abs(a)
            hit = above & (sv >= 0) & (sv <= a) & (tv >= 0) & (tv <= a) & ((sv + tv) <= a)
            parity += hit.sum(axis=1)
        return (parity % 2 == 1) & (P[:, 3] == 0)


class Surface(Mesh):
    """mesh.rs:79-138: within `border` of a vertex, or of a face inside its
    edges' prism."""

    def __init__(self, path, border):
        super().__init__(path)
        self.border = f32(border)

    def bound(self):
        mn, dim = _mesh_bound(self.V)
        mn[:3] = mn[:3] - self.border
        dim[:3] = dim[:3] + self.border * f32(2.0)
        return mn, dim

    @staticmethod
    def _dot(a, b):
        return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]

    @staticmethod
    def _cross(a, b):
        return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                         a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)

    def contains(self, P):
        P3 = P[:, :3]
        out = np.zeros(len(P), bool)
        bb = self.border * self.border
        step = max(1, 4_000_000 // max(len(P), 1))
        for c in range(0, len(self.V), step):
            d = P3[:, None, :] - self.V[None, c:c + step, :]
            out |= (self._dot(d, d) <= bb).any(axis=1)
        V, Fi = self.V, self.Fi
        for c in range(0, len(Fi), step):
            n = self.N[c:c + step]
            a, b, cc = V[Fi[c:c + step, 0]], V[Fi[c:c + step, 1]], V[Fi[c:c + step, 2]]
            d = P3[:, None, :] - a[None]
            near = np.abs(self._dot(d, n[None])) <= np.sqrt(self._dot(n, n))[None] * self.border
            s1, s2, s3, s4 = b - a, cc - a, cc - b, a - b
            d2 = P3[:, None, :] - b[None]
            n1, n2, n3 = self._cross(s1, n), self._cross(s2, n), self._cross(s3, n)
            ok = (near & (_signum(self._dot(d, n1[None])) == _signum(self._dot(s2, n1))[None])
                  & (_signum(self._dot(d, n2[None])) == _signum(self._dot(s1, n2))[None])
                  & (_signum(self._dot(d2, n3[None])) == _signum(self._dot(s4, n3))[None]))
            out |= ok.any(axis=1)
        return out


def parse_base(t):  # config.rs:180-239
    if isinstance(t.get("model"), str):
        b = t.get("border")
        if isinstance(b, float):  # .and_then(as_float): an integer border is no border
            return Surface(t["model"], f32(b))
        return Mesh(t["model"])
    border = f32(_num(t["border"])) if "border" in t else None
    mn = np.zeros(4, f32)
    if isinstance(t.get("dim"), list):
        boxed, dim = True, to_vec4(t["dim"])
    elif isinstance(t.get("radii"), list):
        boxed, dim = False, to_vec4(t["radii"]) * f32(2.0)
    elif isinstance(t.get("diameters"), list):
        boxed, dim = False, to_vec4(t["diameters"])
    else:
        return region_from_mat(t)
    if isinstance(t.get("min"), list):
        mn = to_vec4(t["min"])
    elif isinstance(t.get("center"), list):
        mn = to_vec4(t["center"]) - f32(0.5) * dim
    if boxed:
        return AABB(mn, dim) if border is None else aabb_border(mn, dim, border)
    dim = dim * f32(0.5)
    mn = mn + dim
    return AABE(mn, dim) if border is None else aabe_border(mn, dim, border)


def parse_region(t):  # config.rs:130-178
    base = parse_base(t)
    if not any(k in t for k in ("translation", "scale", "rotation")):
        return base
    trans = vec4_or(t, "translation", [0, 0, 0, 0])
    rv = t.get("rotation")
    rot = np.array([0, 0, 1, rv], f32) if isinstance(rv, float) else vec4_or(t, "rotation", [0, 0, 1, 0])
    sv = t.get("scale")
    scale = np.ones(4, f32)
    if isinstance(sv, float):
        scale[:] = f32(sv)
    elif isinstance(sv, list):
        for i, v in enumerate(sv[:4]):
            scale[i] = f32(_num(v))
    ang = f32(rot[3] * f32(f32(math.pi) / f32(180.0)))  # f32::to_radians
    c, s = f32(_libm.cosf(float(ang))), f32(_libm.sinf(float(ang)))
    u_l = np.sqrt(f32(f32(rot[0] * rot[0] + rot[1] * rot[1]) + rot[2] * rot[2]))
    u = [rot[0] / u_l, rot[1] / u_l, rot[2] / u_l]
    one = f32(1.0)
    m = np.array([
        [c + u[0] * u[0] * (one - c), u[0] * u[1] * (one - c) + u[2] * s, u[0] * u[2] * (one - c) - u[1] * s, 0],
        [u[1] * u[2] * (one - c) - u[1] * s, c + u[1] * u[1] * (one - c), u[1] * u[2] * (one - c) + u[0] * s, 0],
        [u[0] * u[2] * (one - c) + u[1] * s, u[1] * u[2] * (one - c) - u[0] * s, c + u[2] * u[2] * (one - c), 0],
        [0, 0, 0, 1]], f32)
    m = m * scale[:, None]
    return Transformed(base, m, trans)


def region_from_mat(t):  # config.rs:242-252
    for key, node in (("union", Union), ("difference", Difference), ("intersection", Intersection)):
        if isinstance(t.get(key), list):
            regs = [parse_region(e) for e in t[key]]
            if not regs:
                raise SceneError("empty region list")
            acc = regs[0]
            for r in regs[1:]:
                acc = node(acc, r)
            return acc
    if isinstance(t.get("region"), dict):
        return parse_region(t["region"])
    raise SceneError("material has no region")


# ---- seeding (material_region/mod.rs:56-156) -------------------------------------

def _row(x0, h, mn, dim):
    """x0, x0+h, ... while the accumulated value stays within the bound (the
    first value is always taken; the loop stops after the step that leaves)."""
    if dim == 0.0:
        return np.array([x0], f32)
    n = max(int(float(dim) / float(h)), 0) + 4
    while True:
        steps = np.full(n, h, f32)
        steps[0] = x0
        xs = np.add.accumulate(steps, dtype=f32)
        out = (xs[1:] - mn) > dim
        if out.any():
            k = int(np.argmax(out)) + 1
            return xs[:k]
        n *= 2


def gen_particles(region, packing, kernel_h, start_den, vel_fn):
    h = f32(packing * kernel_h)
    bmin, bdim = region.bound()
    sites = []
    z = bmin[2]
    offset2 = f32(0.0)
    sq2, sq3, sq8 = np.sqrt(f32(2.0)), np.sqrt(f32(3.0)), np.sqrt(f32(8.0))
    while True:
        offset = f32(0.0)
        y = f32(bmin[1] + offset2)
        while True:
            xs = _row(f32(bmin[0] + f32(offset + offset2)), h, bmin[0], bdim[0])
            P = np.empty((len(xs), 4), f32)
            P[:, 0], P[:, 1], P[:, 2], P[:, 3] = xs, y, z, bmin[3]
            sites.append(P)
            y = f32(y + f32(h / sq2))
            offset = f32(h / f32(2.0)) if offset == 0.0 else f32(0.0)
            if f32(y - bmin[1]) > bdim[1] or bdim[1] == 0.0:
                break
        z = f32(z + f32(h / sq3))
        offset2 = f32(h / sq8) if offset2 == 0.0 else f32(0.0)
        if f32(z - bmin[2]) > bdim[2] or bdim[2] == 0.0:
            break
    P = np.concatenate(sites)
    keep = region.contains(P)
    content = 1.0
    for i in range(4):
        if bdim[i] > 0.0:
            content = content * float(bdim[i])
    mass = f32(float(start_den) * content / float(len(P)))
    pos = P[keep]
    vel = vel_fn(pos) if vel_fn else np.zeros_like(pos)
    return pos, vel, mass


def _velocity_fn(vel, w, center):  # config.rs:398-423
    def fn(P):
        r = P - center
        out = np.empty_like(P)
        out[:, 0] = w[1] * r[:, 2] - w[2] * r[:, 1] - w[3] * r[:, 3] + vel[0]
        out[:, 1] = w[2] * r[:, 0] - w[0] * r[:, 2] + w[4] * r[:, 3] + vel[1]
        out[:, 2] = w[0] * r[:, 1] - w[1] * r[:, 0] - w[5] * r[:, 3] + vel[2]
        out[:, 3] = w[3] * r[:, 0] - w[4] * r[:, 1] + w[5] * r[:, 3] + vel[3]
        return out
    return fn


MATERIAL_FIELDS = ("immobile", "mass", "start_den", "state_eq", "sound_speed", "target_den", "visc", "bulk_visc",
                   "strain_order", "normal_stiffness", "shear_stiffness", "normal_damp", "shear_damp", "plastic",
                   "yield_strength", "work_hardening", "work_hardening_exp", "kinematic_hardening",
                   "thermal_softening", "relaxation_time")


def _interaction(t, h):  # config.rs:255-277
    return dict(strength=f32(num_or(t, "contact_strength", 10000.0)),
                radius=f32(num_or(t, "contact_radius", num_or(t, "contact_factor", 2.0) * float(h))),
                friction=f32(num_or(t, "friction", 0.0)), dampening=f32(num_or(t, "dampening", 0.0)),
                potential=POTENTIALS.get(t.get("potential"), 2))


def load(path):
    """The scene as dicts and arrays: particles/boundary as field arrays in
    material order, materials as field dicts, interactions as an m x m list of
    dicts or None."""
    with open(path, "rb") as fh:
        top = tomllib.load(fh)
    h = f32(num_or(top, "kernel_radius", 1.0 / 64.0))
    alpha = f32(num_or(top, "artificial_viscocity", 50.0))
    scene = dict(name=top.get("name", "Fluid Test"), h=h, dt=f32(num_or(top, "time_step", 0.01)),
                 subticks=int(top.get("subticks", 1)), alpha=alpha, gravity=f32(num_or(top, "gravity", 1.0)),
                 bounds_min=vec4_or(top, "min", [-1, -1, 0, 0]), bounds_dim=vec4_or(top, "dim", [2, 2, 0, 0]))
    name = str(top.get("integrator", "verlet")).lower()
    if name not in INTEGRATORS:
        raise SceneError("invalid integrator")
    scene["integrator"] = INTEGRATORS[name]

    objs = [(k, v, True) for k, v in sorted(top.get("boundaries", {}).items())]
    objs += [(k, v, False) for k, v in sorted(top.get("objects", {}).items()) if "on_click" not in v]
    inter_map = {}
    mats, parts = [], {True: [], False: []}
    def seed(t, boundary):
        m = dict.fromkeys(MATERIAL_FIELDS, 0)
        vel_fn = None
        if boundary:
            m.update(visc=f32(num_or(t, "friction", 0.0)), start_den=f32(1.0), target_den=f32(1.0), immobile=1)
        else:
            m["start_den"] = f32(num_or(t, "start_density", num_or(t, "density", 1.0)))
            m["target_den"] = f32(num_or(t, "target_density", num_or(t, "density", 1.0)))
            m["sound_speed"] = f32(num_or(t, "speed_of_sound", 0.0))
            m["visc"] = f32(num_or(t, "viscocity", num_or(t, "friction", 0.0)))
            m["bulk_visc"] = f32(num_or(t, "bulk_viscocity", float(f32(alpha * h) * m["sound_speed"])))
            st = t.get("state", t.get("state_equation"))
            if st is None:
                if "speed_of_sound" in t:
                    st_id = 2 if ("start_density" in t or "target_density" in t) else 3
                else:
                    st_id = 0
            elif st in ("Tait", "tait", "Liquid", "liquid"):
                st_id = 3
            elif st in ("Ideal_Gas", "ideal_gas", "gas", "Gas"):
                st_id = 2
            elif st in ("Constant", "constant"):
                st_id = 1
            else:
                raise SceneError("invalid state equation")
            m["state_eq"] = st_id
            m["strain_order"] = int(t.get("strain_order", 2))
            for key, fld in (("normal_stiffness", "normal_stiffness"), ("shear_stiffness", "shear_stiffness"),
                             ("normal_dampening", "normal_damp"), ("shear_dampening", "shear_damp")):
                m[fld] = f32(num_or(t, key, 0.0))
            if "yield_strength" in t or "relaxation_time" in t:
                m.update(plastic=1, yield_strength=f32(num_or(t, "yield_strength", 0.0)),
                         work_hardening=f32(num_or(t, "work_hardening", 0.0)),
                         work_hardening_exp=f32(num_or(t, "work_hardening_exp", 2.0)),
                         kinematic_hardening=f32(num_or(t, "kinematic_hardening", 0.0)),
                         thermal_softening=f32(num_or(t, "thermal_softening", 0.0)),
                         relaxation_time=f32(num_or(t, "relaxation_time", 1.0)))
        region = region_from_mat(t)
        if not boundary:
            w = np.zeros(6, f32)
            for i, v in enumerate(t.get("angular_velocity", [])[:6]):
                w[i] = f32(_num(v))
            bmin, bdim = region.bound()
            vel_fn = _velocity_fn(vec4_or(t, "velocity", [0, 0, 0, 0]), w, bmin + f32(0.5) * bdim)
        packing = f32(num_or(t, "packing", num_or(t, "spacing", 0.5 * float(h)) / float(h)))
        pos, vel, mass = gen_particles(region, packing, h, m["start_den"], vel_fn)
        m["mass"] = mass
        return m, pos, vel

    for idx, (oname, t, boundary) in enumerate(objs):
        m, pos, vel = seed(t, boundary)
        mats.append(m)
        parts[boundary].append(dict(pos=pos, vel=vel, den=np.full(len(pos), m["start_den"], f32),
                                    mat=np.full(len(pos), idx, np.uint32)))
        for k2, v2 in t.items():
            if isinstance(v2, dict) and k2 not in ("region", "union", "intersection", "difference"):
                inter_map[(oname, k2)] = _interaction(v2, h)
    names = [o[0] for o in objs]
    inter = [[inter_map.get((a, b), inter_map.get((b, a))) for b in names] for a in names]

    for flag, key in ((False, "particles"), (True, "boundary")):
        lst = parts[flag]
        scene[key] = dict(pos=np.concatenate([d["pos"] for d in lst]) if lst else np.zeros((0, 4), f32),
                          vel=np.concatenate([d["vel"] for d in lst]) if lst else np.zeros((0, 4), f32),
                          den=np.concatenate([d["den"] for d in lst]) if lst else np.zeros(0, f32),
                          mat=np.concatenate([d["mat"] for d in lst]) if lst else np.zeros(0, np.uint32))
    scene["materials"] = mats
    scene["interactions"] = inter
    scene["on_click"] = []
    for oname, t in sorted(top.get("objects", {}).items()):
        if "on_click" in t:
            m, pos, vel = seed(t, False)
            scene["on_click"].append(dict(name=oname, material=m, pos=pos, vel=vel,
                                          den=np.full(len(pos), m["start_den"], f32),
                                          relative=t["on_click"] == "Relative"))
    return scene
