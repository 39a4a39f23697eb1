"""`FluidSim` over the C ABI, with the reference's method names
(src/soft_body/mod.rs:45-274): new, init, update, particles, time,
kernel_radius, num_materials, add_particles.  Errors raise `ArpError`
carrying the library's status code and message (the reference returns
`GLError` from `new` and panics elsewhere)."""
import ctypes

import numpy as np

from .abi import (PARTICLE_DTYPE, SOLID_DTYPE, MATERIAL_DTYPE, INTERACTION_DTYPE, ArpProfile, ArpStats,
                  ArpDeviceView, check, load_library, ptr, scene_struct)


class FluidSim:
    def __init__(self, scene=None, _handle=None):
        self._L = load_library()
        if _handle is not None:
            self._h = _handle
        else:
            sc, keep = scene_struct(scene)
            h = ctypes.c_void_p()
            check(self._L.arp_sim_create(ctypes.byref(sc), ctypes.byref(h)))
            self._h = h
        self._refresh_counts()

    @classmethod
    def new(cls, scene):
        """FluidSim::new (mod.rs:58-166)."""
        return cls(scene)

    @classmethod
    def batch(cls, scenes):
        """Several independent scenes stepped together (arp_sim_create_batch)."""
        from .abi import ArpScene
        L = load_library()
        structs, keep = [], []
        for sc in scenes:
            st, k = scene_struct(sc)
            structs.append(st)
            keep.append(k)
        arr = (ArpScene * len(structs))(*structs)
        h = ctypes.c_void_p()
        check(L.arp_sim_create_batch(arr, len(structs), ctypes.byref(h)))
        return cls(_handle=h)

    def num_scenes(self):
        t = ctypes.c_uint32()
        check(self._L.arp_sim_num_scenes(self._h, ctypes.byref(t)))
        return t.value

    def scene_range(self, k):
        """(first_particle, n_particles, first_boundary, n_boundary, first_cell, n_cells) of scene k."""
        v = [ctypes.c_uint32() for _ in range(6)]
        check(self._L.arp_sim_scene_range(self._h, int(k), *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    @classmethod
    def from_toml(cls, path):
        L = load_library()
        h = ctypes.c_void_p()
        check(L.arp_sim_create_from_toml(str(path).encode(), ctypes.byref(h)))
        return cls(_handle=h)

    def _refresh_counts(self):
        n, nb, ns = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(self._L.arp_sim_counts(self._h, ctypes.byref(n), ctypes.byref(nb), ctypes.byref(ns)))
        self.n, self.nb, self.ns = n.value, nb.value, ns.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.arp_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        """FluidSim::init (mod.rs:213-233)."""
        check(self._L.arp_sim_init(self._h))

    def update(self):
        """FluidSim::update (mod.rs:235-274): `subticks` steps."""
        check(self._L.arp_sim_update(self._h))

    def step(self, n=1):
        check(self._L.arp_sim_step(self._h, int(n)))

    def time(self):
        t = ctypes.c_float()
        check(self._L.arp_sim_time(self._h, ctypes.byref(t)))
        return t.value

    def kernel_radius(self):
        t = ctypes.c_float()
        check(self._L.arp_sim_kernel_radius(self._h, ctypes.byref(t)))
        return t.value

    def num_materials(self):
        t = ctypes.c_uint32()
        check(self._L.arp_sim_num_materials(self._h, ctypes.byref(t)))
        return t.value

    def dim(self):
        t = ctypes.c_uint32()
        check(self._L.arp_sim_dim(self._h, ctypes.byref(t)))
        return t.value

    def particles(self, out=None):
        """Mobile particle records in caller order (FluidSim::particles)."""
        if out is None:
            out = np.zeros(self.n, dtype=PARTICLE_DTYPE)
        check(self._L.arp_sim_get_particles(self._h, ptr(out), len(out)))
        return out

    def solids(self):
        out = np.zeros(self.ns, dtype=SOLID_DTYPE)
        if self.ns:
            check(self._L.arp_sim_get_solids(self._h, ptr(out), len(out)))
        return out

    def boundary(self):
        out = np.zeros(self.nb, dtype=PARTICLE_DTYPE)
        if self.nb:
            check(self._L.arp_sim_get_boundary(self._h, ptr(out), len(out)))
        return out

    def materials(self):
        out = np.zeros(self.num_materials(), dtype=MATERIAL_DTYPE)
        check(self._L.arp_sim_get_materials(self._h, ptr(out), len(out)))
        return out

    def interactions(self):
        """The n_materials^2 interaction block of a single scene (all blocks,
        flat, for a batch)."""
        m = self.num_materials()
        cap = max(m * m, 1) if self.num_scenes() == 1 else 32 * 32 * self.num_scenes()
        out = np.zeros(cap, dtype=INTERACTION_DTYPE)
        check(self._L.arp_sim_get_interactions(self._h, ptr(out), len(out)))
        return out.reshape(m, m) if self.num_scenes() == 1 else out

    def set_particles(self, p):
        p = np.ascontiguousarray(p, dtype=PARTICLE_DTYPE)
        check(self._L.arp_sim_set_particles(self._h, ptr(p), len(p)))

    def set_particles_async(self, p):
        """arp_sim_set_particles_async: `p` (a contiguous Particle record
        array, page-locked for a truly asynchronous copy) must stay unchanged
        until synchronize()."""
        if p.dtype != PARTICLE_DTYPE or not p.flags["C_CONTIGUOUS"]:
            raise ValueError("set_particles_async needs a contiguous Particle record array")
        check(self._L.arp_sim_set_particles_async(self._h, ptr(p), len(p)))

    def particles_async(self, out):
        """arp_sim_get_particles_async: `out` (a contiguous Particle record
        array) holds the records after synchronize()."""
        if out.dtype != PARTICLE_DTYPE or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("particles_async needs a contiguous Particle record array")
        check(self._L.arp_sim_get_particles_async(self._h, ptr(out), len(out)))
        return out

    def add_particles(self, p, material, offset=None):
        """FluidSim::add_particles (mod.rs:180-206); returns True when a
        material entry was appended."""
        p = np.ascontiguousarray(p, dtype=PARTICLE_DTYPE)
        m = np.ascontiguousarray(np.asarray(material, dtype=MATERIAL_DTYPE).reshape(1))
        off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float32)
        added = ctypes.c_int(0)
        check(self._L.arp_sim_add_particles(self._h, ptr(p), len(p), ptr(m), ptr(off), ctypes.byref(added)))
        self._refresh_counts()
        return bool(added.value)

    def grid(self):
        sub = np.zeros(4, np.uint32)
        nc = ctypes.c_uint32()
        check(self._L.arp_sim_grid(self._h, ptr(sub), ctypes.byref(nc)))
        return sub, nc.value

    def neighbors(self):
        _, nc = self.grid()
        cell_of = np.zeros(self.n, np.uint32)
        start = np.zeros(nc + 1, np.uint32)
        members = np.zeros(max(self.n, 1), np.uint32)
        nbr = np.zeros(self.n, np.uint32)
        check(self._L.arp_sim_neighbors(self._h, ptr(cell_of), ptr(start), ptr(members), ptr(nbr)))
        return dict(cell_of=cell_of, cell_start=start, members=members[:self.n], nbr_count=nbr)

    def boundary_cells(self):
        _, nc = self.grid()
        start = np.zeros(nc + 1, np.uint32)
        members = np.zeros(max(self.nb, 1), np.uint32)
        check(self._L.arp_sim_boundary_cells(self._h, ptr(start), ptr(members)))
        return start, members[:self.nb]

    def set_graph(self, on=True):
        """Replay each step from a captured CUDA graph (one per alternating buffer set)."""
        check(self._L.arp_sim_set_graph(self._h, int(bool(on))))

    def autotune(self):
        v = ctypes.c_int()
        check(self._L.arp_sim_autotune(self._h, ctypes.byref(v)))
        return v.value

    @staticmethod
    def fluid_variant_count():
        """Number of launch shapes of the fluid kernel."""
        from .abi import load_library
        return int(load_library().arp_fluid_variant_count())

    def set_fluid_variant(self, v):
        check(self._L.arp_sim_set_fluid_variant(self._h, int(v)))

    def fluid_variant(self):
        v, blk, pers = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._L.arp_sim_fluid_variant(self._h, ctypes.byref(v), ctypes.byref(blk), ctypes.byref(pers)))
        return dict(variant=v.value, block=blk.value, persistent=bool(pers.value))

    def set_stream(self, stream_handle):
        check(self._L.arp_sim_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def synchronize(self):
        """Waits for the handle's device work and asynchronous copies and
        raises the record-check errors of asynchronous sets."""
        check(self._L.arp_sim_synchronize(self._h))

    def profile_enable(self, on=True, every=1):
        """Per-segment CUDA-event timing on one step in every `every`."""
        check(self._L.arp_sim_profile_enable(self._h, int(every) if on else 0))

    def profile_read(self):
        p = ArpProfile()
        check(self._L.arp_sim_profile_read(self._h, ctypes.byref(p)))
        return {k: getattr(p, k) for k, _ in ArpProfile._fields_}

    def stats(self):
        s = ArpStats()
        check(self._L.arp_sim_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in ArpStats._fields_}

    def launch_count(self):
        c = ctypes.c_uint64()
        check(self._L.arp_sim_launch_count(self._h, ctypes.byref(c)))
        return c.value

    def set_solid_stiffness(self, normal_shear):
        """Per-solid (normal, shear) stiffness, shape (ns, 2) in solid-id order
        (None restores the materials' values)."""
        if normal_shear is None:
            check(self._L.arp_sim_set_solid_stiffness(self._h, None, 0))
            return
        a = np.ascontiguousarray(normal_shear, dtype=np.float32).reshape(-1, 2)
        check(self._L.arp_sim_set_solid_stiffness(self._h, ptr(a), len(a)))

    def tape_begin(self, checkpoint_every=20):
        """Record the following steps for reverse-mode differentiation."""
        check(self._L.arp_tape_begin(self._h, int(checkpoint_every)))

    def tape_end(self):
        check(self._L.arp_tape_end(self._h))

    def tape_steps(self):
        t = ctypes.c_uint64()
        check(self._L.arp_tape_steps(self._h, ctypes.byref(t)))
        return t.value

    def backward(self, dl_dstate):
        """dL/d(state at tape begin) and dL/d(per-solid stiffness) from dL/d(current
        state); states are (n, 8) float arrays (x, y, z, rho, vx, vy, vz, 0) in
        caller order.  Returns (grad_state0 (n, 8), grad_stiffness (ns, 2))."""
        d = np.ascontiguousarray(dl_dstate, dtype=np.float32).reshape(self.n, 8)
        g = np.empty((self.n, 8), np.float32)  # written in full by the library
        gs = np.zeros((max(self.ns, 1), 2), np.float32)
        check(self._L.arp_tape_backward(self._h, ptr(d), ptr(g), ptr(gs)))
        return g, gs[:self.ns]

    def render(self, width, height, view, style):
        """One RGB24 frame (renderer.rs recording path) as a (height, width, 3)
        uint8 array, row 0 at the bottom as glReadnPixels returns it.
        `view`: dict(angle, pos, scale); `style`: dict(render_h, lighting,
        light_pos, light_color, ambient, diffuse, specular, colors (M x 12),
        densities (M))."""
        from .abi import ArpView, ArpRenderStyle
        v = ArpView()
        v.angle = float(view.get("angle", 0.0))
        v.pos[0], v.pos[1] = (float(x) for x in view.get("pos", (0.0, 0.0)))
        v.scale = float(view.get("scale", 1.0))
        colors = np.ascontiguousarray(style["colors"], dtype=np.float32).reshape(-1, 12)
        dens = np.ascontiguousarray(style["densities"], dtype=np.float32).reshape(-1)
        st = ArpRenderStyle()
        st.render_h = float(style["render_h"])
        st.lighting = int(bool(style.get("lighting", False)))
        for k in range(3):
            st.light_pos[k] = float(style.get("light_pos", (-3.0, 3.0, -3.0))[k])
            st.light_color[k] = float(style.get("light_color", (1.0, 1.0, 1.0))[k])
        st.ambient = float(style.get("ambient", 1.0))
        st.diffuse = float(style.get("diffuse", 10.0))
        st.specular = float(style.get("specular", 0.0))
        st.n_materials = len(colors)
        st.colors = ptr(colors)
        st.densities = ptr(dens)
        out = np.zeros((height, width, 3), np.uint8)
        check(self._L.arp_sim_render_rgb24(self._h, ctypes.byref(v), ctypes.byref(st), int(width), int(height),
                                           ptr(out)))
        return out

    def device_state(self):
        v = ArpDeviceView()
        check(self._L.arp_sim_device_state(self._h, ctypes.byref(v)))
        return dict(pos_den=v.pos_den, vel_mat=v.vel_mat, orig_id=v.orig_id, n=v.n)
