"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg.  Parity unpinned (the reference has no golden
vectors); see oracle.cpp for the files it restates.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_step.argtypes = [vp, ctypes.c_uint32]
        L.orc_update.argtypes = [vp]
        L.orc_time.restype = ctypes.c_double
        L.orc_time.argtypes = [vp]
        L.orc_counts.argtypes = [vp, u32p, u32p, u32p, u32p, vp, u32p]
        L.orc_get_state.argtypes = [vp] * 8
        L.orc_set_state.argtypes = [vp] * 5
        L.orc_derivative.argtypes = [vp] * 5
        L.orc_strains.argtypes = [vp, vp]
        L.orc_buckets.argtypes = [vp] * 6
        L.orc_add_particles.argtypes = [vp, vp, ctypes.c_uint32, vp, vp, ctypes.POINTER(ctypes.c_int)]
        L.orc_materials.argtypes = [vp, u32p, vp, ctypes.c_uint32]
        L.orc_interactions.argtypes = [vp, vp]
        L.orc_set_solid_stiffness.argtypes = [vp, vp, ctypes.c_uint32]
        _L = L
    return _L


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """One oracle simulation in float (precision=32) or double (precision=64)."""

    def __init__(self, scene, precision=32, literal=False):
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(HERE), "ar-physics_b200"))
        from arphys.abi import scene_struct
        self._sc, self._keep = scene_struct(scene)
        err = ctypes.create_string_buffer(256)
        self.h = lib().orc_create(ctypes.byref(self._sc), precision, int(literal), err, 256)
        if not self.h:
            raise RuntimeError("oracle: " + err.value.decode())
        self.precision = precision
        n, nb, ns, nc, dim = (ctypes.c_uint32() for _ in range(5))
        sub = np.zeros(4, np.uint32)
        lib().orc_counts(self.h, ctypes.byref(n), ctypes.byref(nb), ctypes.byref(ns), ctypes.byref(nc),
                         _p(sub), ctypes.byref(dim))
        self.n, self.nb, self.ns, self.ncells, self.dim = n.value, nb.value, ns.value, nc.value, dim.value
        self.sub = sub

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def step(self, n=1):
        lib().orc_step(self.h, n)

    def update(self):
        lib().orc_update(self.h)

    @property
    def time(self):
        return lib().orc_time(self.h)

    def _refresh_counts(self):
        n, nb, ns, nc, dim = (ctypes.c_uint32() for _ in range(5))
        lib().orc_counts(self.h, ctypes.byref(n), ctypes.byref(nb), ctypes.byref(ns), ctypes.byref(nc),
                         _p(self.sub), ctypes.byref(dim))
        self.n, self.nb, self.ns = n.value, nb.value, ns.value

    def add_particles(self, particles, material, offset=None):
        """FluidSim::add_particles (src/soft_body/mod.rs:180-206); returns True
        when a material entry was appended."""
        from arphys.abi import PARTICLE_DTYPE, MATERIAL_DTYPE
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        m = np.ascontiguousarray(np.asarray(material, dtype=MATERIAL_DTYPE).reshape(1))
        off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float32)
        added = ctypes.c_int(0)
        lib().orc_add_particles(self.h, _p(p), len(p), _p(m), _p(off), ctypes.byref(added))
        self._refresh_counts()
        return bool(added.value)

    def set_solid_stiffness(self, normal_shear):
        """Per-solid (normal, shear) stiffness overriding the materials' (None clears)."""
        if normal_shear is None:
            lib().orc_set_solid_stiffness(self.h, None, 0)
            return
        a = np.ascontiguousarray(normal_shear, dtype=np.float64).reshape(-1, 2)
        lib().orc_set_solid_stiffness(self.h, _p(a), len(a))

    def materials(self):
        from arphys.abi import MATERIAL_DTYPE
        cnt = ctypes.c_uint32()
        lib().orc_materials(self.h, ctypes.byref(cnt), None, 0)
        out = np.zeros(cnt.value, dtype=MATERIAL_DTYPE)
        lib().orc_materials(self.h, ctypes.byref(cnt), _p(out), cnt.value)
        return out

    def interactions(self):
        m = len(self.materials())
        out = np.zeros((m, m, 5))
        lib().orc_interactions(self.h, _p(out))
        return out

    def state(self):
        den = np.zeros(self.n)
        pos = np.zeros((self.n, 4))
        vel = np.zeros((self.n, 4))
        mat = np.zeros(self.n, np.uint32)
        sid = np.zeros(self.n, np.uint32)
        ref = np.zeros((self.ns, 4))
        pl = np.zeros((self.ns, 16))
        lib().orc_get_state(self.h, _p(den), _p(pos), _p(vel), _p(mat), _p(sid), _p(ref), _p(pl))
        return dict(den=den, pos=pos, vel=vel, mat=mat, solid_id=sid, ref_pos=ref, plastic=pl)

    def set_state(self, den=None, pos=None, vel=None, plastic=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        den, pos, vel, plastic = f(den), f(pos), f(vel), f(plastic)
        lib().orc_set_state(self.h, _p(den), _p(pos), _p(vel), _p(plastic))

    def derivative(self):
        d = dict(den=np.zeros(self.n), pos=np.zeros((self.n, 4)), vel=np.zeros((self.n, 4)),
                 plastic=np.zeros((self.ns, 16)))
        lib().orc_derivative(self.h, _p(d["den"]), _p(d["pos"]), _p(d["vel"]), _p(d["plastic"]))
        return d

    def strains(self):
        out = np.zeros((self.ns, 3, 16))
        lib().orc_strains(self.h, _p(out))
        return out

    def buckets(self):
        counts = np.zeros((self.ncells, 3), np.uint32)
        contents = np.zeros((self.ncells, 128), np.uint32)
        pos_index = np.zeros(self.n, np.uint32)
        ref_index = np.zeros(self.n, np.uint32)
        nbr = np.zeros(self.n, np.uint32)
        lib().orc_buckets(self.h, _p(counts), _p(contents), _p(pos_index), _p(ref_index), _p(nbr))
        return dict(counts=counts, contents=contents, pos_index=pos_index, ref_index=ref_index, nbr_count=nbr)


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def poly6(dim, h, r):
    """W and grad W of the poly6 kernel for displacement rows r (n x 4)."""
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 4)
    n = len(r)
    w = np.zeros(n)
    gw = np.zeros((n, 4))
    k = ctypes.c_double()
    L = lib()
    L.orc_poly6.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p]
    L.orc_poly6(int(dim), float(h), _p(r), n, _p(w), _p(gw), ctypes.byref(k))
    return w, gw, k.value


def norm_const_f32(dim, h):
    L = lib()
    L.orc_norm_const_f32.restype = ctypes.c_float
    L.orc_norm_const_f32.argtypes = [ctypes.c_int, ctypes.c_float]
    return L.orc_norm_const_f32(int(dim), float(h))
