"""ctypes / numpy mirror of include/arphys.h.

The record dtypes are the reference's std430 layouts (`Particle`,
`SolidParticle`, `Material`, `MatInteraction`, src/soft_body/particle_state/
mod.rs:24-35, src/soft_body/material_region/material.rs:11-28,
interaction.rs:10-14), so host arrays built here cross the C ABI unchanged.
"""
import ctypes
import os

import numpy as np

INVALID = 0xFFFFFFFF

PARTICLE_DTYPE = np.dtype([
    ("den", "<f4"), ("mat", "<u4"), ("solid_id", "<u4"), ("_pad0", "<u4"),
    ("pos", "<f4", (4,)), ("vel", "<f4", (4,)),
])
SOLID_DTYPE = np.dtype([
    ("part_id", "<u4"), ("_pad0", "<u4", (3,)), ("ref_pos", "<f4", (4,)), ("stress", "<f4", (16,)),
])
MATERIAL_DTYPE = np.dtype([
    ("immobile", "<u4"), ("mass", "<f4"), ("start_den", "<f4"),
    ("state_eq", "<u4"), ("sound_speed", "<f4"), ("target_den", "<f4"), ("visc", "<f4"), ("bulk_visc", "<f4"),
    ("strain_order", "<i4"), ("normal_stiffness", "<f4"), ("shear_stiffness", "<f4"),
    ("normal_damp", "<f4"), ("shear_damp", "<f4"),
    ("plastic", "<u4"), ("yield_strength", "<f4"), ("work_hardening", "<f4"), ("work_hardening_exp", "<f4"),
    ("kinematic_hardening", "<f4"), ("thermal_softening", "<f4"), ("relaxation_time", "<f4"),
])
INTERACTION_DTYPE = np.dtype([
    ("potential", "<u4"), ("strength", "<f4"), ("radius", "<f4"), ("dampening", "<f4"), ("friction", "<f4"),
])
assert PARTICLE_DTYPE.itemsize == 48 and SOLID_DTYPE.itemsize == 96
assert MATERIAL_DTYPE.itemsize == 80 and INTERACTION_DTYPE.itemsize == 20

EOS_ZERO, EOS_CONSTANT, EOS_IDEAL_GAS, EOS_TAIT = 0, 1, 2, 3
CONTACT_ZERO, CONTACT_CONSTANT, CONTACT_LINEAR, CONTACT_TAIT, CONTACT_LJ, CONTACT_HERTZ = range(6)

INTEGRATORS = {
    "euler": 0, "rk1": 0, "midpoint": 1, "rk2": 1, "heun2": 2, "heun": 2, "ralston": 3,
    "rk3": 4, "heun3": 5, "rk4": 6, "rk_3_8": 7, "verlet": 8,
}

STATUS = {
    0: "ARP_OK", 1: "ARP_ERR_INVALID_ARG", 2: "ARP_ERR_CUDA", 3: "ARP_ERR_NAN_STATE",
    4: "ARP_ERR_CELL_OVERFLOW", 5: "ARP_ERR_TIMEOUT", 6: "ARP_ERR_UNSUPPORTED",
    7: "ARP_ERR_OUT_OF_MEMORY", 8: "ARP_ERR_PARSE", 9: "ARP_ERR_IO", 10: "ARP_ERR_CAPACITY",
}


class ArpAABB(ctypes.Structure):
    _fields_ = [("min", ctypes.c_float * 4), ("dim", ctypes.c_float * 4)]


class ArpScene(ctypes.Structure):
    _fields_ = [
        ("particles", ctypes.c_void_p), ("n_particles", ctypes.c_uint32),
        ("boundary", ctypes.c_void_p), ("n_boundary", ctypes.c_uint32),
        ("materials", ctypes.c_void_p), ("n_materials", ctypes.c_uint32),
        ("interactions", ctypes.c_void_p), ("interaction_given", ctypes.c_void_p),
        ("bounds", ArpAABB), ("kernel_radius", ctypes.c_float), ("integrator", ctypes.c_int32),
        ("timestep", ctypes.c_float), ("subticks", ctypes.c_uint32), ("gravity", ctypes.c_float),
        ("artificial_viscocity", ctypes.c_float),
    ]


class ArpView(ctypes.Structure):
    _fields_ = [("angle", ctypes.c_float), ("pos", ctypes.c_float * 2), ("scale", ctypes.c_float)]


class ArpRenderStyle(ctypes.Structure):
    _fields_ = [
        ("render_h", ctypes.c_float), ("lighting", ctypes.c_int32), ("light_pos", ctypes.c_float * 3),
        ("light_color", ctypes.c_float * 3), ("ambient", ctypes.c_float), ("diffuse", ctypes.c_float),
        ("specular", ctypes.c_float), ("n_materials", ctypes.c_uint32), ("colors", ctypes.c_void_p),
        ("densities", ctypes.c_void_p),
    ]


class ArpProfile(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_uint64), ("launches", ctypes.c_uint64),
        ("neighbor_ms", ctypes.c_double), ("solid_ms", ctypes.c_double), ("fluid_ms", ctypes.c_double),
        ("integrate_ms", ctypes.c_double), ("fluid_launches", ctypes.c_uint64),
        ("neighbor_launches", ctypes.c_uint64), ("solid_launches", ctypes.c_uint64), ("stages", ctypes.c_uint64),
    ]


class ArpStats(ctypes.Structure):
    _fields_ = [
        ("max_cell_occupancy", ctypes.c_uint32), ("overflow_cells", ctypes.c_uint32),
        ("nonfinite_positions", ctypes.c_uint32), ("clamped_coordinates", ctypes.c_uint32),
    ]


class ArpDeviceView(ctypes.Structure):
    _fields_ = [("pos_den", ctypes.c_void_p), ("vel_mat", ctypes.c_void_p), ("orig_id", ctypes.c_void_p),
                ("n", ctypes.c_uint32)]


def ptr(a):
    """Address of a C-contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def scene_struct(scene):
    """Fill an ArpScene from a `Scene`; the returned tuple keeps the arrays alive."""
    s = ArpScene()
    keep = []
    p = np.ascontiguousarray(scene.particles, dtype=PARTICLE_DTYPE)
    b = np.ascontiguousarray(scene.boundary, dtype=PARTICLE_DTYPE)
    m = np.ascontiguousarray(scene.materials, dtype=MATERIAL_DTYPE)
    keep += [p, b, m]
    s.particles, s.n_particles = ptr(p), len(p)
    s.boundary, s.n_boundary = (ptr(b) if len(b) else None), len(b)
    s.materials, s.n_materials = ptr(m), len(m)
    if scene.interactions is not None:
        it = np.ascontiguousarray(scene.interactions, dtype=INTERACTION_DTYPE).reshape(-1)
        keep.append(it)
        s.interactions = ptr(it)
        if scene.interaction_given is not None:
            gv = np.ascontiguousarray(scene.interaction_given, dtype=np.uint8).reshape(-1)
            keep.append(gv)
            s.interaction_given = ptr(gv)
    for i in range(4):
        s.bounds.min[i] = float(scene.bounds_min[i])
        s.bounds.dim[i] = float(scene.bounds_dim[i])
    s.kernel_radius = scene.h
    s.integrator = INTEGRATORS[scene.integrator] if isinstance(scene.integrator, str) else int(scene.integrator)
    s.timestep = scene.dt
    s.subticks = scene.subticks
    s.gravity = scene.gravity
    s.artificial_viscocity = scene.alpha
    return s, keep


_LIB = None


def lib_path():
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(os.path.dirname(here), "libarphys.so")


def load_library():
    """Load the in-tree libarphys.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError(f"libarphys.so not built at {path}: run `make -C ar-physics_b200` "
                           "(or __graft_entry__.build())")
    L = ctypes.CDLL(path)
    c_sim = ctypes.c_void_p
    u32p = ctypes.POINTER(ctypes.c_uint32)
    sig = {
        "arp_sim_create": [ctypes.POINTER(ArpScene), ctypes.POINTER(c_sim)],
        "arp_sim_create_from_toml": [ctypes.c_char_p, ctypes.POINTER(c_sim)],
        "arp_sim_init": [c_sim], "arp_sim_destroy": [c_sim], "arp_sim_update": [c_sim],
        "arp_sim_step": [c_sim, ctypes.c_uint32],
        "arp_sim_time": [c_sim, ctypes.POINTER(ctypes.c_float)],
        "arp_sim_kernel_radius": [c_sim, ctypes.POINTER(ctypes.c_float)],
        "arp_sim_num_materials": [c_sim, u32p],
        "arp_sim_counts": [c_sim, u32p, u32p, u32p],
        "arp_sim_dim": [c_sim, u32p],
        "arp_sim_get_particles": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_get_solids": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_get_boundary": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_get_materials": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_get_interactions": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_set_particles": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_set_particles_async": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_get_particles_async": [c_sim, ctypes.c_void_p, ctypes.c_uint32],
        "arp_sim_device_state": [c_sim, ctypes.POINTER(ArpDeviceView)],
        "arp_sim_add_particles": [c_sim, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.POINTER(ctypes.c_int)],
        "arp_sim_grid": [c_sim, ctypes.c_void_p, u32p],
        "arp_sim_neighbors": [c_sim, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
        "arp_sim_boundary_cells": [c_sim, ctypes.c_void_p, ctypes.c_void_p],
        "arp_sim_set_stream": [c_sim, ctypes.c_void_p],
        "arp_sim_synchronize": [c_sim],
        "arp_sim_profile_enable": [c_sim, ctypes.c_int],
        "arp_sim_profile_read": [c_sim, ctypes.POINTER(ArpProfile)],
        "arp_sim_stats": [c_sim, ctypes.POINTER(ArpStats)],
        "arp_sim_launch_count": [c_sim, ctypes.POINTER(ctypes.c_uint64)],
    }
    sig["arp_sim_create_batch"] = [ctypes.POINTER(ArpScene), ctypes.c_uint32, ctypes.POINTER(c_sim)]
    sig["arp_sim_num_scenes"] = [c_sim, u32p]
    sig["arp_sim_set_graph"] = [c_sim, ctypes.c_int]
    sig["arp_sim_autotune"] = [c_sim, ctypes.POINTER(ctypes.c_int)]
    sig["arp_sim_set_fluid_variant"] = [c_sim, ctypes.c_int]
    sig["arp_fluid_variant_count"] = []
    sig["arp_sim_fluid_variant"] = [c_sim, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]
    sig["arp_sim_scene_range"] = [c_sim, ctypes.c_uint32, u32p, u32p, u32p, u32p, u32p, u32p]
    sig["arp_grid_build_noalloc"] = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ArpAABB), ctypes.c_float,
                                     ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    sig["arp_scene_file_load"] = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]
    sig["arp_scene_file_scene"] = [ctypes.c_void_p, ctypes.POINTER(ArpScene)]
    sig["arp_scene_file_name"] = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p)]
    sig["arp_scene_file_free"] = [ctypes.c_void_p]
    sig["arp_scene_file_on_click_count"] = [ctypes.c_void_p, u32p]
    sig["arp_scene_file_on_click"] = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), u32p,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    sig["arp_sim_set_solid_stiffness"] = [c_sim, ctypes.c_void_p, ctypes.c_uint32]
    sig["arp_sim_render_rgb24"] = [c_sim, ctypes.POINTER(ArpView), ctypes.POINTER(ArpRenderStyle), ctypes.c_uint32,
                                   ctypes.c_uint32, ctypes.c_void_p]
    sig["arp_scene_file_render_settings"] = [ctypes.c_void_p, ctypes.POINTER(ArpView), ctypes.POINTER(ArpRenderStyle)]
    sig["arp_tape_begin"] = [c_sim, ctypes.c_uint32]
    sig["arp_tape_end"] = [c_sim]
    sig["arp_tape_steps"] = [c_sim, ctypes.POINTER(ctypes.c_uint64)]
    sig["arp_tape_backward"] = [c_sim, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.arp_last_error.restype = ctypes.c_char_p
    L.arp_last_error.argtypes = []
    L.arp_abi_version.restype = ctypes.c_uint32
    L.arp_abi_version.argtypes = []
    _LIB = L
    return L


class ArpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def check(code):
    if code != 0:
        msg = load_library().arp_last_error().decode(errors="replace")
        raise ArpError(code, msg)
