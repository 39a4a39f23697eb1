"""CPU checks of the C ABI: the in-tree library loads, exports every entry
point include/arphys.h declares, and rejects bad scenes before touching a
GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from arphys import scenes
from arphys.abi import (PARTICLE_DTYPE, SOLID_DTYPE, MATERIAL_DTYPE, INTERACTION_DTYPE, ArpScene, scene_struct,
                        load_library)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "arphys.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(arp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) > 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_record_layouts_match_std430():
    assert PARTICLE_DTYPE.itemsize == 48 and PARTICLE_DTYPE.fields["pos"][1] == 16
    assert PARTICLE_DTYPE.fields["vel"][1] == 32
    assert SOLID_DTYPE.itemsize == 96 and SOLID_DTYPE.fields["ref_pos"][1] == 16
    assert MATERIAL_DTYPE.itemsize == 80 and INTERACTION_DTYPE.itemsize == 20


def test_abi_version_and_error_string(lib):
    assert lib.arp_abi_version() == 1
    assert isinstance(lib.arp_last_error(), bytes)


def _create(lib, scene):
    sc, keep = scene_struct(scene)
    h = ctypes.c_void_p()
    code = lib.arp_sim_create(ctypes.byref(sc), ctypes.byref(h))
    return code, h, lib.arp_last_error().decode()


def test_null_scene_is_rejected(lib):
    h = ctypes.c_void_p()
    assert lib.arp_sim_create(None, ctypes.byref(h)) == 1
    assert b"null" in lib.arp_last_error()


def test_four_dimensional_box_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.bounds_dim = (0.2, 0.2, 0.0, 0.1)
    code, _, msg = _create(lib, sc)
    assert code == 6 and "4-dimensional" in msg


def test_mobile_particle_with_immobile_material_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.particles["mat"][0] = 0
    code, _, msg = _create(lib, sc)
    assert code == 1 and "immobile" in msg


def test_material_index_out_of_range_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.particles["mat"][1] = 7
    code, _, _ = _create(lib, sc)
    assert code == 1


def test_null_handle_calls_fail_cleanly(lib):
    t = ctypes.c_float()
    assert lib.arp_sim_time(None, ctypes.byref(t)) == 1
    assert lib.arp_sim_step(None, 1) == 1
    assert lib.arp_sim_set_particles_async(None, None, 0) == 1
    assert lib.arp_sim_get_particles_async(None, None, 0) == 1
    assert lib.arp_sim_synchronize(None) == 1
    assert lib.arp_sim_destroy(None) == 0


def test_noalloc_grid_rejects_a_grid_too_large_to_index(lib):
    """A kernel radius tiny against the box would make dim / h overflow a
    32-bit cell count; the call refuses it before touching the device."""
    from arphys.abi import ArpAABB
    b = ArpAABB()
    for i in range(3):
        b.dim[i] = 1.0
    dummy = ctypes.c_void_p(256)  # never dereferenced: the size checks come first
    for h in (1e-12, 2.0 ** -32, 1e-3):
        code = lib.arp_grid_build_noalloc(dummy, 16, ctypes.byref(b), ctypes.c_float(h), dummy, 1 << 22, dummy, None)
        assert code == 10, (h, lib.arp_last_error())
        assert b"4194302" in lib.arp_last_error()


def test_scene_with_a_grid_too_large_to_index_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.h = 1e-12
    code, _, msg = _create(lib, sc)
    assert code == 6 and "2^30" in msg


@pytest.mark.parametrize("h", [0.0, -0.02, float("nan"), float("inf")])
def test_kernel_radius_must_be_positive_and_finite(lib, h):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.h = h
    code, _, msg = _create(lib, sc)
    assert code == 1 and "kernel_radius" in msg


def test_non_finite_timestep_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.dt = float("nan")
    code, _, msg = _create(lib, sc)
    assert code == 1 and "timestep" in msg


def test_unknown_integrator_id_is_rejected(lib):
    s, keep = scene_struct(scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2)))
    s.integrator = 99
    h = ctypes.c_void_p()
    assert lib.arp_sim_create(ctypes.byref(s), ctypes.byref(h)) == 1
    assert b"integrator" in lib.arp_last_error()


def test_box_without_extent_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.bounds_dim = (0.0, 0.0, 0.0, 0.0)
    code, _, msg = _create(lib, sc)
    assert code == 1 and "extent" in msg


def test_velocity_with_a_w_component_is_rejected(lib):
    sc = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    sc.particles["vel"][2, 3] = 1.0
    code, _, msg = _create(lib, sc)
    assert code == 6 and "w component" in msg


def test_batch_scenes_must_share_the_time_step(lib):
    a = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    b = scenes.dam_break_2d(nx=4, ny=4, box=(0.2, 0.2))
    b.dt = a.dt * 2
    sa, ka = scene_struct(a)
    sb, kb = scene_struct(b)
    arr = (ArpScene * 2)(sa, sb)
    h = ctypes.c_void_p()
    assert lib.arp_sim_create_batch(arr, 2, ctypes.byref(h)) == 6
    assert b"share integrator" in lib.arp_last_error()
