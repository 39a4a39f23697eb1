"""The allocation-free grid build, called through the C ABI.

arp_grid_build_noalloc serves callers that cannot call cudaMalloc on this
path (a host framework that owns the device allocator, or a real-time loop
that forbids allocation after start-up): they pass device inputs and outputs they already own, and the call keeps its
scratch in a fixed device array inside the library.  Its output must equal
the grid that the handle-based entry point (arp_sim_neighbors) reports for
the same positions, bit for bit, on consecutive calls that reuse the shared
scratch.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from arphys import FluidSim, scenes
from arphys.abi import ArpAABB, load_library

pytestmark = pytest.mark.gpu


def _bounds(sc):
    b = ArpAABB()
    for i in range(4):
        b.min[i] = float(sc.bounds_min[i])
        b.dim[i] = float(sc.bounds_dim[i])
    return b


def _noalloc_grid(lib, torch, pos_host, sc, nc):
    n = len(pos_host)
    pos = torch.tensor(np.ascontiguousarray(pos_host, dtype=np.float32), device="cuda")
    cell_start = torch.full((nc + 2,), -1, dtype=torch.int32, device="cuda")
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    b = _bounds(sc)
    code = lib.arp_grid_build_noalloc(pos.data_ptr(), n, ctypes.byref(b), float(np.float32(sc.h)),
                                      cell_start.data_ptr(), nc + 2, perm.data_ptr(), stream.cuda_stream)
    assert code == 0, lib.arp_last_error()
    torch.cuda.synchronize()
    return cell_start.cpu().numpy().view(np.uint32), perm.cpu().numpy().view(np.uint32)


def test_noalloc_grid_matches_the_handle_entry_point():
    torch = pytest.importorskip("torch")
    lib = load_library()
    sc = scenes.small_fluid_bar_3d()
    sim = FluidSim(sc)
    sim.init()
    _, nc = sim.grid()
    for call in range(2):  # two calls in a row share the library's scratch array
        sim.step(3)
        ref = sim.neighbors()
        p = sim.particles()
        start, perm = _noalloc_grid(lib, torch, p["pos"], sc, nc)
        np.testing.assert_array_equal(start[:nc + 1], ref["cell_start"])
        assert start[nc + 1] == sc.n  # the last entry closes the non-finite range
        np.testing.assert_array_equal(perm, ref["members"])


def _expected_grid(pos, bmin, bdim, h):
    """The grid a stable counting sort gives: cell of every particle by the
    reference's hash (every operation rounded to f32), members ascending."""
    f32 = np.float32
    sub = [max(1, int(max(f32(1.0), f32(bdim[a]) / f32(h)))) for a in range(3)]
    nc = sub[0] * sub[1] * sub[2]
    p = pos[:, :3].astype(np.float32)
    finite = np.isfinite(p).all(axis=1)
    key = np.full(len(p), nc, np.int64)
    c = np.zeros((len(p), 3), np.int64)
    with np.errstate(invalid="ignore"):
        for a in range(3):
            t = (p[:, a] - f32(bmin[a])) / f32(bdim[a])
            t = np.clip(t, f32(0.0), f32(1.0)) * f32(sub[a])
            c[:, a] = np.minimum(np.floor(np.where(finite, t, 0)).astype(np.int64), sub[a] - 1)
    key[finite] = (c[:, 0] + c[:, 1] * sub[0] + c[:, 2] * sub[0] * sub[1])[finite]
    perm = np.argsort(key, kind="stable").astype(np.uint32)
    start = np.searchsorted(key[perm], np.arange(nc + 2)).astype(np.uint32)
    return nc, start, perm


def test_noalloc_grid_orders_long_runs():
    """Cells holding more particles than one thread sorts (150: one warp;
    700 and a 300-long non-finite run: the block in shared memory; 5,000: the
    block through scratch) still list their members ascending, the same on
    every call."""
    torch = pytest.importorskip("torch")
    lib = load_library()
    rng = np.random.default_rng(8)
    parts = [np.array([0.2, 0.3, 0.4]) + 0.1 * rng.uniform(0.05, 0.95, size=(5000, 3)),
             np.array([0.5, 0.5, 0.5]) + 0.1 * rng.uniform(0.05, 0.95, size=(700, 3)),
             np.array([0.7, 0.2, 0.6]) + 0.1 * rng.uniform(0.05, 0.95, size=(150, 3)),
             rng.uniform(0.0, 1.0, size=(1500, 3)),
             np.full((300, 3), np.nan)]
    xyz = np.concatenate(parts)[rng.permutation(7650)]
    pos = np.zeros((len(xyz), 4), np.float32)
    pos[:, :3] = xyz
    sc = scenes.Scene(particles=None, boundary=None, materials=None, bounds_min=(0.0, 0.0, 0.0, 0.0),
                      bounds_dim=(1.0, 1.0, 1.0, 0.0), h=0.1)
    nc, start_ref, perm_ref = _expected_grid(pos, sc.bounds_min, sc.bounds_dim, sc.h)
    assert np.diff(start_ref).max() >= 5000  # past the 4096 a block sorts in shared memory
    for call in range(2):
        start, perm = _noalloc_grid(lib, torch, pos, sc, nc)
        np.testing.assert_array_equal(start, start_ref)
        np.testing.assert_array_equal(perm, perm_ref)


def test_noalloc_grid_rejects_sizes_beyond_its_maximum():
    lib = load_library()
    sc = scenes.small_fluid_bar_3d()
    b = _bounds(sc)
    dummy = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    code = lib.arp_grid_build_noalloc(dummy, (1 << 20) + 1, ctypes.byref(b), float(np.float32(sc.h)), dummy,
                                      1 << 22, dummy, None)
    assert code == 10
    assert b"1048576" in lib.arp_last_error()
    code = lib.arp_grid_build_noalloc(dummy, 16, ctypes.byref(b), float(np.float32(sc.h)), dummy, 3, dummy, None)
    assert code == 10 and b"n_cells + 2" in lib.arp_last_error()
