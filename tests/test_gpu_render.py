"""Headless rendering (arp_sim_render_rgb24) against the CPU restatement of the
demo renderer's recording path (oracle/render_oracle.py).

Splat mode composites sprites in draw order with 8-bit rounding after every
blend; every operation of the coverage, colour and blend arithmetic is
rounded the same way on both sides, so the frames must be equal byte for
byte.  The lit mode's sphere shading uses contracted multiply-adds on the
GPU: there the bound is one 8-bit level, on every pixel.
"""
import os

import numpy as np
import pytest

from arphys import FluidSim, scenes
from oracle import render_oracle
from oracle.oracle import norm_const_f32

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def style_for(sc, lighting=False, render_h=None):
    m = len(sc.materials)
    colors = np.zeros((m, 12), np.float32)
    rng = np.random.default_rng(1)
    for k in range(m):
        base = np.append(rng.random(3), 1.0)
        colors[k] = np.concatenate([base, [0.1, 0.2, 0.9, 1.0], [0.9, 0.2, 0.1, 0.8]])
    return dict(render_h=render_h or 4.0 * sc.h, lighting=lighting, colors=colors,
                densities=sc.materials["start_den"].astype(np.float32), light_pos=(-0.5, 1.5, -2.0),
                light_color=(1.0, 0.9, 0.8), ambient=0.8, diffuse=2.0, specular=0.5)


def oracle_frame(sim, view, style, w, h):
    return render_oracle.render(sim.boundary(), sim.particles(), view, style, w, h, norm_const_f32(3, 3.0))


@pytest.mark.parametrize("w,h", [(160, 120), (96, 200)])
def test_splat_frames_match_the_oracle(w, h):
    sc = scenes.dam_break_2d(nx=24, ny=24, box=(0.64, 0.32))
    sim = FluidSim(sc)
    sim.init()
    view = dict(angle=0.0, pos=(0.32, -0.16), scale=1.45)  # clip w = 0.55: a 1.8x zoom on the box
    style = style_for(sc)
    for k in range(2):
        img = sim.render(w, h, view, style)
        ref = oracle_frame(sim, view, style, w, h)
        diff = np.count_nonzero(img != ref)
        print(f"{w}x{h} frame {k}: {diff} differing bytes of {img.size}")
        assert diff == 0
        assert (img != 255).any()  # something was drawn
        sim.step(40)  # densities move away from the ramp centre


def test_lit_frames_match_the_oracle():
    sc = scenes.small_fluid_bar_3d()
    sim = FluidSim(sc)
    sim.init()
    sim.step(5)
    b = sc.bounds_min[:3]
    d = sc.bounds_dim[:3]
    view = dict(angle=0.3, pos=(b[0] + 0.5 * d[0], -(b[1] + 0.5 * d[1])), scale=1.45)
    style = style_for(sc, lighting=True)
    w, h = 128, 128
    img = sim.render(w, h, view, style).astype(int)
    ref = oracle_frame(sim, view, style, w, h).astype(int)
    err = np.abs(img - ref)
    print(f"lit: max level difference {err.max()}, pixels differing {np.count_nonzero(err.any(axis=2))}")
    assert (ref != 255).any()
    assert err.max() <= 1


def test_scene_file_settings_render():
    path = os.path.join(HERE, "golden", "scenes", "csg_2d.toml")
    sc = scenes.load_toml(path)
    sim = FluidSim.from_toml(path)
    sim.init()
    r = sc.meta["render"]
    img = sim.render(200, 150, r["view"], r["style"])
    ref = oracle_frame(sim, r["view"], r["style"], 200, 150)
    assert img.shape == (150, 200, 3)
    assert np.count_nonzero(img != ref) == 0
