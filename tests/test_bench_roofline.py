"""The algorithmic-byte figures the bench divides by its measured times, on
the 1,048,576-particle fluid + bar workload (RK2): 96 B per mobile particle
per stage for the fluid launch, n(96 S + 96) + n_solid 196 S + n_boundary 16 S
for the whole step, and the candidate count of the fluid scan."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def scene():
    from arphys import scenes
    return scenes.fluid_bar_3d()


def test_workload_split(scene):
    assert (scene.n + scene.nb, scene.n, scene.n_solids(), scene.nb) == (1048576, 1013760, 129024, 34816)
    assert scene.integrator == "rk2"


def test_step_bytes_follow_the_stated_formula(bench, scene):
    r = bench.step_roofline(scene, 2, 1.0, 6464.3)
    expected = 1013760 * (96 * 2 + 96) + 129024 * 196 * 2 + 34816 * 16 * 2
    assert expected == 343654400
    assert r["alg_bytes_per_step"] == expected
    assert r["achieved"] == pytest.approx(expected / 1e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6464.3)


def test_candidates_of_the_fluid_scan(bench, scene):
    # rows of 5 x-halved search cells, 3 rows in y and z, mobile and boundary
    # candidates, from the seeded initial positions
    c = bench.candidate_count(scene)
    assert c == 175239810
    assert 170 < c / scene.n < 176
