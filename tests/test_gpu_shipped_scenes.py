"""Every scene the reference ships that loads (22 of its 23 example files,
seeded by the library's scene loader into tests/golden/scenes_seeded;
model_import_test names an STL model the reference does not ship), stepped on
the GPU through one update() (the file's subticks, at least 10 steps) against
the float oracle, with the error against the double oracle printed beside it.
Several of these scenes are stiff solids at small time steps, where the float
oracle itself drifts from the double one by ~1e-4 in velocity within tens of
steps: a quantity then may be as close to the double oracle as twice the float
oracle's own distance from it (helpers.compare_with_oracle)."""
import glob
import os

import pytest

from helpers import compare_with_oracle, load_seeded_scene

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "golden", "scenes_seeded", "*.npz")))


def test_every_loadable_shipped_scene_has_a_fixture():
    assert len(NAMES) == 22


@pytest.mark.parametrize("name", NAMES)
def test_shipped_scene_steps_like_the_oracle(name):
    sc = load_seeded_scene(name)
    compare_with_oracle(sc, max(10, sc.subticks), fp32_floor=True)
