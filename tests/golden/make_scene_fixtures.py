"""Seeded scenes of the reference's shipped example files, saved as fixtures
for the GPU tests, which run where the reference tree is absent: every
example that loads.  model_import_test names an STL model
(examples/models/gear3.stl) that the reference does not ship, so it loads
in neither program.  STL paths in the files are relative to the reference's
root, as the demo runs from there.

Each scene file is parsed and seeded by this library's own loader
(arp_scene_file_load, checked bit for bit against the restatement in
oracle/scene_oracle.py by tests/test_scene_loader.py), and the resulting
records are stored: mobile and boundary particles, materials, the resolved
interaction table and the scalars of the scene.

    ARP_REFERENCE_EXAMPLES=<the reference's examples/> python tests/golden/make_scene_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ar-physics_b200"))

from arphys import scenes  # noqa: E402

NAMES = ("car", "cloth", "container_buckling", "esophagus", "flow_over_cylinder_2d", "flow_over_cylinder_3d",
         "ink_drop", "interactivity_test", "liquid_solid_test", "metal_bar", "plastic_test", "raindrop",
         "raindrop_real_time", "rayleigh_taylor", "rope", "siphon", "solid_test", "solid_test_3D", "spinning_ball",
         "stomach", "wave_3d", "wave_3d_real_time")
OUT = os.path.join(HERE, "scenes_seeded")


def main():
    src = os.environ.get("ARP_REFERENCE_EXAMPLES")
    if not src:
        sys.exit("set ARP_REFERENCE_EXAMPLES to the reference's examples directory")
    os.makedirs(OUT, exist_ok=True)
    src = os.path.abspath(src)
    os.chdir(os.path.dirname(src))  # STL paths are relative to the reference's root
    for name in NAMES:
        sc = scenes.load_toml(os.path.join(src, name + ".toml"))
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), particles=sc.particles, boundary=sc.boundary, materials=sc.materials,
            interactions=sc.interactions, interaction_given=sc.interaction_given,
            bounds_min=np.array(sc.bounds_min, np.float32), bounds_dim=np.array(sc.bounds_dim, np.float32),
            scalars=np.array([sc.h, sc.dt, sc.gravity, sc.alpha], np.float32),
            subticks=np.array(sc.subticks), integrator=np.array(sc.integrator), name=np.array(sc.name))
        print(f"{name}: {sc.n} mobile, {sc.nb} boundary, integrator {sc.integrator}")


if __name__ == "__main__":
    main()
