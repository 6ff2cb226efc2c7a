"""Writes tests/golden/ref_scenes/*.npz: four of diff_fem's own data scenes,
loaded by diff_fem_b200.loader from the reference's data directory and saved
as scene descriptors, so that the parity tests can run them where that
directory is absent.

    python tests/golden/make_ref_scenes.py <diff_fem>/data [name ...]

bridgesus  (a suspended bridge: attachments of stiffness 1e20)
baymax     (a soft body dropped on a ground obstacle: obstacle contact)
cloth_ball (a ball mesh and a cloth: springs, cloth without gravity, self-collision)
octopus    (underwater: drag and lift on the outward surface faces)
droneman   (actuator type 3: 48 pneumatic springs from "Volume Verts", and a ball)
baymax_skeleton (actuator type 1: five "Bones" links, the root ALL and four ROTATIONAL)
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from diff_fem_b200 import loader, scene as S  # noqa: E402

SCENES = [("bridgesus", "bridgesus/bridgesus.json", 3), ("baymax", "baymax/baymax.json", 3),
          ("cloth_ball", "cloth_ball/cloth_ball.json", 3), ("octopus", "octopus/octopus.json", 2),
          ("droneman", "droneman/droneman.json", 3), ("baymax_skeleton", "baymax/baymax_skeleton.json", 3)]


def main(data_root: str, names=()) -> None:
    out = os.path.join(HERE, "ref_scenes")
    os.makedirs(out, exist_ok=True)
    for name, rel, nsteps in SCENES:
        if names and name not in names:
            continue
        d = loader.load_scene(rel, nsteps, data_root=data_root).desc
        S.save_npz(d, os.path.join(out, name + ".npz"))
        print(name, d.n_vertices, "vertices", d.n_tets, "tets")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["DIFF_FEM_DATA"], tuple(sys.argv[2:]))
