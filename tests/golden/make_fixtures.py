"""Writes the small scene fixtures of tests/golden/ in diff_fem's file formats:
a JSON scene ("Parameters", "Meshes", "Obstacles"), a tet OBJ ('v' + 't' lines,
0-based tets), a triangle OBJ obstacle ('f' lines, 1-based) and a muscle file
('fibre segment x y z' rows).  The meshes are synthetic (a cube-grid beam and
a ground quad; pneumatic.json drives the beam with "Volume Verts" springs);
run `python tests/golden/make_fixtures.py` to regenerate.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from diff_fem_b200 import scene as S  # noqa: E402


def main():
    out = os.path.join(HERE, "beam_scene")
    os.makedirs(out, exist_ok=True)
    # beam of 6x2x2 unit cubes (scaled by 0.05 in the JSON like the reference's default)
    x0, tets = S.cube_grid(6, 2, 2, 1.0)
    with open(os.path.join(out, "beam_tet.obj"), "w") as f:
        for p in x0:
            f.write("v %.6f %.6f %.6f\n" % tuple(p))
        for t in tets:
            f.write("t %d %d %d %d\n" % tuple(t))
    with open(os.path.join(out, "ground.obj"), "w") as f:
        for p in ([-1, -0.05, -1], [2, -0.05, -1], [2, -0.05, 1], [-1, -0.05, 1]):
            f.write("v %.6f %.6f %.6f\n" % tuple(p))
        f.write("f 1 3 2\nf 1 4 3\n")
    with open(os.path.join(out, "beam.muscle"), "w") as f:
        for fib, (y, z) in enumerate([(0.5, 0.5), (1.5, 1.5)]):
            for k, x in enumerate(np.linspace(0.1, 5.9, 60)):
                f.write("%d\t%d\t%.6f\t%.6f\t%.6f\n" % (fib, k, x, y, z))
    pins = [int(i) for i in np.nonzero(np.isclose(x0[:, 0], 0.0))[0]]
    scene = {
        "Parameters": [{"Simulation HZ": 100, "Handle collision": True, "Self-collision": False,
                        "Gravity": [0.0, -9.8, 0.0], "Max Iteration": 10}],
        "Meshes": [{"Obj filename": "beam_scene/beam_tet.obj", "Scale": 0.05, "Youngs Modulus": 5e4,
                    "Poisson Ratio": 0.3, "Mass": 1.2, "Attach Verts": pins, "Attach Stiffness": 1e8,
                    "Muscle filename": "beam_scene/beam.muscle", "Muscle Stiffness": 5e3, "Actuator type": 2}],
        "Obstacles": [{"Obj filename": "beam_scene/ground.obj"}],
    }
    with open(os.path.join(out, "beam.json"), "w") as f:
        json.dump(scene, f, indent=1)
    # the same beam driven by pneumatic springs (actuator type 3): three
    # "Volume Verts" polylines along x on the beam's top and bottom edges
    lines = []
    for y, z in ((2.0, 0.0), (2.0, 2.0), (0.0, 2.0)):
        on = np.nonzero(np.isclose(x0[:, 1], y) & np.isclose(x0[:, 2], z))[0]
        lines.append([int(i) for i in on[np.argsort(x0[on, 0])]])
    pneu = {
        "Parameters": [{"Simulation HZ": 100, "Handle collision": False, "Self-collision": False,
                        "Gravity": [0.0, -9.8, 0.0], "Max Iteration": 10}],
        "Meshes": [{"Obj filename": "beam_scene/beam_tet.obj", "Scale": 0.05, "Youngs Modulus": 5e4,
                    "Poisson Ratio": 0.3, "Mass": 1.2, "Attach Verts": pins, "Attach Stiffness": 1e8,
                    "Muscle Stiffness": 1e5, "Actuator type": 3, "Volume Verts": lines}],
    }
    with open(os.path.join(out, "pneumatic.json"), "w") as f:
        json.dump(pneu, f, indent=1)


if __name__ == "__main__":
    main()
