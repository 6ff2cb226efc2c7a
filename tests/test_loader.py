"""Scene loading in diff_fem's file formats (CPU)."""
import os

import numpy as np
import pytest

from diff_fem_b200 import loader, scene as S
from diff_fem_b200.engine import host_factor_solve
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# diff_fem's data directory, when available (the tests reading it skip otherwise;
# tests/golden/ref_scenes holds four of its scenes as descriptors)
REF_DATA = os.environ.get("DIFF_FEM_DATA", "")


def test_fixture_scene_loads():
    L = loader.load_scene("beam_scene/beam.json", 3, data_root=GOLDEN)
    d = L.desc
    assert d.n_vertices == 7 * 3 * 3 and d.n_tets == 6 * 2 * 2 * 5
    assert np.isclose(d.mass.sum(), 1.2)                     # "Mass" with Is Mass Same
    assert d.attach_vertex.size == 9 and np.all(d.attach_stiffness == 1e8)
    assert np.isclose(d.time_step, 0.01) and d.max_iterations == 10
    assert d.handle_collision and d.obstacle_faces.shape == (2, 3)
    assert d.n_segments > 0 and d.muscle_segment.size > 0
    assert np.allclose(d.x0.max(axis=0), [0.3, 0.1, 0.1])    # Scale 0.05
    # the engine's host factorisation accepts it and solves
    x, info = host_factor_solve(d, np.ones(3 * d.n_vertices))
    assert np.all(np.isfinite(x))


def test_surface_extraction_and_orientation():
    x0, tets = S.cube_grid(2, 2, 2, 1.0)
    faces, verts = S.surface_of(x0, tets)
    assert faces.shape[0] == 6 * 2 * 2 * 2            # 2 triangles per boundary cube face
    assert len(set(verts.tolist())) == 26              # every vertex but the centre
    c = x0.mean(axis=0)
    for f in faces:                                    # outward normals
        n = np.cross(x0[f[1]] - x0[f[0]], x0[f[2]] - x0[f[0]])
        assert np.dot(n, x0[f].mean(axis=0) - c) > 0


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="DIFF_FEM_DATA not set")
def test_reference_scenes_load():
    """The reference's own data scenes (read in place, not copied)."""
    d = loader.load_scene("bridgesus/bridgesus.json", 3, data_root=REF_DATA).desc
    assert (d.n_vertices, d.n_tets, d.attach_vertex.size) == (212, 668, 65)
    assert np.isclose(d.mass.sum(), 10.0) and np.isclose(d.time_step, 1 / 200)
    o = O.OracleScene(d)  # the oracle accepts it (attach stiffness 1e20)
    r = o.forward(d.x0.reshape(-1).copy(), np.zeros(3 * d.n_vertices), n_steps=2)
    assert np.all(np.isfinite(r["x"]))
    b = loader.load_scene("baymax/baymax.json", 3, data_root=REF_DATA).desc
    assert (b.n_vertices, b.n_tets) == (775, 3078) and b.obstacle_faces.shape[0] > 0
    c = loader.load_scene("cloth_ball/cloth_ball.json", 3, data_root=REF_DATA)
    assert [bd.kind for bd in c.bodies] == ["mesh", "cloth"] and c.desc.spring_weight.size > 0
    assert np.all(c.desc.spring_weight == 200.0) and not c.desc.gravity_mask[c.bodies[1].offset:].any()


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="DIFF_FEM_DATA not set")
def test_reference_underwater_scene_loads():
    """octopus.json sets "Is underwater": its mesh gets drag and lift on its
    outward surface faces instead of gravity; the oracle steps it.  (fish.json
    has a trailing comma that the reference's JSON parser rejects too.)"""
    L = loader.load_scene("octopus/octopus.json", 2, data_root=REF_DATA)
    d = L.desc
    assert d.underwater and d.drag_faces.shape[0] > 0 and d.drag_faces.max() < d.n_vertices
    assert np.array_equal(np.sort(d.drag_faces, axis=1), np.sort(d.contact_faces, axis=1))
    o = O.OracleScene(d)
    v = np.tile([0.3, 0.0, 0.0], d.n_vertices)
    r = o.forward(d.x0.reshape(-1).copy(), v, n_steps=2)
    assert np.all(np.isfinite(r["x"]))
    mom0 = 0.3 * d.mass.sum()
    assert (d.mass * r["v"].reshape(-1, 3)[:, 0]).sum() < mom0   # the water slows it


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="DIFF_FEM_DATA not set")
def test_reference_scene_fixtures_match_the_data():
    """tests/golden/ref_scenes/*.npz are what the loader makes of the data scenes."""
    import dataclasses
    for name, rel, n in [("bridgesus", "bridgesus/bridgesus.json", 3), ("baymax", "baymax/baymax.json", 3),
                         ("cloth_ball", "cloth_ball/cloth_ball.json", 3), ("octopus", "octopus/octopus.json", 2)]:
        a = loader.load_scene(rel, n, data_root=REF_DATA).desc
        b = S.load_npz(os.path.join(GOLDEN, "ref_scenes", name + ".npz"))
        for f in dataclasses.fields(a):
            u, w = getattr(a, f.name), getattr(b, f.name)
            if u is None or w is None:
                assert u is None and w is None, (name, f.name)
            elif isinstance(u, np.ndarray):
                assert np.array_equal(u, w), (name, f.name)
            else:
                assert u == w, (name, f.name)


def test_reference_scene_fixtures_step_in_the_oracle():
    """The four data-scene fixtures (bridgesus: attachments of stiffness 1e20;
    baymax: ground contact; cloth_ball: a cloth and a ball with self-collision;
    octopus: underwater drag) run forward and backward in the oracle."""
    for name in ("bridgesus", "baymax", "cloth_ball", "octopus"):
        d = S.load_npz(os.path.join(GOLDEN, "ref_scenes", name + ".npz"))
        o = O.OracleScene(d)
        x = d.x0.reshape(-1).copy()
        v = np.tile([0.3, 0.0, 0.0], d.n_vertices) if d.underwater else np.zeros_like(x)
        r = o.forward(x, v, n_steps=3)
        assert np.all(np.isfinite(r["x"])), name
        b = o.backward(np.ones_like(x), np.zeros_like(x))
        assert np.all(np.isfinite(b["x"])), name


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_corrupt_scene_files_raise_clear_errors(tmp_path):
    """Malformed JSON, a JSON without bodies, OBJ files with bad lines or
    indices, a malformed muscle row and an attachment out of range are
    refused with SceneFormatError naming the file (and line)."""
    good_obj = "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nt 0 1 2 3\n"
    obj = _write(tmp_path, "m.obj", good_obj)

    count = [0]

    def scene(mesh, extra=""):
        count[0] += 1
        return _write(tmp_path, "s%d.json" % count[0],
                      '{"Parameters": [{"Simulation HZ": 100}], "Meshes": [{"Obj filename": "%s"%s}]}' % (mesh, extra))

    cases = [
        (_write(tmp_path, "bad.json", '{"Parameters": [{"Simulation HZ": 100}], '), "invalid JSON"),
        (_write(tmp_path, "empty.json", '{"Parameters": [{}]}'), "Meshes"),
        (scene(_write(tmp_path, "a.obj", good_obj + "v 1 x 0\n")), "a.obj:6"),
        (scene(_write(tmp_path, "b.obj", good_obj + "t 0 1 2\n")), "b.obj:6"),
        (scene(_write(tmp_path, "c.obj", good_obj + "t 0 1 2 9\n")), "out of range"),
        (scene(_write(tmp_path, "d.obj", "t 0 1 2 3\n")), "no vertices"),
        (scene(obj, ', "Attach Verts": [7], "Attach Stiffness": 1e8'), "attach vertex 7"),
        (scene(obj, ', "Muscle filename": "%s"' % _write(tmp_path, "m.muscle", "0 0 0.1 0.1 0.1\n0 1 nan? 0 0\n")),
         "m.muscle:2"),
    ]
    for path, what in cases:
        with pytest.raises(loader.SceneFormatError) as ex:
            loader.load_scene(path, 1)
        assert what in str(ex.value), (what, str(ex.value))
    with pytest.raises(FileNotFoundError):
        loader.load_scene(str(tmp_path / "missing.json"), 1)


def test_volume_verts_become_pneumatic_springs():
    """Dfobj.h:231-251: one pneumatic spring per consecutive pair of every
    "Volume Verts" polyline (rest length from the scaled mesh, weight =
    "Muscle Stiffness"), each on its own activation channel."""
    import json
    L = loader.load_scene("beam_scene/pneumatic.json", 1, data_root=GOLDEN)
    d = L.desc
    with open(os.path.join(GOLDEN, "beam_scene", "pneumatic.json")) as fh:
        lines = json.load(fh)["Meshes"][0]["Volume Verts"]
    pairs = [(a, b) for line in lines for a, b in zip(line[:-1], line[1:])]
    assert np.array_equal(d.spring_vertices, np.asarray(pairs))
    assert np.array_equal(d.spring_channel, np.arange(len(pairs)))
    assert d.n_segments == len(pairs) and L.bodies[0].n_pneumatic == len(pairs)
    x = d.x0.reshape(-1, 3)
    assert np.allclose(d.spring_rest, [np.linalg.norm(x[a] - x[b]) for a, b in pairs], rtol=0, atol=1e-15)
    assert np.allclose(d.spring_rest, 0.05)  # unit cube edges at "Scale" 0.05
    assert np.all(d.spring_weight == 1e5)


def test_bones_become_skeleton_links(tmp_path):
    """Dfobj.h:254-288: one link per bone (parent, joint type, unscaled joint
    position, normalised axis, the bone's vertices); the joint torques of the
    non-root links are activation channels after the muscle segments."""
    import json
    src = json.load(open(os.path.join(GOLDEN, "beam_scene", "beam.json")))
    mesh = src["Meshes"][0]
    for k in ("Muscle filename", "Attach Verts", "Attach Stiffness"):
        mesh.pop(k)
    mesh["Actuator type"] = 1
    mesh["Obj filename"] = os.path.join(GOLDEN, "beam_scene", "beam_tet.obj")
    mesh["Bones"] = [
        {"Parent ID": -1, "Joint Type": "ALL", "Joint Pos": [0, 0, 0], "Joint Axis": [0, 0, 0], "Vertices": [0, 1, 2]},
        {"Parent ID": 0, "Joint Type": "ROTATIONAL", "Joint Pos": [0.1, 0.05, 0.05], "Joint Axis": [0, 0, 2],
         "Vertices": [30, 31]},
    ]
    src["Parameters"][0]["Handle collision"] = False
    src.pop("Obstacles")
    path = tmp_path / "bones.json"
    path.write_text(json.dumps(src))
    L = loader.load_scene(str(path), 1, data_root=str(tmp_path))
    d = L.desc
    assert list(d.link_parent) == [-1, 0] and list(d.link_type) == [2, 1]
    assert np.array_equal(d.link_offsets, [0, 3, 5]) and np.array_equal(d.link_vertices, [0, 1, 2, 30, 31])
    assert np.allclose(d.link_joint[1], [0.1, 0.05, 0.05]) and np.allclose(d.link_axis[1], [0, 0, 2])
    assert list(d.link_channel) == [-1, 0] and d.n_segments == 1 and L.bodies[0].n_links == 2
    bad = json.loads(path.read_text())
    bad["Meshes"][0]["Bones"][1]["Joint Type"] = "HINGE"
    path.write_text(json.dumps(bad))
    with pytest.raises(loader.SceneFormatError):
        loader.load_scene(str(path), 1, data_root=str(tmp_path))
