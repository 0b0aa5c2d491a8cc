"""Headless scene files: the MSH 4.1 reader/writer, the YAML scene reader's
set-up (TetMeshObject.cpp:21-113, Rod.cpp:10-68, RigidSphere.cpp:8-22,
Simulation.hpp:108-137) and the OBJ/PLY frame writers."""
import os

import numpy as np
import pytest

from avbd_b200 import meshio, scenefile, scenes

# A gmsh-style MSH 4.1 ASCII file with several entity blocks (a point, a
# surface, a volume) out of (dim, tag) order, and a line element to ignore.
GMSH_TEXT = """$MeshFormat
4.1 0 8
$EndMeshFormat
$Entities
1 0 1 1
1 0 0 0 0
$EndEntities
$Nodes
3 5 1 5
3 1 0 1
5
0.3 0.3 0.3
0 1 0 1
1
0 0 0
2 1 0 3
2
3
4
1 0 0
0 1 0
0 0 1
$EndNodes
$Elements
3 6 1 6
3 1 4 2
5 1 2 3 4
6 5 2 3 4
2 1 2 3
2 1 2 3
3 1 3 4
4 2 4 3
1 1 1 1
1 1 2
$EndElements
"""


def test_read_msh_entity_order_and_types(tmp_path):
    p = tmp_path / "m.msh"
    p.write_text(GMSH_TEXT)
    v, t, f = meshio.read_msh(str(p))
    assert np.allclose(v, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.3, 0.3, 0.3]])
    assert t.tolist() == [[0, 1, 2, 3], [4, 1, 2, 3]]
    assert f.tolist() == [[0, 1, 2], [0, 2, 3], [1, 3, 2]]


def cube(n):
    tets = scenes.hex_grid_tets(n).astype(np.int64)
    X = meshio.grid_vertices(n)
    return X, tets, meshio.outward_surface(X, tets)


def test_outward_surface_encloses_the_volume():
    X, tets, faces = cube(3)
    a, b, c = X[faces[:, 0]], X[faces[:, 1]], X[faces[:, 2]]
    assert np.isclose(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0, 1.0)
    assert np.allclose(scenefile.surface_mass_center(X, faces), [0.5, 0.5, 0.5])


def test_msh_round_trip(tmp_path):
    X, tets, faces = cube(3)
    p = str(tmp_path / "c.msh")
    meshio.write_msh(p, X, tets, faces)
    v, t, f = meshio.read_msh(p)
    assert np.array_equal(v, X) and np.array_equal(t, tets) and np.array_equal(f, faces)


def test_msh_rejects_binary_and_bad_tags(tmp_path):
    p = tmp_path / "b.msh"
    p.write_text("$MeshFormat\n4.1 1 8\n$EndMeshFormat\n")
    with pytest.raises(meshio.MshError):
        meshio.read_msh(str(p))
    p.write_text(GMSH_TEXT.replace("3 1 0 1\n5\n", "3 1 0 1\n7\n"))
    with pytest.raises(meshio.MshError):
        meshio.read_msh(str(p))


def _reference_mesh():
    from oracle.ref import REFERENCE_ROOT  # AVBD_REFERENCE_ROOT
    return os.path.join(REFERENCE_ROOT, "resource", "cube2.msh")


@pytest.mark.skipif(not os.path.exists(_reference_mesh()), reason="reference meshes absent")
def test_reference_cube2_matches_golden_element():
    import json
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "neohookean_element0.json")))
    v, t, f = meshio.read_msh(_reference_mesh())
    assert (v.shape, t.shape, f.shape) == ((27, 3), (40, 4), (48, 3))
    assert (t[0] + 1).tolist() == g["element_node_tags"]
    assert np.allclose(v[t[0]], g["vertices"])


def write_scene(tmp_path, objects):
    X, tets, faces = cube(2)
    meshio.write_msh(str(tmp_path / "cube.msh"), X, tets, faces)
    (tmp_path / "s.yaml").write_text("time-step: 5e-3\nsolver-iters: 10\niter-acceleration: 0.5\nobjects:\n" + objects)
    return str(tmp_path / "s.yaml")


def test_tet_mesh_object_setup(tmp_path):
    path = write_scene(tmp_path, """  - type: "TetMeshObject"
    filename: "cube.msh"
    position: [1, 2, 3]
    scaling: [2, 1, 1]
    rotation: [0, 0, 90]
    velocity: [0.5, 0, 0]
    E: 2e5
    nu: 0.3
    density: 500
""")
    sc = scenefile.load_yaml(path)
    assert sc.dt == 5e-3 and sc.solver_iters == 10
    calls = {m: a for m, a, _ in sc.calls}
    X, m = calls["add_particles"]
    assert np.allclose(m.sum(), 500 * 2.0)                       # density x scaled volume (1 m cube, x2)
    assert np.allclose(X.mean(0), [1, 2, 3])                      # centred by mass, then moved
    ext = X.max(0) - X.min(0)
    assert np.allclose(ext, [1, 2, 1])                            # x scaled by 2, then turned 90 deg about z
    idx, lam, mu, kd, Q, V = calls["add_neo_hookean"]
    assert np.allclose(mu, 2e5 / 2.6) and np.allclose(lam, 2e5 * 0.3 / (1.3 * 0.4)) and np.allclose(V.sum(), 2.0)
    _, vel, _ = calls["set_velocities"]
    assert np.allclose(vel, [0.5, 0, 0])
    p, ks, mus, muk = calls["add_ground_collision"]
    assert np.allclose(ks, m / 5e-3 ** 2) and np.allclose(mus, 0.4) and np.allclose(muk, 0.2)
    assert len(sc.meta["surfaces"]) == 48


def test_rod_and_sphere_objects_run_in_the_oracle(tmp_path, oracle_lib):
    path = write_scene(tmp_path, """  - type: "TetMeshObject"
    filename: "cube.msh"
    position: [0, 1, 0]
  - type: "Rod"
    position: [3, 1.5, 0]
    rotation: [90, 0, 0]
    elements: 8
    length: 0.4
    diameter: 0.02
    E: 1e6
  - type: "RigidSphere"
    position: [-3, 0.6, 0]
    radius: 0.2
""")
    sc = scenefile.load_yaml(path)
    assert sc.num_particles == 27 + 9 + 1
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    x0 = o.positions()
    o.step(150)
    x = o.positions()
    assert np.isfinite(x).all()
    assert np.allclose(x[27], x0[27])              # rod base fixed by default
    assert abs(x[-1, 1] - 0.2) < 1e-3                # sphere at rest on the ground
    assert x[:27, 1].min() > -0.05                  # cube caught by the ground


def test_frame_writers(tmp_path):
    X, tets, faces = cube(2)
    meshio.write_obj(str(tmp_path / "f.obj"), X, faces, [[0, 1, 2]])
    txt = (tmp_path / "f.obj").read_text().splitlines()
    assert sum(l.startswith("v ") for l in txt) == len(X) and sum(l.startswith("f ") for l in txt) == len(faces)
    assert txt[-1] == "l 1 2 3"
    meshio.write_ply(str(tmp_path / "f.ply"), X, faces)
    raw = (tmp_path / "f.ply").read_bytes()
    head, body = raw.split(b"end_header\n", 1)
    assert b"element vertex 27" in head and len(body) == 27 * 12 + len(faces) * 13
