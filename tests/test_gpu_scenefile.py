"""A YAML scene (tet mesh + rod + sphere, the reference's scene schema) run
headless by the engine matches the FP64 oracle, and frames are written."""
import os

import numpy as np
import pytest

from avbd_b200 import Context, meshio, scenefile, scenes

pytestmark = pytest.mark.gpu

SCENE = """time-step: 5e-3
solver-iters: 12
iter-acceleration: 0.9
objects:
  - type: "TetMeshObject"
    filename: "cube.msh"
    position: [0, 0.8, 0]
    rotation: [10, 20, 30]
    velocity: [0.5, 0, 0]
    E: 3.5e5
    nu: 0.45
  - type: "Rod"
    position: [2, 1.0, 0]
    rotation: [90, 0, 0]
    velocity: [0, 0, 1]
    base-fixed: false
    elements: 10
    length: 0.5
    diameter: 0.05
    E: 5e6
    nu: 0.4
  - type: "RigidSphere"
    position: [-2, 0.5, 0]
    radius: 0.25
"""


def make(tmp_path):
    tets = scenes.hex_grid_tets(3).astype(np.int64)
    X = meshio.grid_vertices(3)
    meshio.write_msh(str(tmp_path / "cube.msh"), X, tets, meshio.outward_surface(X, tets))
    (tmp_path / "s.yaml").write_text(SCENE)
    return str(tmp_path / "s.yaml")


def test_yaml_scene_engine_matches_oracle(tmp_path, oracle_lib):
    sc = scenefile.load_yaml(make(tmp_path))
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    for _ in range(4):
        e.step(20)
        o.step(20)
        assert np.abs(e.positions() - o.positions()).max() / sc.bbox_diagonal() < 1e-9
    assert o.positions()[:64, 1].min() < 0.05  # the cube reached the ground


def test_headless_frames(tmp_path):
    ctx, sc = scenefile.run(make(tmp_path), steps=20, frames=str(tmp_path / "frames"), every=10)
    files = sorted(os.listdir(tmp_path / "frames"))
    assert files == ["frame_00010.obj", "frame_00020.obj"]
    txt = (tmp_path / "frames" / "frame_00020.obj").read_text().splitlines()
    assert sum(l.startswith("v ") for l in txt) == sc.num_particles
    assert sum(l.startswith("f ") for l in txt) == len(sc.meta["surfaces"])
    assert sum(l.startswith("l ") for l in txt) == 1
