"""The C++ facade (include/avbd/avbd.hpp): a C++ program builds a cube element
by element through Sim::SimulationContext / Energy pools and steps with
Sim::SimulationExecutor::timeStep(); its positions must match the oracle."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from avbd_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class Capture:
    def __init__(self):
        self.calls = {}

    def __getattr__(self, name):
        def f(*a, **k):
            self.calls.setdefault(name, []).append(a)
        return f


def test_cpp_facade_matches_oracle(oracle_lib, tmp_path):
    sc = scenes.cube_fixed_bottom(4)
    cap = Capture()
    sc.load(cap)
    (X, m), = cap.calls["add_particles"]
    (idx, lam, mu, kd, Q, V), = cap.calls["add_neo_hookean"]
    (slots, fl), = cap.calls["set_fixed"]
    fixed = np.zeros(len(X), dtype=np.uint8)
    fixed[np.asarray(slots)] = 1
    blob = bytearray(struct.pack("<I", len(X)))
    for i in range(len(X)):
        blob += struct.pack("<4dB", *X[i], m[i], fixed[i])
    blob += struct.pack("<I", len(idx))
    for t in range(len(idx)):
        blob += struct.pack("<4I", *[int(v) for v in idx[t]])
        blob += struct.pack("<3d", lam[t], mu[t], kd[t])
        blob += struct.pack("<9d", *Q[t])
        blob += struct.pack("<d", V[t])
    blob += struct.pack("<dId", sc.dt, sc.solver_iters, sc.iter_acceleration)
    scene_bin = tmp_path / "scene.bin"
    scene_bin.write_bytes(bytes(blob))
    exe = tmp_path / "facade_step"
    lib_dir = os.path.join(ROOT, "avbd_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "facade_step.cpp"), "-L" + lib_dir, "-lavbd_b200",
                           "-Wl,-rpath," + lib_dir, "-o", str(exe)])
    out = tmp_path / "x.bin"
    steps = 30
    subprocess.check_call([str(exe), str(scene_bin), str(steps), str(out)])
    x = np.fromfile(out, dtype=np.float64).reshape(-1, 3)
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    o.step(steps)
    err = np.abs(x - o.positions()).max() / sc.bbox_diagonal()
    assert err < 1e-5, err
