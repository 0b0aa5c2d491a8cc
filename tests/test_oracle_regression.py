"""The oracle against its own frozen trajectories (tests/golden/
oracle_regression.json, written by tests/golden/make_oracle_regression.py):
colorings, positions, rotations, iteration counts and contact-pool state of
small seeded scenes at recorded steps.  The GPU parity tests hold the kernels
to the oracle; this holds the oracle still.

Bars: integers (colors, iterations, pool counts) exact; positions and
rotations within 1e-9 of the bounding-box diagonal (the oracle is FP64
without contraction, so on one toolchain it reproduces to the last bit; the
margin absorbs a libm that rounds a transcendental differently).
"""
import numpy as np
import pytest

from conftest import golden

CASES = None


def cases():
    global CASES
    if CASES is None:
        from tests.golden import make_oracle_regression as gen
        CASES = {name: (builder, kw) for name, builder, kw, _ in gen.CASES}
    return CASES


@pytest.mark.parametrize("name", ["cube_fixed_bottom4", "batch3_tol", "spheres_on_cube", "rods_on_cube",
                                  "rods_spheres"])
def test_oracle_reproduces_frozen_trajectory(oracle_lib, name):
    ref = golden("oracle_regression.json")[name]
    builder, kw = cases()[name]
    sc = builder()
    o = oracle_lib.Oracle()
    sc.load(o, **kw)
    o.finalize()
    col, nc = o.coloring()
    assert nc == ref["num_colors"]
    assert [int(c) for c in col] == ref["coloring"]
    diag = ref["bbox_diagonal"]
    done = 0
    for snap in ref["snapshots"]:
        o.step(snap["step"] - done)
        done = snap["step"]
        x = o.positions()
        err = np.abs(x - np.asarray(snap["positions"])).max() / diag
        assert err < 1e-9, (snap["step"], err)
        assert int(o.iterations) == snap["iterations"]
        if "rotations" in snap:
            rot = o.rotations()
            for i, q in snap["rotations"].items():
                assert np.abs(rot[int(i)] - np.asarray(q)).max() < 1e-9, (snap["step"], i)
        info = o.dynamic_info()
        assert {k: int(v) for k, v in info.items()} == snap["dynamic_info"], snap["step"]
