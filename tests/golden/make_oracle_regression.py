"""Generates tests/golden/oracle_regression.json: trajectories of the FP64
oracle on small seeded scenes, one per part of the step it restates.  The
oracle is pinned to the reference's own tests (the other fixtures here); this
file freezes what it computes on whole steps, so that a change to the oracle
that moves any of these numbers shows up in the CPU suite
(tests/test_oracle_regression.py) instead of silently moving the bar the GPU
parity tests are held to.  Regenerate deliberately, after such a change has
been checked:

    python tests/golden/make_oracle_regression.py

Cases (scene builders of avbd_b200.scenes, all seeded):
  cube_fixed_bottom4 -- NeoHookean cube, bottom fixed, fixed iterations, Chebyshev;
  batch3_tol         -- three cubes with ground contact run to R <= 1e-4 per scene;
  spheres_on_cube    -- triangle-sphere CCD, the triangle-rigid contact pool, recoloring;
  rods_on_cube       -- Cosserat rods, triangle-rod contacts, 6-DOF solve;
  rods_spheres       -- helical rods hanging from one-sided fixed joints, spheres,
                        rigid-body ground contact.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from avbd_b200 import scenes  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

# (name, builder, load kwargs, steps at which the state is recorded)
CASES = [
    ("cube_fixed_bottom4", lambda: scenes.cube_fixed_bottom(4), {}, [1, 10, 30]),
    ("batch3_tol", lambda: scenes.batched_cubes(num_scenes=3, seed=7, n_min=3, n_max=4),
     {"residual_tolerance": 1e-4, "max_iters": 100}, [1, 6]),
    ("spheres_on_cube", lambda: scenes.spheres_on_cube(n=3, num_spheres=2, seed=2), {}, [1, 20]),
    ("rods_on_cube", lambda: scenes.rods_on_cube(n=3, num_rods=2, segments=6, seed=1), {}, [1, 20]),
    ("rods_spheres", lambda: scenes.rods_and_spheres(num_rods=2, segments=40, num_spheres=2, seed=3, length=0.4),
     {}, [1, 30]),
]


def oriented_indices(sc):
    """Particle indices of the oriented particles, in the order the scene adds them."""
    out, n = [], 0
    for method, args, _ in sc.calls:
        if method == "add_particles":
            n += len(args[1])
        elif method == "add_oriented_particles":
            out.extend(range(n, n + len(args[1])))
            n += len(args[1])
    return out


def run_case(builder, kw, record_at):
    sc = builder()
    oriented = oriented_indices(sc)
    o = Oracle()
    sc.load(o, **kw)
    o.finalize()
    col, nc = o.coloring()
    out = {"coloring": [int(c) for c in col], "num_colors": int(nc), "bbox_diagonal": sc.bbox_diagonal(),
           "load": kw, "snapshots": []}
    done = 0
    for s in record_at:
        o.step(s - done)
        done = s
        snap = {"step": s, "positions": o.positions().tolist(), "iterations": int(o.iterations)}
        if oriented:
            rot = o.rotations()
            snap["rotations"] = {str(i): rot[i].tolist() for i in oriented}
        info = o.dynamic_info()
        snap["dynamic_info"] = {k: int(v) for k, v in info.items()}
        out["snapshots"].append(snap)
    return out


def main():
    data = {name: run_case(b, kw, at) for name, b, kw, at in CASES}
    path = os.path.join(HERE, "oracle_regression.json")
    with open(path, "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
