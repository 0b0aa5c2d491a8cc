"""Writes tests/golden/reference_outputs.npz: outputs of the reference
implementation itself (oracle/_ref/libavbd_ref.so, built from the reference's
unmodified sources by oracle/Makefile) on seeded synthetic scenes of the
benchmark configurations' shapes.

    python tests/golden/make_reference_golden.py

Needs the reference sources (AVBD_REFERENCE_ROOT, default /root/reference)
to build the library; the fixture it writes is what the tests read
everywhere else.  Every scene runs the reference's fixed iteration count with
one worker thread (its parallel paths then run in a fixed order).

Cases (each key prefixed by the case name):
  c1       1 m cube, 8^3 cells, bottom fixed, 10 iterations: colors and
           positions after steps 1, 10 and 100;
  drop8    8^3 cube with ground contact and its 384 surface triangles as
           collision primitives: colors, and after step 1 the LBVH (Morton
           codes, sorted order, children, parents, subtree sizes, node bounds)
           and the candidate pairs; positions after steps 1, 10, 30;
  c2       the 32^3 cube (35,937 vertices, 196,608 tets, 12,288 surface
           triangles, perturbed, E 1e6, nu 0.49) dropped on the ground: colors,
           the step-1 Morton codes, sorted order, tree, SHA-256 of the node
           bounds and candidate pairs (the reference's parallel-refit path,
           n >= 5,000 primitives), and every 16th vertex's position after
           steps 1 and 2;
  rods     4 helical rods of 100 segments on one-sided fixed joints, 4 spheres,
           rigid-body ground contact: positions and rotations after steps 1,
           10, 30;
  sph      spheres on a soft cube (triangle-rigid contacts): positions after
           steps 1 and 30, the contact pool after step 30;
  rodcube  rods on a cube (triangle-rod contacts): positions and rotations
           after step 30, the rod contact pool after step 30;
  c4_<s>   scenes 0, 1 and 7 of the seed-0 1024-cube batch, each in its own
           context, 15 iterations: every 8th vertex's position after steps 1
           and 5.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from avbd_b200 import scenes  # noqa: E402
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_outputs.npz")
LBVH_KEYS = ("morton", "sorted_order", "left", "right", "parent", "subtree_size")


def cases():
    """name -> (scene, {step: [what to record]})"""
    return {
        "c1": (scenes.cube_fixed_bottom(8), {1: ["pos"], 10: ["pos"], 100: ["pos"]}),
        "drop8": (scenes.cube_drop(n=8, surface=True), {1: ["pos", "lbvh"], 10: ["pos"], 30: ["pos"]}),
        "c2": (scenes.cube_drop(n=32, surface=True), {1: ["pos16", "lbvh_digest"], 2: ["pos16"]}),
        "rods": (scenes.rods_and_spheres(num_rods=4, segments=100, num_spheres=4, seed=1),
                 {1: ["pos", "rot"], 10: ["pos", "rot"], 30: ["pos", "rot"]}),
        "sph": (scenes.spheres_on_cube(n=4, num_spheres=4), {1: ["pos"], 30: ["pos", "trc"]}),
        "rodcube": (scenes.rods_on_cube(n=4, num_rods=3, segments=8), {30: ["pos", "rot", "trd"]}),
        **{f"c4_{s}": (scenes.batched_cubes(num_scenes=1024, seed=0, scene_ids=[s]), {1: ["pos8"], 5: ["pos8"]})
           for s in (0, 1, 7)},
    }


def record(sim, what, step, out, name):
    key = f"{name}/s{step}"
    if "pos" in what:
        out[f"{key}/pos"] = sim.positions()
    if "pos16" in what:
        out[f"{key}/pos16"] = sim.positions()[::16].copy()
    if "pos8" in what:
        out[f"{key}/pos8"] = sim.positions()[::8].copy()
    if "rot" in what:
        out[f"{key}/rot"] = sim.rotations()
    if "lbvh" in what or "lbvh_digest" in what:
        t = sim.lbvh()
        for k in LBVH_KEYS:
            out[f"{key}/{k}"] = t[k]
        if "lbvh" in what:
            out[f"{key}/bounds"] = t["bounds"]
        else:  # node bounds as the SHA-256 of their FP64 bytes
            out[f"{key}/bounds_sha256"] = np.frombuffer(hashlib.sha256(t["bounds"].tobytes()).digest(), np.uint8)
        out[f"{key}/pairs"] = t["pairs"]
        out[f"{key}/root"] = np.array([t["root"]], dtype=np.uint32)
    if "trc" in what:
        p = sim.contact_pool()
        out[f"{key}/trc_particles"] = p["particles"]
        out[f"{key}/trc_active"] = p["active"]
        out[f"{key}/trc_k"] = p["k"]
        out[f"{key}/trc_lam"] = p["lam"]
    if "trd" in what:
        p = sim.rod_contact_pool()
        out[f"{key}/trd_particles"] = p["particles"]
        out[f"{key}/trd_active"] = p["active"]
        out[f"{key}/trd_k"] = p["k"]
        out[f"{key}/trd_lam"] = p["lam"]


def main():
    if ref.build() is None:
        raise SystemExit("the reference sources are not present; set AVBD_REFERENCE_ROOT")
    out = {}
    for name, (sc, plan) in cases().items():
        sim = ref.RefSim(sc)
        sc.load(sim)
        sim.finalize()
        colors, nc = sim.coloring()
        out[f"{name}/colors"] = colors
        out[f"{name}/num_colors"] = np.array([nc], dtype=np.uint32)
        done = 0
        for step in sorted(plan):
            sim.step(step - done)
            done = step
            record(sim, plan[step], step, out, name)
        sim.close()
        print(name, "ok", flush=True)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
