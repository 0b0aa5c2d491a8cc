"""Pins of the oracle's LBVH against hand-derived and independent answers.

* The Karras-2012 radix-tree example used by test/test_lbvh.cpp:38-47: the
  expected topology below is derived by hand from the published figure of
  Karras (2012), not produced by the oracle.
* The few-triangle scene of test/test_lbvh.cpp:168-189: Morton codes are
  recomputed here with numpy (IEEE FP64, no fused multiply-add) and the
  candidate-pair set is compared with a brute-force all-pairs AABB test.
"""
import numpy as np

from conftest import golden

INV = 0xFFFFFFFF


def test_karras_example_topology(oracle_lib):
    fx = golden("lbvh_inputs.json")
    o = oracle_lib.Oracle()
    t = o.lbvh_from_codes(np.array(fx["karras_codes_by_slot"], dtype=np.uint64))
    # stable sort of the slot codes
    assert t["sorted_order"].tolist() == [5, 3, 1, 2, 6, 4, 0, 7]
    n = 8
    I = lambda k: n + k  # internal node k
    expect = {I(0): (I(3), I(4)), I(1): (0, 1), I(2): (2, 3), I(3): (I(1), I(2)),
              I(4): (4, I(5)), I(5): (I(6), 7), I(6): (5, 6)}
    assert t["root"] == I(0)
    for node, (l, r) in expect.items():
        assert (t["left"][node], t["right"][node]) == (l, r), node
    parent = {c: p for p, lr in expect.items() for c in lr}
    for node in range(2 * n - 1):
        assert t["parent"][node] == parent.get(node, INV)
    for leaf in range(n):
        assert t["subtree_size"][leaf] == 1
    assert t["subtree_size"][I(0)] == 8 and t["subtree_size"][I(4)] == 4 and t["subtree_size"][I(6)] == 2


def morton_numpy(boxes):
    """LBVHBuilder::computeAABB_MortonCode restated with numpy FP64."""
    boxes = np.asarray(boxes, dtype=np.float64)
    cen = (boxes[:, :3] + boxes[:, 3:]) * 0.5
    smin = boxes[:, :3].min(0)
    smax = boxes[:, 3:].max(0)
    ext = np.maximum(smax - smin, 1e-6)
    nc = (cen - smin) / ext
    q = np.clip(nc * 2097152.0, 0.0, 2097151.0).astype(np.uint64)

    def expand(v):
        v = v & np.uint64(0x1FFFFF)
        for sh, m in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                      (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
            v = (v | (v << np.uint64(sh))) & np.uint64(m)
        return v

    return expand(q[:, 0]) | (expand(q[:, 1]) << np.uint64(1)) | (expand(q[:, 2]) << np.uint64(2))


def brute_pairs(boxes):
    out = set()
    for i in range(len(boxes)):
        for j in range(i + 1, len(boxes)):
            a, b = boxes[i], boxes[j]
            if np.all(a[:3] <= b[3:]) and np.all(a[3:] >= b[:3]):
                out.add((i, j))
    return out


def _triangle_scene(oracle_lib, tris, vel=None, dt=1e-3):
    o = oracle_lib.Oracle()
    o.set_params(dt)
    P = np.asarray(tris, dtype=np.float64).reshape(-1, 3)
    o.add_particles(P, np.zeros(len(P)))
    if vel is not None:
        o.set_velocities(0, vel)
    o.add_triangles(np.arange(len(P)).reshape(-1, 3), 0)
    o.finalize()
    o.collision_stage()
    return o, P


def test_few_triangles(oracle_lib):
    fx = golden("lbvh_inputs.json")
    o, P = _triangle_scene(oracle_lib, fx["triangles"])
    t = o.lbvh(4)
    T = P.reshape(-1, 3, 3)
    boxes = np.concatenate([T.min(1), T.max(1)], axis=1)
    assert (t["morton"] == morton_numpy(boxes)).all()
    assert (t["sorted_order"] == np.argsort(t["morton"], kind="stable")).all()
    got = {tuple(sorted((int(t["sorted_order"][a]), int(t["sorted_order"][b])))) for a, b in t["pairs"]}
    assert got == brute_pairs(boxes)
    assert all(a < b for a, b in t["pairs"])


def test_random_triangles_swept(oracle_lib):
    rng = np.random.default_rng(3)
    n = 300
    c = rng.uniform(0, 1, size=(n, 1, 3))
    tris = c + rng.uniform(-0.03, 0.03, size=(n, 3, 3))
    vel = rng.normal(0, 5, size=(n * 3, 3))
    dt = 1 / 60
    o, P = _triangle_scene(oracle_lib, tris, vel, dt)
    t = o.lbvh(n)
    Pn = P + dt * vel
    both = np.concatenate([P.reshape(-1, 3, 3), Pn.reshape(-1, 3, 3)], axis=1)
    boxes = np.concatenate([both.min(1), both.max(1)], axis=1)
    assert (t["morton"] == morton_numpy(boxes)).all()
    assert (t["sorted_order"] == np.argsort(t["morton"], kind="stable")).all()
    got = {tuple(sorted((int(t["sorted_order"][a]), int(t["sorted_order"][b])))) for a, b in t["pairs"]}
    assert got == brute_pairs(boxes)
    # refit: every internal node bounds the union of its children
    nn = 2 * n - 1
    B = t["bounds"]
    for node in range(n, nn):
        l, r = t["left"][node], t["right"][node]
        assert (B[node, :3] == np.minimum(B[l, :3], B[r, :3])).all()
        assert (B[node, 3:] == np.maximum(B[l, 3:], B[r, 3:])).all()


def test_equal_codes_break_ties_on_index(oracle_lib):
    """commonPrefixLen falls back to the primitive indices (collision/LBVHBuilder.hpp:33-41)."""
    o = oracle_lib.Oracle()
    codes = np.array([7, 7, 7, 3, 7, 3], dtype=np.uint64)
    t = o.lbvh_from_codes(codes)
    assert t["sorted_order"].tolist() == [3, 5, 0, 1, 2, 4]
    # a valid binary tree over 6 leaves
    n = 6
    kids = [t["left"][k] for k in range(n, 2 * n - 1)] + [t["right"][k] for k in range(n, 2 * n - 1)]
    assert sorted(kids) == sorted(set(range(2 * n - 1)) - {t["root"]})
