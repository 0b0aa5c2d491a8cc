"""The oracle's triangle-rod contacts: the closest-point narrow phase
(CollisionDetector::_triangleRod, collision/CollisionDetector.cpp:601-666;
Math::closestPoint_SegmentTriangle, common/Math.hpp:593-681) on cases with
known answers, and the triangle-rod contact pool and recoloring on rods
dropped on a soft cube (invariants the reference code guarantees; its tests
do not cover this path)."""
import numpy as np
import pytest

from avbd_b200 import scenes
from oracle.oracle import Oracle


def detect(p0, p1, radius=0.05, margin=1e-3, q=(1, 0, 0, 0), tri=None):
    o = Oracle()
    o.set_params(0.01, 0.0, margin)
    o.set_solver(1, 0.5)
    T = np.array(tri if tri is not None else [[0, 0, 0], [1, 0, 0], [0, 0, 1.0]])
    o.add_particles(T, np.ones(3))
    o.set_fixed([0, 1, 2], [1, 1, 1])
    o.add_oriented_particles(np.array([p0, p1], dtype=float), np.array([q, q], dtype=float), [1.0, 1.0],
                             np.ones((2, 3)))
    o.add_triangles(np.array([[0, 1, 2]]), 0)
    o.add_rod_segments(np.array([[3, 4]]), radius, 1)
    o.finalize()
    o.collision_stage()
    return o.rod_contacts()


def test_segment_above_the_triangle():
    """A segment 4 cm above the triangle, radius 5 cm: the closest point is an
    end point's projection, the normal points from the centreline down to the
    triangle, the rod point is radius * normal in the rod frame."""
    c = detect([0.2, 0.04, 0.2], [0.6, 0.04, 0.2])
    assert len(c["key"]) == 1
    assert c["tri"].tolist() == [[0, 1, 2]] and c["rod"].tolist() == [[3, 4]]
    assert np.allclose(c["normal"][0], [0, -1, 0], atol=1e-12)
    assert np.allclose(c["cp_local"][0], [0, -0.05, 0], atol=1e-12)
    assert c["s"][0] in (0.0, 1.0)                       # an end point wins the parallel case
    cl = (1 - c["s"][0]) * np.array([0.2, 0.04, 0.2]) + c["s"][0] * np.array([0.6, 0.04, 0.2])
    foot = c["barys"][0] @ np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1.0]])
    assert np.allclose(foot, [cl[0], 0, cl[2]], atol=1e-12)
    assert c["key"][0] == (3 << 59) | (0 << 33) | (1 << 7)  # TriangleRod, primitives 0 and 1


def test_segment_out_of_reach():
    assert len(detect([0.2, 0.06, 0.2], [0.6, 0.06, 0.2])["key"]) == 0   # 6 cm > r + margin


def test_crossing_segment():
    """A segment through the triangle: distance 0 at the crossing, the
    centreline point and the triangle point coincide and the normal falls
    back to +x."""
    c = detect([0.25, -0.1, 0.25], [0.25, 0.1, 0.25])
    assert len(c["key"]) == 1
    assert np.isclose(c["s"][0], 0.5, atol=1e-12)
    assert np.allclose(c["barys"][0], [0.5, 0.25, 0.25], atol=1e-12)
    assert np.allclose(c["normal"][0], [1, 0, 0])


def test_edge_distance_uses_the_segments_parameter():
    """The edge test measures its distance to (1-s) q0 + s q1 (the edge point
    at the segment's parameter, not at the edge's own t).  A segment 3 cm over
    the triangle near vertex b, crossing edge (a, b) at s = 0.5, t = 0.9: the
    edge tests report 0.4, 0.9 and 0.92 instead of 0.03, the end points
    project to 0.20 and 0.077, nothing crosses the plane, so with radius 5 cm
    no contact is reported although the segment is 3 cm away."""
    c = detect([0.9, 0.03, -0.2], [0.9, 0.03, 0.2])
    assert len(c["key"]) == 0
    # with radius 8 cm the nearer end point (0.077 away) gives the contact
    c = detect([0.9, 0.03, -0.2], [0.9, 0.03, 0.2], radius=0.08)
    assert len(c["key"]) == 1 and c["s"][0] == 1.0
    foot = c["barys"][0] @ np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1.0]])
    assert np.allclose(foot, [0.85, 0, 0.15], atol=1e-12)


def make(rounds=None, **kw):
    sc = scenes.rods_on_cube(**kw)
    o = Oracle()
    sc.load(o)
    o.finalize()
    if rounds is not None:
        o.set_recolor_rounds(rounds)
    return sc, o


def test_rod_contacts_form_and_pool_matches_detections():
    sc, o = make()
    seen = 0
    for _ in range(30):
        o.step(1)
        info = o.dynamic_info()
        det = o.rod_contacts()
        pool = o.rod_contact_pool()
        live = np.nonzero(pool["active"])[0]
        assert info["rod_live"] == len(live) == len(det["key"])
        a = sorted(tuple(int(v) for v in pool["particles"][s]) for s in live)
        b = sorted(tuple(int(v) for v in list(det["tri"][k]) + list(det["rod"][k])) for k in range(len(det["key"])))
        assert a == b
        assert info["entries"] == 5 * info["rod_live"] + 4 * info["live"]
        for s in live:
            F = np.stack([pool["n"][s], pool["t"][s], pool["b"][s]])
            assert np.allclose(F @ F.T, np.eye(3), atol=1e-9)
            assert 0.0 <= pool["s"][s] <= 1.0
        seen = max(seen, len(live))
    assert seen > 0


def test_rods_rest_on_the_cube_with_a_valid_coloring():
    sc, o = make()
    adj = o.adjacency()
    static = set()
    for p in range(o.num_particles):
        for q in adj["p_nbr"][adj["p_off"][p]:adj["p_off"][p + 1]]:
            static.add((min(p, int(q)), max(p, int(q))))
    for _ in range(60):
        o.step(1)
        col, _ = o.coloring()
        conf = o.conflicted()
        E = set(static)
        pool = o.rod_contact_pool()
        for s in np.nonzero(pool["active"])[0]:
            ps = [int(v) for v in pool["particles"][s]]
            E |= {(min(a, b), max(a, b)) for i, a in enumerate(ps) for b in ps[i + 1:]}
        for p, q in E:
            assert col[p] != col[q] or (conf[p] and conf[q]), (p, q)
    x = o.positions()
    top = x[:125, 1].max()
    assert np.isfinite(x).all()
    assert np.all(x[125:, 1] > top - 0.02) and np.all(x[125:, 1] < top + 0.1)
