"""DSATUR (ColorList::greedyColor2, common/ColorList.hpp:149-241) in the oracle:
the heap-ordered variant used for large scenes must make exactly the picks of
the verbatim O(V^2) loop, and every coloring must be proper."""
import numpy as np
import pytest

from avbd_b200 import scenes


def _colors(oracle_lib, sc, reference):
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize(reference_dsatur=reference)
    return o


@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_fast_equals_verbatim_on_cubes(oracle_lib, n):
    sc = scenes.cube_fixed_bottom(n)
    a, na = _colors(oracle_lib, sc, False).coloring()
    b, nb = _colors(oracle_lib, sc, True).coloring()
    assert na == nb and (a == b).all()


def test_fast_equals_verbatim_on_perturbed_and_batched(oracle_lib):
    sc = scenes.batched_cubes(num_scenes=6, seed=1, n_min=2, n_max=5)
    a, na = _colors(oracle_lib, sc, False).coloring()
    b, nb = _colors(oracle_lib, sc, True).coloring()
    assert na == nb and (a == b).all()


def test_random_tet_soup(oracle_lib):
    rng = np.random.default_rng(7)
    nv = 200
    o1, o2 = oracle_lib.Oracle(), oracle_lib.Oracle()
    X = rng.uniform(0, 1, (nv, 3))
    tets = np.array([rng.choice(nv, 4, replace=False) for _ in range(400)])
    for o in (o1, o2):
        o.set_params(1e-2)
        o.add_particles(X, np.ones(nv))
        o.add_neo_hookean(tets, np.full(400, 1.0), np.full(400, 1.0), np.zeros(400), np.tile(np.eye(3).ravel(), (400, 1)),
                          np.ones(400))
    o1.finalize(False)
    o2.finalize(True)
    a, na = o1.coloring()
    b, nb = o2.coloring()
    assert na == nb and (a == b).all()
    adj = o1.adjacency()
    for p in range(nv):
        for q in adj["p_nbr"][adj["p_off"][p]:adj["p_off"][p + 1]]:
            assert a[p] != a[q]


def test_adjacency_layout(oracle_lib):
    """Entries grouped by particle, then type, then pool slot
    (StaticParticleAdjacency::buildAdjacency, common/StaticParticleAdjacency.hpp:42-133)."""
    sc = scenes.cube_drop(n=2, surface=False)
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    adj = o.adjacency()
    n = o.num_particles
    for p in range(n):
        b, e = adj["e_off"][p, 0], adj["e_off"][p + 1, 0]
        types = adj["type"][b:e]
        assert (np.diff(types.astype(int)) >= 0).all()
        for t in range(5):
            seg = adj["idx"][adj["e_off"][p, t]:(adj["e_off"][p, t + 1] if t < 4 else adj["e_off"][p + 1, 0])]
            assert (np.diff(seg.astype(np.int64)) > 0).all()
        assert (types == 2).sum() == 1  # one ground energy per vertex
