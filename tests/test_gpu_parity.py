"""Parity of the engine (through its C-ABI) with the FP64 oracle.

Tolerances (max vertex position error relative to the scene's bounding-box
diagonal):
  * FP64 engine vs oracle: 1e-9 -- same algorithm, only the summation order and
    the block-solve factorisation differ;
  * FP32 engine vs oracle: 1e-5 -- FP32 accumulation with the FP64 fallback of
    ill-conditioned blocks.
Integer outputs (coloring) are compared bit for bit.
"""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu

TOL64 = 1e-9
TOL32 = 1e-5


def pair(sc, oracle_lib, precision="fp32", **kw):
    e = Context()
    sc.load(e, precision=precision, **kw)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o, **kw)
    o.finalize()
    return e, o


def rel_err(e, o, sc):
    return np.abs(e.positions() - o.positions()).max() / sc.bbox_diagonal()


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_cube_fixed_bottom_100_steps(oracle_lib, precision, tol):
    sc = scenes.cube_fixed_bottom(8)
    e, o = pair(sc, oracle_lib, precision)
    ce, nce = e.coloring()
    co, nco = o.coloring()
    assert nce == nco and (ce == co).all()
    x0 = o.positions()
    for _ in range(10):
        e.step(10)
        o.step(10)
        assert rel_err(e, o, sc) < tol
    assert np.abs(o.positions() - x0).max() > 1e-3  # the cube moved
    np.testing.assert_allclose(e.velocities(), o.velocities(), atol=tol * sc.bbox_diagonal() * 60 * 10)


def oracle_sensitivity(sc, oracle_lib, steps):
    """How far the FP64 oracle itself moves when its initial positions are
    rounded to FP32: the floor below which no FP32 engine can be expected to
    track a contact scene whose friction switches stick/slip discretely."""
    a = oracle_lib.Oracle()
    sc.load(a)
    a.finalize()
    b = oracle_lib.Oracle()
    sc.load(b)
    b.finalize()
    b.set_positions_raw(0, a.positions().astype(np.float32).astype(np.float64))
    a.step(steps)
    b.step(steps)
    return np.abs(a.positions() - b.positions()).max() / sc.bbox_diagonal()


def test_cube_drop_ground_contact_fp64(oracle_lib):
    sc = scenes.cube_drop(n=6, iters=20, surface=True)
    e, o = pair(sc, oracle_lib, "fp64")
    for _ in range(6):
        e.step(10)
        o.step(10)
    assert o.positions()[:, 1].min() < 0.05  # it reached the ground
    assert rel_err(e, o, sc) < TOL64


def test_cube_drop_ground_contact_fp32(oracle_lib):
    """FP32 with contact: within 1e-5 of the bbox diagonal before touchdown;
    after touchdown within 3x the oracle's own sensitivity to FP32 rounding of
    its inputs (and never above 1e-3)."""
    sc = scenes.cube_drop(n=6, iters=20, surface=True)
    e, o = pair(sc, oracle_lib, "fp32")
    e.step(10)
    o.step(10)
    assert rel_err(e, o, sc) < TOL32  # free fall
    e.step(50)
    o.step(50)
    err = rel_err(e, o, sc)
    floor = oracle_sensitivity(sc, oracle_lib, 60)
    assert err < max(TOL32, 3 * floor) and err < 1e-3, (err, floor)


def test_damping_fp64(oracle_lib):
    sc = scenes.Scene(name="damped", dt=1 / 60, solver_iters=10, iter_acceleration=0.5)
    scenes.add_tet_cube(sc, 4, E=1e5, nu=0.4, kd=10.0, fix_bottom=True)
    e, o = pair(sc, oracle_lib, "fp64")
    e.step(30)
    o.step(30)
    assert rel_err(e, o, sc) < TOL64


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_block_gradient_hessian(oracle_lib, precision):
    """avbd_debug_block vs the oracle's accumulate at a perturbed state (the
    scalar-vs-AVX comparison of test/test_neohookean_accumulate.cpp:51-84)."""
    sc = scenes.cube_drop(n=4, surface=False)
    e, o = pair(sc, oracle_lib, precision)
    rng = np.random.default_rng(0)
    X = o.positions() + rng.uniform(-0.02, 0.02, size=(o.num_particles, 3))
    if precision == "fp32":
        X = X.astype(np.float32).astype(np.float64)
    e.set_positions(0, X)
    o.set_positions_raw(0, X)
    rtol = 1e-10 if precision == "fp64" else 2e-4
    for p in rng.choice(o.num_particles, 12, replace=False):
        Ge, He = e.debug_block(int(p))
        Go, Ho = o.debug_block(int(p))
        scale_g = np.abs(Go).max() + 1e-12
        scale_h = np.abs(Ho).max()
        assert np.abs(Ge - Go).max() <= rtol * max(scale_g, scale_h * 1e-2) + 1e-9, (p, Ge, Go)
        assert np.abs(He - Ho).max() <= rtol * scale_h, (p, He, Ho)


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32 * 10)])
def test_batched_scenes(oracle_lib, precision, tol):
    sc = scenes.batched_cubes(num_scenes=7, seed=3, n_min=2, n_max=5, iters=15)
    e, o = pair(sc, oracle_lib, precision)
    ce, nce = e.coloring()
    co, nco = o.coloring()
    assert nce == nco and (ce == co).all()
    e.step(20)
    o.step(20)
    assert rel_err(e, o, sc) < tol


def test_coloring_bit_exact_large(oracle_lib):
    sc = scenes.cube_drop(n=16, surface=False)
    e, o = pair(sc, oracle_lib, "fp32")
    ce, nce = e.coloring()
    co, nco = o.coloring()
    assert nce == nco and (ce == co).all()


def test_residual_matches_oracle(oracle_lib):
    sc = scenes.cube_drop(n=4, surface=False)
    e, o = pair(sc, oracle_lib, "fp64")
    e.step(3)
    o.step(3)
    assert abs(e.residual() - o.residual()) <= 1e-8 * max(1.0, o.residual())


def test_run_to_tolerance(oracle_lib):
    sc = scenes.cube_fixed_bottom(6)
    e, o = pair(sc, oracle_lib, "fp64", residual_tolerance=1e-4, max_iters=500)
    e.step(5)
    o.step(5)
    st = e.stats()
    assert st["last_residual"] <= 1e-4
    assert st["iterations"] == o.iterations
    assert rel_err(e, o, sc) < 1e-7


@pytest.mark.parametrize("n", [4, 8])
def test_mixed_precision_tracks_oracle(oracle_lib, n):
    """Mixed mode (FP64 state and gradient, FP32 records and Hessian): the FP32
    rounding of the element data perturbs the model by ~1e-7 relative."""
    sc = scenes.cube_fixed_bottom(n)
    e, o = pair(sc, oracle_lib, "mixed")
    e.step(50)
    o.step(50)
    assert rel_err(e, o, sc) < 1e-6


def test_mixed_run_to_tolerance_on_stiff_batch(oracle_lib):
    """Stiff scenes reach R <= 1e-4 in the mixed mode with about the oracle's
    iteration count, while FP32 stalls on its rounding floor."""
    sc = scenes.batched_cubes(num_scenes=4, seed=5, n_min=5, n_max=8)
    e, o = pair(sc, oracle_lib, "mixed", residual_tolerance=1e-4, max_iters=300)
    for step in range(7):
        e.step(1)
        o.step(1)
        # every scene's iterations of every step within 2 of the oracle's
        ie, io = e.scene_iterations().astype(int), o.scene_iterations().astype(int)
        assert np.abs(ie - io).max() <= 2, (step, ie, io)
    assert e.stats()["last_residual"] <= 1e-4


def test_per_scene_tolerance_batch_fp64(oracle_lib):
    """Every scene of a batch iterates to its own residual: the FP64 engine
    spends the oracle's scene-iterations and ends in the oracle's state."""
    sc = scenes.batched_cubes(num_scenes=6, seed=2, n_min=3, n_max=6)
    e, o = pair(sc, oracle_lib, "fp64", residual_tolerance=1e-4, max_iters=200)
    for _ in range(5):
        e.step(1)
        o.step(1)
    st = e.stats()
    assert abs(st["iterations"] - o.iterations) <= 2, (st["iterations"], o.iterations)
    assert rel_err(e, o, sc) < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_piece_launches_match_slab_launches(monkeypatch, precision):
    """Run-to-tolerance sweeps launch one block per (color, scene) piece of
    at most 512 vertices (fewer here, to cut scenes into several pieces);
    AVBD_SOLVE_CHUNK=0 launches whole slabs.  Both update the same vertices
    with the same arithmetic: the states and iteration counts agree."""
    sc = scenes.batched_cubes(num_scenes=6, seed=3, n_min=3, n_max=7)
    runs = {}
    for chunk in ("40", "0"):
        monkeypatch.setenv("AVBD_SOLVE_CHUNK", chunk)
        e = Context()
        sc.load(e, precision=precision, residual_tolerance=1e-4, max_iters=150)
        e.finalize()
        e.step(5)
        runs[chunk] = (e.positions(), e.stats()["iterations"])
    (xa, ia), (xb, ib) = runs["40"], runs["0"]
    assert abs(ia - ib) <= 2, (ia, ib)
    assert np.abs(xa - xb).max() / sc.bbox_diagonal() < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_iteration_loop_matches_host_loop(monkeypatch, precision):
    """A run-to-tolerance step is one CUDA graph whose iteration loop is a
    conditional while node (index and Chebyshev weight in device memory);
    AVBD_GRAPH=0 runs the same launches from a host loop that reads the count
    of scenes still iterating after every iteration.  The per-scene sums of
    residuals are atomic, so the two agree to rounding: states, iteration
    counts and launch counts (the graph adds one loop-control kernel per
    iteration)."""
    sc = scenes.batched_cubes(num_scenes=6, seed=5, n_min=3, n_max=7)
    runs = {}
    for graph in ("1", "0"):
        monkeypatch.setenv("AVBD_GRAPH", graph)
        e = Context()
        sc.load(e, precision=precision, residual_tolerance=1e-4, max_iters=150)
        e.finalize()
        e.step(2)
        e.step(4)  # the second call replays the recorded graph
        st = e.stats()
        runs[graph] = (e.positions(), st["iterations"], st["kernel_launches"], st["capped_scene_steps"])
        e.close()
    (xa, ia, la, ca), (xb, ib, lb, cb) = runs["1"], runs["0"]
    assert ia > 6 * 6 and abs(ia - ib) <= 2, (ia, ib)
    assert ca == cb
    assert np.abs(xa - xb).max() / sc.bbox_diagonal() < 1e-7
    assert lb < la < 1.2 * lb, (la, lb)


def test_stats_and_no_fallback_on_c1(oracle_lib):
    sc = scenes.cube_fixed_bottom(8)
    e, _ = pair(sc, oracle_lib, "fp32")
    e.step(5)
    st = e.stats()
    assert st["iterations"] == 50 and st["kernel_launches"] > 0 and st["num_colors"] >= 4
