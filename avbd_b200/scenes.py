"""Procedural scene builders for the engine's workloads.

A Scene records the set-up calls a host application makes against a
SimulationContext (particles, energies, collision primitives, parameters) and
replays them into any object exposing the same method names -- the engine's
avbd_b200.Context or the FP64 oracle used by the tests.

The per-object set-up math restates the reference's scene objects, which
build their particles and energies with plain FP64 arithmetic:
  * TetMeshObject::setup (simobject/TetMeshObject.cpp:21-113): Lame
    parameters mu = E/(2(1+nu)), lambda = E nu/((1+nu)(1-2nu)); per tet
    X = [v1-v4, v2-v4, v3-v4], Q = X^-1, V = |det X|/6; lumped mass V rho/4;
  * per-vertex ground contact (simulation/Simulation.hpp:117-126):
    k_start = m/dt^2, mu_s = 0.4, mu_k = 0.2;
  * Rod::Rod (simobject/Rod.cpp:10-68) and RigidSphere (simobject/rigid/
    RigidSphere.cpp:8-22) for the oriented particles.
Meshes are generated here (a hex grid split into 6 tets per cell) instead of
being read from gmsh files.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np


@dataclass
class Scene:
    name: str
    dt: float
    g_accel: float = 9.81
    collision_margin: float = 1e-3
    solver_iters: int = 10
    iter_acceleration: float = 0.5
    calls: list = field(default_factory=list)
    num_particles: int = 0
    num_tets: int = 0
    num_primitives: int = 0
    num_scenes: int = 1
    meta: dict = field(default_factory=dict)

    def record(self, method: str, *args, **kwargs):
        self.calls.append((method, args, kwargs))

    def load(self, target: Any, residual_tolerance: float = 0.0, max_iters: int = 0, precision=None):
        target.set_params(self.dt, self.g_accel, self.collision_margin)
        target.set_solver(self.solver_iters, self.iter_acceleration, residual_tolerance, max_iters, precision)
        for method, args, kwargs in self.calls:
            getattr(target, method)(*args, **kwargs)
        return target

    def bbox_diagonal(self) -> float:
        return float(self.meta.get("bbox_diagonal", 1.0))


def lame(E: float, nu: float):
    """TetMeshObject::setup (simobject/TetMeshObject.cpp:44-45)."""
    mu = E / (2 * (1 + nu))
    lam = (E * nu) / ((1 + nu) * (1 - 2 * nu))
    return lam, mu


def hex_grid_tets(n: int):
    """Vertex grid (n+1)^3 (x fastest) and 6 tets per cell (Kuhn split along the
    (0,0,0)-(1,1,1) cell diagonal, the same diagonal in every cell)."""
    m = n + 1

    def vid(i, j, k):
        return i + m * (j + m * k)

    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    corner = lambda a, b, c: vid(ii + a, jj + b, kk + c)
    e = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    tets = []
    for perm in [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]:
        p1 = e[perm[0]]
        p2 = tuple(e[perm[0]][t] + e[perm[1]][t] for t in range(3))
        tets.append(np.stack([corner(0, 0, 0), corner(*p1), corner(*p2), corner(1, 1, 1)], axis=1))
    # cell-major order: all 6 tets of a cell are consecutive
    T = np.stack(tets, axis=1).reshape(-1, 4)
    return T.astype(np.uint32)


def surface_triangles(tets: np.ndarray) -> np.ndarray:
    """Boundary faces of a tet mesh (faces used by exactly one tet)."""
    f = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    key = np.sort(f, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    once = cnt[inv.ravel()] == 1
    return f[once].astype(np.uint32)


def tet_setup(X: np.ndarray, tets: np.ndarray, E, nu, density):
    """Q, rest volume and lumped masses of TetMeshObject::setup
    (simobject/TetMeshObject.cpp:62-97)."""
    v1, v2, v3, v4 = (X[tets[:, k]] for k in range(4))
    a, b, c = v1 - v4, v2 - v4, v3 - v4  # columns of X
    # X^-1 rows are the cross products of the columns over det X
    r0, r1, r2 = np.cross(b, c), np.cross(c, a), np.cross(a, b)
    det = np.einsum("ij,ij->i", a, r0)
    Q = np.stack([r0, r1, r2], axis=1) / det[:, None, None]
    V = np.abs(det / 6.0)
    lam, mu = lame(E, nu)
    masses = np.bincount(tets.ravel(), weights=np.repeat(0.25 * V * density, 4), minlength=len(X))
    return Q, V, lam, mu, masses


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def add_tet_cube(sc: Scene, n: int, size: float = 1.0, origin=(0.0, 0.0, 0.0), E=1e5, nu=0.45,
                 density=1000.0, kd=0.0, perturb=0.0, rng=None, rotation=None,
                 fix_bottom=False, ground=False, surface=False, object_id=0, velocity=None, bottom_at=None):
    """Adds one cube of n^3 hex cells (6 tets each) to the scene."""
    m = n + 1
    h = size / n
    g = np.arange(m) * h
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    # vertex id = i + m*(j + m*k): x fastest
    X = np.stack([gx.transpose(2, 1, 0).ravel(), gy.transpose(2, 1, 0).ravel(), gz.transpose(2, 1, 0).ravel()], axis=1)
    jidx = (np.arange(m ** 3) // m) % m
    if perturb > 0:
        rng = rng if rng is not None else np.random.default_rng(0)
        X = X + rng.uniform(-perturb * h, perturb * h, size=X.shape)
    if rotation is not None:
        c = np.full(3, size / 2)
        X = (X - c) @ np.asarray(rotation).T + c
    X = X + np.asarray(origin, dtype=np.float64)
    if bottom_at is not None:
        X[:, 1] += bottom_at - X[:, 1].min()
    tets = hex_grid_tets(n)
    Q, V, lam, mu, masses = tet_setup(X, tets, E, nu, density)
    base = sc.num_particles
    sc.record("add_particles", X, masses)
    if velocity is not None:
        vel = np.tile(np.asarray(velocity, dtype=np.float64), (len(X), 1))
        sc.record("set_velocities", base, vel, vel)
    gt = tets.astype(np.int64) + base
    nt = len(tets)
    sc.record("add_neo_hookean", gt, np.full(nt, lam), np.full(nt, mu), np.full(nt, kd), Q.reshape(-1, 9), V)
    if fix_bottom:
        slots = np.nonzero(jidx == 0)[0] + base
        sc.record("set_fixed", slots, np.ones(len(slots), dtype=np.uint8))
    if ground:
        ks = masses / (sc.dt * sc.dt)
        sc.record("add_ground_collision", np.arange(len(X)) + base, ks, np.full(len(X), 0.4), np.full(len(X), 0.2))
    if surface:
        tri = surface_triangles(tets).astype(np.int64) + base
        sc.record("add_triangles", tri, object_id)
        sc.num_primitives += len(tri)
    sc.num_particles += len(X)
    sc.num_tets += nt
    lo, hi = X.min(0), X.max(0)
    sc.meta.setdefault("boxes", []).append((lo, hi))
    allb = sc.meta["boxes"]
    glo = np.min([b[0] for b in allb], axis=0)
    ghi = np.max([b[1] for b in allb], axis=0)
    sc.meta["bbox_diagonal"] = float(np.linalg.norm(ghi - glo))
    return base


def cube_fixed_bottom(n: int = 8, steps_dt: float = 1.0 / 60.0, iters: int = 10, rho: float = 0.5) -> Scene:
    """Single NeoHookean cube, bottom face fixed, no collision:
    1 m cube of n^3 cells, rho 1000 kg/m^3, E 1e5 Pa, nu 0.45, g 9.81, dt 1/60,
    10 iterations per step (n = 8: 729 vertices, 3072 tets)."""
    sc = Scene(name=f"cube{n}_fixed", dt=steps_dt, solver_iters=iters, iter_acceleration=rho)
    add_tet_cube(sc, n, E=1e5, nu=0.45, density=1000.0, fix_bottom=True)
    return sc


def cube_drop(n: int = 32, seed: int = 0, iters: int = 20, rho: float = 0.5, dt: float = 1.0 / 60.0,
              height: float = 0.5, surface: bool = True) -> Scene:
    """Cube dropped onto the ground plane with self-collision candidates:
    1 m cube of n^3 cells (n = 32: 35,937 vertices, 196,608 tets, 12,288
    surface triangles), E 1e6, nu 0.49, rho 1000, every vertex perturbed by
    seeded uniform noise of +-0.2 cell, bottom face at y = height, per-vertex
    ground contact, 20 iterations per step."""
    sc = Scene(name=f"cube{n}_drop", dt=dt, solver_iters=iters, iter_acceleration=rho)
    rng = np.random.default_rng(seed)
    add_tet_cube(sc, n, origin=(0.0, height, 0.0), E=1e6, nu=0.49, density=1000.0, perturb=0.2, rng=rng,
                 ground=True, surface=surface)
    return sc


def batched_cube_params(seed: int, s: int, n_min: int = 4, n_max: int = 24):
    """Parameters of scene s of a batch: drawn from a generator seeded by
    (seed, s), so any subset of a batch is reproduced exactly."""
    rng = np.random.default_rng([seed, s])
    n = int(rng.integers(n_min, n_max + 1))
    E = float(10 ** rng.uniform(4, 7))
    nu = float(rng.uniform(0.3, 0.49))
    R = random_rotation(rng)
    return n, E, nu, R


def batched_cubes(num_scenes: int = 1024, seed: int = 0, n_min: int = 4, n_max: int = 24, iters: int = 15,
                  rho: float = 0.5, dt: float = 1.0 / 60.0, spacing: float = 2.0, scene_ids=None) -> Scene:
    """Many independent cubes of uneven size advanced together: cell counts
    n ~ U{n_min..n_max} per side (6 n^3 tets), E log-uniform in [1e4, 1e7],
    nu ~ U(0.3, 0.49), random initial rotation, per-vertex ground contact,
    15 iterations per step.  Each cube is its own scene (own coloring).
    scene_ids selects a subset of the batch (same cubes, same placement)."""
    ids = list(range(num_scenes)) if scene_ids is None else list(scene_ids)
    sc = Scene(name=f"batch{num_scenes}", dt=dt, solver_iters=iters, iter_acceleration=rho)
    side = int(np.ceil(np.sqrt(num_scenes)))
    cells = []
    for k, s in enumerate(ids):
        if k > 0:
            sc.record("begin_scene")
        n, E, nu, R = batched_cube_params(seed, s, n_min, n_max)
        cells.append(n)
        ox, oz = (s % side) * spacing, (s // side) * spacing
        add_tet_cube(sc, n, size=1.0, origin=(ox, 0.0, oz), E=E, nu=nu, density=1000.0, rotation=R, ground=True,
                     bottom_at=0.3)
    sc.num_scenes = len(ids)
    sc.meta["cells"] = cells
    return sc
