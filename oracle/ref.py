"""ctypes binding of the reference implementation itself (oracle/_ref).

TEST INFRASTRUCTURE: oracle/Makefile compiles the reference's unmodified
hot-path sources (simulation/VBDSolver.hpp, simulation/SimulationExecutor.hpp,
energy/**, common/*.hpp, collision/{CollisionDetector,LBVHBuilder,LBVH}.cpp)
against the project's Eigen-API shim (oracle/eigen_shim) into
oracle/_ref/libavbd_ref.so, driven by oracle/ref_harness.cpp.  Only tests/ and
the CPU legs of bench.py load it: it pins the FP64 restatement
(oracle/oracle.py) to the reference, and it is the reference arm of the CPU
baseline.  The library is built only where the reference sources are present
(`build()`); elsewhere `available()` is False.

`RefSim` takes the same set-up calls as `oracle.Oracle` and
`avbd_b200.Context`, so a scene description loads into any of them.  The
reference has no residual and no run-to-tolerance mode: it runs the fixed
iteration count of `set_solver`.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libavbd_ref.so")
# where the reference sources are read from when the library is built
REFERENCE_ROOT = os.environ.get("AVBD_REFERENCE_ROOT", "/root/reference")
_lib = None


def build(force: bool = False) -> str | None:
    """Compiles oracle/_ref/libavbd_ref.so when the reference sources are
    present; returns the library path, or None without them."""
    if not os.path.isdir(os.path.join(REFERENCE_ROOT, "simulation")):
        return LIB_PATH if os.path.exists(LIB_PATH) else None
    args = ["make", "-s", "-C", _HERE, f"REF={REFERENCE_ROOT}", "_ref/libavbd_ref.so"]
    if force:
        args.insert(2, "-B")
    subprocess.check_call(args)
    return LIB_PATH


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} is missing (build it with oracle.ref.build())")
        L = C.CDLL(LIB_PATH)
        vp, dp, up, u8p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint), C.POINTER(C.c_uint8)
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_create": (vp, [C.c_uint] * 6),
            "ref_destroy": (None, [vp]),
            "ref_set_params": (None, [vp, C.c_double, C.c_double, C.c_double]),
            "ref_set_solver": (None, [vp, C.c_uint, C.c_double]),
            "ref_particles_add": (C.c_uint, [vp, C.c_uint, dp, dp]),
            "ref_particles_add_oriented": (C.c_uint, [vp, C.c_uint, dp, dp, dp, dp]),
            "ref_set_fixed": (None, [vp, C.c_uint, up, u8p]),
            "ref_set_velocities": (None, [vp, C.c_uint, C.c_uint, dp, dp]),
            "ref_set_angular_velocities": (None, [vp, C.c_uint, C.c_uint, dp]),
            "ref_neo_hookean_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp, dp, dp]),
            "ref_cosserat_rod_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp]),
            "ref_ground_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp]),
            "ref_rigid_ground_add": (C.c_uint, [vp, C.c_uint, up, u8p, dp, dp, dp, dp, dp]),
            "ref_joint_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp, dp]),
            "ref_add_triangles": (C.c_uint, [vp, C.c_uint, up, C.c_uint]),
            "ref_add_rod_segments": (C.c_uint, [vp, C.c_uint, up, C.c_double, C.c_uint]),
            "ref_add_spheres": (C.c_uint, [vp, C.c_uint, up, dp, up]),
            "ref_finalize": (C.c_int, [vp]),
            "ref_step": (C.c_int, [vp, C.c_uint]),
            "ref_set_iterations": (C.c_int, [vp, C.c_uint]),
            "ref_time_steps": (C.c_double, [vp, C.c_uint]),
            "ref_num_particles": (C.c_uint, [vp]),
            "ref_get_positions": (None, [vp, dp]),
            "ref_get_velocities": (None, [vp, dp]),
            "ref_get_rotations": (None, [vp, dp]),
            "ref_get_angular_velocities": (None, [vp, dp]),
            "ref_get_coloring": (None, [vp, up, up]),
            "ref_num_primitives": (C.c_uint, [vp]),
            "ref_collect_pairs": (C.c_uint, [vp]),
            "ref_get_lbvh": (None, [vp, C.POINTER(C.c_uint64), up, up, up, up, up, dp, up, up]),
            "ref_dynamic_info": (None, [vp, up]),
            "ref_get_trc": (None, [vp, up, u8p, dp]),
            "ref_get_trd": (None, [vp, up, u8p, dp]),
            "ref_get_conflicted": (None, [vp, u8p]),
            "ref_debug_block": (C.c_int, [vp, C.c_uint, dp, dp, C.POINTER(C.c_int)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _u(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def capacities(scene) -> dict:
    """Pool capacities for a scene description: the largest pool it fills,
    with room for the dynamic contact pools."""
    counts = {"particles": 0, "oriented": 0, "energies": 1, "prims": 1, "sdf": 1}
    per_pool = {}
    width = {"add_particles": 3, "add_oriented_particles": 3, "add_neo_hookean": 4, "add_cosserat_rod": 2,
             "add_triangles": 3, "add_rod_segments": 2}
    for method, args, _ in scene.calls:
        if not method.startswith("add_") or not args:
            continue
        n = np.asarray(args[0]).size // width.get(method, 1)
        if method == "add_particles":
            counts["particles"] += n
        elif method == "add_oriented_particles":
            counts["particles"] += n
            counts["oriented"] += n
        elif method in ("add_triangles", "add_rod_segments", "add_spheres"):
            counts["prims"] += n
            counts["sdf"] += n if method == "add_spheres" else 1
        elif method.startswith("add_"):
            per_pool[method] = per_pool.get(method, 0) + n
    counts["energies"] = max([1] + list(per_pool.values()) + [64 * counts["prims"]])
    return counts


class RefSim:
    """One reference SimulationContext + SimulationExecutor (FP64, CPU)."""

    def __init__(self, scene=None, threads: int = 1, particles=0, oriented=0, energies=0, prims=0, sdf=0):
        self.L = lib()
        if scene is not None:
            c = capacities(scene)
            particles, oriented = max(particles, c["particles"]), max(oriented, c["oriented"])
            energies, prims, sdf = max(energies, c["energies"]), max(prims, c["prims"]), max(sdf, c["sdf"])
        self.h = self.L.ref_create(particles, oriented, energies, prims, sdf, threads)
        self.dt = 1.0 / 60.0

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"reference error: {self.L.ref_last_error().decode()}")

    # ---- set-up (the names of avbd_b200.Context and oracle.Oracle)
    def set_params(self, dt, g_accel=9.81, collision_margin=1e-3):
        self.dt = dt
        self.L.ref_set_params(self.h, dt, g_accel, collision_margin)

    def set_solver(self, solver_iters, iter_acceleration, residual_tolerance=0.0, max_iters=0, precision=None):
        if residual_tolerance:
            raise ValueError("the reference has no residual tolerance; it runs a fixed iteration count")
        self.L.ref_set_solver(self.h, solver_iters, iter_acceleration)

    def begin_scene(self):
        raise ValueError("one reference context holds one scene")

    def add_particles(self, positions, masses):
        x, m = _d(positions, (-1, 3)), _d(masses)
        return self.L.ref_particles_add(self.h, len(m), _p(x, C.c_double), _p(m, C.c_double))

    def add_oriented_particles(self, positions, rotations, masses, inertias):
        x, q, m, I = _d(positions, (-1, 3)), _d(rotations, (-1, 4)), _d(masses), _d(inertias, (-1, 3))
        return self.L.ref_particles_add_oriented(self.h, len(m), _p(x, C.c_double), _p(q, C.c_double),
                                                 _p(m, C.c_double), _p(I, C.c_double))

    def set_fixed(self, slots, fixed):
        s, f = _u(slots), np.ascontiguousarray(fixed, dtype=np.uint8)
        self.L.ref_set_fixed(self.h, len(s), _p(s, C.c_uint), _p(f, C.c_uint8))

    def set_velocities(self, first, velocities, previous_velocities=None):
        v = _d(velocities, (-1, 3))
        vp = _d(previous_velocities, (-1, 3)) if previous_velocities is not None else None
        self.L.ref_set_velocities(self.h, first, len(v), _p(v, C.c_double), _p(vp, C.c_double))

    def set_angular_velocities(self, first, w):
        w = _d(w, (-1, 3))
        self.L.ref_set_angular_velocities(self.h, first, len(w), _p(w, C.c_double))

    def add_neo_hookean(self, indices, lam, mu, kd, Q, V):
        idx = _u(indices).reshape(-1, 4)
        return self.L.ref_neo_hookean_add(self.h, len(idx), _p(idx, C.c_uint), _p(_d(lam), C.c_double),
                                          _p(_d(mu), C.c_double), _p(_d(kd), C.c_double),
                                          _p(_d(Q, (-1, 9)), C.c_double), _p(_d(V), C.c_double))

    def add_cosserat_rod(self, indices, stiffness, rest_length, precurvature):
        idx = _u(indices).reshape(-1, 2)
        return self.L.ref_cosserat_rod_add(self.h, len(idx), _p(idx, C.c_uint),
                                           _p(_d(stiffness, (-1, 6)), C.c_double), _p(_d(rest_length), C.c_double),
                                           _p(_d(precurvature, (-1, 3)), C.c_double))

    def add_ground_collision(self, particle_index, k_start, mu_s, mu_k):
        p = _u(particle_index)
        return self.L.ref_ground_add(self.h, len(p), _p(p, C.c_uint), _p(_d(k_start), C.c_double),
                                     _p(_d(mu_s), C.c_double), _p(_d(mu_k), C.c_double))

    def add_rigid_body_ground_collision(self, particle_index, shape_type, shape_radius, cp_rb_local, k_start,
                                        mu_s, mu_k):
        p = _u(particle_index)
        st = np.ascontiguousarray(shape_type, dtype=np.uint8)
        return self.L.ref_rigid_ground_add(self.h, len(p), _p(p, C.c_uint), _p(st, C.c_uint8),
                                           _p(_d(shape_radius), C.c_double), _p(_d(cp_rb_local, (-1, 3)), C.c_double),
                                           _p(_d(k_start), C.c_double), _p(_d(mu_s), C.c_double),
                                           _p(_d(mu_k), C.c_double))

    def add_one_sided_fixed_joint(self, particle_index, position_offset, rotation_offset, ref_position,
                                  ref_rotation):
        p = _u(particle_index)
        return self.L.ref_joint_add(self.h, len(p), _p(p, C.c_uint), _p(_d(position_offset, (-1, 3)), C.c_double),
                                    _p(_d(rotation_offset, (-1, 4)), C.c_double),
                                    _p(_d(ref_position, (-1, 3)), C.c_double),
                                    _p(_d(ref_rotation, (-1, 4)), C.c_double))

    def add_triangles(self, indices, object_id=0):
        idx = _u(indices).reshape(-1, 3)
        return self.L.ref_add_triangles(self.h, len(idx), _p(idx, C.c_uint), object_id)

    def add_rod_segments(self, indices, radius, object_id=0):
        idx = _u(indices).reshape(-1, 2)
        return self.L.ref_add_rod_segments(self.h, len(idx), _p(idx, C.c_uint), radius, object_id)

    def add_spheres(self, particle_index, radius, object_id):
        p = _u(particle_index)
        return self.L.ref_add_spheres(self.h, len(p), _p(p, C.c_uint), _p(_d(radius), C.c_double),
                                      _p(_u(object_id), C.c_uint))

    def finalize(self):
        self._check(self.L.ref_finalize(self.h))

    # ---- stepping and queries
    def step(self, n=1):
        self._check(self.L.ref_step(self.h, n))

    def set_iterations(self, iters):
        """The fixed iteration count of the following steps."""
        self._check(self.L.ref_set_iterations(self.h, int(iters)))

    def time_steps(self, n) -> float:
        t = self.L.ref_time_steps(self.h, n)
        if t < 0:
            raise RuntimeError(f"reference error: {self.L.ref_last_error().decode()}")
        return t

    @property
    def num_particles(self):
        return self.L.ref_num_particles(self.h)

    def _vec(self, fn, width):
        out = np.zeros((self.num_particles, width))
        fn(self.h, _p(out, C.c_double))
        return out

    def positions(self):
        return self._vec(self.L.ref_get_positions, 3)

    def velocities(self):
        return self._vec(self.L.ref_get_velocities, 3)

    def rotations(self):
        return self._vec(self.L.ref_get_rotations, 4)

    def angular_velocities(self):
        return self._vec(self.L.ref_get_angular_velocities, 3)

    def coloring(self):
        out = np.zeros(self.num_particles, dtype=np.uint32)
        nc = C.c_uint(0)
        self.L.ref_get_coloring(self.h, _p(out, C.c_uint), C.byref(nc))
        return out, nc.value

    def lbvh(self):
        """Morton codes, sorted order, tree arrays and candidate leaf pairs of
        the last step's collision stage (the pool's totalSize() primitives)."""
        n = self.L.ref_num_primitives(self.h)
        nn = 2 * n - 1
        npairs = self.L.ref_collect_pairs(self.h)
        out = dict(
            morton=np.zeros(n, dtype=np.uint64), sorted_order=np.zeros(n, dtype=np.uint32),
            left=np.zeros(nn, dtype=np.uint32), right=np.zeros(nn, dtype=np.uint32),
            parent=np.zeros(nn, dtype=np.uint32), subtree_size=np.zeros(nn, dtype=np.uint32),
            bounds=np.zeros((nn, 6)), pairs=np.zeros((npairs, 2), dtype=np.uint32))
        root = C.c_uint(0)
        self.L.ref_get_lbvh(self.h, _p(out["morton"], C.c_uint64), _p(out["sorted_order"], C.c_uint),
                            _p(out["left"], C.c_uint), _p(out["right"], C.c_uint), _p(out["parent"], C.c_uint),
                            _p(out["subtree_size"], C.c_uint), _p(out["bounds"], C.c_double), C.byref(root),
                            _p(out["pairs"], C.c_uint))
        out["root"] = root.value
        return out

    def dynamic_info(self):
        out = np.zeros(8, dtype=np.uint32)
        self.L.ref_dynamic_info(self.h, _p(out, C.c_uint))
        return dict(zip(["live", "pool_size", "colors", "conflicted", "dirty", "entries", "rod_live", "rod_pool_size"],
                        (int(v) for v in out)))

    def contact_pool(self):
        n = self.dynamic_info()["pool_size"]
        p4 = np.zeros((n, 4), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 24))
        self.L.ref_get_trc(self.h, _p(p4, C.c_uint), _p(act, C.c_uint8), _p(d, C.c_double))
        return {"particles": p4, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "k": d[:, 15:19], "lam": d[:, 19:23],
                "flags": d[:, 23].astype(np.uint8)}

    def rod_contact_pool(self):
        n = self.dynamic_info()["rod_pool_size"]
        p5 = np.zeros((n, 5), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 25))
        self.L.ref_get_trd(self.h, _p(p5, C.c_uint), _p(act, C.c_uint8), _p(d, C.c_double))
        return {"particles": p5, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "s": d[:, 15], "k": d[:, 16:20], "lam": d[:, 20:24],
                "flags": d[:, 24].astype(np.uint8)}

    def conflicted(self):
        out = np.zeros(self.num_particles, dtype=np.uint8)
        self.L.ref_get_conflicted(self.h, _p(out, C.c_uint8))
        return out.astype(bool)

    def debug_block(self, p):
        G, H = np.zeros(6), np.zeros(36)
        dof = C.c_int(0)
        self._check(self.L.ref_debug_block(self.h, p, _p(G, C.c_double), _p(H, C.c_double), C.byref(dof)))
        d = dof.value
        return G[:d].copy(), H[: d * d].reshape(d, d).copy()
