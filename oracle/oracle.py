"""ctypes binding of the FP64 oracle (oracle/avbd_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The engine never loads
this module.  The oracle is pinned to the reference implementation itself
(compiled from its own sources into oracle/_ref, see oracle/ref.py and
tests/test_ref_pinning.py); the header of avbd_oracle.cpp lists the pins.

The method names mirror the engine's Python facade (avbd_b200.Context), so a
scene description can be loaded into either with the same calls.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

NEO_HOOKEAN, COSSERAT_ROD, GROUND, RIGID_GROUND, JOINT = range(5)


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (g++, no CUDA)."""
    src = os.path.join(_HERE, "avbd_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"])
    return _LIB_PATH


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        up = C.POINTER(C.c_uint)
        u8p = C.POINTER(C.c_uint8)
        sig = {
            "orc_create": (vp, []),
            "orc_destroy": (None, [vp]),
            "orc_set_params": (None, [vp, C.c_double, C.c_double, C.c_double]),
            "orc_set_solver": (None, [vp, C.c_uint, C.c_double, C.c_double, C.c_uint]),
            "orc_set_threads": (None, [vp, C.c_int]),
            "orc_begin_scene": (None, [vp]),
            "orc_particles_add": (C.c_uint, [vp, C.c_uint, dp, dp]),
            "orc_particles_add_oriented": (C.c_uint, [vp, C.c_uint, dp, dp, dp, dp]),
            "orc_set_fixed": (None, [vp, C.c_uint, up, u8p]),
            "orc_set_velocities": (None, [vp, C.c_uint, C.c_uint, dp, dp]),
            "orc_set_positions_raw": (None, [vp, C.c_uint, C.c_uint, dp]),
            "orc_set_rotations_raw": (None, [vp, C.c_uint, C.c_uint, dp]),
            "orc_set_angular_velocities": (None, [vp, C.c_uint, C.c_uint, dp]),
            "orc_get_positions": (None, [vp, dp]),
            "orc_get_velocities": (None, [vp, dp]),
            "orc_get_rotations": (None, [vp, dp]),
            "orc_get_contacts": (C.c_uint, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint), dp]),
            "orc_get_angular_velocities": (None, [vp, dp]),
            "orc_dynamic_info": (None, [vp, up]),
            "orc_get_trc": (None, [vp, up, u8p, dp]),
            "orc_get_trd": (None, [vp, up, u8p, dp]),
            "orc_get_rod_contacts": (C.c_uint, [vp, C.POINTER(C.c_uint64), up, dp]),
            "orc_get_conflicted": (None, [vp, u8p]),
            "orc_set_recolor_rounds": (None, [vp, C.c_uint]),
            "orc_num_particles": (C.c_uint, [vp]),
            "orc_neo_hookean_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp, dp, dp]),
            "orc_cosserat_rod_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp]),
            "orc_ground_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp]),
            "orc_rigid_ground_add": (C.c_uint, [vp, C.c_uint, up, u8p, dp, dp, dp, dp, dp]),
            "orc_joint_add": (C.c_uint, [vp, C.c_uint, up, dp, dp, dp, dp]),
            "orc_add_triangles": (C.c_uint, [vp, C.c_uint, up, C.c_uint]),
            "orc_add_rod_segments": (C.c_uint, [vp, C.c_uint, up, C.c_double, C.c_uint]),
            "orc_add_spheres": (C.c_uint, [vp, C.c_uint, up, dp, up]),
            "orc_finalize": (C.c_int, [vp, C.c_int]),
            "orc_step": (C.c_int, [vp, C.c_uint]),
            "orc_time_steps": (C.c_double, [vp, C.c_uint]),
            "orc_collision_stage": (C.c_int, [vp]),
            "orc_after_time_step": (None, [vp]),
            "orc_get_coloring": (None, [vp, up, up]),
            "orc_num_entries": (C.c_uint, [vp]),
            "orc_num_neighbors": (C.c_uint, [vp]),
            "orc_get_adjacency": (None, [vp, up, u8p, up, C.POINTER(C.c_uint16), up, up]),
            "orc_num_pairs": (C.c_uint, [vp]),
            "orc_get_lbvh": (None, [vp, C.POINTER(C.c_uint64), up, up, up, up, up, dp, up, up]),
            "orc_lbvh_from_codes": (C.c_int, [vp, C.c_uint, C.POINTER(C.c_uint64), dp]),
            "orc_debug_block": (C.c_int, [vp, C.c_uint, dp, dp, C.POINTER(C.c_int)]),
            "orc_energy": (C.c_double, [vp, C.c_int, C.c_uint]),
            "orc_element_accumulate": (None, [vp, C.c_int, C.c_uint, C.c_uint, dp, dp]),
            "orc_residual": (C.c_double, [vp]),
            "orc_last_residual": (C.c_double, [vp]),
            "orc_iterations": (C.c_ulonglong, [vp]),
            "orc_scene_iterations": (C.c_uint, [vp, up]),
            "orc_exp_s3": (None, [dp, dp]),
            "orc_quat_from_xyz_euler": (None, [dp, dp]),
            "orc_plus_s3": (None, [dp, dp, dp]),
            "orc_last_error": (C.c_char_p, []),
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


def quat_from_xyz_euler(deg) -> np.ndarray:
    """Math::QuaternionFromXYZEulerAngles (common/Math.hpp:298-318), (w,x,y,z)."""
    out = np.zeros(4)
    lib().orc_quat_from_xyz_euler(_p(_d(deg), C.c_double), _p(out, C.c_double))
    return out


def exp_s3(v) -> np.ndarray:
    out = np.zeros(4)
    lib().orc_exp_s3(_p(_d(v), C.c_double), _p(out, C.c_double))
    return out


def plus_s3(q, v) -> np.ndarray:
    out = np.zeros(4)
    lib().orc_plus_s3(_p(_d(q), C.c_double), _p(_d(v), C.c_double), _p(out, C.c_double))
    return out


class Oracle:
    """FP64 CPU restatement of one SimulationContext + SimulationExecutor."""

    def __init__(self, threads: int = 1):
        self.L = lib()
        self.h = self.L.orc_create()
        self.threads = threads
        if threads > 1:
            self.L.orc_set_threads(self.h, threads)

    def __del__(self):
        try:
            if self.h:
                self.L.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {self.L.orc_last_error().decode()}")

    # ---- set-up (same names as avbd_b200.Context)
    def set_params(self, dt, g_accel=9.81, collision_margin=1e-3):
        self.dt = dt
        self.L.orc_set_params(self.h, dt, g_accel, collision_margin)

    def set_solver(self, solver_iters, iter_acceleration, residual_tolerance=0.0, max_iters=0, precision=None):
        self.L.orc_set_solver(self.h, solver_iters, iter_acceleration, residual_tolerance, max_iters)

    def begin_scene(self):
        self.L.orc_begin_scene(self.h)

    def add_particles(self, positions, masses):
        x = _d(positions, (-1, 3))
        m = _d(masses)
        return self.L.orc_particles_add(self.h, len(m), _p(x, C.c_double), _p(m, C.c_double))

    def add_oriented_particles(self, positions, rotations, masses, inertias):
        x = _d(positions, (-1, 3))
        q = _d(rotations, (-1, 4))
        m = _d(masses)
        I = _d(inertias, (-1, 3))
        return self.L.orc_particles_add_oriented(self.h, len(m), _p(x, C.c_double), _p(q, C.c_double),
                                                 _p(m, C.c_double), _p(I, C.c_double))

    def set_fixed(self, slots, fixed):
        s = _u(slots)
        f = np.ascontiguousarray(fixed, dtype=np.uint8)
        self.L.orc_set_fixed(self.h, len(s), _p(s, C.c_uint), _p(f, C.c_uint8))

    def set_velocities(self, first, velocities, previous_velocities=None):
        v = _d(velocities, (-1, 3))
        vp = _d(previous_velocities, (-1, 3)) if previous_velocities is not None else None
        self.L.orc_set_velocities(self.h, first, len(v), _p(v, C.c_double), _p(vp, C.c_double) if vp is not None else None)

    def set_positions_raw(self, first, positions):
        x = _d(positions, (-1, 3))
        self.L.orc_set_positions_raw(self.h, first, len(x), _p(x, C.c_double))

    def set_angular_velocities(self, first, w):
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1, 3)
        self.L.orc_set_angular_velocities(self.h, first, len(w), _p(w, C.c_double))

    def set_rotations_raw(self, first, rotations):
        q = _d(rotations, (-1, 4))
        self.L.orc_set_rotations_raw(self.h, first, len(q), _p(q, C.c_double))

    def add_neo_hookean(self, indices, lam, mu, kd, Q, V):
        idx = _u(indices).reshape(-1, 4)
        n = len(idx)
        return self.L.orc_neo_hookean_add(self.h, n, _p(idx, C.c_uint), _p(_d(lam), C.c_double), _p(_d(mu), C.c_double),
                                          _p(_d(kd), C.c_double), _p(_d(Q, (-1, 9)), C.c_double), _p(_d(V), C.c_double))

    def add_cosserat_rod(self, indices, stiffness, rest_length, precurvature):
        idx = _u(indices).reshape(-1, 2)
        return self.L.orc_cosserat_rod_add(self.h, len(idx), _p(idx, C.c_uint), _p(_d(stiffness, (-1, 6)), C.c_double),
                                           _p(_d(rest_length), C.c_double), _p(_d(precurvature, (-1, 3)), C.c_double))

    def add_ground_collision(self, particle_index, k_start, mu_s, mu_k):
        p = _u(particle_index)
        return self.L.orc_ground_add(self.h, len(p), _p(p, C.c_uint), _p(_d(k_start), C.c_double),
                                     _p(_d(mu_s), C.c_double), _p(_d(mu_k), C.c_double))

    def add_rigid_body_ground_collision(self, particle_index, shape_type, shape_radius, cp_rb_local, k_start, mu_s, mu_k):
        p = _u(particle_index)
        st = np.ascontiguousarray(shape_type, dtype=np.uint8)
        return self.L.orc_rigid_ground_add(self.h, len(p), _p(p, C.c_uint), _p(st, C.c_uint8), _p(_d(shape_radius), C.c_double),
                                           _p(_d(cp_rb_local, (-1, 3)), C.c_double), _p(_d(k_start), C.c_double),
                                           _p(_d(mu_s), C.c_double), _p(_d(mu_k), C.c_double))

    def add_one_sided_fixed_joint(self, particle_index, position_offset, rotation_offset, ref_position, ref_rotation):
        p = _u(particle_index)
        return self.L.orc_joint_add(self.h, len(p), _p(p, C.c_uint), _p(_d(position_offset, (-1, 3)), C.c_double),
                                    _p(_d(rotation_offset, (-1, 4)), C.c_double), _p(_d(ref_position, (-1, 3)), C.c_double),
                                    _p(_d(ref_rotation, (-1, 4)), C.c_double))

    def add_triangles(self, indices, object_id=0):
        idx = _u(indices).reshape(-1, 3)
        return self.L.orc_add_triangles(self.h, len(idx), _p(idx, C.c_uint), object_id)

    def add_rod_segments(self, indices, radius, object_id=0):
        idx = _u(indices).reshape(-1, 2)
        return self.L.orc_add_rod_segments(self.h, len(idx), _p(idx, C.c_uint), radius, object_id)

    def add_spheres(self, particle_index, radius, object_id):
        p = _u(particle_index)
        return self.L.orc_add_spheres(self.h, len(p), _p(p, C.c_uint), _p(_d(radius), C.c_double), _p(_u(object_id), C.c_uint))

    def finalize(self, reference_dsatur: bool = False):
        self._check(self.L.orc_finalize(self.h, 1 if reference_dsatur else 0))

    # ---- stepping / queries
    def step(self, n=1):
        self._check(self.L.orc_step(self.h, n))

    def time_steps(self, n) -> float:
        return self.L.orc_time_steps(self.h, n)

    def collision_stage(self):
        self._check(self.L.orc_collision_stage(self.h))

    def after_time_step(self):
        self.L.orc_after_time_step(self.h)

    @property
    def num_particles(self):
        return self.L.orc_num_particles(self.h)

    def positions(self):
        out = np.zeros((self.num_particles, 3))
        self.L.orc_get_positions(self.h, _p(out, C.c_double))
        return out

    def velocities(self):
        out = np.zeros((self.num_particles, 3))
        self.L.orc_get_velocities(self.h, _p(out, C.c_double))
        return out

    def rotations(self):
        out = np.zeros((self.num_particles, 4))
        self.L.orc_get_rotations(self.h, _p(out, C.c_double))
        return out

    def contacts(self):
        """Triangle-sphere contacts of the last collision stage, ascending key:
        dict of key [k], tri [k, 3], rigid [k], normal / barys / cp_local [k, 3]."""
        n = self.L.orc_get_contacts(self.h, None, None, None)
        keys = np.zeros(n, dtype=np.uint64)
        idx = np.zeros((n, 4), dtype=np.uint32)
        vec = np.zeros((n, 9))
        if n:
            self.L.orc_get_contacts(self.h, _p(keys, C.c_uint64), _p(idx, C.c_uint), _p(vec, C.c_double))
        return {"key": keys, "tri": idx[:, :3], "rigid": idx[:, 3], "normal": vec[:, 0:3], "barys": vec[:, 3:6],
                "cp_local": vec[:, 6:9]}

    def dynamic_info(self):
        """Contact pool and recoloring state: live contacts, pool size, colors,
        conflicted particles, particles still dirty, dynamic adjacency entries."""
        out = np.zeros(8, dtype=np.uint32)
        self.L.orc_dynamic_info(self.h, _p(out, C.c_uint))
        return dict(zip(["live", "pool_size", "colors", "conflicted", "dirty", "entries", "rod_live", "rod_pool_size"],
                        (int(v) for v in out)))

    def contact_pool(self):
        """Triangle-rigid contact pool by slot: particles [s, 4], active [s],
        and per slot n, t, b, barys, cp_local [s, 3], k (k_start, k_n, k_t,
        k_b) [s, 4], lam (lam_n, lam_t, lam_b, C_n_prev) [s, 4], flags [s]
        (1 static friction, 2 unclamped)."""
        n = self.dynamic_info()["pool_size"]
        p4 = np.zeros((n, 4), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 24))
        if n:
            self.L.orc_get_trc(self.h, _p(p4, C.c_uint), _p(act, C.c_uint8), _p(d, C.c_double))
        return {"particles": p4, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "k": d[:, 15:19], "lam": d[:, 19:23],
                "flags": d[:, 23].astype(np.uint8)}

    def set_recolor_rounds(self, rounds):
        self.L.orc_set_recolor_rounds(self.h, rounds)

    def rod_contact_pool(self):
        """Triangle-rod contact pool by slot: particles [s, 5], active [s], and
        per slot n, t, b, barys, cp_local [s, 3], s [s], k [s, 4], lam [s, 4],
        flags [s]."""
        n = self.dynamic_info()["rod_pool_size"]
        p5 = np.zeros((n, 5), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 25))
        if n:
            self.L.orc_get_trd(self.h, _p(p5, C.c_uint), _p(act, C.c_uint8), _p(d, C.c_double))
        return {"particles": p5, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "s": d[:, 15], "k": d[:, 16:20], "lam": d[:, 20:24],
                "flags": d[:, 24].astype(np.uint8)}

    def rod_contacts(self):
        """Triangle-rod contacts of the last collision stage, ascending key:
        key [k], tri [k, 3], rod [k, 2], normal / barys / cp_local [k, 3], s [k]."""
        n = self.L.orc_get_rod_contacts(self.h, None, None, None)
        keys = np.zeros(n, dtype=np.uint64)
        idx = np.zeros((n, 5), dtype=np.uint32)
        vec = np.zeros((n, 10))
        if n:
            self.L.orc_get_rod_contacts(self.h, _p(keys, C.c_uint64), _p(idx, C.c_uint), _p(vec, C.c_double))
        return {"key": keys, "tri": idx[:, :3], "rod": idx[:, 3:5], "normal": vec[:, 0:3], "barys": vec[:, 3:6],
                "cp_local": vec[:, 6:9], "s": vec[:, 9]}

    def conflicted(self):
        out = np.zeros(self.num_particles, dtype=np.uint8)
        self.L.orc_get_conflicted(self.h, _p(out, C.c_uint8))
        return out.astype(bool)

    def angular_velocities(self):
        out = np.zeros((self.num_particles, 3))
        self.L.orc_get_angular_velocities(self.h, _p(out, C.c_double))
        return out

    def coloring(self):
        out = np.zeros(self.num_particles, dtype=np.uint32)
        nc = C.c_uint(0)
        self.L.orc_get_coloring(self.h, _p(out, C.c_uint), C.byref(nc))
        return out, nc.value

    def adjacency(self):
        n = self.num_particles
        ne = self.L.orc_num_entries(self.h)
        nn = self.L.orc_num_neighbors(self.h)
        e_off = np.zeros((n + 1) * 5, dtype=np.uint32)
        typ = np.zeros(ne, dtype=np.uint8)
        idx = np.zeros(ne, dtype=np.uint32)
        loc = np.zeros(ne, dtype=np.uint16)
        p_off = np.zeros(n + 1, dtype=np.uint32)
        p_nbr = np.zeros(nn, dtype=np.uint32)
        self.L.orc_get_adjacency(self.h, _p(e_off, C.c_uint), _p(typ, C.c_uint8), _p(idx, C.c_uint),
                                 _p(loc, C.c_uint16), _p(p_off, C.c_uint), _p(p_nbr, C.c_uint))
        return dict(e_off=e_off.reshape(n + 1, 5), type=typ, idx=idx, local=loc, p_off=p_off, p_nbr=p_nbr)

    def lbvh(self, num_primitives):
        n = num_primitives
        nn = max(2 * n - 1, 0)
        npairs = self.L.orc_num_pairs(self.h)
        out = dict(
            morton=np.zeros(n, dtype=np.uint64), sorted_order=np.zeros(n, dtype=np.uint32),
            left=np.zeros(nn, dtype=np.uint32), right=np.zeros(nn, dtype=np.uint32),
            parent=np.zeros(nn, dtype=np.uint32), subtree_size=np.zeros(nn, dtype=np.uint32),
            bounds=np.zeros((nn, 6)), pairs=np.zeros((npairs, 2), dtype=np.uint32))
        root = C.c_uint(0)
        self.L.orc_get_lbvh(self.h, _p(out["morton"], C.c_uint64), _p(out["sorted_order"], C.c_uint),
                            _p(out["left"], C.c_uint), _p(out["right"], C.c_uint), _p(out["parent"], C.c_uint),
                            _p(out["subtree_size"], C.c_uint), _p(out["bounds"], C.c_double), C.byref(root),
                            _p(out["pairs"], C.c_uint))
        out["root"] = root.value
        return out

    def lbvh_from_codes(self, codes, boxes=None):
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        b = _d(boxes, (-1, 6)) if boxes is not None else None
        self._check(self.L.orc_lbvh_from_codes(self.h, len(codes), _p(codes, C.c_uint64),
                                               _p(b, C.c_double) if b is not None else None))
        return self.lbvh(len(codes))

    def debug_block(self, p):
        G = np.zeros(6)
        H = np.zeros(36)
        dof = C.c_int(0)
        self.L.orc_debug_block(self.h, p, _p(G, C.c_double), _p(H, C.c_double), C.byref(dof))
        d = dof.value
        return G[:d].copy(), H[: d * d].reshape(d, d).copy()

    def energy(self, etype, slot):
        return self.L.orc_energy(self.h, etype, slot)

    def element_accumulate(self, etype, slot, local):
        G = np.zeros(6)
        H = np.zeros(36)
        self.L.orc_element_accumulate(self.h, etype, slot, local, _p(G, C.c_double), _p(H, C.c_double))
        d = 3 if etype == NEO_HOOKEAN else 6
        return G[:d].copy(), H[: d * d].reshape(d, d).copy()

    def residual(self):
        return self.L.orc_residual(self.h)

    @property
    def last_residual(self):
        return self.L.orc_last_residual(self.h)

    @property
    def iterations(self):
        return self.L.orc_iterations(self.h)

    def scene_iterations(self):
        """Iterations each scene ran in the last run-to-tolerance step."""
        buf = np.zeros(1 << 16, dtype=np.uint32)
        n = self.L.orc_scene_iterations(self.h, _p(buf, C.c_uint))
        return buf[:n].copy()
