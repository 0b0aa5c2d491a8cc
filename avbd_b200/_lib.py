"""ctypes binding of libavbd_b200.so (the C-ABI of include/avbd.h).

The library is loaded from this package's directory.  There is no fallback:
if the shared library is missing or cannot be loaded, importing the engine
fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libavbd_b200.so")

AVBD_OK = 0
ERRORS = {
    1: "AVBD_ERR_INVALID_ARG", 2: "AVBD_ERR_CAPACITY", 3: "AVBD_ERR_COLORS", 4: "AVBD_ERR_UNSUPPORTED_PAIR",
    5: "AVBD_ERR_NAN", 6: "AVBD_ERR_BARRIER_TIMEOUT", 7: "AVBD_ERR_CUDA", 8: "AVBD_ERR_STATE",
    9: "AVBD_ERR_UNSUPPORTED", 10: "AVBD_ERR_NO_DEVICE",
}
DEFAULT_WAIT_POLLS = 1 << 22
PRECISION_FP32 = 0
PRECISION_FP64 = 1
PRECISION_MIXED = 2
SHAPE_TRIANGLE, SHAPE_ROD_SEGMENT, SHAPE_SPHERE = 0, 1, 2
# learned warm start (include/avbd.h): feature rows of 32 BF16, target rows of 4 FP32
MLP_IN, MLP_IN_PAD, MLP_HIDDEN, MLP_OUT, MLP_OUT_PAD, MLP_NPARAMS = 27, 32, 128, 3, 16, 39312


class AvbdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("dt", C.c_double), ("end_time", C.c_double), ("g_accel", C.c_double),
                ("viewer_refresh_time_ms", C.c_double), ("collision_margin", C.c_double)]


class SolverParams(C.Structure):
    _fields_ = [("solver_iters", C.c_uint), ("iter_acceleration", C.c_double), ("residual_tolerance", C.c_double),
                ("max_iters", C.c_uint), ("precision", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("kernel_launches", C.c_ulonglong), ("iterations", C.c_ulonglong), ("fp64_fallbacks", C.c_ulonglong),
                ("candidate_pairs", C.c_ulonglong), ("last_residual", C.c_double), ("num_colors", C.c_uint),
                ("num_scenes", C.c_uint), ("capped_scene_steps", C.c_ulonglong),
                ("warmstart_applied", C.c_ulonglong)]


# name -> argtypes (all return int unless listed in _RESTYPE)
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint)
_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_fp = C.POINTER(C.c_float)
SIGNATURES = {
    "avbd_create": [C.POINTER(_vp), C.c_int, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint],
    "avbd_destroy": [_vp],
    "avbd_set_stream": [_vp, _vp],
    "avbd_set_params": [_vp, C.POINTER(Params)],
    "avbd_set_solver": [_vp, C.POINTER(SolverParams)],
    "avbd_begin_scene": [_vp, _up],
    "avbd_particles_add": [_vp, C.c_uint, _dp, _dp, _up],
    "avbd_particles_add_oriented": [_vp, C.c_uint, _dp, _dp, _dp, _dp, _up],
    "avbd_particles_set_fixed": [_vp, C.c_uint, _up, _u8p],
    "avbd_set_positions": [_vp, C.c_uint, C.c_uint, _dp],
    "avbd_set_velocities": [_vp, C.c_uint, C.c_uint, _dp, _dp],
    "avbd_set_state": [_vp, _dp, _dp],
    "avbd_get_positions": [_vp, C.c_uint, C.c_uint, _dp],
    "avbd_get_velocities": [_vp, C.c_uint, C.c_uint, _dp],
    "avbd_get_rotations": [_vp, C.c_uint, C.c_uint, _dp],
    "avbd_get_angular_velocities": [_vp, C.c_uint, C.c_uint, _dp],
    "avbd_num_particles": [_vp, _up],
    "avbd_neo_hookean_add": [_vp, C.c_uint, _up, _dp, _dp, _dp, _dp, _dp, _up],
    "avbd_cosserat_rod_add": [_vp, C.c_uint, _up, _dp, _dp, _dp, _up],
    "avbd_ground_collision_add": [_vp, C.c_uint, _up, _dp, _dp, _dp, _up],
    "avbd_rigid_body_ground_collision_add": [_vp, C.c_uint, _up, _u8p, _dp, _dp, _dp, _dp, _dp, _up],
    "avbd_one_sided_fixed_joint_add": [_vp, C.c_uint, _up, _dp, _dp, _dp, _dp, _up],
    "avbd_collision_add_triangles": [_vp, C.c_uint, _up, C.c_uint, _up],
    "avbd_collision_add_rod_segments": [_vp, C.c_uint, _up, C.c_double, C.c_uint, _up],
    "avbd_collision_add_spheres": [_vp, C.c_uint, _up, _dp, _up, _up],
    "avbd_finalize": [_vp],
    "avbd_step": [_vp, C.c_uint],
    "avbd_synchronize": [_vp],
    "avbd_collision_stage": [_vp],
    "avbd_get_stats": [_vp, C.POINTER(Stats)],
    "avbd_get_coloring": [_vp, _up, _up],
    "avbd_get_lbvh": [_vp, _up, _u64p, _up, _up, _up, _up, _up, _dp, _up],
    "avbd_get_candidate_pairs": [_vp, C.c_uint, _up, _up],
    "avbd_get_contacts": [_vp, C.c_uint, _u64p, _up, _dp, _up],
    "avbd_dynamic_info": [_vp, _up],
    "avbd_get_contact_pool": [_vp, C.c_uint, _up, _u8p, _dp, _up],
    "avbd_get_rod_contact_pool": [_vp, C.c_uint, _up, _u8p, _dp, _up],
    "avbd_get_rod_contacts": [_vp, C.c_uint, _u64p, _up, _dp, _up],
    "avbd_debug_set_recolor_rounds": [_vp, C.c_uint],
    "avbd_debug_set_pair_capacity": [_vp, C.c_uint],
    "avbd_debug_set_wait_limit": [C.c_int, C.c_uint],
    "avbd_debug_block": [_vp, C.c_uint, _dp, _dp, C.POINTER(C.c_int)],
    "avbd_residual": [_vp, _dp],
    "avbd_get_scene_iterations": [_vp, _up],
    "avbd_profile_solve": [_vp, C.c_uint, _dp, _dp, _up],
    "avbd_profile_step": [_vp, _dp, _dp, _up, _up],
    "avbd_lbvh_morton_sort_noalloc": [_vp, C.c_uint, _vp, _vp, _vp],
    "avbd_gemm_bf16": [_vp, C.c_uint, _vp, C.c_uint, _vp, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _vp],
    "avbd_mlp_create": [C.POINTER(_vp), C.c_int, _fp],
    "avbd_mlp_forward": [_vp, _vp, C.c_uint, _vp, _vp],
    "avbd_mlp_destroy": [_vp],
    "avbd_mlp_trainer_create": [C.POINTER(_vp), C.c_int, C.c_uint, _fp],
    "avbd_mlp_trainer_step": [_vp, _vp, _vp, C.c_float, _fp],
    "avbd_mlp_trainer_grad": [_vp, _vp, _vp, _fp, _fp],
    "avbd_mlp_trainer_get_params": [_vp, _fp],
    "avbd_mlp_trainer_destroy": [_vp],
    "avbd_set_warmstart": [_vp, C.c_int, _fp],
    "avbd_warmstart_sample": [_vp, _vp, _vp, _up],
    "avbd_set_initial_guess": [_vp, _dp],
    "avbd_last_error_string": [],
    "avbd_version": [],
}
_RESTYPE = {"avbd_last_error_string": C.c_char_p, "avbd_version": C.c_char_p}

_lib = None


def load():
    """Loads the engine library (built in-tree by avbd_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m avbd_b200.build` "
                          "(nvcc for sm_100a); the engine has no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _RESTYPE.get(name, C.c_int)
    _lib = lib
    return lib


def check(rc: int):
    if rc != AVBD_OK:
        raise AvbdError(rc, load().avbd_last_error_string().decode())
