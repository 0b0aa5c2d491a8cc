"""avbd_lbvh_morton_sort_noalloc: the LBVH Morton codes and sorted order for
callers that cannot allocate device memory while they run (a loop being
recorded into a CUDA graph, a real-time loop on a fixed memory budget, an
application whose device memory belongs to another framework's allocator).

The entry point allocates nothing: the caller owns inputs and outputs (here
torch CUDA tensors) and the scratch lives in the library's file-scope device
arrays.  Its results must equal the context path's (avbd_collision_stage +
avbd_get_lbvh) bit for bit, on two calls in a row that share that scratch.
"""
import ctypes as C

import numpy as np
import pytest

from avbd_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu


def _context_lbvh(sc, X, V):
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    e.set_positions(0, X)
    e.set_velocities(0, V)
    e.collision_stage()
    t = e.lbvh()
    e.close()
    return t


def _swept_boxes(sc, X, V, tris):
    """CollisionPrimitivePool::speculativeGlobalBounds for triangles, in numpy
    FP64 (a multiply then an add for p + dt v, as on the device)."""
    P = X[tris]                  # (m, 3, 3)
    Pn = X[tris] + sc.dt * V[tris]
    both = np.concatenate([P, Pn], axis=1)
    return np.ascontiguousarray(np.concatenate([both.min(1), both.max(1)], axis=1))


def _noalloc(boxes):
    import torch
    L = _lib.load()
    n = len(boxes)
    d_boxes = torch.from_numpy(boxes).cuda()
    d_morton = torch.empty(n, dtype=torch.int64, device="cuda")
    d_sorted = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.avbd_lbvh_morton_sort_noalloc(C.c_void_p(d_boxes.data_ptr()), n, C.c_void_p(d_morton.data_ptr()),
                                         C.c_void_p(d_sorted.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    assert rc == 0, L.avbd_last_error_string()
    return d_morton.cpu().numpy().view(np.uint64), d_sorted.cpu().numpy().view(np.uint32)


class _Tris:
    def __init__(self):
        self.tris = None

    def __getattr__(self, name):
        def f(*a, **k):
            if name == "add_triangles":
                self.tris = np.asarray(a[0], dtype=np.int64)
        return f


def test_noalloc_matches_context_path_twice():
    sc = scenes.cube_drop(n=10, surface=True)
    cap = _Tris()
    sc.load(cap)
    tris = cap.tris
    rng = np.random.default_rng(11)
    base = None
    for call in range(2):  # two calls in a row share the scratch arrays
        o = Context()
        sc.load(o, precision="fp64")
        X0 = o.positions() if base is None else base
        o.close()
        base = X0
        X = X0 + rng.uniform(-0.02, 0.02, size=X0.shape)
        V = rng.normal(0, 1.0 + call, size=X0.shape)
        ref = _context_lbvh(sc, X, V)
        boxes = _swept_boxes(sc, X, V, tris)
        morton, order = _noalloc(boxes)
        assert (morton == ref["morton"]).all(), f"call {call}: Morton codes differ"
        assert (order == ref["sorted_order"]).all(), f"call {call}: sorted order differs"


def test_noalloc_at_the_primitive_limit():
    """AVBD_NOALLOC_MAX_PRIMITIVES (262,144) random boxes, twice: the
    single-block scan then runs over all 256 x 1,024 digit-histogram entries.
    Codes are checked against a NumPy restatement of the Morton arithmetic
    (LBVHBuilder.cpp:98-127; every step is one IEEE operation, so numpy
    reproduces it) and the order against a stable sort of the codes."""
    n = 262144
    rng = np.random.default_rng(2026)
    for call in range(2):
        lo = rng.uniform(-3.0, 3.0, size=(n, 3))
        boxes = np.ascontiguousarray(np.concatenate([lo, lo + rng.uniform(0, 0.05, size=(n, 3))], axis=1))
        morton, order = _noalloc(boxes)
        smin, smax = boxes[:, :3].min(0), boxes[:, 3:].max(0)
        ext = np.maximum(smax - smin, 1e-6)
        c = (boxes[:, :3] + boxes[:, 3:]) * 0.5
        q = np.clip((c - smin) / ext * 2097152.0, 0.0, 2097151.0).astype(np.uint64)

        def expand(v):
            v = v & np.uint64(0x1FFFFF)
            for sh, m in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                          (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
                v = (v | (v << np.uint64(sh))) & np.uint64(m)
            return v

        codes = expand(q[:, 0]) | (expand(q[:, 1]) << np.uint64(1)) | (expand(q[:, 2]) << np.uint64(2))
        assert (morton == codes).all(), f"call {call}: Morton codes differ"
        assert (order == np.argsort(codes, kind="stable")).all(), f"call {call}: sorted order differs"


def test_noalloc_rejects_oversized_input():
    import torch
    L = _lib.load()
    n = 262144 + 1
    d = torch.empty(16, dtype=torch.float64, device="cuda")
    rc = L.avbd_lbvh_morton_sort_noalloc(C.c_void_p(d.data_ptr()), n, C.c_void_p(d.data_ptr()),
                                         C.c_void_p(d.data_ptr()), None)
    assert rc == 2  # AVBD_ERR_CAPACITY
