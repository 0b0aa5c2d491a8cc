"""Error paths of the C-ABI, provoked without faulting the GPU.

The reference reports these conditions by throwing (TombstonePool.hpp:61-65
"Pool has exceeded capacity", ColorList.hpp:184-185 "Ran out of colors!") or
not at all (a NaN state, a lost collision pair).  The engine returns integer
status codes instead; each test below makes one of them happen on the host
side or through a short wait limit and checks the code, then that the
context (or the device) is still usable.
"""
import ctypes as C

import numpy as np
import pytest

from avbd_b200 import Context, _lib, scenes
from avbd_b200._lib import AvbdError

pytestmark = pytest.mark.gpu

ERR_CAPACITY, ERR_COLORS, ERR_NAN, ERR_TIMEOUT = 2, 3, 5, 6


def test_nan_state_is_reported_on_the_next_step():
    sc = scenes.cube_fixed_bottom(n=3)
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    X = e.positions()
    X[-1, 1] = np.nan
    e.set_positions(0, X)
    with pytest.raises(AvbdError) as ex:
        e.step(1)
        e.synchronize()
    assert ex.value.code == ERR_NAN
    e.close()


def test_particle_pool_over_capacity():
    e = Context(particles_capacity=8)
    e.add_particles(np.zeros((8, 3)), np.ones(8))
    with pytest.raises(AvbdError) as ex:
        e.add_particles(np.zeros((1, 3)), np.ones(1))
    assert ex.value.code == ERR_CAPACITY
    assert "capacity" in str(ex.value)
    e.close()


def test_energy_pool_over_capacity():
    sc = scenes.cube_fixed_bottom(n=2)
    e = Context(energies_capacity=10)   # the 2^3 cube has 48 tets
    with pytest.raises(AvbdError) as ex:
        sc.load(e, precision="fp64")
    assert ex.value.code == ERR_CAPACITY
    e.close()


def test_more_than_256_colors():
    """257 oriented particles joined pairwise by Cosserat rods: the vertex
    graph is complete, so a proper coloring needs 257 colors."""
    n = 257
    e = Context(energies_capacity=1 << 16)
    X = np.stack([np.arange(n) * 0.1, np.zeros(n), np.zeros(n)], axis=1)
    q = np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))
    e.add_oriented_particles(X, q, np.ones(n), np.full((n, 3), 1e-3))
    i, j = np.triu_indices(n, 1)
    m = len(i)
    e.add_cosserat_rod(np.stack([i, j], 1), np.ones((m, 6)), np.full(m, 0.1), np.zeros((m, 3)))
    with pytest.raises(AvbdError) as ex:
        e.finalize()
    assert ex.value.code == ERR_COLORS
    e.close()


def test_candidate_pair_overflow_is_an_error():
    """A traversal that finds more pairs than the pair buffer holds fails the
    step instead of dropping collisions; with the default capacity the same
    scene runs."""
    sc = scenes.cube_drop(n=4, surface=True)
    e = Context()
    sc.load(e, precision="fp64")
    e.set_pair_capacity(16)
    e.finalize()
    with pytest.raises(AvbdError) as ex:
        e.collision_stage()
    assert ex.value.code == ERR_CAPACITY
    e.close()
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    e.collision_stage()
    assert 16 < len(e.candidate_pairs()) <= max(1024, 64 * sc.num_primitives)
    e.close()


def test_barrier_wait_gives_up_with_a_status():
    """A wait limit of zero polls makes the MLP kernel's tensor-core barrier
    wait give up at once: the call returns AVBD_ERR_BARRIER_TIMEOUT, and after
    the limit is restored the same object computes the same outputs as
    before."""
    torch = pytest.importorskip("torch")
    from avbd_b200 import warmstart
    L = _lib.load()
    rng = np.random.default_rng(5)
    p = warmstart.init_params(3)
    warmstart.view(p, "W4")[:3] = rng.normal(0, 0.2, size=(3, 128))
    X = np.zeros((1000, 32), dtype=np.float32)
    X[:, :27] = rng.normal(size=(1000, 27))
    feat = torch.tensor(X, device="cuda").to(torch.bfloat16).contiguous()
    m = warmstart.MLP(p)
    ref = m.forward(feat).cpu().numpy()
    try:
        assert L.avbd_debug_set_wait_limit(0, 0) == 0
        with pytest.raises(AvbdError) as ex:
            m.forward(feat)
        assert ex.value.code == ERR_TIMEOUT
        A = torch.ones((128, 32), device="cuda", dtype=torch.bfloat16)
        Cm = torch.zeros((128, 128), device="cuda", dtype=torch.float32)
        rc = L.avbd_gemm_bf16(C.c_void_p(A.data_ptr()), 32, C.c_void_p(A.data_ptr()), 32,
                              C.c_void_p(Cm.data_ptr()), 128, 128, 128, 32, 0, None)
        assert rc == ERR_TIMEOUT
    finally:
        assert L.avbd_debug_set_wait_limit(0, _lib.DEFAULT_WAIT_POLLS) == 0
    again = m.forward(feat).cpu().numpy()
    assert np.array_equal(again, ref)
    m.close()
