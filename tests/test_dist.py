"""Multi-process plumbing on CPU (gloo, world size 2): the sharded run is the
union of independent per-rank runs, reductions give the max/sum over ranks,
and a rank that leaves makes the other's next collective fail instead of
hanging."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    try:
        from avbd_b200 import dist, scenes
        dist.init("gloo", timeout_s=20)
        if mode == "shard":
            seed = dist.shard_seed(0, rank)
            from oracle.oracle import Oracle
            sc = scenes.batched_cubes(num_scenes=2, seed=seed, n_min=2, n_max=3)
            o = Oracle()
            sc.load(o, residual_tolerance=1e-4, max_iters=50)
            o.finalize()
            o.step(2)
            x = o.positions()
            mx, sm = dist.reduce([float(rank + 1), float(x.shape[0])], "max"), dist.reduce([float(x.shape[0])], "sum")
            dist.barrier()
            q.put((rank, seed, float(np.abs(x).sum()), mx, sm))
        elif mode == "leave":
            if rank == 1:
                q.put((rank, "left"))
                q.close()
                q.join_thread()
                os._exit(0)  # leaves between steps: no collective in flight
            try:
                dist.barrier(timeout_s=3)
                q.put((rank, "no error"))
            except Exception as exc:  # the barrier fails instead of hanging
                q.put((rank, "error", str(exc)[:200]))
            q.close()
            q.join_thread()
            os._exit(0)
        dist.shutdown()
    except Exception as exc:
        q.put((rank, "exception", repr(exc)))


def _run(mode, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = []
    for _ in range(world):
        out.append(q.get(timeout=timeout))
    for p in ps:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


def test_sharded_run_equals_independent_runs():
    from avbd_b200 import dist, scenes
    from oracle.oracle import Oracle
    res = _run("shard")
    assert [r[0] for r in res] == [0, 1]
    assert res[0][1] != res[1][1]  # distinct scene seeds per rank
    n = []
    for rank, seed, checksum, mx, sm in res:
        assert seed == dist.shard_seed(0, rank)
        sc = scenes.batched_cubes(num_scenes=2, seed=seed, n_min=2, n_max=3)
        o = Oracle()
        sc.load(o, residual_tolerance=1e-4, max_iters=50)
        o.finalize()
        o.step(2)
        assert np.isclose(float(np.abs(o.positions()).sum()), checksum, rtol=0, atol=1e-12)
        n.append(o.num_particles)
        assert mx[0] == 2.0
    for r in res:
        assert r[3][1] == max(n) and r[4][0] == sum(n)


def test_rank_leaving_fails_the_next_collective():
    res = _run("leave")
    assert res[1][1] == "left"
    assert res[0][1] == "error", res[0]
    assert "1" in res[0][2]  # names the missing rank
