#!/usr/bin/env python
"""Benchmark: batched AVBD steps to residual 1e-4 on B200.

Workload (default): 1024 independent NeoHookean cubes of uneven size
(n ~ U{4..24} cells per side, 6 n^3 tets, E log-uniform 1e4..1e7,
nu ~ U(0.3, 0.49), random rotation, ground contact), all advanced together;
every step runs AVBD iterations until the residual R <= 1e-4 (at most
--max-iters).  One step of the batch counts as `scenes` scene-steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload batch_cubes|rods_spheres|contacts]

The batched-cubes line times two arms on identically built contexts: plain
AVBD (the adaptive inertial guess) and the learned warm start (the fused
tensor-core MLP corrects the guess before the same iterations); `value` is
the learned arm, `config.arms` holds both with their iterations per
scene-step, the fraction of scene-steps stopped at max_iters and the p50/p99
latency of one batch step (CUDA events around every step).

`--workload rods_spheres` measures the rod scene instead: 256 Cosserat rods
of 100 segments hanging from one-sided fixed joints plus 64 rigid spheres,
all with rigid-body ground contact, 20 iterations per step, FP32 (steps/s).

`--workload contacts` measures the dynamic contacts: 24 Cosserat rods of 32
segments dropped flat on a 32^3-cell tet cube (35,937 vertices, 196,608 tets,
12,288 surface triangles) resting on the ground; every step runs the LBVH
broad phase over triangles and rod segments, the triangle-rod narrow phase,
the contact pool merge (up to ~3,900 live contacts), the incremental
recoloring and the contact energies inside 20 iterations, FP32 (steps/s).
(Spheres on such a cube drift into each other within tens of steps, and
the reference throws on sphere-sphere candidates.)

Prints one JSON line.  `value` is scene-steps/s over all ranks with the state
resident in HBM; `e2e` repeats the measurement through the C-ABI with the
state uploaded from pinned host memory and the positions read back every
step; `roofline` reports the per-color vertex-solve kernel against the
measured HBM bandwidth on the launches a timed step uses; `cpu_baseline`
times the reference's own CPU solver (compiled from its sources into
oracle/_ref; the FP64 port where that library is absent) on the host cores,
on a stratified sample of the same batch, each scene-step running the
iterations the residual needs.  `--impl reference` prints that measurement
over the same --steps / --warmup window as its own line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s to residual 1e-4: learned+batched vs plain AVBD, same B200"
UNIT = "scene-steps/s"
DTYPES = {"fp32": "f32", "fp64": "f64", "mixed": "f64 state+gradient / f32 element records+Hessian"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--scenes", type=int, default=1024)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--tol", type=float, default=1e-4)
    p.add_argument("--max-iters", type=int, default=100)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--split", default="strong", choices=["strong", "weak"],
                   help="multi-GPU batch_cubes: one batch split across the ranks by tets (strong), or one "
                        "batch per rank with a rank-specific seed (weak)")
    p.add_argument("--precision", default=None, choices=["fp32", "mixed", "fp64"],
                   help="default: mixed for batch_cubes, fp32 for rods_spheres and contacts")
    p.add_argument("--workload", default="batch_cubes", choices=["batch_cubes", "rods_spheres", "contacts"])
    p.add_argument("--warmstart", default="learned", choices=["learned", "none"],
                   help="batch_cubes: time the learned warm start beside plain AVBD (value = learned)")
    p.add_argument("--weights", default=os.path.join(ROOT, "avbd_b200", "data", "warmstart_mlp.npz"))
    a = p.parse_args()
    if a.precision is None:
        a.precision = "mixed" if a.workload == "batch_cubes" else "fp32"
    return a


class Workload:
    """The scene set one rank advances, and how its steps are counted."""

    def __init__(self, args, seed, rank=0, world=1):
        from avbd_b200 import dist, scenes
        self.rods = args.workload == "rods_spheres"
        self.contacts = args.workload == "contacts"
        self.single = self.rods or self.contacts   # one scene, fixed iterations, working set within L2
        if self.rods:
            self.scene = scenes.rods_and_spheres(seed=seed)
            self.name = "rods256x100_spheres64"
            self.units = 1
            self.unit = "steps/s"
            self.tol, self.max_iters = 0.0, 0
            self.method = "plain AVBD, 20 fixed iterations per step"
        elif self.contacts:
            self.scene = scenes.rods_on_cube(n=32, num_rods=24, segments=32, rod_length=0.9, seed=seed)
            self.name = "cube32_rods24x32_contacts"
            self.units = 1
            self.unit = "steps/s"
            self.tol, self.max_iters = 0.0, 0
            self.method = ("plain AVBD with triangle-rod contacts (narrow phase, contact pool, "
                           "incremental recoloring), 20 fixed iterations per step")
        else:
            # strong scaling: this rank's tet-balanced part of one batch;
            # weak scaling: a whole batch of this rank's own seed
            ids = dist.batch_partition(args.scenes, seed, world)[rank] if args.split == "strong" else None
            self.scene = scenes.batched_cubes(num_scenes=args.scenes, seed=seed, scene_ids=ids)
            self.name = f"batch{args.scenes}_cubes"
            self.units = len(ids) if ids is not None else args.scenes
            self.unit = UNIT
            self.tol, self.max_iters = args.tol, args.max_iters
            self.method = "plain AVBD (no warm start)"


def measured_bf16():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        """Starts the sampler and returns once it has written its first sample,
        so its start-up (hundreds of ms) stays out of the timed region."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def traffic_for(workload: str, bytes_per_launch: float):
    """Per-launch DRAM bytes of the solve kernel: the DRAM/algorithmic ratio of
    the committed ncu capture times the algorithmic bytes per launch."""
    path = os.path.join(ROOT, "profiles", "solve_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        ratio = d[workload]["dram_over_algorithmic"]
        return ratio * bytes_per_launch
    except Exception:
        return None


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def stratified_sample(num_scenes, seed, size, pick_seed=20251):
    """Scenes of the batch in 8 strata (cells per side 4-8 / 9-13 / 14-18 /
    19-24 x E below / above 10^5.5); each stratum gets a share of the sample
    proportional to its population (at least one scene), drawn with a fixed
    generator.  Returns the scene ids and each one's weight (the stratum's
    population over its sampled count), so that sum(weight * t) estimates a
    per-scene total over the whole batch."""
    import numpy as np
    from avbd_b200.scenes import batched_cube_params
    strata = {}
    for s in range(num_scenes):
        n, E, _, _ = batched_cube_params(seed, s)
        strata.setdefault((min(3, (n - 4) // 5), int(np.log10(E) >= 5.5)), []).append(s)
    keys = sorted(strata)
    size = max(size, len(keys))
    share = {k: max(1, int(round(size * len(strata[k]) / num_scenes))) for k in keys}
    rng = np.random.default_rng(pick_seed)
    ids, weights = [], []
    for k in keys:
        m = min(share[k], len(strata[k]))
        for s in sorted(rng.choice(strata[k], size=m, replace=False).tolist()):
            ids.append(int(s))
            weights.append(len(strata[k]) / m)
    return ids, weights


def reference_batch(args, seed, warmup, steps, workers):
    """The reference's own CPU solver (oracle/_ref, compiled from its sources)
    on a stratified sample of the batch, each scene in its own
    SimulationContext, `workers` scenes at a time on the host cores.

    The reference has no residual: it runs a fixed iteration count.  Each
    sampled scene's step therefore runs exactly the iterations that this
    project's residual (evaluated by the FP64 port, which matches the
    reference's trajectory to 1e-12) needs to reach the tolerance in that step,
    at most max_iters -- the same count the GPU runs.  Steps 1..warmup run
    untimed, steps warmup+1..warmup+steps are timed (wall clock per step).
    Without oracle/_ref (no reference sources where it was built) the FP64
    port itself is timed.  Returns the line's fields."""
    import concurrent.futures as cf
    import numpy as np
    from avbd_b200 import scenes
    from oracle import ref
    from oracle.oracle import Oracle
    ids, weights = stratified_sample(args.scenes, seed, max(8, workers))
    total = warmup + steps

    def counts(s):  # iterations each step needs (untimed)
        sc = scenes.batched_cubes(num_scenes=args.scenes, seed=seed, scene_ids=[s])
        o = Oracle()
        sc.load(o, residual_tolerance=args.tol, max_iters=args.max_iters)
        o.finalize()
        out = []
        for _ in range(total):
            o.step(1)
            out.append(int(o.scene_iterations()[0]))
        return out

    use_ref = ref.available()

    def timed(s, its):
        sc = scenes.batched_cubes(num_scenes=args.scenes, seed=seed, scene_ids=[s])
        if use_ref:
            r = ref.RefSim(sc)
            sc.load(r)
            r.finalize()
        else:
            r = Oracle()
            sc.load(r, residual_tolerance=args.tol, max_iters=args.max_iters)
            r.finalize()
        t = 0.0
        for k, it in enumerate(its):
            if use_ref:
                r.set_iterations(it)
            dt = r.time_steps(1)
            if k >= warmup:
                t += dt
        verts = sc.num_particles
        if use_ref:
            r.close()
        return t / steps, verts

    t0 = time.time()
    with cf.ThreadPoolExecutor(workers) as ex:
        its = list(ex.map(counts, ids))
        res = list(ex.map(timed, ids, its))
    wall = time.time() - t0
    w = np.asarray(weights)
    t_scene = np.array([r[0] for r in res])            # s per step, one core
    verts = np.array([r[1] for r in res], dtype=np.float64)
    it_mean = np.array([np.mean(i[warmup:]) for i in its])
    T1 = float((w * t_scene).sum())                   # one batch step on one core
    value = args.scenes * workers / T1                 # scene-steps/s on `workers` cores
    capped = np.array([np.mean([x >= args.max_iters for x in i[warmup:]]) for i in its])
    return {
        "value": value,
        "iterations_per_scene_step": float((w * it_mean).sum() / w.sum()),
        "vertex_iterations_per_s": float((w * verts * it_mean).sum() * workers / T1),
        "capped_fraction": float((w * capped).sum() / w.sum()),
        "kind": "reference" if use_ref else "port",
        "cores": workers,
        "sample": (f"{len(ids)} of {args.scenes} scenes of the same batch, stratified by size and stiffness "
                   f"(weights = stratum population / sampled), steps {warmup + 1}-{total} of each "
                   f"({steps} timed), each step running the iterations the residual needs (<= {args.max_iters}); "
                   f"{'the reference compiled from its own sources' if use_ref else 'the FP64 port'}, "
                   f"{workers} scenes at a time; {wall:.0f} s wall"),
        "scene_ids": ids,
    }


def run_reference(args):
    from avbd_b200 import dist
    rank, world, _ = dist.env()
    if rank != 0:
        return
    workers = min(host_cores(), 32)
    wl = Workload(args, args.seed)
    if wl.single:
        v, kind, sample, it_ps = single_scene_reference(args, wl, args.warmup, args.steps, workers)
        extra = {}
    else:
        rb = reference_batch(args, args.seed, args.warmup, args.steps, workers)
        v, kind, sample = rb["value"], rb["kind"], rb["sample"]
        extra = {k: rb[k] for k in ("iterations_per_scene_step", "vertex_iterations_per_s", "capped_fraction",
                                    "scene_ids")}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": wl.unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wl.units / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "residual_tolerance": wl.tol, "max_iters": wl.max_iters, **extra},
            "cpu_baseline": {"value": v, "unit": wl.unit, "cores": workers, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": wl.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def single_scene_reference(args, wl, warmup, steps, threads):
    """The reference (or, without oracle/_ref, the FP64 port) on the
    single-scene workloads, with its own worker threads: steps/s."""
    from oracle import ref
    from oracle.oracle import Oracle
    sc = wl.scene
    if ref.available():
        r = ref.RefSim(sc, threads=threads)
        kind = "reference"
    else:
        r = Oracle(threads=threads)
        kind = "port"
    sc.load(r)
    r.finalize()
    r.step(max(1, warmup))
    n, t = 0, 0.0
    while n < steps and (t < args.cpu_seconds or n == 0):
        t += r.time_steps(1)
        n += 1
    what = "the reference compiled from its own sources" if kind == "reference" else "the FP64 port"
    return n / t, kind, f"the same scene, {n} steps after {max(1, warmup)} untimed, {what}, {threads} threads", None


def make_context(wl, args, local, stream):
    from avbd_b200 import Context
    e = Context(device=local)
    e.set_stream(stream.cuda_stream)
    wl.scene.load(e, residual_tolerance=wl.tol, max_iters=wl.max_iters, precision=args.precision)
    e.finalize()
    return e


def time_steps(e, stream, steps, flush=None, scene_verts=None):
    """Device time (ms) of `steps` steps on the engine's stream, with the
    counters they moved.  With `flush` (a tensor larger than L2) every step
    is preceded by a write of it and timed alone.  With `scene_verts` (the
    vertex count of every scene of a run-to-tolerance batch) each step's
    per-scene iteration counts are read after it (outside its events) and
    summed into vertex-iterations."""
    import numpy as np
    import torch
    st0 = e.stats()
    evs = []
    vert_it = 0.0
    for _ in range(steps):
        if flush is not None:
            with torch.cuda.stream(stream):
                flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.step(1)
        b.record(stream)
        evs.append((a, b))
        if scene_verts is not None:
            vert_it += float((e.scene_iterations().astype(np.float64) * scene_verts).sum())
    stream.synchronize()
    per = [a.elapsed_time(b) for a, b in evs]
    ms = sum(per)
    st1 = e.stats()
    d = {k: st1[k] - st0[k] for k in ("kernel_launches", "iterations", "capped_scene_steps", "warmstart_applied")}
    d["p50_ms"], d["p99_ms"] = float(np.percentile(per, 50)), float(np.percentile(per, 99))
    d["vertex_iterations"] = vert_it
    return ms, d


def time_e2e(e, stream, steps, n):
    """The same steps through the C-ABI with the state in pinned host memory:
    positions and velocities uploaded before and read back after every step."""
    import torch
    x_host = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    v_host = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    x_host[:] = e.positions()
    v_host[:] = e.velocities()
    torch.cuda.synchronize()
    st0 = e.stats()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        e.set_state(x_host, v_host)
        e.step(1)
        e.positions(out=x_host)
        e.velocities(out=v_host)
    b.record(stream)
    b.synchronize()
    st1 = e.stats()
    return a.elapsed_time(b), st1["iterations"] - st0["iterations"]


def mlp_roofline(e, n, local, peak):
    """Tensor-core roofline of the fused MLP kernel on this step's feature
    rows: 2 (27*128 + 2*128^2 + 128*3) FLOP per row over CUDA-event time."""
    import torch
    from avbd_b200 import warmstart
    F = torch.empty((n, 32), dtype=torch.bfloat16, device=torch.device("cuda", local))
    e.warmstart_sample(F, None)
    m = warmstart.MLP(e._ws_params, local)
    st = torch.cuda.Stream(device=local)
    for _ in range(3):
        m.forward(F, st.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    a.record(st)
    for _ in range(reps):
        m.forward(F, st.cuda_stream)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b) / reps
    m.close()
    flop = 2.0 * (27 * 128 + 2 * 128 * 128 + 128 * 3) * n
    tf = flop / (ms / 1e3) / 1e12
    return {"bound": "tensor", "kernel": "k_mlp_apply (fused MLP, tcgen05)", "achieved": tf, "peak": peak,
            "unit": "TFLOP/s", "frac": tf / peak, "traffic": None, "ms_per_launch": ms, "rows": n,
            "peak_source": "measured bf16_tflops (burst)"}


def run_engine(args):
    import numpy as np
    import torch

    from avbd_b200 import dist, warmstart

    rank, world, local = dist.env()
    torch.cuda.set_device(local)
    dist.init("nccl")
    seed = dist.shard_seed(args.seed, rank) if args.split == "weak" else args.seed
    dev = torch.device("cuda", local)

    t0 = time.time()
    wl = Workload(args, seed, rank, world)
    sc = wl.scene
    n = sc.num_particles
    stream = torch.cuda.Stream(device=local)
    learned = not wl.single and args.warmstart == "learned"
    params = warmstart.load_params(args.weights) if learned else None

    def build():
        e = make_context(wl, args, local, stream)
        if params is not None:
            e.set_warmstart(2, params)
            e._ws_params = params
        return e

    ep = make_context(wl, args, local, stream)       # plain AVBD
    el = build() if learned else None                # learned warm start, same scenes
    ee = build()                                     # the timed arm again, for the end-to-end run
    setup_s = time.time() - t0
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev) if wl.single else None

    for e in (ep, el, ee):
        if e is not None:
            e.step(args.warmup)
            e.synchronize()

    # ---- device-resident timing: plain, then learned
    dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    verts = None if wl.single else np.array([(c + 1) ** 3 for c in sc.meta["cells"]], dtype=np.float64)
    ms_plain, c_plain = time_steps(ep, stream, args.steps, flush, verts)
    ms_learn, c_learn = time_steps(el, stream, args.steps, flush, verts) if el is not None else (None, None)
    dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    main_e, ms, cnt = (el, ms_learn, c_learn) if el is not None else (ep, ms_plain, c_plain)

    # ---- end to end through the C-ABI with pinned host buffers, on a context
    # built and warmed like the timed arm, so it runs the same simulation steps
    dist.barrier()
    clocks_e2e = Clocks(local)
    clocks_e2e.start()
    ms_e2e, it_e2e = time_e2e(ee, stream, args.steps, n)
    clk_e2e = clocks_e2e.stop()
    dist.barrier()

    # ---- rooflines: the per-color vertex solve on the launches the timed step
    # uses (run-to-tolerance: per-scene pieces, converged scenes gated out;
    # fixed iterations: whole color slabs), and the MLP on the tensor cores
    sum_sweep_bytes = 0.0
    if wl.tol > 0:
        solve_ms, solve_bytes, solve_launches, prof_iters = ep.profile_step()
        sum_sweep_bytes = ep.profile_solve(1)[1]   # one whole-slab sweep: every scene's data
    else:
        solve_ms, solve_bytes, solve_launches = ep.profile_solve(2)
        prof_iters = 2
    ep.synchronize()
    peak, peak_kind = measured_peaks()
    roof_mlp = mlp_roofline(el, n, local, measured_bf16()) if el is not None else None

    red = dist.reduce([ms, ms_e2e, ms_plain], "max", device=dev)
    ms_max, ms_e2e_max, ms_plain_max = red
    units_all = dist.reduce([float(wl.units)], "sum", device=dev)[0]   # scenes all ranks advance
    value = units_all * args.steps / (ms_max / 1e3)
    value_e2e = units_all * args.steps / (ms_e2e_max / 1e3)
    value_plain = units_all * args.steps / (ms_plain_max / 1e3)

    if rank == 0:
        per_launch_ms = solve_ms / max(1, solve_launches)
        per_launch_bytes = solve_bytes / max(1, solve_launches)
        achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
        workload = wl.name
        # one solve launch per iteration: the persistent sweep (every color of
        # the iteration in one cooperative launch)
        persistent = wl.tol > 0 and not wl.rods and solve_launches == prof_iters
        kernel = ("k_solve_rod (per-color 6-DOF vertex block solve)" if wl.rods
                  else "k_sweep_persistent (vertex block solve, every color of an iteration in one launch)"
                  if persistent else "k_solve_tet (per-color vertex block solve)")
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic_for(workload, per_launch_bytes), "kernel": kernel,
                "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms, "peak_source": peak_kind,
                "launch_shape": ("one run-to-tolerance step as timed: one persistent sweep per iteration, "
                                 "blocks drawing the per-scene pieces of each color slab in turn, converged "
                                 f"scenes gated out ({solve_launches} launches, {prof_iters} iterations)"
                                 if persistent else
                                 "one run-to-tolerance step as timed: per-scene pieces of every color slab, "
                                 f"converged scenes gated out ({solve_launches} launches, {prof_iters} iterations)"
                                 if wl.tol > 0 else f"whole color slabs ({solve_launches} launches, "
                                 f"{prof_iters} iterations)")}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            workers = min(host_cores(), 32)
            if wl.single:
                v_cpu, kind, what, _ = single_scene_reference(args, wl, args.warmup, 3, workers)
                cpu = {"value": v_cpu, "unit": wl.unit, "cores": workers, "kind": kind, "sample": what}
            else:
                rb = reference_batch(args, seed, args.warmup, min(args.steps, 3), workers)
                cpu = {"value": rb["value"], "unit": wl.unit, "cores": workers, "kind": rb["kind"],
                       "sample": rb["sample"], "iterations_per_scene_step": rb["iterations_per_scene_step"],
                       "vertex_iterations_per_s": rb["vertex_iterations_per_s"]}
        su = args.steps * wl.units
        def arm(val, ms_arm, c):
            a = {"value": val, "ms_per_step": ms_arm / args.steps,
                 "step_latency_ms": {"p50": c["p50_ms"], "p99": c["p99_ms"]},
                 "iterations_per_scene_step": c["iterations"] / su}
            if wl.tol > 0:
                a["capped_fraction"] = c["capped_scene_steps"] / su
                a["converged_scene_steps_per_s"] = val * (1 - c["capped_scene_steps"] / su)
                a["vertex_iterations_per_s"] = c["vertex_iterations"] * world / (ms_arm / 1e3)
            return a

        arms = {"plain": arm(value_plain, ms_plain_max, c_plain)}
        if el is not None:
            arms["learned"] = arm(value, ms_max, c_learn)
            arms["learned"]["corrections_applied_fraction"] = c_learn["warmstart_applied"] / (args.steps * n)
        method = (wl.method if el is None else
                  "learned warm start (MLP 27-128-128-128-3, BF16 tcgen05) + plain AVBD iterations")
        line = {
            "metric": METRIC, "value": value, "unit": wl.unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if (args.split == "strong" and not wl.single) else "weak",
            "vs_baseline": None, "dtype": DTYPES[args.precision], "data": "synthetic",
            "config": {"workload": workload, "scenes_per_gpu": wl.units, "vertices_per_gpu": n,
                       "tets_per_gpu": sc.num_tets, "residual_tolerance": wl.tol, "max_iters": wl.max_iters,
                       "method": method, "arms": arms, "precision": args.precision,
                       "l2": (f"L2 flushed (256 MB write) before every timed step; "
                              f"{solve_bytes / prof_iters / 1e6:.1f} MB of solve data per iteration" if wl.single else
                              f"inputs larger than L2: {sum_sweep_bytes / 1e9:.2f} GB of solve data in a sweep of "
                              "every scene"),
                       "parallelism": (f"dp{world}: one batch split across the GPUs, balanced by tets"
                                       if args.split == "strong" and not wl.single else
                                       f"dp{world}: independent scenes per GPU"),
                       "setup_s": round(setup_s, 1)},
            "clocks": clk, "gpu_launches": cnt["kernel_launches"],
            "e2e": {"value": value_e2e, "unit": wl.unit, "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": 48 * n,
                    "iterations_per_scene_step": it_e2e / su, "clocks": clk_e2e},
            "roofline": roof, "roofline_mlp": roof_mlp, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    for e in (ep, el, ee):
        if e is not None:
            e.close()
    dist.shutdown()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
