"""Benchmark of the Sim.step hot path (body-steps/s) on B200.

Contract: ``python bench.py --gpus N --steps K --warmup W`` prints one JSON line. A step is one
frame (all substeps) of every scene of the workload. Default workload: the uneven batch (2048
independent scenes, log-uniform 8-512 boxes each plus one 2-40 link revolute chain and a ground
plane, 240 fps, 4 substeps, 12 iterations), stepped as one batch per substep launch sequence and
replayed from a CUDA graph. Inputs are seeded synthetic scenes (no dataset exists for this path).

``--impl reference`` times the reference algorithm on the host cores instead: the CPU oracle (a
restatement of the reference's WGSL; the reference itself needs a WebGPU adapter and a JS runtime,
neither of which exists here), over a bounded sample of the same scenes, all cores in parallel.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (generator kwargs, description)
    "uneven_batch_2048": dict(n_scenes=2048),
    "uneven_batch_256": dict(n_scenes=256),
    "uneven_batch_512": dict(n_scenes=512),  # loaded case (several blocks per SM) for profiler captures
    "uneven_batch_64": dict(n_scenes=64),  # small case for profiler captures
    # Single large scenes (the plain method at scale): one block runs each scene's prepare and solve.
    "convex_pour_8192": dict(n_scenes=1, single="convex_pour"),  # 8192 hulls, boxes, capsules in a bin
    "quadrupeds_1024": dict(n_scenes=1, single="quadrupeds"),  # 1024 quadrupeds + 64 x 40-link chains
    "boxes_64": dict(n_scenes=1, single="boxes"),  # 64 boxes on a plane
    # Serving: resident instances of the articulation workload's sizes (1-4 quadrupeds, or one
    # 40-link chain, on a plane; 500 fps), mixed so that instances differ in size.
    "serve_quadrupeds_4096": dict(n_scenes=4096, serve=True),
}


def _build_single(kind: str, seed: int):
    from steel_webgpu_b200 import pack, synth
    from steel_webgpu_b200.sim import auto_caps
    if kind == "convex_pour":
        sc = synth.convex_pour(n=8192, seed=seed)
        caps = auto_caps(sc)  # the settled pour needs more than the uneven batch's 8 pairs per shape
        caps.update(MAXP=1 << 18, MAXC=1 << 18, MAXU=1 << 18, UH=1 << 18, WH=1 << 19, AH=1 << 18)
        return [pack(sc, caps=caps)]
    sc = synth.quadrupeds(n_quad=1024, n_chains=64, chain_links=40, seed=seed) if kind == "quadrupeds" \
        else synth.boxes_on_plane(64, seed=seed)
    return [pack(sc, caps=auto_caps(sc))]


def _build_chunk(args):
    seed, lo, hi, n_total, caps_mode, fp64 = args
    from steel_webgpu_b200 import pack, synth
    from steel_webgpu_b200.sim import auto_caps
    # Every scene draws from its own generator seeded by (seed, index), so chunks are independent.
    opts = {"solver": {"articulation_fp64": True}} if fp64 else None
    out = []
    for i in range(lo, hi):
        if n_total < 0:  # serving instances
            kind = i % 5
            sc = synth.quadrupeds(n_quad=kind + 1 if kind < 4 else 0, n_chains=1 if kind == 4 else 0, chain_links=40,
                                  seed=seed * 1000003 + i)
            out.append(pack(sc, opts=opts, caps=auto_caps(sc)))
            continue
        sc = synth.uneven_batch(n_scenes=1, seed=seed * 1000003 + i)[0]
        out.append(pack(sc, opts=opts, caps=auto_caps(sc) if caps_mode == "auto" else None))
    return out


def build_workload(name: str, seed: int, caps_mode: str = "auto", nproc: int | None = None, limit: int | None = None,
                   fp64: bool = False):
    """The workload's packed scenes. fp64: the articulated-inertia pass's D factor/inverse and root
    inertia accumulation in FP64 (the uneven batch's stated precision split)."""
    if "single" in WORKLOADS[name]:
        return _build_single(WORKLOADS[name]["single"], seed)
    n = WORKLOADS[name]["n_scenes"]
    if limit is not None:
        n = min(n, limit)
    nproc = nproc or min(os.cpu_count() or 1, 32)
    chunk = max(1, math.ceil(n / (nproc * 4)))
    total = -1 if WORKLOADS[name].get("serve") else n
    jobs = [(seed, lo, min(lo + chunk, n), total, caps_mode, fp64) for lo in range(0, n, chunk)]
    if nproc <= 1 or len(jobs) == 1:
        parts = [_build_chunk(j) for j in jobs]
    else:
        with mp.get_context("spawn").Pool(nproc) as pool:
            parts = pool.map(_build_chunk, jobs)
    return [p for part in parts for p in part]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"steel_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for k, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def trace_summary(batch, pks) -> dict:
    """One traced frame (steel_trace): for the last prepare and solve launches, the launch span, the
    longest block and its scene, the mean block time and the most blocks resident at once; the span
    over the work per slot says how far the launch is from a balanced one."""
    batch.trace(True)
    batch.step(1)
    rec = batch.trace_read()
    batch.trace(False)
    out = {}
    for k in ("prepare", "solve"):
        r = rec[k]
        ran = r[:, 0] > 0
        st, en = r[ran, 0], r[ran, 1]
        dur = (en - st) / 1e3
        ev = sorted([(t, 1) for t in st] + [(t, -1) for t in en], key=lambda x: (x[0], x[1]))
        cur = peak = 0
        for _, d in ev:
            cur += d
            peak = max(peak, cur)
        i = int(np.argmax(dur))
        scene = int(np.nonzero(ran)[0][i])
        out[k] = {"span_us": round(float((en.max() - st.min()) / 1e3), 1), "longest_block_us": round(float(dur[i]), 1),
                  "longest_scene": {"links": pks[scene].NL, "bodies": pks[scene].NB},
                  "mean_block_us": round(float(dur.mean()), 1), "max_resident_blocks": peak,
                  "balanced_span_us": round(float(dur.sum() / max(peak, 1)), 1)}
    out["what"] = ("steel_trace of one frame after the timed regions: block start/end from the global timer, "
                   "last launch of the frame; balanced_span_us = summed block time / max resident blocks")
    return out


def scene_counts(batch, pks):
    """Run-measured per-scene counts for the algorithmic byte model (last substep)."""
    tot = dict(NB=0, NS=0, NL=0, pairs=0, contacts=0, rows=0, hull_bytes=0)
    for i, pk in enumerate(pks):
        st = batch.stats(i)
        meta = batch.read_words("sched", batch.layout("S_META", i), 1, scene=i, dtype=np.uint32)[0]
        rows = batch.read_words("sched", batch.layout("S_USTART", i) + int(meta), 1, scene=i, dtype=np.uint32)[0]
        tot["NB"] += pk.NB
        tot["NS"] += pk.NS
        tot["NL"] += pk.NL
        tot["pairs"] += st["max_pairs"]
        tot["contacts"] += st["contacts"]
        tot["rows"] += int(rows)
    return tot


# DRAM bytes (read + write) per body and launch, from one ncu capture of the 512-scene uneven batch
# (80,090 bodies, FP64 D-inverse, the 64-thread kernel instances and 12.9 KB staging budget the
# autotuner picks for the bench batch; cold cache). Scaled by a batch's body count for the bench
# line's roofline traffic; the narrow stage is k_narrow + k_narrow_jobs.
NCU_TRAFFIC_PER_BODY = {"narrow": 2031.0, "prepare": 1902.0, "solve": 1575.0}


def kernel_bytes(k: str, c: dict, rows_vec4: int, iterations: int) -> float:
    """Algorithmic bytes per launch of kernel k over the whole batch (one substep).

    Terms follow the per-substep byte budget of the path: body static record 128 B and COM pose +
    twist 64 B read and written; shape record 112 B read, pose + AABB 64 B written; a pair 8 B
    written and read; a contact record 96 B written by narrow, read and written by the sort, read by
    prepare; a row ROWS x 16 B written once and read every sweep with its 16 B impulse written; a
    link block 1072 B read and written once, and per sweep 24 B twist read/written plus 432 B of
    motion subspace, U and D^-1 read.
    """
    NB, NS, NP, NC, NK, NL = c["NB"], c["NS"], c["pairs"], c["contacts"], c["rows"], c["NL"]
    I = iterations
    if k == "shapes":
        return NS * (112 + 64) + NB * 32
    if k == "broad":
        return NS * 64 + NP * 8
    if k == "narrow":
        return NP * (8 + 2 * 112 + 2 * 32) + NC * 96
    if k == "csort":
        return NC * (96 + 96 + 16)
    if k == "prepare":
        return NB * (128 + 64) + NC * 96 + NK * rows_vec4 * 16 + NL * 2 * 1072
    if k == "solve":
        return NK * rows_vec4 * 16 * (1 + I) + NK * 16 * (1 + I) + NB * (128 + 2 * 64) + NL * (2 * 1072 + I * (2 * 24 + 432))
    return 0.0


def _oracle_worker(conn, pks):
    from oracle.oracle import OracleSim
    sims = [OracleSim(pk) for pk in pks]
    conn.send("ready")
    while True:
        frames = conn.recv()
        if frames is None:
            break
        for s in sims:
            s.step(frames)
        conn.send("done")


class OraclePool:
    """CPU oracle sims spread over worker processes (spawned), built once, stepped on command."""

    def __init__(self, pks, nproc: int):
        ctx = mp.get_context("spawn")
        self.workers = []
        shares = [pks[i::nproc] for i in range(nproc)]
        for share in shares:
            if not share:
                continue
            a, b = ctx.Pipe()
            p = ctx.Process(target=_oracle_worker, args=(b, share), daemon=True)
            p.start()
            self.workers.append((p, a))
        for _, a in self.workers:
            a.recv()
        self.bodies = sum(pk.NB for pk in pks)

    def step(self, frames: int) -> float:
        t0 = time.perf_counter()
        for _, a in self.workers:
            a.send(frames)
        for _, a in self.workers:
            a.recv()
        return time.perf_counter() - t0

    def close(self):
        for p, a in self.workers:
            a.send(None)
            p.join(10)


def cpu_baseline_sample(pks, frames: int):
    """The CPU oracle on a bounded sample, one thread: body-steps/s and the stepping time."""
    from oracle.oracle import OracleSim
    sims = [OracleSim(pk) for pk in pks]
    t0 = time.perf_counter()
    for s in sims:
        s.step(frames)
    dt = time.perf_counter() - t0
    return sum(pk.NB for pk in pks) * frames / dt, dt


def dist_setup(n_gpus: int, backend: str = "nccl"):
    """Rank, world size and local device from the torchrun environment (single process otherwise)."""
    if n_gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0
    import torch
    import torch.distributed as dist
    import datetime
    rank, world, local = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]), int(os.environ.get("LOCAL_RANK", 0))
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(x: float, world: int, local: int = 0) -> float:
    """The maximum of x over all ranks (x itself for one rank): times are max-over-ranks."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def whole_job_rate(world: int, units_per_rank: int, steps: int, seconds: float) -> float:
    """Units of all ranks per second of the slowest rank (every rank steps the same workload size)."""
    return world * units_per_rank * steps / seconds


def plain_path_sample(pks, frames: int, device: int):
    """The plain path: each scene alone, one batch of one scene per launch sequence; body-steps/s."""
    from steel_webgpu_b200.sim import Batch
    bodies, ms = 0, 0.0
    for pk in pks:
        b = Batch([pk], device=device)
        b.step(3)
        ms += b.step_timed(frames)
        bodies += pk.NB * frames
        b.close()
    return bodies / (ms / 1000.0)


def single_scenes(device: int, frames: int = 3, warmup: int = 3) -> dict:
    """The plain method at scale on one scene each: the 8192-body convex pour (240 fps) and 1024
    quadrupeds with 64 40-link chains (500 fps), created from their scene files through the C ABI
    (packed in C++), tiles from the autotuner; device-timed body-steps/s."""
    import json as _json
    from steel_webgpu_b200 import synth
    from steel_webgpu_b200.sim import Batch, auto_caps
    out = {}
    for name, make, extra_caps in (
            ("convex_pour_8192", lambda: synth.convex_pour(n=8192, seed=0),
             dict(MAXP=1 << 18, MAXC=1 << 18, MAXU=1 << 18, UH=1 << 18, WH=1 << 19, AH=1 << 18)),
            ("quadrupeds_1024", lambda: synth.quadrupeds(n_quad=1024, n_chains=64, chain_links=40, seed=0), {})):
        t0 = time.perf_counter()
        sc = make()
        caps = auto_caps(sc)
        caps.update(extra_caps)
        b = Batch.from_files([(_json.dumps(sc.json).encode(), sc.bin, {"capacities": caps})], device=device)
        build_s = time.perf_counter() - t0
        tiles, _ = b.autotune(2)
        b.step(warmup)
        ms = b.step_timed(frames) / frames
        nb = sc.json["bodies"]["count"]
        out[name] = {"body_steps_per_s": nb / (ms / 1000.0), "ms_per_frame": ms, "bodies": nb,
                     "fps": sc.json["fps"], "tiles": tiles, "team_blocks": b.team(), "build_s": round(build_s, 1),
                     "timed": f"{frames} frames after {warmup} warm-up frames, CUDA events"}
        b.close()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    nproc = min(os.cpu_count() or 1, 64)
    # Bounded sample: the first scenes of the same workload with the reference's capacities.
    sample = build_workload(args.workload, args.seed, caps_mode="reference", limit=args.ref_scenes)
    nb = sum(pk.NB for pk in sample)
    pool = OraclePool(sample, nproc)
    for _ in range(args.warmup):
        pool.step(1)
    times = [pool.step(1) for _ in range(args.steps)]
    pool.close()
    step_s = statistics.mean(times)
    value = nb / step_s
    line = {"metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "sample_scenes": len(sample), "sample_bodies": nb,
                       "precision": "FP32 throughout, the reference's own arithmetic",
                       "fps": sample[0].params["fps"], "substeps": sample[0].params["substeps"], "iterations": sample[0].params["iterations"]},
            "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": nproc, "kind": "port",
                             "sample": f"{len(sample)} scenes ({nb} bodies) of {args.workload}, 1 frame per step"},
            "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_steel(args):
    import torch
    rank, world, local = dist_setup(args.gpus)
    from steel_webgpu_b200.sim import Batch
    t_build = time.perf_counter()
    fp64 = args.fp64_dinv == "on"
    pks = build_workload(args.workload, args.seed + rank, fp64=fp64)
    build_s = time.perf_counter() - t_build
    batch = Batch(pks, device=local)
    nbodies = sum(pk.NB for pk in pks)
    iterations = pks[0].params["iterations"]
    substeps = pks[0].params["substeps"]
    # Tile configuration: the autotuner's short timed search (it resets the batch afterwards), or
    # the configuration given on the command line. Outside the timed region.
    t_tune = time.perf_counter()
    if args.tiles == "auto":
        tiles, tune_ms = batch.autotune(args.tune_frames)
    else:
        batch.set_tiles(*[int(x) for x in args.tiles.split(",")])
        tiles, tune_ms = batch.tiles(), None
    tune_s = time.perf_counter() - t_tune
    batch.step(max(args.warmup, 3))
    batch.sync()
    barrier(world)
    torch.cuda.synchronize(local)
    with ClockSampler(local) as clk:
        ms = batch.step_timed(args.steps)
    torch.cuda.synchronize(local)
    ms = max_over_ranks(ms, world, local)
    value = whole_job_rate(world, nbodies, args.steps, ms / 1000.0)
    # End to end through the C ABI with pinned host buffers: joint targets in, body poses out. The
    # batch restarts from its initial state and takes the same warm-up, so these K frames are the
    # frames the device-timed region covered (the piles grow denser as a run goes on).
    batch.reset()
    batch.step(max(args.warmup, 3) - 1)
    nd = sum(pk.ND for pk in pks)
    npose = sum(pk.NB * 8 for pk in pks)
    h_tgt = torch.zeros(max(nd, 1), dtype=torch.float32, pin_memory=True).numpy()[:nd]
    h_pose = torch.zeros(npose, dtype=torch.float32, pin_memory=True).numpy()
    rng = np.random.default_rng(1)
    batch.step_io(1, h_tgt if nd else None, h_pose)
    barrier(world)
    frame_ms = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f0 = time.perf_counter()
        h_tgt[:] = rng.uniform(-0.5, 0.5, nd).astype(np.float32)
        batch.step_io(1, h_tgt if nd else None, h_pose)
        frame_ms.append((time.perf_counter() - f0) * 1000.0)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, local)
    e2e = whole_job_rate(world, nbodies, args.steps, e2e_s)
    # Roofline of the dominant kernel: per-launch device time from CUDA events around each launch,
    # over the first frames of the timed region (restart and warm-up as above).
    batch.reset()
    batch.step(max(args.warmup, 3))
    prof = batch.profile_kernels(max(2, min(args.steps, 8)))
    counts = scene_counts(batch, pks)
    # Capacities change results only when a buffer overflows; count the scenes where one did.
    overflow_scenes = sum(1 for i in range(len(pks)) if batch.stats(i)["overflow"])
    block_trace = trace_summary(batch, pks) if pks and pks[0].NB else None
    rows_vec4 = pks[0].C["ROWS"]
    total_ms = sum(prof.values())
    dom = max(prof, key=prof.get)
    peak, peak_kind = measured_peaks()
    bytes_dom = kernel_bytes(dom, counts, rows_vec4, iterations)
    achieved = bytes_dom / (prof[dom] / 1000.0) / 1e9
    if rank != 0:
        return
    plain = plain_path_sample(pks[:args.plain_scenes], 2, local) if args.plain_scenes > 0 else None
    singles = single_scenes(local) if (args.single_scenes == "on" and world == 1) else None
    cpu_sample = pks[:args.cpu_scenes]
    cpu_val, cpu_dt = cpu_baseline_sample(cpu_sample, args.cpu_frames)
    clocks = clk.summary()
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes, no dataset)",
        "config": {"workload": args.workload, "scenes_per_gpu": len(pks), "bodies_per_gpu": nbodies,
                   "fps": pks[0].params["fps"], "substeps": substeps, "iterations": iterations, "parallelism": f"replicas x{world}",
                   "graph": True, "l2": "per-scene state is resident and re-read every substep; no L2 flush",
                   "contact_steps_per_s": world * counts["contacts"] * substeps * args.steps / (ms / 1000.0),
                   "build_s": round(build_s, 1), "overflow_scenes": overflow_scenes,
                   "fp64_dinv": fp64 and "single" not in WORKLOADS[args.workload],
                   "placement": "each scene's boxes on a 0.4 m grid, dropped from 0.3-1.3 m onto its plane (a 2x2x2 m "
                                "volume cannot hold 512 boxes of half-extents 0.05-0.15 m without overlaps)",
                   "tiles": dict(tiles, source="autotuner" if args.tiles == "auto" else "command line",
                                 tuning_ms_per_frame=tune_ms, tuning_s=round(tune_s, 2),
                                 team_blocks=batch.team()),
                   "frame_latency_ms": {"p50": float(np.percentile(frame_ms, 50)),
                                        "p99": float(np.percentile(frame_ms, 99)),
                                        "what": "one frame of the whole batch through steel_step_io, host clock"},
                   "plain_path": None if plain is None else {
                       "body_steps_per_s": plain, "batched_over_plain": value / world / plain,
                       "sample": f"first {args.plain_scenes} scenes, each alone (one scene per launch sequence), 2 frames"}},
        "e2e": {"value": e2e, "unit": "body-steps/s", "h2d_bytes_per_step": 4 * nd, "d2h_bytes_per_step": 4 * npose},
        "gpu_launches": args.steps * (substeps * 8 + 1),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": NCU_TRAFFIC_PER_BODY[dom] * nbodies if dom in NCU_TRAFFIC_PER_BODY else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of uneven_batch_512 "
                                       "(64-thread tiles, FP64 D-inverse), per body, scaled to this batch",
                     "algorithmic_bytes_per_launch": bytes_dom, "ms_per_launch": prof[dom],
                     "kernel_share": {k: round(v / total_ms, 4) for k, v in prof.items()}},
        "single_scenes": singles,
        "block_trace": block_trace,
        "cpu_baseline": {"value": cpu_val, "unit": "body-steps/s", "cores": 1, "kind": "port",
                         "sample": f"{len(cpu_sample)} scenes x {args.cpu_frames} frames on the CPU oracle "
                                   f"({cpu_dt:.1f} s)"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _serve_at_rate(batch, pks, rate: float, n: int, seed: int, max_active: int, budget: int) -> dict:
    """Poisson arrivals at `rate` requests/s of n requests (1-32 frames each, random instances),
    continuous batching through steel_serve_*; latency from submit to completion."""
    from steel_webgpu_b200.sim import Server
    srv = Server(batch, max_active=max_active, budget_bytes=budget)
    rng = np.random.default_rng(seed)
    arrive = np.cumsum(rng.exponential(1.0 / rate, n))
    inst = rng.integers(0, len(pks), n)
    frames = rng.integers(1, 33, n)
    done, k, lat, body_frames, ticks, active = 0, 0, [], 0, 0, []
    t0 = time.perf_counter()
    while done < n:
        now = time.perf_counter() - t0
        while k < n and arrive[k] <= now:
            srv.submit(int(inst[k]), int(frames[k]))
            body_frames += pks[int(inst[k])].NB * int(frames[k])
            k += 1
        stepped = srv.tick()
        if stepped == 0 and k < n:
            time.sleep(max(0.0, min(arrive[k] - (time.perf_counter() - t0), 0.001)))
        else:
            ticks += 1
            active.append(stepped)
        for _, _, ms in srv.poll():
            lat.append(ms)
            done += 1
    wall = time.perf_counter() - t0
    srv.close()
    return {"rate_per_s": rate, "requests": n, "completed_per_s": n / wall, "body_steps_per_s": body_frames / wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "ticks": ticks, "mean_admitted": float(np.mean(active)) if active else 0.0, "wall_s": round(wall, 2)}


def run_serve(args):
    """Serving: resident instances, Poisson arrivals of 1-32-frame requests for random instances at
    each rate of a sweep, continuous batching (steel_serve_*) with admission by an HBM budget;
    p50/p99 request latency and served body-steps/s per rate, beside the plain per-scene path."""
    from steel_webgpu_b200.sim import Batch
    pks = build_workload(args.workload, args.seed, limit=args.serve_instances)
    batch = Batch(pks)
    batch.step(2)
    batch.sync()
    inst_bytes = [batch.scene_bytes(i) for i in range(len(pks))]
    budget = int(args.serve_budget_mb * 1e6)
    rates = [float(r) for r in args.serve_rates.split(",")]
    sweep = []
    for r in rates:
        n = int(min(max(r * args.serve_seconds, 300), args.serve_requests))
        sweep.append(_serve_at_rate(batch, pks, r, n, args.seed, args.serve_max_active, budget))
        print(json.dumps(sweep[-1]), file=sys.stderr, flush=True)
    plain = plain_path_sample(pks[:16], 4, 0)
    print(json.dumps({
        "metric": "served body-steps/s", "value": max(x["body_steps_per_s"] for x in sweep), "unit": "body-steps/s",
        "n_gpus": 1, "higher_is_better": True, "data": "synthetic (seeded scenes, no dataset)",
        "config": {"workload": args.workload, "instances": len(pks), "bodies": sum(pk.NB for pk in pks),
                   "instance_mb": {"min": min(inst_bytes) / 1e6, "max": max(inst_bytes) / 1e6,
                                   "total": sum(inst_bytes) / 1e6},
                   "hbm_budget_mb": args.serve_budget_mb, "max_active": args.serve_max_active or len(pks),
                   "frames_per_request": "uniform 1-32", "arrivals": "Poisson"},
        "sweep": sweep,
        "plain_path": {"body_steps_per_s": plain, "sample": "16 instances, each alone (one scene per launch sequence)"},
    }), flush=True)
    batch.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="steel", choices=["steel", "reference"])
    ap.add_argument("--workload", default="uneven_batch_2048", choices=list(WORKLOADS))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-scenes", type=int, default=128)
    ap.add_argument("--cpu-frames", type=int, default=8)
    ap.add_argument("--ref-scenes", type=int, default=128)
    ap.add_argument("--plain-scenes", type=int, default=16)
    ap.add_argument("--mode", default="bench", choices=["bench", "serve"])
    ap.add_argument("--tiles", default="auto",
                    help='"auto" (autotuner) or block_threads,smem_budget,narrow_blocks_per_sm')
    ap.add_argument("--tune-frames", type=int, default=3)
    ap.add_argument("--single-scenes", default="on", choices=["on", "off"],
                    help="also time the 8192-body pour and the 1024-quadruped scene (one scene each)")
    ap.add_argument("--fp64-dinv", default="on", choices=["on", "off"],
                    help="FP64 in the articulated-inertia D factor/inverse and root inertia (uneven batch)")
    ap.add_argument("--serve-instances", type=int, default=4096)
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-rates", default="1000,3000,10000,20000,50000")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-budget-mb", type=float, default=0.0)
    ap.add_argument("--serve-max-active", type=int, default=0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "serve":
        if args.workload == "uneven_batch_2048":
            args.workload = "serve_quadrupeds_4096"
        run_serve(args)
    else:
        run_steel(args)


if __name__ == "__main__":
    main()
