"""Particle-substeps/s of the plain PBF dam break (1,048,576 particles) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one frame of the scene: 2 substeps of predict -> cell-key sort -> 4 PBF iterations ->
velocity update.  `value` times K frames replayed from one CUDA graph with the state resident in
HBM (device time, CUDA events, max over ranks).  `e2e` times the same frames through the C ABI
with the particle state uploaded from pinned host memory and read back every frame (the
reference's enableBlockingReadback behaviour).  Under torchrun each rank steps its own replica
of the scene (the single-scene substep does not shard), so `scaling` is "weak".

--impl reference times the reference's CPU implementation of the same path on the same full
workload.  The reference's own solver is Vulkan/D3D12 HLSL behind Diligent Engine and cannot run
here, so its CPU restatement (the oracle under oracle/, pinned to the reference's own shaders) is
timed on the host cores with every thread it can use; the scene comes from oracle/cn_scenes.py,
so that arm loads no product library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cressim-neo_b200"))

import numpy as np  # noqa: E402

METRIC = "particle-substeps/s"
WORKLOAD = "pbf_dam_break_128x64x128"
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=0, help="frames of the e2e run (0: the timed frames again)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dims", type=str, default="128,64,128", help="fluid lattice (profiling runs use smaller ones)")
    ap.add_argument("--serve-scenes", type=int, default=512, help="tissue scenes of the served/batched pool (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="Poisson arrival window of the served run")
    ap.add_argument("--serve-rate", type=float, default=20000.0, help="offered frames per second")
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable-rollout measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the XPBD cube / mixed scene measurements")
    ap.add_argument("--serve-substeps", type=int, default=1)
    ap.add_argument("--serve-iterations", type=int, default=20)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def max_over_ranks(value: float, world: int, device="cuda") -> float:
    """The largest `value` over all ranks (the slowest rank's time); identity for one rank."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(particles: int, substeps: int, steps: int, world: int, seconds: float) -> float:
    """Particle-substeps/s of the whole job: every rank steps its own replica of the scene."""
    return float(particles) * substeps * steps * world / seconds


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    MEM_FIELDS = ",clocks.mem,clocks.max.mem"

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        fields = self.FIELDS
        try:  # the memory clock too, where this nvidia-smi knows the fields
            probe = subprocess.run(["nvidia-smi", f"--query-gpu={fields}{self.MEM_FIELDS}", "--format=csv,noheader,nounits"],
                                   capture_output=True, text=True, timeout=20)
            if probe.returncode == 0:
                fields += self.MEM_FIELDS
        except (FileNotFoundError, subprocess.TimeoutExpired):
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, mem, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            if self.uuid and self.uuid not in parts[0]:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            try:
                mem.append(float(parts[9]))
            except (ValueError, IndexError):
                pass
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "mem_mhz": statistics.median(mem) if mem else None, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        p = json.loads(MEASURED_PEAKS.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# Algorithmic bytes per particle of one launch of each fluid kernel (compulsory traffic; neighbour
# entries count 4 B).  Neighbour build + density: position P (16) + cell entry (16) + metadata (16)
# + kind/material (4) + boundary mask (8), list writes 4*nbar, count (4), constraint write (16).
# The first iteration of a substep also writes the superset list (4*nsup + 4 for its count);
# the later iterations read it back instead of walking the cells (4*nsup + 4).
# Delta + apply + clamp: P (16) + x (16) + accumulated delta r/w (32) + constraint (16) + list reads
# 4*nbar + count (4) + kind/material (4) + boundary mask (8) + packed delta write (16 when kept).
def kernel_bytes(name: str, nbar: float, nsup: float = 0.0) -> float | None:
    if name == "fluid_neighbors_density":
        return 80.0 + 4.0 * nbar + (4.0 * nsup + 4.0 if nsup > 0 else 0.0)
    if name == "fluid_neighbors_superset":
        return 84.0 + 4.0 * nbar + 4.0 * nsup
    if name == "fluid_delta_apply_clamp":
        return 96.0 + 4.0 * nbar
    if name == "fluid_gather":
        return 4.0 + 16.0 + 16.0 + 16.0 + 16.0
    if name == "predict_keys":
        return 16 + 16 + 16 + 16 + 16 + 16 + 4 + 4 + 4  # x r/w, v r/w, x_prev w, entry w, key w, kinds
    return None


def substep_bytes(nbar: float, iters: int) -> float:
    """The substep byte model: 232 + I * (140 + 12 nbar) bytes per particle."""
    return 232.0 + iters * (140.0 + 12.0 * nbar)


def traffic_from_profiles():
    f = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(f.read_text())
    except Exception:
        return {}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from cn_physics import Solver, scenes

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dims = tuple(int(v) for v in args.dims.split(","))
    w, desc, dt = scenes.dam_break(nx=dims[0], ny=dims[1], nz=dims[2])
    soa = w.soa()
    n = soa.particle_count
    solver = Solver(desc, device=local)
    free0 = torch.cuda.mem_get_info(local)[0]
    solver.sync_world(soa)
    # A dedicated stream: the C ABI reads a NULL stream as "the solver's own stream", and torch's
    # default stream has handle 0, so stepping on it would leave the events below unordered.
    stream = torch.cuda.Stream(device=local)
    sh = stream.cuda_stream
    assert sh != 0
    solver.step_many(dt, max(args.warmup, 0), sh)
    torch.cuda.synchronize()
    resident_gb = (free0 - torch.cuda.mem_get_info(local)[0]) / 1e9   # the solver's device state
    x0, v0, _ = solver.read_particles()  # the timed frames are replayed below for the kernel split
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    marks[0].record(stream)
    for i in range(args.steps):
        solver.step_many(dt, 1, sh)
        marks[i + 1].record(stream)
    torch.cuda.synchronize()
    start, end = marks[0], marks[-1]
    step_ms = sorted(marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps))
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(start.elapsed_time(end), world)
    substeps = desc.substeps
    value = whole_job_rate(n, substeps, args.steps, world, ms / 1e3)
    meta = solver.validate_gpu_meta()
    kernels_per_frame, _ = solver.graph_stats()
    counts, sup_counts = solver_neighbor_mean(solver)

    # Kernel split: the same frames again from the same state, with event probes around every
    # kernel group of the captured frame, read back after each frame and averaged.
    solver.write_particles(x0, v0)
    solver.set_timing(True)
    ktimes = {}
    for _ in range(args.steps):
        solver.step_many(dt, 1, sh)
        for k, (t, launches) in solver.kernel_times().items():
            acc = ktimes.setdefault(k, [0.0, 0])
            acc[0] += t / args.steps
            acc[1] += launches / args.steps
    solver.set_timing(False)
    probe_frame_ms = sum(t for t, _ in ktimes.values())

    # e2e through the C ABI: the timed frames again, from the same state, with the pinned host
    # state uploaded and read back every frame
    xh = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    vh = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    solver.write_particles(x0, v0)
    xh.numpy()[:] = x0
    vh.numpy()[:] = v0
    lib = solver._lib
    import ctypes as C
    xp = C.cast(xh.data_ptr(), C.POINTER(C.c_float))
    vp = C.cast(vh.data_ptr(), C.POINTER(C.c_float))
    e2e_steps = args.steps if args.e2e_steps <= 0 else max(1, min(args.e2e_steps, args.steps))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        # upload x, v -> frame -> read x, v back, in order on the stream, one wait per frame
        assert lib.cn_solver_step_io(solver._h, C.c_float(dt), xp, vp, xp, vp, C.c_void_p(sh)) == 0
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = whole_job_rate(n, substeps, e2e_steps, world, e2e_s)

    def pct(q):
        return round(step_ms[min(len(step_ms) - 1, int(q * len(step_ms)))], 4)

    hbm, peak_kind = peaks()
    dominant = max((k for k in ktimes if kernel_bytes(k, counts) is not None), key=lambda k: ktimes[k][0], default=None)
    roofline = None
    if dominant:
        tot_ms, launches = ktimes[dominant]
        per_launch_s = tot_ms / launches / 1e3
        algo = kernel_bytes(dominant, counts, sup_counts) * n
        achieved = algo / per_launch_s / 1e9
        tr = traffic_from_profiles().get(dominant)
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": hbm,
                    "peak_kind": f"{peak_kind} copy bandwidth", "unit": "GB/s", "frac": round(achieved / hbm, 4),
                    "traffic": tr, "algorithmic_bytes_per_launch": algo, "launch_ms": round(tot_ms / launches, 4)}
    per_kernel = {}
    for k, (tot_ms, launches) in ktimes.items():
        b = kernel_bytes(k, counts, sup_counts)
        if b is not None and tot_ms > 0:
            per_kernel[k] = {"launch_ms": round(tot_ms / launches, 4),
                             "achieved_gbs": round(b * n / (tot_ms / launches / 1e3) / 1e9, 1)}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "particle-substeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "step_latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "max": round(step_ms[-1], 4)},
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD if dims == (128, 64, 128) else f"pbf_dam_break_{dims[0]}x{dims[1]}x{dims[2]}",
                   "particles": n, "substeps": substeps, "fluid_iterations": desc.fluid_iterations,
                   "frame_dt": dt, "parallelism": f"replicas{world}", "l2": f"working set > L2 ({resident_gb:.2f} GB resident on the device)",
                   "mean_neighbors": round(counts, 2), "mean_superset": round(sup_counts, 2)},
        "e2e": {"value": round(e2e_value, 1), "unit": "particle-substeps/s", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "steps": e2e_steps},
        "gpu_launches": int(kernels_per_frame) * args.steps,
        "roofline": roofline,
        "kernel_ms_per_frame": {k: round(t, 4) for k, (t, _) in sorted(ktimes.items(), key=lambda kv: -kv[1][0])},
        "kernel_split_frame_ms": round(probe_frame_ms, 4),
        "kernel_roofline": per_kernel,
        "substep_model_bytes_per_particle": substep_bytes(counts, desc.fluid_iterations),
        "clocks": clk,
        "meta_status": meta["status"],
    }
    # the batched / served form shards its scene pool across the ranks; the differentiable form
    # and the other configurations are single-GPU workloads of their own
    if args.serve_scenes > 0:
        served = run_served(args, stream, sh, rank, world)
        if rank == 0:
            line["served"] = served
    if world == 1 and not args.no_diff:
        line["differentiation"] = run_diff(stream, cpu_sample=not args.no_cpu_baseline)
    if world == 1 and not args.no_configs:
        line["other_configs"] = run_other_configs(stream, sh, cpu=not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(budget_s=15.0)
    if world > 1:
        dist.barrier()
        solver.close()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_served(args, stream, sh, rank: int = 0, world: int = 1) -> dict:
    """The batched and served forms on a pool of soft-tissue scenes (2K-60K tets, log-uniform),
    against the plain per-scene drop-in (one cn_solver per scene) on the same pool.

    plain: one frame of every scene, scene after scene, each through its own solver;
    batched: one tick stepping every scene together (saturated);
    served: Poisson arrivals of 1-8-frame requests with drifting tool poses, replayed in real
    time through the server (admission by a device-memory budget, continuous batching).

    With several ranks the pool is sharded at scene granularity (scene k on rank k mod N, its
    requests with it; no collective on the data path): each rank runs its shard, times are the
    slowest rank's and counts add up (the pool is fixed: strong scaling).  Returns the whole-job
    figures on rank 0, None elsewhere."""
    import torch
    import torch.distributed as dist
    from cn_physics import Batch, Server, Solver, batch_desc, serving

    count = args.serve_scenes
    mine = list(range(rank, count, world))
    pool = serving.tissue_pool(count, seed=0, indices=mine)
    P = sum(sc.particles for sc in pool)
    T = sum(sc.tets for sc in pool)
    E = sum(sc.world.counts()["edges"] for sc in pool)
    desc = serving.serving_solver_desc(args.serve_substeps, args.serve_iterations)
    sub = desc.substeps
    dt = 1.0 / 60.0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    # plain per-scene drop-in
    solvers = []
    for sc in pool:
        sv = Solver(desc)
        sv.sync_world(sc.world.soa())
        solvers.append(sv)
    serving.plain_round(pool, solvers, dt, sh)  # graph capture + warm-up
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev[0].record(stream)
    serving.plain_round(pool, solvers, dt, sh)
    ev[1].record(stream)
    torch.cuda.synchronize()
    plain_ms = max_over_ranks(ev[0].elapsed_time(ev[1]), world)
    for sv in solvers:
        sv.close()
    del solvers

    # batched: every scene resident, created with colour tables so that the autotuner times the
    # gather schedule (per-phase and fused) against colour Jacobi; saturated ticks
    from cn_physics._abi import XPBD_COLOUR_JACOBI, XPBD_GATHER
    budget = 120 << 30
    bdesc = type(desc).from_buffer_copy(desc)
    bdesc.soft.xpbd_schedule = XPBD_COLOUR_JACOBI
    bd = batch_desc(bdesc, memory_budget_bytes=budget, max_scenes=len(pool) + 8, particle_capacity=P + 4096,
                    edge_capacity=E + 4096, tet_capacity=T + 4096)
    b = Batch(bd)
    ids = [b.add_scene(sc.world.soa()) for sc in pool]
    tune = b.autotune(ids, dt)

    def time_ticks(n=5):
        b.step(ids, dt, sh)
        torch.cuda.synchronize()
        out = []
        for _ in range(n):
            if world > 1:
                dist.barrier()
            ev[0].record(stream)
            b.step(ids, dt, sh)
            ev[1].record(stream)
            torch.cuda.synchronize()
            out.append(max_over_ranks(ev[0].elapsed_time(ev[1]), world))
        return out

    ticks = time_ticks()
    tick_ms = float(np.median(ticks))
    # both schedules at the tuned tile shape, per-phase kernels (the state moves on: timing only)
    by_schedule = {}
    b.set_fused(0)
    for name, sched in (("gather", XPBD_GATHER), ("colour_jacobi", XPBD_COLOUR_JACOBI)):
        b.set_xpbd_schedule(sched)
        by_schedule[name] = round(float(np.median(time_ticks(3))), 3)
    b.close()

    # served: a fresh batch (same schedule) behind the server, Poisson load in real time
    bdesc.soft.xpbd_schedule = tune["xpbd_schedule"]
    bd.solver = bdesc
    bd.tile_elements, bd.blocks_per_sm = tune["tile_elements"], tune["blocks_per_sm"]
    bd.fused_cluster_ctas = tune["cluster_ctas"]
    b = Batch(bd)
    srv = Server(b, dt)
    sids = [srv.register(sc.world.soa()) for sc in pool]
    # warm start: the even-numbered half of the pool is resident before the clock starts; the
    # other half is admitted against the budget by the server when its first request arrives
    prefetched = sum(1 for j, k in enumerate(sids) if mine[j] % 2 == 0 and srv.admit(k))
    poses = [serving.tool_start(d) for d in serving.pool_dims(count, seed=0)]
    reqs = serving.poisson_requests(poses, steps_per_second=args.serve_rate, duration_s=args.serve_seconds, seed=1)
    _, reqs = serving.shard(reqs, count, rank, world)
    if world > 1:
        dist.barrier()
    out = serving.serve(srv, pool, sids, reqs, sh)
    bstats = b.stats()
    srv.close()
    b.close()
    part = {"out": out, "P": P, "T": T, "E": E, "prefetched": prefetched, "budget_bytes": bstats["budget_bytes"],
            "budget_used_bytes": bstats["budget_used_bytes"], "tune": tune}
    cpu = served_cpu_baseline(pool, desc, dt) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    parts = [part]
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, part)
    if rank != 0:
        return None
    merged = serving.merge_served([q["out"] for q in parts])
    P = sum(q["P"] for q in parts)
    T = sum(q["T"] for q in parts)
    E = sum(q["E"] for q in parts)
    prefetched = sum(q["prefetched"] for q in parts)
    plain_rate = P * sub / (plain_ms / 1e3)
    batched_rate = P * sub / (tick_ms / 1e3)
    served_rate = merged["particle_substeps"] / merged["elapsed_s"]
    tick_p = [q["out"]["stats"] for q in parts]
    return {
        "workload": f"tissue_pool_{count}: XPBD tissue blocks, tets log-uniform 2K-60K, per-tet compliance "
                    f"log-normal (sigma 0.5), kinematic capsule tool, dt 1/60, {sub} substep x "
                    f"{desc.default_iterations} iterations",
        "scenes": count, "particles": P, "tets": T, "edges": E, "unit": "particle-substeps/s",
        "ranks": world, "sharding": "scene k on rank k mod N, no data-path collective" if world > 1 else None,
        "plain": {"value": round(plain_rate, 1), "round_ms": round(plain_ms, 3),
                  "method": "one cn_solver per scene, one frame of every scene in turn (CUDA-graph replays)"},
        "batched": {"value": round(batched_rate, 1), "tick_ms_p50": round(tick_ms, 3),
                    "tick_ms_max": round(max(ticks), 3), "schedule": {"tile_elements": tune["tile_elements"],
                                                                      "blocks_per_sm": tune["blocks_per_sm"],
                                                                      "fused_cluster_ctas": tune["cluster_ctas"],
                                                                      "xpbd_schedule": ["gather", "colour_jacobi"][
                                                                          tune["xpbd_schedule"]]},
                    "tick_ms_per_phase_by_xpbd_schedule": by_schedule,
                    "autotune_candidates": tune["candidates"]},
        "batched_over_plain": round(batched_rate / plain_rate, 2),
        "served": {"offered_frames_per_s": args.serve_rate, "arrival_window_s": args.serve_seconds,
                   "requests": merged["requests"], "frames": merged["frames"], "value": round(served_rate, 1),
                   "frames_per_s": round(merged["frames"] / merged["elapsed_s"], 1),
                   "elapsed_s": round(merged["elapsed_s"], 3),
                   "request_latency_ms": {"p50": round(merged["latency_ms_p50"], 3),
                                          "p99": round(merged["latency_ms_p99"], 3)},
                   "step_latency_ms": {"p50": round(max(x["tick_ms_p50"] for x in tick_p), 3),
                                       "p99": round(max(x["tick_ms_p99"] for x in tick_p), 3)},
                   "ticks": merged["ticks"], "prefetched_scenes": prefetched,
                   "admissions_during_run": merged["admissions"] - prefetched, "evictions": merged["evictions"],
                   "budget_bytes": sum(q["budget_bytes"] for q in parts),
                   "budget_used_bytes": sum(q["budget_used_bytes"] for q in parts)},
        "cpu_baseline": cpu,
    }


def _oracle_module():
    sys.path.insert(0, str(ROOT / "oracle"))
    import cn_oracle
    return cn_oracle, cn_oracle.set_threads(os.cpu_count() or 1)


def served_cpu_baseline(pool, desc, dt, budget_s: float = 8.0) -> dict:
    """The oracle stepping the pool's scenes one after another, one frame each (the per-scene CPU
    stepping a served pool replaces), in pool order until the time budget is spent."""
    cn_oracle, threads = _oracle_module()
    lat, particles = [], 0
    t0 = time.perf_counter()
    for sc in pool:
        o = cn_oracle.Oracle(desc, sc.world.soa())
        o.set_kinematic_target(sc.tool, tuple(float(v) for v in sc.tool_pose))
        t1 = time.perf_counter()
        o.step(dt)
        lat.append((time.perf_counter() - t1) * 1e3)
        particles += sc.particles
        if time.perf_counter() - t0 > budget_s:
            break
    el = sum(lat) / 1e3
    return {"value": round(particles * desc.substeps / el, 1), "unit": "particle-substeps/s", "cores": threads,
            "kind": "port", "frame_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                                         "p99": round(float(np.percentile(lat, 99)), 3)},
            "sample": f"one frame of each of the first {len(lat)} pool scenes ({particles} particles), {el:.1f} s"}


def run_other_configs(stream, sh, cpu: bool = True) -> dict:
    """The plain XPBD cube (16^3 vertices, 16,875 tets, 10 substeps x 20 iterations, ground), a pile
    of 4,096 dynamic rigid bodies in 4 layers with 4 proxy-particle bodies (rigid broadphase and
    contacts), and
    the mixed surgical scene (60x30x60 tissue, 256^2 cloth, 64 strands of 129, 64^3 fluid,
    kinematic capsule on a seeded path, 8 substeps), each timed over frames replayed from its CUDA
    graph; the cube also beside the oracle on the host cores (the reference's CPU-runnable case)."""
    import torch
    from cn_physics import Solver, scenes
    out = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(solver, dt, frames, tool=None):
        for k in range(3):
            if tool is not None:
                solver.set_kinematic_target(tool, scenes.tool_path(dt * (k + 1)))
            solver.step_many(dt, 1, sh)
        torch.cuda.synchronize()
        ev[0].record(stream)
        if tool is None:
            solver.step_many(dt, frames, sh)
        else:
            for k in range(frames):
                solver.set_kinematic_target(tool, scenes.tool_path(dt * (k + 4)))
                solver.step_many(dt, 1, sh)
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / frames

    w, desc, dt = scenes.xpbd_cube()
    soa = w.soa()
    sv = Solver(desc)
    sv.sync_world(soa)
    ms = timed(sv, dt, 100)
    kernels, _ = sv.graph_stats()
    n = soa.particle_count
    cube = {"workload": "xpbd_cube_16: 4,096 particles, 16,875 tets, 10 substeps x 20 iterations, dt 1/60, ground",
            "value": round(n * desc.substeps / (ms / 1e3), 1), "unit": "particle-substeps/s",
            "ms_per_frame": round(ms, 4), "kernels_per_frame": kernels,
            "us_per_kernel": round(ms * 1e3 / max(kernels, 1), 3)}
    sv.close()
    # the same cube under the other XPBD schedules (all opt-in): fused iterations (one cluster
    # kernel per substep) and the graph-coloured Jacobi / Gauss-Seidel schedules
    cube["schedules"] = {}
    for label, sched, fused in (("gather_fused", 0, 1), ("colour_jacobi", 1, 0), ("colour_jacobi_fused", 1, 1),
                                ("gauss_seidel", 2, 0), ("gauss_seidel_fused", 2, 1)):
        w2, d2, dt2 = scenes.xpbd_cube()
        d2.soft.xpbd_schedule, d2.soft.fused_iterations = sched, fused
        s2 = Solver(d2)
        s2.sync_world(w2.soa())
        ms2 = timed(s2, dt2, 20)
        cube["schedules"][label] = {"ms_per_frame": round(ms2, 4), "kernels_per_frame": s2.graph_stats()[0],
                                    "fused": s2.schedule_info()["fused_iterations"]}
        s2.close()
    if cpu:
        cn_oracle, threads = _oracle_module()
        w2, d2, dt2 = scenes.xpbd_cube()
        o = cn_oracle.Oracle(d2, w2.soa())
        t0, frames = time.perf_counter(), 0
        while frames < 50 and time.perf_counter() - t0 < 10.0:
            o.step(dt2)
            frames += 1
        el = time.perf_counter() - t0
        cube["cpu_baseline"] = {"value": round(n * d2.substeps * frames / el, 1), "unit": "particle-substeps/s",
                                "cores": threads, "kind": "port", "sample": f"{frames} frames of the same cube"}
    out["xpbd_cube"] = cube

    # dynamic rigid bodies: 4,096 spheres / capsules / boxes dropped in 4 layers of 32 x 32 plus 4
    # bodies of 27 proxy particles; timed once the pile has formed (frames 60-119)
    w, desc, dt, bodies = scenes.rigid_pile()
    soa = w.soa()
    sv = Solver(desc)
    sv.sync_world(soa)
    sv.step_many(dt, 57, sh)
    ms = timed(sv, dt, 60)
    meta = sv.validate_gpu_meta()
    c = w.counts()
    pos = sv.read_rigid_bodies()[0]
    out["rigid_pile"] = {
        "workload": f"rigid pile: {len(bodies) - 4} dynamic spheres / capsules / boxes in 4 layers + 4 bodies of "
                    f"27 proxy particles, {c['colliders']} colliders, ground box, {desc.substeps} substeps x "
                    f"{desc.default_iterations} iterations, dt 1/60",
        "value": round(c["bodies"] * desc.substeps / (ms / 1e3), 1), "unit": "body-substeps/s",
        "ms_per_frame": round(ms, 3), "kernels_per_frame": sv.graph_stats()[0],
        "rigid_rigid_pairs": meta["rigid_rigid_candidate_count"],
        "proxy_contacts": meta["proxy_rigid_contact_count"], "meta_status": meta["status"],
        "lowest_body_y": round(float(pos[1:, 1].min()), 4)}
    sv.close()

    w, desc, dt, tool = scenes.mixed_surgical()
    soa = w.soa()
    c = w.counts()
    sv = Solver(desc)
    sv.sync_world(soa)
    ms = timed(sv, dt, 10, tool)
    meta = sv.validate_gpu_meta()
    n = soa.particle_count
    # surface render passes (skinning, normals, bounds) of the frame, from the event probes
    sv.set_timing(True)
    surf_ms = 0.0
    for k in range(3):
        sv.set_kinematic_target(tool, scenes.tool_path(dt * (k + 20)))
        sv.step_many(dt, 1, sh)
        surf_ms += sv.kernel_times().get("surface_render", (0.0, 0))[0] / 3
    sv.set_timing(False)
    sr = soa.surface_render.contents
    V, T, I = sr.vertex_count, sr.triangle_count, sr.vertex_triangle_index_count
    surf_particles = sum(int(sr.surface_particle_ranges[2 * k + 1]) for k in range(sr.surface_count))
    chunks = sum((int(sr.surface_particle_ranges[2 * k + 1]) + 63) // 64 for k in range(sr.surface_count))
    # binding 32 + 4 gathered positions + output per vertex; 3 gathered positions + indices + output
    # per triangle; range + incident index and face normal + output per vertex; positions + chunk
    # and surface AABBs for the bounds
    surf_bytes = V * 112 + T * 80 + V * 32 + I * 20 + surf_particles * 16 + chunks * 64 + sr.surface_count * 32
    out["mixed_surgical"] = {
        "workload": f"mixed: {c['tets']} tets, {c['dihedrals']} dihedrals, {c['segments']} "
                    f"strand segments, {n} particles in all (tissue, cloth, strands, 64^3 fluid), kinematic capsule, "
                    f"{desc.substeps} substeps x {desc.default_iterations} iterations, dt 1/60",
        "value": round(n * desc.substeps / (ms / 1e3), 1), "unit": "particle-substeps/s",
        "ms_per_frame": round(ms, 3), "meta_status": meta["status"],
        "surface_render": {"render_vertices": V, "render_triangles": T, "surfaces": sr.surface_count,
                           "ms_per_frame": round(surf_ms, 4), "algorithmic_bytes": surf_bytes,
                           "achieved_gbs": round(surf_bytes / max(surf_ms, 1e-6) / 1e6, 1)}}
    sv.close()
    if cpu:
        # the oracle on the same scene for one frame of 2 substeps at the substep dt of the
        # 8-substep frame: the work per particle-substep is that of the full frame
        cn_oracle, threads = _oracle_module()
        w2, d2, dt2, tool2 = scenes.mixed_surgical()
        sub = d2.substeps
        d2.substeps = 2
        o = cn_oracle.Oracle(d2, w2.soa())
        o.set_kinematic_target(tool2, scenes.tool_path(dt2))
        t0 = time.perf_counter()
        o.step(dt2 * 2 / sub)
        el = time.perf_counter() - t0
        out["mixed_surgical"]["cpu_baseline"] = {
            "value": round(n * 2 / el, 1), "unit": "particle-substeps/s", "cores": threads, "kind": "port",
            "sample": f"one frame of 2 substeps (substep dt 1/{int(round(sub / dt2))}) of the same scene, {el:.1f} s"}
    return out


def _diff_block(dims, spacing=0.1, base=1e-11, seed=0):
    """Pinned soft block whose per-tet compliances (log-normal, sigma 0.5) carry its stiffness."""
    from cn_physics import World
    rx, ry, rz = dims
    w = World()
    size = ((rx - 1.25) * spacing, (ry - 1.25) * spacing, (rz - 1.25) * spacing)
    pinned = [x * ry * rz + z for x in range(rx) for z in range(rz)]
    w.add_soft_body_grid(size, spacing, position=(0.0, size[1] * 0.5, 0.0), radius=0.4 * spacing,
                         edge_compliance=1e-4, volume_compliance=base, static_particles=pinned)
    w.soa()
    comp = w.array("tets").view(np.float32)[:, 5]
    comp[:] = (base * np.random.default_rng(seed).lognormal(0.0, 0.5, comp.shape[0])).astype(np.float32)
    return w


def run_diff(stream, cpu_sample: bool = True) -> dict:
    """Differentiation: a 28x14x28-vertex block (47,385 tets), 32 substeps x 20 iterations,
    surface-vertex MSE against a target rolled out with log-normal (sigma 0.3) per-tet stiffness;
    gradient with respect to per-tet compliance and initial velocities, checkpoint every 8
    substeps.  The adjoint is checked against FP64 central differences (eps 1e-6) on a
    9x8x8-vertex (1,960-tet) instance."""
    import torch
    from cn_physics import diff

    def inputs(w, dtype):
        x0 = torch.as_tensor(w.positions().copy(), device="cuda", dtype=dtype)
        comp = torch.as_tensor(w.array("tets").view(np.float32)[:, 5].copy(), device="cuda", dtype=dtype)
        v = np.zeros((x0.shape[0], 4))
        v[:, :3] = np.random.default_rng(1).normal(0.0, 0.05, (x0.shape[0], 3))
        v0 = torch.as_tensor(v, device="cuda", dtype=dtype)
        v0[x0[:, 3] <= 0] = 0
        return comp, x0, v0

    def loss_grad(r, comp, x0, v0, target, surf):
        out = torch.empty_like(x0)
        r.forward(comp, x0, v0, out)
        d = out[surf, :3] - target[surf, :3]
        g = torch.zeros_like(out)
        g[surf, :3] = 2.0 * d / d.numel()
        gc, gv = torch.zeros_like(comp), torch.zeros_like(v0)
        r.backward(g, None, gc, None, gv)
        return float((d * d).mean()), gc, gv

    dims = (28, 14, 28)
    w = _diff_block(dims)
    surf = torch.as_tensor(diff.lattice_surface(dims), device="cuda")
    kw = dict(substeps=32, iterations=20, substep_dt=1.0 / 480.0, checkpoint_interval=8)
    r = diff.Rollout(w, **kw)
    comp, x0, v0 = inputs(w, torch.float32)
    true = comp * torch.as_tensor(np.random.default_rng(2).lognormal(0.0, 0.3, comp.shape[0]), device="cuda",
                                  dtype=torch.float32)
    target = torch.empty_like(x0)
    r.forward(true, x0, v0, target)
    loss_grad(r, comp, x0, v0, target, surf)  # warm-up
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    out = torch.empty_like(x0)
    g = torch.zeros_like(x0)
    g[surf, :3] = 1e-3
    gc, gv = torch.zeros_like(comp), torch.zeros_like(v0)
    ev[0].record(stream)
    r.forward(comp, x0, v0, out)
    ev[1].record(stream)
    r.backward(g, None, gc, None, gv)
    ev[2].record(stream)
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    kept = r.memory_bytes()
    n, t = w.counts()["particles"], w.counts()["tets"]
    e = w.counts()["edges"]
    tape = 32 * 20 * (2 * n * 16 + (e + t) * 4) + 32 * 2 * n * 16   # every iteration state of every substep
    r.close()

    # FD check on the small instance in FP64
    sd = (9, 8, 8)
    ws = _diff_block(sd)
    ssurf = torch.as_tensor(diff.lattice_surface(sd), device="cuda")
    kws = dict(substeps=32, iterations=10, substep_dt=1.0 / 480.0, checkpoint_interval=8)
    r64 = diff.Rollout(ws, precision=8, **kws)
    c64, x64, v64 = inputs(ws, torch.float64)
    rng = np.random.default_rng(7)
    t64 = torch.empty_like(x64)
    r64.forward(c64 * torch.as_tensor(rng.lognormal(0.0, 0.3, c64.shape[0]), device="cuda"), x64, v64, t64)
    _, g64, _ = loss_grad(r64, c64, x64, v64, t64, ssurf)
    u = torch.as_tensor(rng.normal(0.0, 1.0, c64.shape[0]), device="cuda") * c64
    eps = 1e-6

    def L(c):
        o = torch.empty_like(x64)
        r64.forward(c, x64, v64, o)
        d = o[ssurf, :3] - t64[ssurf, :3]
        return float((d * d).mean())
    fd = (L(c64 + eps * u) - L(c64 - eps * u)) / (2 * eps)
    an = float((g64 * u).sum())
    r64.close()

    # CPU: the oracle's float32 XPBD substep on the same block, 4 of the 32 substeps; a
    # central-difference gradient with respect to every compliance costs 2 T rollouts
    cpu = None
    if cpu_sample:
        from cn_physics import solver_desc
        cn_oracle, threads = _oracle_module()
        o = cn_oracle.Oracle(solver_desc(substeps=4, default_iterations=20, soft_internal_relaxation=0.2), w.soa())
        t0 = time.perf_counter()
        o.step(4.0 / 480.0)
        sub_s = (time.perf_counter() - t0) / 4
        cpu = {"value": round(n / sub_s, 1), "unit": "particle-substeps/s", "cores": threads, "kind": "port",
               "rollout_s": round(sub_s * 32, 3), "fd_gradient_s": round(sub_s * 32 * 2 * t, 1),
               "sample": "4 substeps x 20 iterations of the same block (float32); rollout = 32 substeps, "
                         f"fd_gradient = 2 x {t} rollouts"}
    return {"workload": f"XPBD block {dims[0]}x{dims[1]}x{dims[2]} vertices ({t} tets, {n} particles), 32 substeps x "
                        f"20 iterations, checkpoint every 8 substeps, surface MSE vs a log-normal (sigma 0.3) "
                        f"stiffness target; gradients w.r.t. per-tet compliance and initial velocities",
            "forward_ms": round(fwd_ms, 3), "backward_ms": round(bwd_ms, 3),
            "particle_substeps_per_s_forward": round(n * 32 / (fwd_ms / 1e3), 1),
            "adjoint_state_bytes": kept, "full_tape_bytes": tape,
            "fd_check": {"instance": "9x8x8 vertices (1,960 tets), FP64, eps 1e-6, random log-space direction",
                         "adjoint": an, "central_difference": fd, "relative_error": abs(an - fd) / abs(fd)},
            "cpu_baseline": cpu}


def solver_neighbor_mean(solver) -> tuple:
    c = solver.debug_read("fluid_neighbor_counts").view(np.uint32)
    sc = solver.debug_read("fluid_superset_counts").view(np.uint32)
    return (float(c.mean()) if c.size else 0.0), (float(sc.mean()) if sc.size else 0.0)


def cpu_baseline(budget_s: float = 15.0, dims=(64, 32, 64), max_frames: int = 8):
    """The oracle (CPU restatement, all host threads) on a lattice sample of the same scene."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import cn_oracle
    from cn_physics import scenes

    threads = cn_oracle.set_threads(os.cpu_count() or 1)
    w, desc, dt = scenes.dam_break(nx=dims[0], ny=dims[1], nz=dims[2])
    soa = w.soa()
    ora = cn_oracle.Oracle(desc, soa)
    frames, t0 = 0, time.perf_counter()
    while frames < max_frames and (time.perf_counter() - t0) < budget_s:
        ora.step(dt)
        frames += 1
    el = time.perf_counter() - t0
    v = soa.particle_count * desc.substeps * frames / el
    return {"value": round(v, 1), "unit": "particle-substeps/s", "cores": threads, "kind": "port",
            "sample": f"{dims[0]}x{dims[1]}x{dims[2]} lattice ({soa.particle_count} particles) of the same dam break, "
                      f"{frames} frames x {desc.substeps} substeps, {el:.1f} s"}


def run_reference(args, dims=(128, 64, 128)):
    """The reference's CPU implementation of the path on this workload: the oracle (the C++
    restatement of the reference's substep, pinned bit for bit to the reference's own shaders run
    on the host) on the full 128 x 64 x 128 dam break, every host thread.  The scene is built by
    oracle/cn_scenes.py, so this arm loads no product library."""
    rank, local, world = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import cn_oracle
    import cn_scenes

    threads = cn_oracle.set_threads(os.cpu_count() or 1)
    scene = cn_scenes.DamBreak(*dims)
    soa, desc, dt = scene.soa(), scene.desc, scene.frame_dt
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(max(args.warmup, 0)):
        ora.step(dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ora.step(dt)
    el = time.perf_counter() - t0
    n = soa.particle_count
    value = n * desc.substeps * args.steps / el
    sample = (f"the full workload: {n} particles, {args.steps} frames x {desc.substeps} substeps after "
              f"{args.warmup} warm-up frames, {el:.1f} s; the oracle (C++ restatement of the reference's "
              "HLSL passes, bit-identical to them with the shaders' quotients) on the host cores, as the "
              "reference's own Vulkan path cannot run here")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "particle-substeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if tuple(dims) == (128, 64, 128) else
                       f"pbf_dam_break_{dims[0]}x{dims[1]}x{dims[2]}", "particles": n, "substeps": desc.substeps,
                       "fluid_iterations": desc.fluid_iterations, "frame_dt": dt, "parallelism": "host threads"},
            "cpu_baseline": {"value": round(value, 1), "unit": "particle-substeps/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 1), "unit": "particle-substeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
