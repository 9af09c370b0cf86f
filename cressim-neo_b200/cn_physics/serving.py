"""Seeded soft-tissue scene pools and Poisson request streams for the batched / served forms.

A pool scene is one XPBD tissue block (regular-grid 5-tet split, bottom face pinned, per-tet
volume compliance log-normal around 1e-6), a ground plane and a kinematic capsule tool hovering
over the block.  Requests ask for 1-8 frames of one scene and carry the tool's target pose for
each frame: a seeded random walk from the scene's last tool pose.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch, Server, Solver, World, scenes, solver_desc

SPACING = 0.01          # 1 cm lattice
TOOL_RADIUS = 0.01
TOOL_HALF_HEIGHT = 0.05


def serving_solver_desc(substeps: int = 8, iterations: int = 10):
    """Settings shared by every pool scene (dt = 1/60 s frames)."""
    return solver_desc(substeps=substeps, default_iterations=iterations, enable_blocking_readback=0)


@dataclass
class TissueScene:
    world: World
    tool: int                    # rigid-body index of the tool in the scene
    cells: tuple
    tets: int
    particles: int
    tool_pose: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))


def tool_start(cells) -> np.ndarray:
    """Initial tool pose of a pool scene: resting just above the lattice top."""
    cy = max(int(cells[1]), 1)
    top = (cy - 0.25) * SPACING + 0.002
    return np.array([0.0, top + TOOL_RADIUS + 0.004, 0.0], np.float32)


def tissue_scene(cells=(10, 6, 10), seed: int = 0, compliance_sigma: float = 0.5) -> TissueScene:
    cx, cy, cz = (max(int(c), 1) for c in cells)
    rng = np.random.default_rng(seed)
    w = World()
    # extents a quarter cell short of whole cells, so ceil(extent / spacing) = cells exactly
    size = ((cx - 0.25) * SPACING, (cy - 0.25) * SPACING, (cz - 0.25) * SPACING)
    rx, ry, rz = cx + 1, cy + 1, cz + 1
    pinned = [x * ry * rz + z for x in range(rx) for z in range(rz)]  # y = 0 layer
    w.add_soft_body_grid(size, SPACING, position=(0.0, size[1] * 0.5 + 0.002, 0.0), radius=0.4 * SPACING,
                         edge_compliance=1e-5, volume_compliance=1e-6, static_particles=pinned, friction=0.3)
    scenes.ground(w)
    tool_pos = tool_start((cx, cy, cz))
    tool = w.add_rigid_body("kinematic", position=tuple(float(v) for v in tool_pos))
    w.add_collider(tool, "capsule", (TOOL_RADIUS, TOOL_HALF_HEIGHT), local_orientation=(0.0, 0.0, 0.7071068, 0.7071068),
                   friction=0.2)
    w.soa()
    tets = w.array("tets")
    comp = tets.view(np.float32)[:, 5]
    comp[:] = (1e-6 * rng.lognormal(0.0, compliance_sigma, size=comp.shape[0])).astype(np.float32)
    x = w.positions()
    x[:, :3] += rng.uniform(-1e-5, 1e-5, size=(x.shape[0], 3)).astype(np.float32) * (x[:, 3:4] > 0)
    c = w.counts()
    return TissueScene(w, tool, (cx, cy, cz), c["tets"], c["particles"], tool_pos)


def pool_dims(count: int = 512, seed: int = 0, tet_range=(2000, 60000)) -> list:
    """Seeded lattice dims of the pool's scenes (tet counts log-uniform in `tet_range`)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        target = math.exp(rng.uniform(math.log(tet_range[0]), math.log(tet_range[1])))
        cells = target / 5.0
        a = rng.uniform(0.7, 1.4, size=3)
        a = a / np.cbrt(np.prod(a))
        side = np.cbrt(cells)
        out.append(tuple(max(2, int(round(side * r))) for r in a))
    return out


def tissue_pool(count: int = 512, seed: int = 0, tet_range=(2000, 60000), indices=None) -> list:
    """`count` scenes with tet counts log-uniform in `tet_range`, built from seeded lattice dims;
    with `indices`, only those scenes of the pool (a rank's shard), each as the whole pool has it."""
    dims = pool_dims(count, seed, tet_range)
    ks = range(count) if indices is None else indices
    return [tissue_scene(dims[k], seed=seed * 100003 + k) for k in ks]


def shard(requests: list, count: int, rank: int, world: int):
    """Scene-granular partition of a pool of `count` scenes: scene k is served by rank k mod world.
    Returns the rank's global scene indices and its requests, re-indexed into its shard (arrival
    times unchanged)."""
    mine = list(range(rank, count, world))
    local = {g: i for i, g in enumerate(mine)}
    return mine, [Request(r.arrival, local[r.scene], r.steps, r.targets) for r in requests if r.scene in local]


def merge_served(parts: list) -> dict:
    """Whole-job figures of a sharded run from every rank's serve() result: frames and
    particle-substeps add up, the wall time is the slowest rank's, latency percentiles are taken
    over every request."""
    lat = np.concatenate([np.asarray(p["latencies_ms"], np.float64) for p in parts]) if parts else np.zeros(0)
    st = [p["stats"] for p in parts]
    return {"elapsed_s": max(p["elapsed_s"] for p in parts), "requests": sum(p["requests"] for p in parts),
            "frames": sum(x["scene_steps"] for x in st), "particle_substeps": sum(x["particle_substeps"] for x in st),
            "ticks": sum(x["ticks"] for x in st), "admissions": sum(x["admissions"] for x in st),
            "evictions": sum(x["evictions"] for x in st),
            "latency_ms_p50": float(np.percentile(lat, 50)) if lat.size else None,
            "latency_ms_p99": float(np.percentile(lat, 99)) if lat.size else None}


@dataclass
class Request:
    arrival: float
    scene: int
    steps: int
    targets: np.ndarray          # steps x 7: position xyz, orientation xyzw


def poisson_requests(pool: list, steps_per_second: float = 20000.0, duration_s: float = 1.0, seed: int = 0,
                     drift: float = 0.001) -> list:
    """Poisson arrivals carrying `steps_per_second` frames per second in total (1-8 frames each).
    `pool`: the scenes, or their initial tool poses."""
    rng = np.random.default_rng(seed)
    rate = steps_per_second / 4.5
    t, out = 0.0, []
    poses = [np.array(sc.tool_pose if hasattr(sc, "tool_pose") else sc, np.float32) for sc in pool]
    quat = np.array([0.0, 0.0, 0.7071068, 0.7071068], np.float32)
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            return out
        s = int(rng.integers(len(pool)))
        k = int(rng.integers(1, 9))
        tg = np.zeros((k, 7), np.float32)
        for j in range(k):
            poses[s] = poses[s] + rng.normal(0.0, drift, 3).astype(np.float32)
            poses[s][1] = min(max(poses[s][1], 0.0), 0.3)
            tg[j, :3] = poses[s]
            tg[j, 3:] = quat
        out.append(Request(t, s, k, tg))


def serve(server: Server, pool: list, pool_ids: list, requests: list, stream: int = 0) -> dict:
    """Replays `requests` in real time: each is submitted once its arrival time has passed on the
    wall clock, and the server ticks while any work is pending."""
    t0 = time.perf_counter()
    nxt = 0
    while nxt < len(requests) or server.stats()["pending"]:
        now = time.perf_counter() - t0
        while nxt < len(requests) and requests[nxt].arrival <= now:
            r = requests[nxt]
            server.submit(pool_ids[r.scene], r.steps, tool_body=pool[r.scene].tool, targets=r.targets)
            nxt += 1
        if server.tick(stream) == 0 and nxt < len(requests):
            time.sleep(max(0.0, min(requests[nxt].arrival - (time.perf_counter() - t0), 0.001)))
    server.drain(stream)
    elapsed = time.perf_counter() - t0
    done = server.poll()
    lat = np.array([d["done_s"] - d["submit_s"] for d in done]) * 1e3
    st = server.stats()
    return {"elapsed_s": elapsed, "requests": len(done), "stats": st, "latencies_ms": lat.tolist(),
            "latency_ms_p50": float(np.percentile(lat, 50)) if lat.size else None,
            "latency_ms_p99": float(np.percentile(lat, 99)) if lat.size else None}


def plain_round(pool: list, solvers: list, dt: float, stream: int = 0) -> None:
    """One frame of every scene through its own cn_solver (the plain per-scene drop-in)."""
    for sc, sv in zip(pool, solvers):
        sv.step_many(dt, 1, stream)
