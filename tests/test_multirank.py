"""Host logic of the multi-rank bench on CPU: two gloo ranks on 127.0.0.1.

The single-scene substep does not shard (replicas only): every rank steps its own copy, the
timing is the slowest rank's, and the whole-job rate counts every rank's particles.  The
reference arm runs on rank 0 only.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    slowest = bench.max_over_ranks(10.0 + rank, world, device="cpu")
    rate = bench.whole_job_rate(1000, 2, 5, world, slowest)
    # the reference arm: rank 0 alone does work and prints; the others return at once
    class Args:
        steps, warmup = 1, 0
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(Args, dims=(6, 4, 6))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, slowest, rate, buf.getvalue()))


def test_two_gloo_ranks_take_the_slowest_time_and_sum_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, v0, o0), (r1, s1, v1, o1) = res
    assert s0 == s1 == 11.0                        # max over ranks
    assert v0 == v1 == pytest.approx(1000 * 2 * 5 * 2 / 11.0)
    assert '"impl": "reference"' in o0 and o1 == ""


def _served_rank_main(rank, world, port, out):
    """A rank of the sharded served form: its scenes and requests, then the whole-job merge."""
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT / "cressim-neo_b200"))
    from cn_physics import serving
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    count = 12
    poses = [serving.tool_start(d) for d in serving.pool_dims(count, seed=0)]
    reqs = serving.poisson_requests(poses, steps_per_second=2000.0, duration_s=0.5, seed=1)
    mine, local = serving.shard(reqs, count, rank, world)
    # a stand-in for serve(): every request completes after (rank + 1) ms per frame
    lat = [float((rank + 1) * r.steps) for r in local]
    part = {"elapsed_s": 0.5 + rank, "requests": len(local), "latencies_ms": lat,
            "stats": {"scene_steps": sum(r.steps for r in local), "particle_substeps": 100 * len(local),
                      "ticks": len(local), "admissions": len(mine), "evictions": 0}}
    parts = [None] * world
    dist.all_gather_object(parts, part)
    merged = serving.merge_served(parts) if rank == 0 else None
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, mine, [(r.scene, r.steps) for r in local], len(reqs), sum(r.steps for r in reqs), merged))


def test_sharded_serving_partitions_scenes_and_merges_whole_job_figures():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_served_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=240) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, mine0, loc0, n, frames, merged), (_, mine1, loc1, _, _, _) = res
    assert sorted(mine0 + mine1) == list(range(12)) and not set(mine0) & set(mine1)   # each scene once
    assert len(loc0) + len(loc1) == n                                                    # every request once
    assert all(0 <= s < len(mine0) for s, _ in loc0) and all(0 <= s < len(mine1) for s, _ in loc1)
    assert merged["requests"] == n and merged["frames"] == frames
    assert merged["elapsed_s"] == 1.5                                                    # slowest rank
    assert merged["particle_substeps"] == 100 * n
