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
