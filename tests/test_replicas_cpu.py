"""The multi-GPU path is replicas only (every rank renders its own frames, no
data exchange): bench.py's barrier and max-over-ranks timing, run as two
gloo ranks on the CPU."""
import os
import socket
from datetime import timedelta

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    bench.barrier(world)
    ms = bench.max_over_ranks(100.0 + 25.0 * rank, world)      # rank 1 is the slow replica
    q.put((rank, ms, bench.replicas_value(1_000_000, ms, world)))
    dist.destroy_process_group()


def test_two_gloo_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 125.0
        # 2 replicas x 1M paths in 125 ms
        assert abs(value - 2 * 1_000_000 / 0.125 / 1e6) < 1e-9
