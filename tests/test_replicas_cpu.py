"""The multi-GPU path is replicas only (every rank renders its own frames, no
data exchange): bench.py's barrier, max-over-ranks timing and per-rank frame
numbering, run as two gloo ranks on the CPU, the second test with each rank
rendering its frames (through the CPU oracle, as no GPU is present)."""
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


def _render_rank(rank: int, world: int, port: int, q) -> None:
    """One replica: renders its own frames of a small scene (the CPU oracle
    stands in for the GPU pass here), times them and reports the slowest
    rank's time the way bench.py does."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import time

    import numpy as np
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    from oracle import oracle as orc
    from tests.helpers import oracle_image
    from tfg_b200 import bvh as hbvh
    from tfg_b200 import scenes
    scene = scenes.box_icosphere(32, 24, subdiv=2)
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    steps = 2
    bench.barrier(world)
    t0 = time.perf_counter()
    imgs = [oracle_image(orc, scene, hb, bench.replica_frame(rank, s, steps), nthreads=2) for s in range(steps)]
    ms = (time.perf_counter() - t0) * 1e3
    ms_max = bench.max_over_ranks(ms, world)
    q.put((rank, ms, ms_max, [bench.replica_frame(rank, s, steps) for s in range(steps)], np.stack(imgs)))
    dist.destroy_process_group()


def test_two_gloo_replicas_render_their_own_frames():
    import numpy as np

    from oracle import oracle as orc
    from tests.helpers import oracle_image
    from tfg_b200 import bvh as hbvh
    from tfg_b200 import scenes
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_render_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=180) for _ in range(2)), key=lambda x: x[0])
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    (_, ms0, max0, frames0, img0), (_, ms1, max1, frames1, img1) = got
    assert max0 == max1 == max(ms0, ms1)               # both ranks report the slowest replica
    assert not set(frames0) & set(frames1)             # distinct frames, distinct work
    assert frames0[0] == 1                              # rank 0 renders the single-GPU run's frames
    assert not np.array_equal(img0, img1)
    scene = scenes.box_icosphere(32, 24, subdiv=2)
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    for frames, imgs in ((frames0, img0), (frames1, img1)):
        for f, im in zip(frames, imgs):
            np.testing.assert_array_equal(im, oracle_image(orc, scene, hb, f, nthreads=2))
