"""The multi-GPU path is replicas: each rank denoises its own clip with no data-path collective,
and the job's throughput is the frames of all ranks over the max-over-ranks time. This runs that
path with two `gloo` ranks on the CPU: each rank denoises its own seeded clip with the oracle (the
GPU engine is the same code per rank), and bench.py's aggregation reduces the timings."""

import os
import sys
import time
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench
    import oracle

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(bench.replica_seed(rank))
        frames = [np.clip(0.5 + rng.normal(0, 0.04, (24, 32, 1)), 0, 1).astype(np.float32) for _ in range(3)]
        t0 = time.perf_counter()
        outs = oracle.nlm_stream_repeat(frames, 1, 2, 1, oracle.h2_inv_norm(6.0, 1))
        local = time.perf_counter() - t0
        dist.barrier()
        times, values = bench.replica_throughput([local, 2 * local], len(frames), world, device="cpu")
        out.put((rank, local, times, values, float(np.asarray(outs).sum())))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_timings_to_the_max():
    world, port = 2, 29000 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    locals_ = [r[1] for r in results]
    for rank, local, times, values, checksum in results:
        assert times[0] == max(locals_) and times[1] == 2 * max(locals_)
        assert values[0] == 3 * world / times[0]
    # Independent units: each rank denoised a different clip.
    assert results[0][4] != results[1][4]
