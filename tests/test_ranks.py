"""The multi-GPU plumbing of the measurement, on CPU: two gloo ranks take
disjoint, reproducible batches of systems and combine their timings as
max-over-ranks and their move counts as a sum (what bench.py does under
torchrun with NCCL). No collective is on the data path."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from raspa2_b200 import ranks, systems


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    w, r, _ = ranks.rank_env()
    batch = systems.batched_co2_systems(3, seed=ranks.batch_seed(2, r))
    t, n = ranks.reduce_time_and_count(1.0 + r, 10.0 * (r + 1))
    out.put((r, w, t, n, [s.name for s in batch], [float(s.frac.sum()) for s in batch]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, t0, n0, names0, f0), (r1, w1, t1, n1, names1, f1) = res
    assert (w0, w1) == (2, 2)
    assert t0 == t1 == 2.0          # max of 1.0 and 2.0
    assert n0 == n1 == 30.0         # 10 + 20
    assert f0 != f1                 # each rank its own frameworks
    # a rank's batch is reproducible
    again = systems.batched_co2_systems(3, seed=ranks.batch_seed(2, 1))
    np.testing.assert_allclose([float(s.frac.sum()) for s in again], f1)


def test_single_process_reduction_is_identity():
    assert ranks.reduce_time_and_count(1.5, 7.0) == (1.5, 7.0)
