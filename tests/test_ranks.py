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


def test_placement_by_footprint():
    rng = np.random.default_rng(5)
    fp = rng.integers(1, 1000, 40)
    work = rng.uniform(1.0, 10.0, 40)
    parts = ranks.place(fp, work, 3, budget=8000)
    assert sorted(i for p in parts for i in p) == list(range(40))
    assert all(sum(fp[i] for i in p) <= 8000 for p in parts)
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= work.max()
    assert parts == ranks.place(fp, work, 3, budget=8000)     # the same on every rank
    assert [len(p) for p in ranks.place(fp, work, 4, max_items=10)] == [10, 10, 10, 10]
    with pytest.raises(ValueError):
        ranks.place([10, 10], [1, 1], 1, budget=15)


class OracleServer:
    """Stands in for the GPU server on CPU: each job's MC steps by the oracle
    on the job's own random stream (seed, job id), as the engine keys it."""

    def run(self, jobs, realtime=True):
        from oracle import oracle as O
        for j in jobs:
            o = O.Oracle.from_system(j.system, maxmol=j.maxmol)
            o.set_molecules(np.zeros((0, j.system.molecule.n_atoms, 3)))
            st = O.MCState()
            o.mc_run(O.mc_params(j.system, j.seed, j.id), st, 0, j.steps)
            j.result = {"nmol": o.nmol, "u": list(st.u), "attempts": list(st.attempts), "accepted": list(st.accepted),
                        "xyz": o.molecules().tolist()}
        return {"jobs": len(jobs)}


def _jobs():
    from raspa2_b200 import serve
    base = [systems.tiny_co2_system(seed=7), systems.tiny_co2_system(seed=8, n_atoms=64, cell=24.0),
            systems.methane_like_system(seed=3, n_atoms=96)]
    import dataclasses
    out = []
    for i in range(6):
        s = dataclasses.replace(base[i % 3], pressure=1e5 * (i + 1), name=f"job{i}")
        out.append(serve.Job(id=i, system=s, steps=150, seed=100 + i, maxmol=32))
    return out


def _serve_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from raspa2_b200 import serve
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    mine, stats, allres = serve.serve_placed(_jobs(), rank, world, make_server=OracleServer, realtime=False)
    out.put((rank, mine, allres))
    dist.barrier()
    dist.destroy_process_group()


def test_jobs_placed_on_two_gloo_ranks_give_the_results_of_single_runs():
    """One job list served over two ranks (placement by footprint, one
    server per rank, results gathered on rank 0): every job runs on exactly
    one rank and its result equals the job run alone."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, mine0, all0), (_, mine1, all1) = res
    assert all1 is None and sorted(mine0 + mine1) == list(range(6)) and mine0 and mine1
    alone = _jobs()
    OracleServer().run(alone)
    for j in alone:
        assert all0[j.id] == j.result, j.id
