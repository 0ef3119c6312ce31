"""The multi-GPU host path on CPUs: two gloo ranks split a molecule list with
replicas.shard, run their molecules' SCFs with the CPU oracle, and combine
the job's time as the max over ranks and its molecule count as the sum -- the
arithmetic bench.py applies to device timings under torchrun."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mopac_gpu_b200.replicas import shard


def test_shard_is_disjoint_complete_and_balanced():
    rng = np.random.default_rng(0)
    costs = rng.integers(20, 123, size=101) ** 3
    parts = [shard(costs, r, 4) for r in range(4)]
    allidx = sorted(i for p in parts for i in p)
    assert allidx == list(range(101))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) / min(loads) < 1.1
    assert shard(costs, 0, 1) == list(range(101))
    with pytest.raises(ValueError):
        shard(costs, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import time
    import torch.distributed as dist
    from mopac_gpu_b200 import workloads
    from mopac_gpu_b200.replicas import max_over_ranks, shard, sum_over_ranks
    from oracle import scf_oracle as so
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mols = workloads.alkane_batch(6, seed=5, nmin=3, nmax=5)
    costs = [len(m[0]) ** 3 for m in mols]
    mine = shard(costs, rank, world)
    t0 = time.perf_counter()
    heats = {i: so.iter_scf(so.make_system(*mols[i])).escf for i in mine}
    dt = time.perf_counter() - t0
    tmax = max_over_ranks(dt, dist)
    n = sum_over_ranks(len(mine), dist)
    out.put((rank, sorted(heats.items()), dt, tmax, n))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_split_the_batch_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    idx = sorted(i for r in res for i, _ in r[1])
    assert idx == list(range(6))                     # every molecule ran once
    assert res[0][4] == res[1][4] == 6               # summed count
    tmax = max(r[2] for r in res)
    assert res[0][3] == res[1][3] == pytest.approx(tmax)   # both ranks see the max
