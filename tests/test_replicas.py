"""The multi-GPU path is replicas: independent columns per rank and a maximum
of the timings over ranks.  Exercised here with 2 gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from ibis_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(size),
                      LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    from ibis_b200 import synth
    W = replicas.world_from_env()
    replicas.init(W, "gloo", timeout_s=60)
    # each replica builds its own columns from its own seed
    wl = synth.make_workload(64, 2, seed=replicas.replica_seed(1000, W.rank))
    mine = torch.tensor([float(wl.stat["sand"].sum())], dtype=torch.float64)
    both = [torch.zeros(1, dtype=torch.float64) for _ in range(size)]
    dist.all_gather(both, mine)
    replicas.barrier(W)
    m = replicas.max_over_ranks(W, [1.0 + W.rank, 10.0 - W.rank, 3.5])
    out[rank] = (m, [float(b) for b in both])
    replicas.finish(W)


def test_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == [2.0, 10.0, 3.5]
    sums = res[0][1]
    assert sums == res[1][1] and sums[0] != sums[1]          # different columns on each rank


def test_single_process_world():
    W = replicas.World(0, 1, 0)
    assert not W.multi
    assert replicas.max_over_ranks(W, [1, 2]) == [1.0, 2.0]
    assert replicas.replica_seed(1000, 3) == 1003
