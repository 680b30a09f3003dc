"""Multi-rank replica logic on CPU with the gloo backend (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from pennsylvaniagpugraphclustering_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = replicas.max_over_ranks([10.0 + rank, 5.0 - rank])
        best = replicas.best_trial(0.5 + 0.1 * rank)
        out[rank] = (times, best, replicas.replica_seed(7, rank))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        times, best, seed = out[r]
        assert times == [11.0, 5.0]
        assert best[0] == 1 and abs(best[1] - 0.6) < 1e-12
        assert seed == 7 + r


def test_single_process_identity():
    from pennsylvaniagpugraphclustering_b200 import replicas
    assert replicas.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]
    assert replicas.best_trial(0.3) == (0, 0.3)
