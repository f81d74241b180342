"""The N>1 bench path on CPU: two gloo ranks, barrier + max-over-ranks timing (replicas only,
no collective on the data path)."""
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


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    dist.barrier()
    ms = 10.0 + 5.0 * rank
    out[rank] = bench.max_over_ranks(ms, world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo_two_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1] == 15.0
