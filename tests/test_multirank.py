# -*- coding: utf-8 -*-
"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the timing
reduction takes the max over ranks, every rank takes the same collective
steps, and the reference arm runs on rank 0 only. Signals are sharded by
rank (weak scaling) with no collective on the data path, so the reduction
is the only cross-rank traffic."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # per-rank step times: the reported time is the slowest rank's
        a, b = bench.max_over_ranks([1.0 + rank, 10.0 - rank], torch.device('cpu'))
        dist.barrier()
        out[rank] = (a, b)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_two_gloo_ranks():
    world = 2
    mgr = mp.get_context('spawn').Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                       start_method='spawn', join=True)
    assert out[0] == (2.0, 10.0) and out[1] == (2.0, 10.0)


def test_max_over_ranks_single_process_is_identity():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.5, 1.25], torch.device('cpu')) == [3.5, 1.25]


def test_reference_arm_runs_on_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv('RANK', '1')
    args = type('A', (), dict(steps=1, warmup=0, gpus=2))()
    assert bench.run_reference(args) == 0  # returns at once, no work, no output
