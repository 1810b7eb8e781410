"""The multi-GPU path on CPU ranks (gloo, world size 2).

The batch path shards by frames with no collective on the data path: each
rank processes its own frames, and only the timing is reduced (max over
ranks).  These tests run two gloo ranks on the CPU with the oracle standing
in for the GPU kernels and check that (1) processing the two halves of a
batch on two ranks gives, frame by frame, exactly the single-process result,
and (2) bench.py's max-over-ranks reduction returns the slowest rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import torch

    import bench
    import digholo_oracle as O
    from helpers import config_for, make_case
    hol = make_case("plain_320x256_f32_1pol", 4)
    cfg = config_for(hol, 0)
    shard = hol.frames[rank * 2:(rank + 1) * 2]
    res = O.process_batch(shard, cfg, quantised=True)
    coefs = torch.from_numpy(np.ascontiguousarray(res["coefs"]).view(np.float64))
    gathered = [torch.zeros_like(coefs) for _ in range(world)]
    dist.all_gather(gathered, coefs)
    slowest = bench.max_over_ranks(10.0 + 5.0 * rank)
    if rank == 0:
        out["coefs"] = np.concatenate([g.numpy() for g in gathered]).view(np.complex128)
        out["slowest"] = slowest
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_sharding_matches_single_process():
    import sys
    for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import digholo_oracle as O
    from helpers import config_for, make_case
    # the manager process is shut down when the block ends, not at interpreter exit
    with mp.get_context("spawn").Manager() as manager:
        shared = manager.dict()
        port = _free_port()
        mp.start_processes(_worker, args=(2, port, shared), nprocs=2, start_method="spawn", join=True)
        out = dict(shared)
    hol = make_case("plain_320x256_f32_1pol", 4)
    cfg = config_for(hol, 0)
    full = O.process_batch(hol.frames, cfg, quantised=True)["coefs"]
    np.testing.assert_array_equal(out["coefs"].reshape(full.shape), full)
    assert out["slowest"] == 15.0


def test_max_over_ranks_without_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.shard_seed(1, 2) != bench.shard_seed(0, 2)
