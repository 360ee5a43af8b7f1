"""Multi-rank sample sharding on CPU (gloo, world size 2): the ranks' FP64
sums, all-reduced, equal the single-process mean over the same samples."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nectarrender_b200.sharding import combine_sums, shard_samples


def test_shard_cover():
    for count in range(0, 23):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                s = shard_samples(5, count, world, r)
                seen += list(range(s.first, s.first + s.count))
            assert seen == list(range(5, 5 + count))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from nectarrender_b200 import scenes
    spec = scenes.cornell(res=16, spp=6)
    sh = shard_samples(1, 6, world, rank)
    _, _, _, _, b64 = oracle.Oracle().render(spec, sh.first, count=sh.count, mode=1, draw_rtl=0,
                                             fp64=True, threads=1)
    t = torch.from_numpy(b64)
    mean = combine_sums(t, 6, dist.all_reduce)
    if rank == 0:
        np.save(out, mean.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_combine_equals_single(tmp_path):
    import oracle
    from nectarrender_b200 import scenes
    out = str(tmp_path / "mean.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    spec = scenes.cornell(res=16, spp=6)
    _, _, _, _, b64 = oracle.Oracle().render(spec, 1, count=6, mode=1, draw_rtl=0, fp64=True)
    assert np.allclose(np.load(out), b64 / 6.0, rtol=1e-12, atol=0)
