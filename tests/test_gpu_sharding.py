"""Two ranks (processes, gloo over the host) each render their shard of the
sample indices through the product's own path (capi.Render with FP64 sums on
the GPU) and combine the sums with one all-reduce; the combined mean equals
one process rendering every sample index. Both ranks use the one GPU of the
machine; neither waits on the other's kernels (the only exchange is the
host-side all-reduce after both have finished rendering)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
FIRST, COUNT = 1, 7


def _spec():
    from nectarrender_b200 import scenes
    return scenes.mesh_stress(levels=3, res_h=48, res_w=48, spp=FIRST + COUNT, depth=8,
                              n_spheres=12, hdri_size=(64, 32), scene_seed=11)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    from nectarrender_b200 import capi
    from nectarrender_b200.sharding import combine_sums, render_shard
    spec = _spec()
    r = capi.Render(capi.Scene(spec), fp64_accumulate=1)
    s, n = render_shard(r, FIRST, COUNT, world, rank)
    t = torch.from_numpy(s)
    cnt = torch.tensor([n], dtype=torch.int64)
    dist.all_reduce(cnt)
    mean = combine_sums(t, int(cnt.item()), dist.all_reduce)
    if rank == 0:
        np.save(out, mean.numpy())
        np.save(out + ".n.npy", cnt.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_combine_to_the_single_render(tmp_path):
    from nectarrender_b200 import capi
    out = str(tmp_path / "mean.npy")
    _spec()  # writes the scene's files before the ranks read them
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    r = capi.Render(capi.Scene(_spec()), fp64_accumulate=1)
    r.samples(FIRST, COUNT)
    whole = r.beauty_fp64()
    assert int(np.load(out + ".n.npy")[0]) == COUNT
    np.testing.assert_allclose(np.load(out), whole, rtol=1e-12, atol=1e-300)
