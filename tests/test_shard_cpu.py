"""Sharding logic of droplet_b200.shard on gloo ranks (CPU, world size 2):
view assignment and the gathers that put results back in global order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from droplet_b200 import shard
    from droplet_b200.api import BlockMaskBuffer, VoxelizeResult
    from droplet_b200.types import Bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n_views = 7
        ids = shard.views_of_rank(n_views, rank, world)
        # stand-in images: view v is (v + 1) * 11 pixels of value v
        imgs = [np.full((v + 1) * 11 * 4, v, np.uint8) for v in ids]
        got = shard.gather_images(ids, imgs, n_views, dst=0)
        # stand-in voxel shards: rank r holds blocks 100 r + k, k < r + 2
        k = np.arange(rank + 2, dtype=np.uint32)
        local = VoxelizeResult(BlockMaskBuffer(100 * rank + k, k + 1, k * 3), Bounds((0, 0, 0), (1, 1, 1)),
                               0.05, 5.0, 5.0, 5.0)
        blocks = shard.gather_blocks(local, dst=0)
        if rank == 0:
            assert len(got) == n_views
            for v, im in enumerate(got):
                assert im.size == (v + 1) * 11 * 4 and np.all(im == v)
            exp = np.concatenate([100 * r + np.arange(r + 2) for r in range(world)]).astype(np.uint32)
            assert np.array_equal(blocks.buffer.blockIdx, exp)
            assert blocks.buffer.count == exp.size and blocks.numBlocksZ == 5.0
            open(os.path.join(out_dir, "ok"), "w").write("ok")
        else:
            assert got is None and blocks is None
    finally:
        dist.destroy_process_group()


def test_views_round_robin_partition():
    from droplet_b200 import shard
    for world in (1, 2, 3, 8):
        seen = sorted(v for r in range(world) for v in shard.views_of_rank(64, r, world))
        assert seen == list(range(64))
    with pytest.raises(ValueError):
        shard.views_of_rank(4, 2, 2)


def test_gathers_on_two_gloo_ranks(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert (tmp_path / "ok").exists()
