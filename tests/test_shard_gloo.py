"""Sample-range sharding of one frame over ranks (cudaraytracer_b200.shard),
as world_size-2 gloo process groups on the CPU. Each rank's renderer here is
the CPU oracle (the product renders on the GPU); what is checked is the
partition and the sum-reduce: the reduced frame equals the frame rendered
with all samples in one call."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cudaraytracer_b200.shard import reduce_sample_shards, sample_range


def test_sample_ranges_tile_exactly():
    for spp in (0, 1, 5, 16, 17, 4096):
        for world in (1, 2, 3, 4, 8):
            got = [sample_range(spp, r, world, first_sample=7) for r in range(world)]
            nxt = 7
            for first, count in got:
                assert first == nxt and count >= 0
                nxt += count
            assert nxt == 7 + spp
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        sample_range(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, scene_json, spp, all_ranks, out_path):
    import torch.distributed as dist
    from datetime import timedelta

    import oracle
    from oracle import scene as osc

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ref = osc.load_scene(scene_json)
    cam = osc.orbit_camera(ref)

    def render(first, count):
        d, i, q = oracle.render(ref, cam, spp=count, first_sample=first, seed=3, nthreads=1)
        return torch.from_numpy(d), torch.from_numpy(i), torch.from_numpy(q)

    d, i, q = reduce_sample_shards(render, spp, all_ranks=all_ranks)
    np.savez(f"{out_path}.{rank}.npz", d=d.numpy(), i=i.numpy(), q=q.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("all_ranks", [False, True])
def test_sharded_frame_equals_single_render(tmp_path, all_ranks):
    import oracle
    from oracle import scene as osc

    from cudaraytracer_b200 import scenes

    path = scenes.cornell_box(width=24, height=24, max_bounces=4).write(str(tmp_path), "cb")
    spp, world = 5, 2
    out = str(tmp_path / "acc")
    mp.start_processes(_worker, args=(world, _free_port(), path, spp, all_ranks, out), nprocs=world,
                       join=True, start_method="spawn")
    ref = osc.load_scene(path)
    d, i, q = oracle.render(ref, osc.orbit_camera(ref), spp=spp, seed=3, nthreads=2)
    r0 = np.load(f"{out}.0.npz")
    for got, want in ((r0["d"], d), (r0["i"], i), (r0["q"], q)):
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)
    if all_ranks:
        r1 = np.load(f"{out}.1.npz")
        for k in ("d", "i", "q"):
            np.testing.assert_array_equal(r1[k], r0[k])
