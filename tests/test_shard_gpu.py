"""render_sharded on one GPU through a one-rank NCCL group: the reduce path
runs on the device and the frame equals render_device with all samples."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_render_sharded_single_rank_nccl(tmp_path, crt_ctx):
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from cudaraytracer_b200 import Scene, scenes
    from cudaraytracer_b200.shard import render_sharded

    sc = Scene.load(crt_ctx, scenes.cornell_box(width=64, height=64).write(str(tmp_path), "cb"))
    sc.set_render_params(seed=17)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=timedelta(seconds=30))
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", crt_ctx.device))
    try:
        d, i, q = render_sharded(sc, 6, with_sumsq=True)
        torch.cuda.synchronize()
        shape = d.shape
        wd = torch.zeros(shape, device="cuda")
        wi = torch.zeros(shape, device="cuda")
        wq = torch.zeros(shape, device="cuda")
        sc.render_device(wd, wi, 6, sumsq=wq)
        torch.cuda.synchronize()
        for a, b in ((d, wd), (i, wi), (q, wq)):
            np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=1e-5, atol=1e-6)
        assert float(d.sum()) > 0
    finally:
        dist.destroy_process_group()
        sc.close()
