"""The learned denoiser trained on tracer-generated pairs (seeded Cornell
variants, GPU training by the project's own kernels) and what it gains over
the raw image and over SVGF on unseen test scenes."""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_kpcn_beats_raw_and_svgf_on_unseen_scenes(crt_ctx):
    from cudaraytracer_b200 import denoise as D
    from cudaraytracer_b200 import kpcn
    from cudaraytracer_b200.kpcn import Kpcn

    data = D.build_dataset(crt_ctx, range(100, 112), 1, 128, 128, [2, 4, 8], ref_spp=512, seed=1)
    net = Kpcn(crt_ctx, seed=0)
    losses = D.train(net, data, steps=300, batch=8, crop=64, lr=1e-3)
    kpcn.check_device_errors(crt_ctx)  # no convolution gave up a bounded wait
    first, last = sum(losses[:30]), sum(losses[-30:])
    assert last < 0.5 * first, (first, last, losses[::30])
    tab = D.evaluate(crt_ctx, net, range(200, 203), 128, 128, [4], svgf_spp=4, ref_spp=1024)
    net.close()
    # the network removes most of the noise of a 4-spp image ...
    assert tab["kpcn_4"] < 0.25 * tab["raw_4"]
    # ... and does better than SVGF on the same 4-spp image
    assert tab["kpcn_4"] < tab["svgf_4"]
