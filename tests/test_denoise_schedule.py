"""The denoiser's training loop (cudaraytracer_b200.denoise.train) on the
CPU with a stand-in network that records each step's learning rate: a
linear ramp over the first 10% of the steps (at most 30), then a cosine
decay to 5% of the base rate. The ramp keeps the first Adam steps from
overshooting, which left some GPU training runs in a state they never
recovered from."""
import math
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from cudaraytracer_b200 import denoise as D


class Recorder:
    def __init__(self):
        self.lrs = []
        self.shapes = []

    def train_step(self, f, nz, rf, lr):
        self.lrs.append(lr)
        self.shapes.append((tuple(f.shape), tuple(nz.shape), tuple(rf.shape)))
        return 1.0


def example(h=24, w=20):
    return types.SimpleNamespace(feat=torch.zeros((h, w, 16)), noisy=torch.zeros((h, w, 4)),
                                 ref=torch.zeros((h, w, 4)))


@pytest.mark.parametrize("steps", [300, 1500, 12])
def test_learning_rate_ramps_then_decays(steps):
    net = Recorder()
    losses = D.train(net, [example(), example()], steps=steps, batch=3, crop=8, lr=1e-3)
    assert len(losses) == steps and len(net.lrs) == steps
    warm = max(1, min(30, steps // 10))
    lrs = np.array(net.lrs)
    for k in range(steps):
        want = 1e-3 * min(1.0, (k + 1) / warm) * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * k / steps)))
        assert lrs[k] == pytest.approx(want, rel=1e-12)
    assert np.all(np.diff(lrs[:warm]) > 0)          # the ramp rises
    assert np.all(np.diff(lrs[warm:]) <= 0)         # then the cosine falls
    assert lrs[-1] < 0.1e-3                         # towards 5% of the base rate (reached at step `steps`)
    assert net.shapes[0] == ((3, 8, 8, 16), (3, 8, 8, 4), (3, 8, 8, 4))
