"""Learned kernel-predicting denoiser (KPCN) on the tensor-core convolution
kernels of libcrt.so.

The tensor-level entry points take CUDA torch tensors (torch provides device
memory and streams only): activations NHWC torch.bfloat16, 3x3 weights
(9, cout, cin) torch.bfloat16, biases and weight gradients float32.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .tracer import _torch_stream


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _check_act(x, name):
    import torch

    if not (x.is_cuda and x.dtype == torch.bfloat16 and x.dim() == 4 and x.is_contiguous()):
        raise ValueError(f"{name}: expected a contiguous CUDA bfloat16 tensor (n, h, w, c)")


def conv3x3_forward(ctx, x, w, bias=None, relu=False, out=None, out_f32=None, stream=None):
    """3x3 convolution (stride 1, zero padding 1) on the tensor cores:
    out[p, o] = bias[o] + sum_{t, c} x[p + off(t), c] * w[t][o][c] (ReLU if
    relu). Returns the BF16 output (and fills out_f32 when given)."""
    import torch

    _check_act(x, "x")
    n, h, wd, cin = x.shape
    cout = w.shape[1]
    if out is None and out_f32 is None:
        out = torch.empty((n, h, wd, cout), dtype=torch.bfloat16, device=x.device)
    _lib.call("crt_conv3x3_forward", ctx.handle, _ptr(x), n, h, wd, cin, _ptr(w), _ptr(bias), cout, 1 if relu else 0,
              _ptr(out), _ptr(out_f32), C.c_void_p(_torch_stream(x.device, stream)))
    return out


def conv3x3_backward_data(ctx, g, wt, mask=None, out=None, stream=None):
    """grad_x[q, c] = sum_{t, o} g[q - off(t), o] * wt[t][c][o] (wt = w
    transposed per tap), times (mask > 0) when mask is given."""
    import torch

    _check_act(g, "g")
    n, h, wd, cout = g.shape
    cin = wt.shape[1]
    if out is None:
        out = torch.empty((n, h, wd, cin), dtype=torch.bfloat16, device=g.device)
    _lib.call("crt_conv3x3_backward_data", ctx.handle, _ptr(g), n, h, wd, cout, _ptr(wt), cin, _ptr(mask), _ptr(out),
              C.c_void_p(_torch_stream(g.device, stream)))
    return out


def conv3x3_backward_weights(ctx, x, g, dw=None, stream=None):
    """dw[t][o][c] += sum_p x[p + off(t), c] * g[p, o] (float32)."""
    import torch

    _check_act(x, "x")
    _check_act(g, "g")
    n, h, wd, cin = x.shape
    cout = g.shape[3]
    if dw is None:
        dw = torch.zeros((9, cout, cin), dtype=torch.float32, device=x.device)
    _lib.call("crt_conv3x3_backward_weights", ctx.handle, _ptr(x), _ptr(g), n, h, wd, cin, cout, _ptr(dw),
              C.c_void_p(_torch_stream(x.device, stream)))
    return dw


def check_device_errors(ctx) -> None:
    """Raises CrtError if a kernel of ctx recorded a device-side error since
    the last check (CRT_ERR_TIMEOUT: a tensor-core kernel gave up a bounded
    wait)."""
    _lib.call("crt_check_device_errors", ctx.handle)


class Kpcn:
    """The kernel-predicting denoiser (crt_kpcn_*): a 3-level U-Net on the
    tensor-core convolutions predicting a 5x5 filter per pixel. Tensors are
    CUDA torch tensors: features (n, h, w, 16) bfloat16, radiance (n, h, w, 4)
    float32 (rgb, unused); h and w multiples of 4."""

    LAYERS = ["e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "d1a", "d1b", "d0a", "d0b", "out"]
    SPEC = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (160, 64), (64, 64), (96, 32), (32, 32),
            (32, 32)]

    def __init__(self, ctx, seed: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        _lib.call("crt_kpcn_create", ctx.handle, int(seed), C.byref(h))
        self._h = h
        ctx._adopt(self)
        n = C.c_int64()
        _lib.call("crt_kpcn_num_params", self._h, C.byref(n))
        self.num_params = n.value

    def close(self):
        if self._h:
            _lib.lib().crt_kpcn_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        import numpy as np

        p = np.empty(self.num_params, np.float32)
        _lib.call("crt_kpcn_get_params", self._h, p.ctypes.data)
        return p

    def set_params(self, p):
        import numpy as np

        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        _lib.call("crt_kpcn_set_params", self._h, p.ctypes.data)

    def get_grads(self):
        import numpy as np

        g = np.empty(self.num_params, np.float32)
        _lib.call("crt_kpcn_get_grads", self._h, g.ctypes.data)
        return g

    def forward(self, features, noisy, out=None, stream=None):
        import torch

        n, h, w, _ = features.shape
        if out is None:
            out = torch.empty((n, h, w, 4), dtype=torch.float32, device=features.device)
        _lib.call("crt_kpcn_forward", self._h, n, h, w, _ptr(features), _ptr(noisy), _ptr(out),
                  C.c_void_p(_torch_stream(features.device, stream)))
        return out

    def train_step(self, features, noisy, target, lr: float, stream=None) -> float:
        """Forward, relMSE loss, backward and (lr > 0) an Adam step; returns
        the batch loss (synchronises)."""
        n, h, w, _ = features.shape
        loss = C.c_float()
        _lib.call("crt_kpcn_train_step", self._h, n, h, w, _ptr(features), _ptr(noisy), _ptr(target), float(lr),
                  C.byref(loss), C.c_void_p(_torch_stream(features.device, stream)))
        return loss.value

    def debug_tensor(self, which: int, shape, dtype):
        """Internal tensor of the last forward (0..9 layer outputs, 10 logits,
        11 pool0, 12 pool1, 13 cat1, 14 cat0) as a numpy array."""
        import numpy as np

        a = np.empty(shape, dtype)
        _lib.call("crt_kpcn_debug_tensor", self._h, int(which), a.ctypes.data, int(a.nbytes))
        return a


def make_features(scene, gbuffer: dict, direct, indirect, spp: int, depth_scale: float, stream=None, out=None):
    """Network input of one rendered view: (features (h, w, 16) bfloat16,
    noisy radiance (h, w, 4) float32 = (direct + indirect) / spp) from the
    render accumulators and the view's G-buffer (Scene.gbuffer()). direct
    and indirect are CUDA tensors (h, w, 4), or device addresses (ints) of
    such float4 planes when `out` = (feat, noisy) gives the output tensors
    to fill."""
    import torch

    from .tracer import _gbuffer_struct

    if out is not None:
        feat, noisy = out
        h, w = feat.shape[0], feat.shape[1]
        dev = feat.device
    else:
        h, w = direct.shape[0], direct.shape[1]
        dev = direct.device
        feat = torch.empty((h, w, 16), dtype=torch.bfloat16, device=dev)
        noisy = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
    dp = C.c_void_p(direct) if isinstance(direct, int) else _ptr(direct)
    ip = C.c_void_p(indirect) if isinstance(indirect, int) else _ptr(indirect)
    gb = _gbuffer_struct(gbuffer)
    _lib.call("crt_kpcn_features", scene.handle, C.byref(gb), dp, ip, int(spp), h * w, float(depth_scale), _ptr(feat),
              _ptr(noisy), C.c_void_p(_torch_stream(dev, stream)))
    return feat, noisy
