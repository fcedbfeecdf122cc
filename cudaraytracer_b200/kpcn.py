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
    """Raises CrtError (CRT_ERR_TIMEOUT) if a tensor-core kernel gave up a
    bounded wait since the last check."""
    _lib.call("crt_check_device_errors", ctx.handle)
