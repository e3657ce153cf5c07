"""Small 3-D CNN of the learned gradient preconditioner on the engine's BF16
tensor-core convolutions (efwi_conv3d_forward / efwi_conv3d_wgrad).

Four 3x3x3 convolutions with 16 channels (ReLU after the first three),
BF16 weights and activations, FP32 accumulation; inputs of fewer than 16
channels are zero-padded.  Activations are channels-last [D][H][W][16].  The
FP32 master weights are cast to BF16 at every forward pass, so any torch
optimizer trains them.  No reference counterpart.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from ._lib import lib

C16 = 16


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def conv3d_raw(x: torch.Tensor, wb: torch.Tensor, bias, relu: bool, out_f32: bool = False):
    """x [D,H,W,16] bf16, wb [27,16,16] bf16 -> [D,H,W,16] (bf16, or f32)."""
    assert x.dtype == torch.bfloat16 and x.is_contiguous() and x.shape[-1] == C16
    assert wb.dtype == torch.bfloat16 and wb.is_contiguous() and tuple(wb.shape) == (27, C16, C16)
    D, H, W = x.shape[:3]
    yb = None if out_f32 else torch.empty_like(x)
    yf = torch.empty(x.shape, device=x.device, dtype=torch.float32) if out_f32 else None
    b = bias.float().contiguous() if bias is not None else None
    with torch.cuda.device(x.device):
        rc = lib().efwi_conv3d_forward(_ptr(x), _ptr(wb), _ptr(b), D, H, W, int(relu), _ptr(yb),
                                       _ptr(yf), _stream(x.device))
    if rc:
        raise RuntimeError(f"efwi_conv3d_forward failed ({rc})")
    return yf if out_f32 else yb


CONV_FORMS = {"mma": 0, "tcgen05": 1, "tcgen05-tma": 2, "tcgen05-tma3": 3, "tcgen05-ws": 4,
              "tcgen05-ws3": 5}


def set_conv_kernel(form: str) -> None:
    """Kernel of every later forward / input-gradient convolution of this
    process: 'mma' (mma.sync m16n8k16), 'tcgen05' (tensor-memory accumulator,
    one MMA per tap for 128 voxels, tile staged by loads), 'tcgen05-tma'
    (the same MMAs, tiles staged by bulk tensor copies two stages deep, the
    next tile's MMAs overlapping this tile's epilogue; the default),
    'tcgen05-tma3' (three stages, fewer CTAs per SM), 'tcgen05-ws' /
    'tcgen05-ws3' (warp-specialised: one warp issues the copies and MMAs,
    four drain the accumulators, mbarriers between them; two / three
    stages)."""
    if form not in CONV_FORMS:
        raise ValueError(f"unknown convolution kernel form {form!r}")
    lib().efwi_conv3d_set_kernel(CONV_FORMS[form])


def set_wgrad_kernel(form: str) -> None:
    """'tcgen05' (eight taps per MMA, accumulators in tensor memory; the
    default) or 'mma' (mma.sync) for every later weight-gradient
    convolution."""
    if form not in ("tcgen05", "mma"):
        raise ValueError(f"unknown weight-gradient kernel form {form!r}")
    lib().efwi_conv3d_set_wgrad_kernel(1 if form == "tcgen05" else 0)


def conv3d_status(device=None) -> bool:
    """True when a tcgen05 convolution since the last call gave up waiting for
    its tensor cores (its outputs are then incomplete); clears the flag."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    flag = C.c_int(0)
    with torch.cuda.device(dev):
        rc = lib().efwi_conv3d_status(C.byref(flag), _stream(dev))
    if rc:
        raise RuntimeError(f"efwi_conv3d_status failed ({rc})")
    return bool(flag.value)


def conv3d_wgrad(x: torch.Tensor, dy: torch.Tensor, nparts: int = 592) -> torch.Tensor:
    """dW[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci] (f32)."""
    D, H, W = x.shape[:3]
    partial = torch.empty(nparts * 27 * C16 * C16, device=x.device, dtype=torch.float32)
    dw = torch.empty(27, C16, C16, device=x.device, dtype=torch.float32)
    with torch.cuda.device(x.device):
        rc = lib().efwi_conv3d_wgrad(_ptr(x), _ptr(dy), D, H, W, _ptr(partial), nparts, _ptr(dw),
                                     _stream(x.device))
    if rc:
        raise RuntimeError(f"efwi_conv3d_wgrad failed ({rc})")
    return dw


class Conv3dBF16(torch.autograd.Function):
    """One layer: y = relu?(conv(x, w) + b) with BF16 operands."""

    @staticmethod
    def forward(ctx, x, w, b, relu, out_f32):
        wb = w.to(torch.bfloat16).contiguous()
        y = conv3d_raw(x, wb, b, relu, out_f32)
        ctx.save_for_backward(x, wb, y)
        ctx.relu = relu
        return y

    @staticmethod
    def backward(ctx, gy):
        x, wb, y = ctx.saved_tensors
        g = gy.float()
        if ctx.relu:
            g = g * (y > 0)
        dyb = g.to(torch.bfloat16).contiguous()
        wt = wb.flip(0).transpose(1, 2).contiguous()  # w'[t][a][b] = w[26-t][b][a]
        dx = conv3d_raw(dyb, wt, None, False) if ctx.needs_input_grad[0] else None
        dw = conv3d_wgrad(x, dyb)
        db = g.sum(dim=(0, 1, 2))
        return dx, dw, db, None, None


def to_channels_last(feats: torch.Tensor) -> torch.Tensor:
    """[C, D, H, W] f32 -> [D, H, W, 16] bf16 (channels zero-padded)."""
    c = feats.shape[0]
    x = torch.zeros(feats.shape[1:] + (C16,), device=feats.device, dtype=torch.bfloat16)
    x[..., :c] = feats.permute(1, 2, 3, 0).to(torch.bfloat16)
    return x


class Preconditioner(torch.nn.Module):
    """(gradient, model, illumination) -> update direction."""

    def __init__(self, cin: int = 3, seed: int = 0, layers: int = 4):
        super().__init__()
        gen = torch.Generator().manual_seed(seed)
        ws, bs = [], []
        for k in range(layers):
            fan_in = 27 * (cin if k == 0 else C16)
            w = torch.randn(27, C16, C16, generator=gen) * math.sqrt(2.0 / fan_in)
            if k == 0:
                w[:, :, cin:] = 0.0
            if k == layers - 1:
                w[:, 1:, :] = 0.0
                w *= 0.1
            ws.append(torch.nn.Parameter(w))
            bs.append(torch.nn.Parameter(torch.zeros(C16)))
        self.w = torch.nn.ParameterList(ws)
        self.b = torch.nn.ParameterList(bs)

    def forward(self, feats: torch.Tensor) -> torch.Tensor:
        """feats [C, D, H, W] f32 on a GPU -> [D, H, W] f32."""
        h = to_channels_last(feats)
        n = len(self.w)
        for k in range(n):
            last = k == n - 1
            h = Conv3dBF16.apply(h, self.w[k], self.b[k], not last, last)
        return h[..., 0]
