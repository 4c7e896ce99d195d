"""Learned warm start for the PCG solve: a small 3D U-Net that maps (log kappa, Y) on a 64^3
grid to an initial guess of u, trained and evaluated with the library's own tensor-core
kernels (libripley_gpu.so, rg_ws_*).

Activations are torch bf16 CUDA tensors of shape (N, D+2, H, W, C): channels-last with one
zero slice before and after every sample along depth, the layout the convolution kernels
read through TMA.  torch only provides the memory.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L

BF16 = torch.bfloat16


def new_act(n, d, h, w, c, device="cuda"):
    """Zeroed activation tensor (the depth halo slices must stay zero)."""
    return torch.zeros((n, d + 2, h, w, c), dtype=BF16, device=device)


def act_struct(t):
    n, dz, h, w, c = t.shape
    return L.rg_act(t.data_ptr(), n, dz - 2, h, w, c)


def interior(t):
    """View of the interior slices: (N, D, H, W, C)."""
    return t[:, 1:-1]


class DeviceError:
    """Device-side error flag shared by the network kernels (bounded waits that gave up)."""

    def __init__(self, device="cuda"):
        self.t = torch.zeros(1, dtype=torch.int32, device=device)

    def ptr(self):
        return C.c_void_p(self.t.data_ptr())

    def check(self):
        if int(self.t.item()):
            raise L.RipleyGPUError("a bounded wait inside a warm-start network kernel gave up")


def conv3(x, weights, bias, y, relu=True, mask=None, err=None):
    """y = act(conv3x3x3(x, weights) + bias); weights bf16 [27][Cout][Cin] contiguous."""
    err = err or DeviceError(x.device)
    xs, ys = act_struct(x), act_struct(y)
    ms = act_struct(mask) if mask is not None else None
    L.set_stream_from_torch()
    L.check(L.lib().rg_ws_conv3(C.byref(xs), C.c_void_p(weights.data_ptr()),
                                C.c_void_p(bias.data_ptr()) if bias is not None else None,
                                C.byref(ys), int(relu), C.byref(ms) if ms is not None else None, err.ptr()))
    return y
