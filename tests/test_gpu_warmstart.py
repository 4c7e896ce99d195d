"""Warm-start network kernels against plain PyTorch fp32 references of the same ops.

Tolerance: outputs are bf16 (8-bit mantissa), inputs bf16, accumulation fp32; results must
agree with the fp32 reference to 2e-2 of the reference's largest magnitude.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from esys_b200 import warmstart as W

pytestmark = pytest.mark.gpu
TOL = 2e-2


def ref_conv(x, w27, b, relu, mask=None):
    """x: (N, D, H, W, Cin) fp32; w27: (27, Cout, Cin) with tap = kw + 3 kh + 9 kd."""
    n, d, h, ww, cin = x.shape
    cout = w27.shape[1]
    wt = w27.reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2)  # (Cout, Cin, kd, kh, kw)
    y = F.conv3d(x.permute(0, 4, 1, 2, 3), wt, b, padding=1).permute(0, 2, 3, 4, 1)
    if relu:
        y = torch.relu(y)
    if mask is not None:
        y = y * (mask > 0)
    return y


@pytest.mark.parametrize("n,dhw,cin,cout,relu,use_mask", [
    (1, (8, 8, 8), 16, 16, True, False),
    (2, (16, 16, 16), 32, 48, False, False),
    (1, (32, 32, 32), 80, 32, True, True),
    (1, (16, 16, 16), 112, 48, True, False),
    (1, (64, 64, 64), 16, 16, True, False),
    (1, (8, 8, 8), 64, 64, False, True),
    (2, (16, 16, 16), 48, 112, True, False),
])
def test_conv3_matches_torch(cuda, n, dhw, cin, cout, relu, use_mask):
    torch.manual_seed(0)
    d, h, w = dhw
    x = W.new_act(n, d, h, w, cin)
    xv = torch.randn(n, d, h, w, cin, device="cuda").to(torch.bfloat16)
    W.interior(x).copy_(xv)
    wt = (torch.randn(27, cout, cin, device="cuda") * (1.0 / (27 * cin) ** 0.5)).to(torch.bfloat16).contiguous()
    b = torch.randn(cout, device="cuda")
    mask = None
    if use_mask:
        mask = W.new_act(n, d, h, w, cout)
        W.interior(mask).copy_((torch.rand(n, d, h, w, cout, device="cuda") - 0.5).to(torch.bfloat16))
    y = W.new_act(n, d, h, w, cout)
    err = W.DeviceError()
    W.conv3(x, wt, b, y, relu=relu, mask=mask, err=err)
    torch.cuda.synchronize()
    err.check()
    ref = ref_conv(xv.float().cpu(), wt.float().cpu(), b.cpu(), relu,
                   W.interior(mask).float().cpu() if use_mask else None)
    got = W.interior(y).float().cpu()
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= TOL * scale
    # halo slices untouched
    assert not bool(y[:, 0].any()) and not bool(y[:, -1].any())
