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
    # the persistent kernel (weights resident, two TMEM accumulators): several tiles per CTA,
    # two input chunks, two samples, 64 output channels
    (1, (64, 64, 64), 32, 16, True, True),
    (2, (32, 32, 16), 16, 32, False, False),
    (1, (16, 16, 16), 32, 64, True, True),
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


def _act_from(t, device="cuda"):
    """activation tensor holding t (N, D, H, W, C) as bf16."""
    n, d, h, w, c = t.shape
    a = W.new_act(n, d, h, w, c, device=device)
    W.interior(a).copy_(t.to(torch.bfloat16))
    return a


@pytest.mark.parametrize("n,dhw,cin,cout", [
    (1, (8, 8, 8), 16, 16),
    (2, (16, 16, 16), 32, 48),
    (1, (16, 16, 16), 80, 32),
    (1, (32, 32, 32), 16, 16),
    (1, (8, 8, 8), 112, 48),
    (1, (16, 16, 8), 48, 64),
    (1, (8, 16, 16), 16, 128),
])
def test_conv3_wgrad_matches_torch(cuda, n, dhw, cin, cout):
    """dW[tap][co][ci] = sum_p g(p, co) x(p + off(tap), ci), against torch autograd of conv3d."""
    torch.manual_seed(1)
    d, h, w = dhw
    xv = torch.randn(n, d, h, w, cin, device="cuda").to(torch.bfloat16)
    gv = torch.randn(n, d, h, w, cout, device="cuda").to(torch.bfloat16)
    x, g = _act_from(xv), _act_from(gv)
    dw = torch.full((27, cout, cin), 7.0, device="cuda")
    partials = torch.zeros(1 << 22, device="cuda")
    err = W.DeviceError()
    W.conv3_wgrad(x, g, dw, partials, err=err)
    torch.cuda.synchronize()
    err.check()
    w27 = torch.zeros(27, cout, cin, dtype=torch.float64, requires_grad=True)
    y = ref_conv(xv.double().cpu(), w27, None, relu=False)
    (y * gv.double().cpu()).sum().backward()
    ref = w27.grad
    got = dw.double().cpu()
    assert (got - ref).abs().max().item() <= 1e-3 * ref.abs().max().item()
    # accumulate adds onto the previous result
    W.conv3_wgrad(x, g, dw, partials, accumulate=True, err=err)
    torch.cuda.synchronize()
    assert (dw.double().cpu() - 2 * ref).abs().max().item() <= 2e-3 * ref.abs().max().item()


def test_conv3_wgrad_small_partials_buffer(cuda):
    """a partials buffer for one split still gives the full sum."""
    torch.manual_seed(2)
    xv = torch.randn(1, 16, 16, 16, 16, device="cuda").to(torch.bfloat16)
    gv = torch.randn(1, 16, 16, 16, 16, device="cuda").to(torch.bfloat16)
    dw_big, dw_small = torch.zeros(27, 16, 16, device="cuda"), torch.zeros(27, 16, 16, device="cuda")
    x, g = _act_from(xv), _act_from(gv)
    W.conv3_wgrad(x, g, dw_big, torch.zeros(1 << 22, device="cuda"))
    mtiles = (27 + 7) // 8
    W.conv3_wgrad(x, g, dw_small, torch.zeros(mtiles * 128 * 16, device="cuda"))
    torch.cuda.synchronize()
    assert torch.allclose(dw_big, dw_small, rtol=1e-4, atol=1e-3)


def test_memory_bound_layers_match_torch(cuda):
    torch.manual_seed(3)
    n, d, h, w, c = 2, 8, 16, 16, 32
    sv = torch.randn(n, d, h, w, c, device="cuda").relu().to(torch.bfloat16)
    s = _act_from(sv)
    # pooling
    p = W.new_act(n, d // 2, h // 2, w // 2, c)
    W.avgpool(s, p)
    ref_p = sv.float().reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).mean(dim=(2, 4, 6))
    assert torch.allclose(W.interior(p).float(), ref_p, atol=2e-2, rtol=1e-2)
    # pooling backward with a skip gradient at channel offset 16 of a 48-channel tensor
    dpv = torch.randn(n, d // 2, h // 2, w // 2, c, device="cuda").to(torch.bfloat16)
    dskv = torch.randn(n, d, h, w, 48, device="cuda").to(torch.bfloat16)
    din = W.new_act(n, d, h, w, c)
    W.avgpool_bwd(_act_from(dpv), s, _act_from(dskv), 16, din)
    up = dpv.float().repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3) / 8
    ref = (up + dskv.float()[..., 16:48]) * (sv.float() > 0)
    assert torch.allclose(W.interior(din).float(), ref, atol=2e-2, rtol=1e-2)
    # upsample + concat and its backward with the mask of the upsampled tensor
    av = torch.randn(n, d // 2, h // 2, w // 2, 48, device="cuda").relu().to(torch.bfloat16)
    cat = W.new_act(n, d, h, w, 48 + c)
    W.upcat(_act_from(av), s, cat)
    upa = av.float().repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3)
    assert torch.equal(W.interior(cat).float(), torch.cat([upa, sv.float()], dim=-1))
    dcv = torch.randn(n, d, h, w, 48 + c, device="cuda").to(torch.bfloat16)
    da = W.new_act(n, d // 2, h // 2, w // 2, 48)
    W.upcat_bwd(_act_from(dcv), _act_from(av), da)
    ref = dcv.float()[..., :48].reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, 48).sum(dim=(2, 4, 6)) * (av.float() > 0)
    assert torch.allclose(W.interior(da).float(), ref, atol=5e-2, rtol=1e-2)
    # head, its input gradient and the column sums
    hw = torch.randn(c, device="cuda")
    hb = torch.randn(1, device="cuda")
    out = torch.empty(n, d, h, w, device="cuda")
    W.head(s, hw, hb, out)
    assert torch.allclose(out, sv.float() @ hw + hb, atol=1e-3, rtol=1e-4)
    dout = torch.randn(n, d, h, w, device="cuda")
    dx = W.new_act(n, d, h, w, c)
    W.head_bwd_x(s, hw, dout, dx)
    ref = dout[..., None] * hw * (sv.float() > 0)
    assert torch.allclose(W.interior(dx).float(), ref, atol=2e-2, rtol=1e-2)
    work = torch.zeros(592 * 128, device="cuda")
    cs = torch.zeros(c, device="cuda")
    W.colsum(s, None, cs, work)
    assert torch.allclose(cs, sv.float().sum(dim=(0, 1, 2, 3)), rtol=1e-4, atol=1e-2)
    W.colsum(s, dout, cs, work)
    assert torch.allclose(cs, (sv.float() * dout[..., None]).sum(dim=(0, 1, 2, 3)), rtol=1e-4, atol=1e-2)
    # halos untouched everywhere
    for t in (p, din, cat, da, dx):
        assert not bool(t[:, 0].any()) and not bool(t[:, -1].any())


def test_mse_adam_and_weight_copies(cuda):
    torch.manual_seed(4)
    out = torch.randn(3, 8, 8, 8, device="cuda")
    t = torch.randn(3, 8, 8, 8, device="cuda")
    dout = torch.empty_like(out)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    dsum = torch.zeros(1, device="cuda")
    W.mse(out, t, dout, loss, dsum, torch.zeros(1184, dtype=torch.float64, device="cuda"))
    e = (out - t).double()
    assert abs(loss.item() - (e * e).mean().item()) <= 1e-12 * (e * e).mean().item() + 1e-15
    assert torch.allclose(dout, (2 * e / e.numel()).float(), rtol=1e-6, atol=1e-9)
    assert abs(dsum.item() - (2 * e / e.numel()).sum().item()) <= 1e-5
    # Adam (bias corrected), two steps, against the textbook update in float64
    wv = torch.randn(1000, device="cuda")
    g1, g2 = torch.randn(1000, device="cuda"), torch.randn(1000, device="cuda")
    m, v = torch.zeros_like(wv), torch.zeros_like(wv)
    w0 = wv.double().clone()
    from esys_b200 import _lib as Lb
    for step, g in ((1, g1), (2, g2)):
        Lb.check(Lb.lib().rg_ws_adam(W._p(wv), W._p(g), W._p(m), W._p(v), 1000, 1e-2, 0.9, 0.999, 1e-8, step))
    mr, vr, wr = torch.zeros_like(w0), torch.zeros_like(w0), w0.clone()
    for step, g in ((1, g1.double()), (2, g2.double())):
        mr = 0.9 * mr + 0.1 * g
        vr = 0.999 * vr + 0.001 * g * g
        wr -= 1e-2 * (mr / (1 - 0.9 ** step)) / ((vr / (1 - 0.999 ** step)).sqrt() + 1e-8)
    assert torch.allclose(wv.double(), wr, rtol=1e-5, atol=1e-6)
    # bf16 forward copy and flipped/transposed data-gradient copy
    w = torch.randn(27, 48, 32, device="cuda")
    wf = torch.zeros(27, 48, 32, dtype=torch.bfloat16, device="cuda")
    wd = torch.zeros(27, 32, 48, dtype=torch.bfloat16, device="cuda")
    W.weights_bf16(w, wf, wd)
    assert torch.equal(wf, w.to(torch.bfloat16))
    assert torch.equal(wd, w.to(torch.bfloat16).flip(0).transpose(1, 2))


def test_data_gradient_is_conv_with_flipped_weights(cuda):
    """conv3 of the output gradient with rg_ws_weights_bf16's flipped copy and the mask of
    the layer below equals torch's input gradient."""
    torch.manual_seed(6)
    n, d, h, w, cin, cout = 1, 16, 16, 16, 48, 32
    xv = torch.randn(n, d, h, w, cin, device="cuda").relu().to(torch.bfloat16)
    gv = torch.randn(n, d, h, w, cout, device="cuda").to(torch.bfloat16)
    wt = torch.randn(27, cout, cin, device="cuda") * 0.05
    wf = torch.zeros(27, cout, cin, dtype=torch.bfloat16, device="cuda")
    wd = torch.zeros(27, cin, cout, dtype=torch.bfloat16, device="cuda")
    W.weights_bf16(wt, wf, wd)
    x = _act_from(xv)
    dx = W.new_act(n, d, h, w, cin)
    W.conv3(_act_from(gv), wd, None, dx, relu=False, mask=x)
    torch.cuda.synchronize()
    xr = xv.double().cpu().requires_grad_(True)
    y = ref_conv(xr, wf.double().cpu(), None, relu=False)
    (y * gv.double().cpu()).sum().backward()
    ref = xr.grad * (xv.double().cpu() > 0)
    got = W.interior(dx).double().cpu()
    assert (got - ref).abs().max().item() <= TOL * ref.abs().max().item()


def test_field_maps_are_consistent(cuda):
    """stats, input packing (with 2x coarsening), nodal targets and the nodal guess."""
    torch.manual_seed(7)
    fine, f = (16, 16, 16), 2
    kappa = torch.exp(torch.randn(1, *fine, device="cuda"))
    y = torch.randn(1, *fine, device="cuda")
    fm = W.FieldMap(1, fine, f)
    x0 = W.new_act(1, 8, 8, 8, 16)
    fm.pack(kappa, y, x0)
    st = fm.stats.cpu()
    mu = torch.log(kappa.double()).mean().item()
    sy = y.abs().max().item()
    h = 1.0 / 8
    assert abs(st[0].item() - mu) < 1e-5 and abs(st[1].item() - sy) < 1e-6
    assert abs(st[3].item() - 10 * sy * h * h / np.exp(mu)) < 1e-5 * st[3].item()
    lk = torch.log(kappa).reshape(1, 8, 2, 8, 2, 8, 2).mean(dim=(2, 4, 6)) - mu
    yy = y.reshape(1, 8, 2, 8, 2, 8, 2).mean(dim=(2, 4, 6)) / sy
    xi = W.interior(x0).float()
    assert torch.allclose(xi[..., 0], lk, atol=2e-2, rtol=1e-2)
    assert torch.allclose(xi[..., 1], yy, atol=2e-2, rtol=1e-2)
    c = (torch.arange(8, device="cuda", dtype=torch.float32) + 0.5) / 8
    assert torch.allclose(xi[0, :, 0, 0, 2], c, atol=4e-3)
    assert torch.allclose(xi[0, 0, :, 0, 3], c, atol=4e-3)
    assert torch.allclose(xi[0, 0, 0, :, 4], c, atol=4e-3)
    assert not bool(xi[..., 5:].any())
    # a linear nodal field: cell means are exact, and interpolating them back reproduces
    # every node at least half a cell away from the faces
    nn = fine[0] + 1
    zz, yy_, xx = torch.meshgrid(*(torch.arange(nn, device="cuda", dtype=torch.float64) / fine[0],) * 3,
                                 indexing="ij")
    u = (0.3 + 2.0 * xx - 1.0 * yy_ + 0.5 * zz).reshape(-1)
    t = torch.zeros(1, 8, 8, 8, device="cuda")
    fm.targets(u, t)
    c = (torch.arange(8, device="cuda", dtype=torch.float64) + 0.5) / 8
    cz, cy, cx = torch.meshgrid(c, c, c, indexing="ij")
    ref_t = (0.3 + 2.0 * cx - 1.0 * cy + 0.5 * cz) / st[3].item()
    assert torch.allclose(t.double()[0], ref_t, rtol=1e-5, atol=1e-5)
    q = torch.zeros(nn ** 3, dtype=torch.float64, device="cuda")
    q[(nn - 1) * nn * nn:] = 1
    g = torch.zeros(nn ** 3, dtype=torch.float64, device="cuda")
    fm.guess(t, q, g)
    g3, u3 = g.reshape(nn, nn, nn), u.reshape(nn, nn, nn)
    inner = slice(1, nn - 2)
    assert torch.allclose(g3[inner, inner, inner], u3[inner, inner, inner], rtol=1e-5, atol=1e-5)
    assert not bool(g3[-1].any())


def _oracle_params(net):
    """the network's parameters as the GPU uses them: bf16 weights, fp32 biases/head."""
    p = {}
    for name, _, _ in net.layers:
        p[name + ".w"] = net.wf[name].double().cpu().numpy()
        p[name + ".b"] = net.p[name + ".b"].double().cpu().numpy()
    p["head.w"] = net.p["head.w"].double().cpu().numpy()
    p["head.b"] = net.p["head.b"].double().cpu().numpy()
    return p


def test_network_gradients_match_cpu_oracle(cuda):
    """forward output, loss and every parameter gradient of the GPU training pass against
    the float64 CPU oracle with the same bf16 weights and input.  bf16 activations and
    gradients between layers bound the agreement: 3e-2 relative (norm-wise) per tensor."""
    from oracle import unet_oracle as U
    torch.manual_seed(8)
    n, d, h, w = 1, 16, 64, 64
    net = W.UNet(seed=3)
    # non-zero biases so that every bias path is exercised
    for name, _, cout in net.layers:
        net.p[name + ".b"].copy_(torch.randn(cout) * 0.05)
    net.refresh()
    ws = W.Workspace(n, d, h, w)
    xin = torch.zeros(n, d, h, w, 16, device="cuda")
    xin[..., :2] = torch.randn(n, d, h, w, 2, device="cuda")
    W.interior(ws.x0).copy_(xin.to(torch.bfloat16))
    ws.target.copy_(torch.randn(n, d, h, w, device="cuda") * 0.1)
    net.forward(ws)
    net.loss_and_backward(ws)
    torch.cuda.synchronize()
    net.err.check()
    p = _oracle_params(net)
    loss, grads, out = U.loss_and_grads(p, W.interior(ws.x0).double().cpu().numpy(), ws.target.double().cpu().numpy())
    got_out = ws.out.double().cpu().numpy()
    assert np.linalg.norm(got_out - out) <= 3e-2 * np.linalg.norm(out)
    assert abs(net.loss.item() - loss) <= 3e-2 * loss
    worst = {}
    for k, ref in grads.items():
        gg = net.g[k].double().cpu().numpy()
        if k == "enc0a.w":       # only the two live input channels carry gradient
            ref, gg = ref[..., :2], gg[..., :2]
        worst[k] = np.linalg.norm(gg - ref) / max(np.linalg.norm(ref), 1e-30)
    bad = {k: v for k, v in worst.items() if v > 3e-2}
    assert not bad, f"relative gradient errors above 3e-2: {bad}; all: {worst}"


def test_training_steps_reduce_the_loss(cuda):
    """Adam on one fixed batch: the loss falls by more than half in 40 steps."""
    torch.manual_seed(9)
    net = W.UNet(seed=1)
    ws = W.Workspace(2, 16, 64, 64)
    xin = torch.zeros(2, 16, 64, 64, 16, device="cuda")
    xin[..., :2] = torch.randn(2, 16, 64, 64, 2, device="cuda")
    W.interior(ws.x0).copy_(xin.to(torch.bfloat16))
    # a smooth target that depends on the input
    ws.target.copy_(torch.nn.functional.avg_pool3d(xin[..., 1][:, None], 5, 1, 2)[:, 0] + 0.3)
    losses = []
    for _ in range(40):
        net.forward(ws)
        net.loss_and_backward(ws)
        losses.append(net.loss.item())
        net.adam_step(2e-3)
    torch.cuda.synchronize()
    net.err.check()
    assert losses[-1] < 0.5 * losses[0], losses


def test_h1_loss_matches_torch(cuda):
    torch.manual_seed(10)
    n, d, h, w, lam = 2, 8, 16, 16, 5.0
    out = torch.randn(n, d, h, w, device="cuda")
    t = torch.randn(n, d, h, w, device="cuda")
    dout = torch.empty_like(out)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    dsum = torch.zeros(1, device="cuda")
    W.h1_loss(out, t, lam, dout, loss, dsum, torch.zeros(1184, dtype=torch.float64, device="cuda"))
    o = out.double().cpu().requires_grad_(True)
    e = o - t.double().cpu()
    ref = (e * e).sum()
    for ax in (1, 2, 3):
        ref = ref + lam * (torch.diff(e, dim=ax) ** 2).sum()
    ref = ref / e.numel()
    ref.backward()
    assert abs(loss.item() - ref.item()) <= 1e-6 * ref.item()
    assert torch.allclose(dout.double().cpu(), o.grad, rtol=1e-4, atol=1e-7)
    assert abs(dsum.item() - o.grad.sum().item()) <= 1e-5
