"""Learned warm start for the PCG solve: a small 3D U-Net that maps (log kappa, Y) on a 64^3
grid to an initial guess of u, trained and evaluated with the library's own tensor-core and
memory-bound kernels (libripley_gpu.so, rg_ws_*).

Activations are torch bf16 CUDA tensors of shape (N, D+2, H, W, C): channels-last with one
zero slice before and after every sample along depth, the layout the convolution kernels
read through TMA.  torch only provides the memory; every layer, gradient and optimiser step
is a library kernel.

Network (4 levels, 16/32/48/64 channels, 3x3x3 convolutions with ReLU, average pooling,
nearest upsampling with skip concatenation, 1x1x1 head; bf16 weights and activations, fp32
accumulation, fp32 master weights and Adam state).  The solve keeps its tolerance: the
guess only changes where PCG starts, and the solver drops a guess whose residual exceeds the
right hand side's (rg_diag.guess_rejected).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import torch

from . import _lib as L

BF16 = torch.bfloat16
LEVELS = (16, 32, 48, 64)
IN_CH = 16
WEIGHTS_FILE = os.path.join(os.path.dirname(__file__), "data", "warmstart_unet.npz")


def layer_table():
    """(name, c_in, c_out) of every 3x3x3 convolution, in forward order."""
    c0, c1, c2, c3 = LEVELS
    return [("enc0a", IN_CH, c0), ("enc0b", c0, c0), ("enc1a", c0, c1), ("enc1b", c1, c1),
            ("enc2a", c1, c2), ("enc2b", c2, c2), ("bota", c2, c3), ("botb", c3, c3),
            ("dec2a", c3 + c2, c2), ("dec2b", c2, c2), ("dec1a", c2 + c1, c1), ("dec1b", c1, c1),
            ("dec0a", c1 + c0, c0), ("dec0b", c0, c0)]


# ---------------------------------------------------------------------------------------------
# activations and thin wrappers of the C entry points
# ---------------------------------------------------------------------------------------------

def new_act(n, d, h, w, c, device="cuda"):
    """Zeroed activation tensor (the depth halo slices must stay zero)."""
    return torch.zeros((n, d + 2, h, w, c), dtype=BF16, device=device)


def act_struct(t):
    n, dz, h, w, c = t.shape
    return L.rg_act(t.data_ptr(), n, dz - 2, h, w, c)


def interior(t):
    """View of the interior slices: (N, D, H, W, C)."""
    return t[:, 1:-1]


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _a(t):
    return C.byref(act_struct(t)) if t is not None else None


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
    L.set_stream_from_torch()
    L.check(L.lib().rg_ws_conv3(_a(x), _p(weights), _p(bias), _a(y), int(relu), _a(mask), err.ptr()))
    return y


def conv3_wgrad(x, g, dw, partials, accumulate=False, err=None):
    """dw (fp32 [27][Cout][Cin]) = weight gradient of conv3 for the output gradient g."""
    err = err or DeviceError(x.device)
    L.set_stream_from_torch()
    L.check(L.lib().rg_ws_conv3_wgrad(_a(x), _a(g), _p(dw), _p(partials), partials.numel(),
                                      int(accumulate), err.ptr()))
    return dw


def avgpool(x, out):
    L.check(L.lib().rg_ws_avgpool(_a(x), _a(out)))
    return out


def avgpool_bwd(dout, x, dskip, skip_off, din):
    L.check(L.lib().rg_ws_avgpool_bwd(_a(dout), _a(x), _a(dskip), int(skip_off), _a(din)))
    return din


def upcat(a, b, out):
    L.check(L.lib().rg_ws_upcat(_a(a), _a(b), _a(out)))
    return out


def upcat_bwd(dcat, a, da):
    L.check(L.lib().rg_ws_upcat_bwd(_a(dcat), _a(a), _a(da)))
    return da


def head(x, w, b, out):
    L.check(L.lib().rg_ws_head(_a(x), _p(w), _p(b), _p(out)))
    return out


def head_bwd_x(x, w, dout, dx):
    L.check(L.lib().rg_ws_head_bwd_x(_a(x), _p(w), _p(dout), _a(dx)))
    return dx


def colsum(v, dout, out, work, accumulate=False):
    L.check(L.lib().rg_ws_colsum(_a(v), _p(dout), _p(out), _p(work), int(accumulate)))
    return out


def mse(out, target, dout, loss, dsum, work):
    L.check(L.lib().rg_ws_mse(_p(out), _p(target), out.numel(), _p(dout), _p(loss), _p(dsum), _p(work)))


def h1_loss(out, target, lam, dout, loss, dsum, work):
    n, d, h, w = out.shape
    L.check(L.lib().rg_ws_h1_loss(_p(out), _p(target), n, d, h, w, float(lam), _p(dout), _p(loss), _p(dsum),
                                  _p(work)))


def weights_bf16(w, w_fwd, w_dgrad):
    _, cout, cin = w.shape
    L.check(L.lib().rg_ws_weights_bf16(_p(w), _p(w_fwd), _p(w_dgrad), cout, cin))


# ---------------------------------------------------------------------------------------------
# the network
# ---------------------------------------------------------------------------------------------

class Workspace:
    """Activations and gradients of one batch shape (n samples of d x h x w cells)."""

    def __init__(self, n, d, h, w, device="cuda", train=True):
        for s in (d, h, w):
            if s % 8:
                raise ValueError("network grid sizes must be multiples of 8")
        self.shape = (n, d, h, w)
        c0, c1, c2, c3 = LEVELS
        lv = [(d >> k, h >> k, w >> k) for k in range(4)]

        def A(level, c):
            return new_act(n, *lv[level], c, device=device)

        self.x0 = A(0, IN_CH)
        self.a0, self.s0 = A(0, c0), A(0, c0)
        self.p1, self.a1, self.s1 = A(1, c0), A(1, c1), A(1, c1)
        self.p2, self.a2, self.s2 = A(2, c1), A(2, c2), A(2, c2)
        self.p3, self.a3, self.b3 = A(3, c2), A(3, c3), A(3, c3)
        self.u2, self.d2a, self.d2 = A(2, c3 + c2), A(2, c2), A(2, c2)
        self.u1, self.d1a, self.d1 = A(1, c2 + c1), A(1, c1), A(1, c1)
        self.u0, self.d0a, self.d0 = A(0, c1 + c0), A(0, c0), A(0, c0)
        self.out = torch.zeros((n, d, h, w), dtype=torch.float32, device=device)
        self.train = train
        if train:
            self.target = torch.zeros_like(self.out)
            self.dout = torch.zeros_like(self.out)
            self.g_d0, self.g_d0a, self.dU0 = A(0, c0), A(0, c0), A(0, c1 + c0)
            self.g_d1, self.g_d1a, self.dU1 = A(1, c1), A(1, c1), A(1, c2 + c1)
            self.g_d2, self.g_d2a, self.dU2 = A(2, c2), A(2, c2), A(2, c3 + c2)
            self.g_b3, self.g_a3, self.dP3 = A(3, c3), A(3, c3), A(3, c2)
            self.g_s2, self.g_a2, self.dP2 = A(2, c2), A(2, c2), A(2, c1)
            self.g_s1, self.g_a1, self.dP1 = A(1, c1), A(1, c1), A(1, c0)
            self.g_s0, self.g_a0 = A(0, c0), A(0, c0)


class UNet:
    """Parameters (fp32 master copy, bf16 forward and data-gradient copies, Adam state) and
    the forward/backward passes through the library's kernels."""

    def __init__(self, device="cuda", seed=0):
        self.device = torch.device(device)
        self.layers = layer_table()
        shapes = []
        for name, cin, cout in self.layers:
            shapes += [(name + ".w", (27, cout, cin)), (name + ".b", (cout,))]
        shapes += [("head.w", (LEVELS[0],)), ("head.b", (1,))]
        offs, o = {}, 0
        for key, shp in shapes:
            cnt = int(np.prod(shp))
            offs[key] = (o, cnt, shp)
            o += (cnt + 3) // 4 * 4
        self.count = o
        self.flat = torch.zeros(o, dtype=torch.float32, device=self.device)
        self.grad = torch.zeros_like(self.flat)
        self.m = torch.zeros_like(self.flat)
        self.v = torch.zeros_like(self.flat)
        self.keys = [k for k, _ in shapes]
        self.p = {k: self.flat[a:a + c].view(s) for k, (a, c, s) in offs.items()}
        self.g = {k: self.grad[a:a + c].view(s) for k, (a, c, s) in offs.items()}
        self.wf = {n: torch.zeros((27, co, ci), dtype=BF16, device=self.device) for n, ci, co in self.layers}
        self.wd = {n: torch.zeros((27, ci, co), dtype=BF16, device=self.device) for n, ci, co in self.layers}
        self.step_count = 0
        self.err = DeviceError(self.device)
        self.partials = torch.zeros(1 << 24, dtype=torch.float32, device=self.device)
        self.work = torch.zeros(592 * 128, dtype=torch.float32, device=self.device)
        self.work64 = torch.zeros(2 * 592, dtype=torch.float64, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.init(seed)

    # -- parameters
    def init(self, seed=0):
        """He-normal weights (fan-in 27 c_in; 27 x 5 for the five live input channels), zero
        biases, small head."""
        gen = torch.Generator().manual_seed(seed)
        for name, cin, cout in self.layers:
            fan = 27 * (5 if name == "enc0a" else cin)
            w = torch.randn((27, cout, cin), generator=gen) * math.sqrt(2.0 / fan)
            self.p[name + ".w"].copy_(w)
            self.p[name + ".b"].zero_()
        self.p["head.w"].copy_(torch.randn((LEVELS[0],), generator=gen) * 0.1)
        self.p["head.b"].zero_()
        self.m.zero_()
        self.v.zero_()
        self.step_count = 0
        self.refresh()

    def refresh(self):
        """bf16 copies of the fp32 master weights (forward and flipped/transposed)."""
        L.set_stream_from_torch()
        for name, _, _ in self.layers:
            weights_bf16(self.p[name + ".w"], self.wf[name], self.wd[name])

    def state_dict(self):
        return {k: self.p[k].detach().cpu().numpy().copy() for k in self.keys}

    def load_state_dict(self, d):
        for k in self.keys:
            self.p[k].copy_(torch.as_tensor(np.asarray(d[k]), dtype=torch.float32))
        self.refresh()

    def save(self, path, **meta):
        np.savez(path, **self.state_dict(), **{"meta." + k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path=WEIGHTS_FILE, device="cuda"):
        net = cls(device=device)
        with np.load(path) as z:
            net.load_state_dict({k: z[k] for k in net.keys})
            net.meta = {k[5:]: z[k] for k in z.files if k.startswith("meta.")}
        return net

    # -- passes
    def _conv(self, x, name, y):
        conv3(x, self.wf[name], self.p[name + ".b"], y, relu=True, err=self.err)

    def forward(self, ws):
        """ws.out = network(ws.x0)."""
        L.set_stream_from_torch()
        c = self._conv
        c(ws.x0, "enc0a", ws.a0); c(ws.a0, "enc0b", ws.s0)
        avgpool(ws.s0, ws.p1); c(ws.p1, "enc1a", ws.a1); c(ws.a1, "enc1b", ws.s1)
        avgpool(ws.s1, ws.p2); c(ws.p2, "enc2a", ws.a2); c(ws.a2, "enc2b", ws.s2)
        avgpool(ws.s2, ws.p3); c(ws.p3, "bota", ws.a3); c(ws.a3, "botb", ws.b3)
        upcat(ws.b3, ws.s2, ws.u2); c(ws.u2, "dec2a", ws.d2a); c(ws.d2a, "dec2b", ws.d2)
        upcat(ws.d2, ws.s1, ws.u1); c(ws.u1, "dec1a", ws.d1a); c(ws.d1a, "dec1b", ws.d1)
        upcat(ws.d1, ws.s0, ws.u0); c(ws.u0, "dec0a", ws.d0a); c(ws.d0a, "dec0b", ws.d0)
        head(ws.d0, self.p["head.w"], self.p["head.b"], ws.out)
        return ws.out

    def _bwd(self, name, x, g, dx, mask):
        """weight and bias gradients of layer `name` (input x, masked output gradient g) and,
        when dx is given, the masked gradient reaching x."""
        conv3_wgrad(x, g, self.g[name + ".w"], self.partials, err=self.err)
        colsum(g, None, self.g[name + ".b"], self.work)
        if dx is not None:
            conv3(g, self.wd[name], None, dx, relu=False, mask=mask, err=self.err)

    def loss_and_backward(self, ws, grad_weight=0.0):
        """self.loss = mse(ws.out, ws.target) (+ grad_weight x the squared differences of the
        error between adjacent cells); self.grad = its gradient (forward must have run)."""
        L.set_stream_from_torch()
        if grad_weight > 0:
            h1_loss(ws.out, ws.target, grad_weight, ws.dout, self.loss, self.g["head.b"], self.work64)
        else:
            mse(ws.out, ws.target, ws.dout, self.loss, self.g["head.b"], self.work64)
        colsum(ws.d0, ws.dout, self.g["head.w"], self.work)
        head_bwd_x(ws.d0, self.p["head.w"], ws.dout, ws.g_d0)
        b = self._bwd
        b("dec0b", ws.d0a, ws.g_d0, ws.g_d0a, ws.d0a)
        b("dec0a", ws.u0, ws.g_d0a, ws.dU0, None)
        upcat_bwd(ws.dU0, ws.d1, ws.g_d1)
        b("dec1b", ws.d1a, ws.g_d1, ws.g_d1a, ws.d1a)
        b("dec1a", ws.u1, ws.g_d1a, ws.dU1, None)
        upcat_bwd(ws.dU1, ws.d2, ws.g_d2)
        b("dec2b", ws.d2a, ws.g_d2, ws.g_d2a, ws.d2a)
        b("dec2a", ws.u2, ws.g_d2a, ws.dU2, None)
        upcat_bwd(ws.dU2, ws.b3, ws.g_b3)
        b("botb", ws.a3, ws.g_b3, ws.g_a3, ws.a3)
        b("bota", ws.p3, ws.g_a3, ws.dP3, None)
        avgpool_bwd(ws.dP3, ws.s2, ws.dU2, LEVELS[3], ws.g_s2)
        b("enc2b", ws.a2, ws.g_s2, ws.g_a2, ws.a2)
        b("enc2a", ws.p2, ws.g_a2, ws.dP2, None)
        avgpool_bwd(ws.dP2, ws.s1, ws.dU1, LEVELS[2], ws.g_s1)
        b("enc1b", ws.a1, ws.g_s1, ws.g_a1, ws.a1)
        b("enc1a", ws.p1, ws.g_a1, ws.dP1, None)
        avgpool_bwd(ws.dP1, ws.s0, ws.dU0, LEVELS[1], ws.g_s0)
        b("enc0b", ws.a0, ws.g_s0, ws.g_a0, ws.a0)
        b("enc0a", ws.x0, ws.g_a0, None, None)
        return self.loss

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        L.set_stream_from_torch()
        L.check(L.lib().rg_ws_adam(_p(self.flat), _p(self.grad), _p(self.m), _p(self.v), self.count,
                                   float(lr), float(beta1), float(beta2), float(eps), self.step_count))
        self.refresh()


# ---------------------------------------------------------------------------------------------
# fields <-> network
# ---------------------------------------------------------------------------------------------

class FieldMap:
    """Per-sample normalisation and the maps between per-element fields, network cells and
    the nodal solution (rg_ws_field_stats / pack_input / nodes_to_cells / cells_to_nodes)."""

    def __init__(self, nsamples, fine, factor, device="cuda"):
        self.n = nsamples
        self.fine = tuple(fine)            # (fd, fh, fw) elements of the PDE grid
        self.factor = int(factor)
        self.net = tuple(s // self.factor for s in self.fine)
        self.stats = torch.zeros(4 * nsamples, dtype=torch.float32, device=device)
        self.work = torch.zeros(128 * nsamples, dtype=torch.float64, device=device)

    def pack(self, kappa, y, x0):
        """kappa, y: fp32 per element (n, fd, fh, fw); fills stats and the network input."""
        per = int(np.prod(self.fine))
        h_net = 1.0 / self.net[2]
        L.set_stream_from_torch()
        L.check(L.lib().rg_ws_field_stats(_p(kappa), _p(y), self.n, per, h_net, _p(self.stats), _p(self.work)))
        L.check(L.lib().rg_ws_pack_input(_p(kappa), _p(y), self.factor, _a(x0), _p(self.stats)))

    def targets(self, u_nodes, target):
        d, h, w = self.net
        L.check(L.lib().rg_ws_nodes_to_cells(_p(u_nodes), self.factor, self.n, d, h, w, _p(self.stats),
                                             _p(target)))

    def guess(self, cells, q, u_nodes):
        d, h, w = self.net
        nd, nh, nw = (s + 1 for s in self.fine)
        L.check(L.lib().rg_ws_cells_to_nodes(_p(cells), self.n, d, h, w, _p(self.stats), nd, nh, nw, _p(q),
                                             _p(u_nodes)))


class WarmStart:
    """Initial guesses for Brick problems from a trained network (inference only)."""

    def __init__(self, net: UNet, net_grid=64):
        self.net = net
        self.net_grid = net_grid
        self._ws = {}

    def guess(self, kappa_elem, y_elem, fine, q=None, out=None):
        """Nodal fp64 guess ((fd+1)(fh+1)(fw+1),) for one sample; kappa_elem and y_elem fp32 per
        element (x fastest); q the Dirichlet mask on the nodes (or None)."""
        fine = tuple(int(s) for s in fine)
        factor = max(1, fine[2] // self.net_grid)
        key = (fine, factor)
        if key not in self._ws:
            fm = FieldMap(1, fine, factor, device=self.net.device)
            self._ws[key] = (fm, Workspace(1, *fm.net, device=self.net.device, train=False))
        fm, ws = self._ws[key]
        fm.pack(kappa_elem, y_elem, ws.x0)
        self.net.forward(ws)
        if out is None:
            out = torch.empty(int(np.prod([s + 1 for s in fine])), dtype=torch.float64, device=self.net.device)
        fm.guess(ws.out, q, out)
        return out


# ---------------------------------------------------------------------------------------------
# synthetic problems (GPU)
# ---------------------------------------------------------------------------------------------

def _shape3(ne):
    """(nx, ny, nz) from an edge length or a 3-tuple."""
    return (ne, ne, ne) if isinstance(ne, int) else tuple(int(v) for v in ne)


def gaussian_random_field(n, ne, corr_cells, gen, device="cuda"):
    """n zero-mean, unit-variance fields on ne^3 (or nx x ny x nz) cells: white noise
    smoothed by a periodic Gaussian of standard deviation corr_cells cells,
    (n, nz, ny, nx) fp32, x fastest."""
    nx, ny, nz = _shape3(ne)
    noise = torch.randn((n, nz, ny, nx), generator=gen, device=device, dtype=torch.float32)
    fz = torch.fft.fftfreq(nz, device=device) * (2 * math.pi)
    fy = torch.fft.fftfreq(ny, device=device) * (2 * math.pi)
    fx = torch.fft.rfftfreq(nx, device=device) * (2 * math.pi)
    k2 = fz[:, None, None] ** 2 + fy[None, :, None] ** 2 + fx[None, None, :] ** 2
    g = torch.fft.irfftn(torch.fft.rfftn(noise, dim=(1, 2, 3)) * torch.exp(-0.5 * corr_cells ** 2 * k2),
                         s=(nz, ny, nx), dim=(1, 2, 3))
    g = g - g.mean(dim=(1, 2, 3), keepdim=True)
    # a correlation length of the order of the grid leaves (almost) a constant: zero field
    return g / g.std(dim=(1, 2, 3), keepdim=True).clamp_min(1e-6)


def gaussian_blobs(n, ne, width_cells, gen, nblobs=4, device="cuda"):
    """sum of nblobs Gaussian blobs per sample, amplitudes U(-1, 1), centres uniform in the
    domain, sampled at the element centres of ne^3 (or nx x ny x nz) unit cells scaled to
    the unit cube (cell sizes 1/nx, 1/ny, 1/nz; widths in cells of each axis);
    (n, nz, ny, nx) fp32."""
    nx, ny, nz = _shape3(ne)
    amps = torch.rand((n, nblobs), generator=gen, device=device) * 2 - 1
    ctr = torch.rand((n, nblobs, 3), generator=gen, device=device)
    y = torch.zeros((n, nz, ny, nx), device=device)
    axes = []
    for cnt in (nx, ny, nz):
        axes.append((torch.arange(cnt, device=device, dtype=torch.float32) + 0.5) / cnt)
    for b in range(nblobs):
        f = []
        for d, cnt in enumerate((nx, ny, nz)):
            w2 = 2 * (width_cells / cnt) ** 2
            f.append(torch.exp(-(axes[d][None, :] - ctr[:, b, d:d + 1]) ** 2 / w2))
        y += amps[:, b, None, None, None] * f[2][:, :, None, None] * f[1][:, None, :, None] * f[0][:, None, None, :]
    return y


class BrickProblem:
    """-div(kappa grad u) = Y on a Brick of ne^3 (or nx x ny x nz) elements on [0,1]^3 (each
    axis), u = 0 on the top face z = 1, with kappa and Y per element, assembled and solved
    through the C entry points."""

    def __init__(self, ne, device="cuda"):
        lib = L.lib()
        self.shape = _shape3(ne)
        self.ne = ne
        nx, ny, nz = self.shape
        self.nel = nx * ny * nz
        self.device = torch.device(device)
        self.dom = C.c_void_p()
        L.set_stream_from_torch()
        L.check(lib.rg_domain_create(3, (C.c_int64 * 3)(nx, ny, nz), (C.c_double * 3)(0, 0, 0),
                                     (C.c_double * 3)(1, 1, 1), C.byref(self.dom)))
        n = C.c_int64()
        L.check(lib.rg_domain_info(self.dom, C.byref(n), None, None, None, None))
        self.n = n.value
        self.mat = C.c_void_p()
        L.check(lib.rg_matrix_create(self.dom, C.byref(self.mat)))
        self.rhs = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        self.x = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        self.q = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        self.q[nz * (nx + 1) * (ny + 1):] = 1.0
        self.A = torch.zeros((self.nel, 3, 3), dtype=torch.float64, device=self.device)
        self.Y = torch.zeros(self.nel, dtype=torch.float64, device=self.device)

    def close(self):
        lib = L.lib()
        if self.mat:
            lib.rg_matrix_destroy(self.mat)
            self.mat = None
        if self.dom:
            lib.rg_domain_destroy(self.dom)
            self.dom = None

    def assemble(self, kappa_elem, y_elem=None):
        """Matrix for kappa (per element); right hand side for y_elem when given."""
        lib = L.lib()
        for i in range(3):
            self.A[:, i, i] = kappa_elem.reshape(-1)
        L.set_stream_from_torch()
        L.check(lib.rg_matrix_reset(self.mat))
        self.set_rhs(y_elem if y_elem is not None else torch.zeros(self.nel, device=self.device),
                     with_matrix=True)

    def set_rhs(self, y_elem, with_matrix=False):
        lib = L.lib()
        self.Y.copy_(y_elem.reshape(-1))
        self.rhs.zero_()
        e = L.rg_coef(None, 0)
        cA = L.rg_coef(self.A.data_ptr(), L.RG_COEF_PER_ELEMENT) if with_matrix else e
        cY = L.rg_coef(self.Y.data_ptr(), L.RG_COEF_PER_ELEMENT)
        L.set_stream_from_torch()
        if with_matrix:
            L.check(lib.rg_assemble_single(self.mat, _p(self.rhs), C.byref(cA), C.byref(e), C.byref(e),
                                           C.byref(e), C.byref(e), C.byref(cY)))
            L.check(lib.rg_insert_constraint(self.mat, _p(self.rhs), _p(self.q), None, 0))
        else:
            # right hand side only: the matrix keeps its values and balancing
            L.check(lib.rg_assemble_single(self.mat, _p(self.rhs), C.byref(e), C.byref(e), C.byref(e),
                                           C.byref(e), C.byref(e), C.byref(cY)))
            L.check(lib.rg_insert_constraint(self.mat, _p(self.rhs), _p(self.q), None, 1))

    def solve(self, tol=1e-8, fp32=True, guess=None, iter_max=100000, guess_sweeps=0):
        lib = L.lib()
        o = L.rg_solver_opts()
        lib.rg_solver_opts_default(C.byref(o))
        o.tolerance = tol
        o.iter_max = iter_max
        o.mode = L.RG_MODE_STANDARD
        o.precision = L.RG_PREC_FP32_REFINE if fp32 else L.RG_PREC_FP64
        o.layout = L.RG_LAYOUT_BAND if fp32 else L.RG_LAYOUT_CSR
        if guess is not None:
            o.initial_guess = guess.data_ptr()
            o.guess_sweeps = guess_sweeps
        d = L.rg_diag()
        L.set_stream_from_torch()
        L.check(lib.rg_solve(self.mat, _p(self.rhs), _p(self.x), C.byref(o), C.byref(d)))
        return d
