"""CPU oracle (test infrastructure only) of the warm-start network: float64 numpy forward
and backward passes of the 4-level 3D U-Net that maps (log kappa, Y) to an initial guess.

The network has no counterpart in the reference (esys-escript solves from a zero or user
guess; paso/src/Solver.cpp:181 starts from the Jacobi step); it is restated here from its
definition so that the GPU training kernels' gradients can be checked:

* activations (N, D, H, W, C), channels last; every 3x3x3 convolution pads with zeros and is
  followed by ReLU; weights (27, C_out, C_in) with tap = kw + 3 kh + 9 kd, i.e. the output at
  p reads the input at p + (kd - 1, kh - 1, kw - 1);
* encoder: two convolutions per level at 16, 32, 48 channels, 2x2x2 average pooling between
  levels, two 64-channel convolutions at the bottom;
* decoder: nearest-neighbour 2x upsampling, concatenation [upsampled, skip], two
  convolutions per level back to 48, 32, 16 channels;
* head: 1x1x1 convolution 16 -> 1 without activation; loss = mean squared error.

Only tests import this module.
"""
from __future__ import annotations

import numpy as np

LEVELS = (16, 32, 48, 64)
IN_CH = 16


def layer_table():
    c0, c1, c2, c3 = LEVELS
    return [("enc0a", IN_CH, c0), ("enc0b", c0, c0), ("enc1a", c0, c1), ("enc1b", c1, c1),
            ("enc2a", c1, c2), ("enc2b", c2, c2), ("bota", c2, c3), ("botb", c3, c3),
            ("dec2a", c3 + c2, c2), ("dec2b", c2, c2), ("dec1a", c2 + c1, c1), ("dec1b", c1, c1),
            ("dec0a", c1 + c0, c0), ("dec0b", c0, c0)]


def _taps():
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                yield kw + 3 * kh + 9 * kd, kd, kh, kw


def conv3(x, w, b):
    """zero-padded 3x3x3 convolution: y[p] = b + sum_tap w[tap] @ x[p + off(tap)]."""
    n, d, h, ww, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    y = np.broadcast_to(b, (n, d, h, ww, w.shape[1])).copy()
    for tap, kd, kh, kw in _taps():
        y += xp[:, kd:kd + d, kh:kh + h, kw:kw + ww, :] @ w[tap].T
    return y


def conv3_backward(x, w, g):
    """gradients of conv3 for the output gradient g: (dx, dw, db)."""
    n, d, h, ww, cin = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    g2 = g.reshape(-1, g.shape[-1])
    for tap, kd, kh, kw in _taps():
        xs = xp[:, kd:kd + d, kh:kh + h, kw:kw + ww, :]
        dw[tap] = g2.T @ xs.reshape(-1, cin)
        dxp[:, kd:kd + d, kh:kh + h, kw:kw + ww, :] += g @ w[tap]
    return dxp[:, 1:-1, 1:-1, 1:-1, :], dw, g2.sum(axis=0)


def pool(x):
    n, d, h, w, c = x.shape
    return x.reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4, 6))


def pool_backward(g):
    return np.repeat(np.repeat(np.repeat(g, 2, axis=1), 2, axis=2), 2, axis=3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def up_backward(g):
    n, d, h, w, c = g.shape
    return g.reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4, 6))


def relu(x):
    return np.maximum(x, 0.0)


def forward(params, x):
    """Returns (output (N, D, H, W), cache of activations)."""
    a = {"x0": x}

    def cr(name, src, dst):
        a[dst] = relu(conv3(a[src], params[name + ".w"], params[name + ".b"]))

    cr("enc0a", "x0", "a0"); cr("enc0b", "a0", "s0")
    a["p1"] = pool(a["s0"]); cr("enc1a", "p1", "a1"); cr("enc1b", "a1", "s1")
    a["p2"] = pool(a["s1"]); cr("enc2a", "p2", "a2"); cr("enc2b", "a2", "s2")
    a["p3"] = pool(a["s2"]); cr("bota", "p3", "a3"); cr("botb", "a3", "b3")
    a["u2"] = np.concatenate([up(a["b3"]), a["s2"]], axis=-1); cr("dec2a", "u2", "d2a"); cr("dec2b", "d2a", "d2")
    a["u1"] = np.concatenate([up(a["d2"]), a["s1"]], axis=-1); cr("dec1a", "u1", "d1a"); cr("dec1b", "d1a", "d1")
    a["u0"] = np.concatenate([up(a["d1"]), a["s0"]], axis=-1); cr("dec0a", "u0", "d0a"); cr("dec0b", "d0a", "d0")
    out = a["d0"] @ params["head.w"] + params["head.b"][0]
    return out, a


def loss_and_grads(params, x, target):
    """MSE loss and the gradient of every parameter (same keys as params)."""
    out, a = forward(params, x)
    e = out - target
    loss = float(np.mean(e * e))
    dout = 2.0 * e / e.size
    grads = {"head.w": np.tensordot(a["d0"], dout, axes=([0, 1, 2, 3], [0, 1, 2, 3])),
             "head.b": np.array([dout.sum()])}

    def back(name, src, dst, gout):
        """gradient through relu(conv(src)) whose output is a[dst]; returns d src."""
        g = gout * (a[dst] > 0)
        dx, dw, db = conv3_backward(a[src], params[name + ".w"], g)
        grads[name + ".w"] = dw
        grads[name + ".b"] = db
        return dx

    g = dout[..., None] * params["head.w"]
    g = back("dec0b", "d0a", "d0", g)
    du0 = back("dec0a", "u0", "d0a", g)
    c1 = LEVELS[1]
    g = back("dec1b", "d1a", "d1", up_backward(du0[..., :c1]))
    du1 = back("dec1a", "u1", "d1a", g)
    c2 = LEVELS[2]
    g = back("dec2b", "d2a", "d2", up_backward(du1[..., :c2]))
    du2 = back("dec2a", "u2", "d2a", g)
    c3 = LEVELS[3]
    g = back("botb", "a3", "b3", up_backward(du2[..., :c3]))
    dp3 = back("bota", "p3", "a3", g)
    g = back("enc2b", "a2", "s2", pool_backward(dp3) + du2[..., c3:])
    dp2 = back("enc2a", "p2", "a2", g)
    g = back("enc1b", "a1", "s1", pool_backward(dp2) + du1[..., c2:])
    dp1 = back("enc1a", "p1", "a1", g)
    g = back("enc0b", "a0", "s0", pool_backward(dp1) + du0[..., c1:])
    back("enc0a", "x0", "a0", g)
    return loss, grads, out
