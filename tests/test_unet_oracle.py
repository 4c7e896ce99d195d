"""The CPU oracle of the warm-start network checks itself: its analytic gradients against
central finite differences of its own loss (float64, tiny grid)."""
import numpy as np

from oracle import unet_oracle as U


def _params(rng):
    p = {}
    for name, cin, cout in U.layer_table():
        p[name + ".w"] = rng.standard_normal((27, cout, cin)) * np.sqrt(2.0 / (27 * cin))
        p[name + ".b"] = rng.standard_normal(cout) * 0.1
    p["head.w"] = rng.standard_normal(U.LEVELS[0]) * 0.3
    p["head.b"] = np.array([0.05])
    return p


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    p = _params(rng)
    x = rng.standard_normal((1, 8, 8, 8, U.IN_CH))
    t = rng.standard_normal((1, 8, 8, 8))
    loss, grads, _ = U.loss_and_grads(p, x, t)
    assert set(grads) == set(p)
    eps = 1e-6
    for key in ["enc0a.w", "enc1b.w", "bota.w", "botb.b", "dec2a.w", "dec1b.b", "dec0a.w", "head.w", "head.b"]:
        flat = p[key].reshape(-1)
        for i in rng.choice(flat.size, size=min(3, flat.size), replace=False):
            old = flat[i]
            flat[i] = old + eps
            lp = U.loss_and_grads(p, x, t)[0]
            flat[i] = old - eps
            lm = U.loss_and_grads(p, x, t)[0]
            flat[i] = old
            fd = (lp - lm) / (2 * eps)
            an = grads[key].reshape(-1)[i]
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(fd)), (key, i, fd, an)


def test_oracle_conv_matches_direct_sum():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((1, 3, 4, 5, 2))
    w = rng.standard_normal((27, 3, 2))
    b = rng.standard_normal(3)
    y = U.conv3(x, w, b)
    # direct definition at one interior and one corner position
    for (d, h, ww) in [(1, 2, 2), (0, 0, 4)]:
        ref = b.copy()
        for kd in range(3):
            for kh in range(3):
                for kw in range(3):
                    dd, hh, wx = d + kd - 1, h + kh - 1, ww + kw - 1
                    if 0 <= dd < 3 and 0 <= hh < 4 and 0 <= wx < 5:
                        ref += w[kw + 3 * kh + 9 * kd] @ x[0, dd, hh, wx]
        assert np.allclose(y[0, d, h, ww], ref, rtol=1e-12, atol=1e-12)
