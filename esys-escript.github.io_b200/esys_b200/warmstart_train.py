"""Training of the warm-start network on the GPU.

Data: seeded (kappa, Y) pairs on Brick 64^3 (kappa = exp(g), g a unit-variance Gaussian random
field; Y = 4 Gaussian blobs), each solved by the library's GPU PCG to rtol 1e-10.  Half of the
kappa fields have a correlation length of 8 cells with blobs 3 cells wide (the 64^3
problems), half 4 cells with blobs 1.5 cells wide (what a 128^3 problem with 8-cell
correlation and 3-cell blobs looks like after 2x coarsening).  Several right hand sides share
one kappa (one assembly and balancing per kappa).

    python -m esys_b200.warmstart_train --samples 20000 --epochs 4 --out weights.npz

Every layer, gradient and Adam step runs in libripley_gpu.so; torch holds the memory and
draws the random fields.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import warmstart as W

NET = 64


def generate(nsamples, rhs_per_kappa, seed, device="cuda", tol=1e-10, log=print, time_limit=None):
    """(x (n, 64, 64, 64, 2) bf16 network inputs, t (n, 64, 64, 64) fp32 targets, info)."""
    gen = torch.Generator(device=device).manual_seed(seed)
    prob = W.BrickProblem(NET, device=device)
    fm = W.FieldMap(1, (NET,) * 3, 1, device=device)
    x_tmp = W.new_act(1, NET, NET, NET, W.IN_CH, device=device)
    xs = torch.zeros((nsamples, NET, NET, NET, 2), dtype=torch.bfloat16, device=device)
    ts = torch.zeros((nsamples, NET, NET, NET), dtype=torch.float32, device=device)
    iters, t0, i = [], time.time(), 0
    while i < nsamples:
        fine_scale = (i // rhs_per_kappa) % 2 == 1
        corr, width = (4.0, 1.5) if fine_scale else (8.0, 3.0)
        kappa = torch.exp(W.gaussian_random_field(1, NET, corr, gen, device=device))[0]
        ys = W.gaussian_blobs(rhs_per_kappa, NET, width, gen, device=device)
        prob.assemble(kappa.double(), ys[0].double())
        for r in range(rhs_per_kappa):
            if i >= nsamples:
                break
            if r:
                prob.set_rhs(ys[r].double())
            d = prob.solve(tol=tol, fp32=False)
            if not d.converged:
                raise RuntimeError(f"training solve {i} did not converge")
            iters.append(int(d.num_iter))
            fm.pack(kappa[None], ys[r][None], x_tmp)
            xs[i] = W.interior(x_tmp)[0, ..., :2]
            fm.targets(prob.x, ts[i:i + 1])
            i += 1
        if log and (i // rhs_per_kappa) % 200 == 0:
            log(f"generated {i}/{nsamples} samples, {time.time() - t0:.1f} s, mean PCG iterations "
                f"{np.mean(iters):.0f}")
        if time_limit and time.time() - t0 > time_limit:
            xs, ts = xs[:i], ts[:i]
            break
    torch.cuda.synchronize()
    prob.close()
    return xs, ts, {"samples": int(xs.shape[0]), "gen_s": time.time() - t0, "mean_iters": float(np.mean(iters)),
                    "tol": tol, "rhs_per_kappa": rhs_per_kappa, "seed": seed}


def cell_centres(ne, device="cuda"):
    """(ne, ne, ne, 3) cell-centre coordinates (z, y, x) in the unit cube: the input channels
    2..4 that rg_ws_pack_input writes."""
    c = (torch.arange(ne, device=device, dtype=torch.float32) + 0.5) / ne
    z, y, x = torch.meshgrid(c, c, c, indexing="ij")
    return torch.stack([z, y, x], dim=-1)


def train(net, xs, ts, epochs, batch, lr, val_frac=0.02, log=print, time_limit=None, seed=0, grad_weight=0.0,
          warmup=300):
    """Adam with a linear warm-up over `warmup` steps and a cosine decay to 1% of lr."""
    n = xs.shape[0]
    nval = max(batch, int(n * val_frac)) if n > 4 * batch else 0
    ntr = n - nval
    ws = W.Workspace(batch, NET, NET, NET, device=net.device)
    steps = max(1, epochs * ntr // batch)
    g = torch.Generator(device="cpu").manual_seed(seed)
    t0, step, hist = time.time(), 0, []
    W.interior(ws.x0).zero_()
    W.interior(ws.x0)[..., 2:5].copy_(cell_centres(NET, net.device).to(torch.bfloat16))
    while step < steps:
        perm = torch.randperm(ntr, generator=g)
        for b0 in range(0, ntr - batch + 1, batch):
            idx = perm[b0:b0 + batch].to(net.device)
            W.interior(ws.x0)[..., :2].copy_(xs.index_select(0, idx))
            ws.target.copy_(ts.index_select(0, idx))
            net.forward(ws)
            net.loss_and_backward(ws, grad_weight)
            cur = lr * 0.5 * (1 + math.cos(math.pi * step / steps)) * min(1.0, (step + 1) / max(warmup, 1))
            net.adam_step(max(cur, lr * 0.01))
            step += 1
            if step % 200 == 0 or step == steps:
                loss = net.loss.item()
                hist.append((step, loss))
                if log:
                    log(f"step {step}/{steps} loss {loss:.4e} lr {cur:.2e} {time.time() - t0:.1f} s")
            if step >= steps or (time_limit and time.time() - t0 > time_limit):
                steps = step
                break
    torch.cuda.synchronize()
    net.err.check()
    train_s = time.time() - t0
    val = None
    if nval:
        num = den = 0.0
        for b0 in range(ntr, n - batch + 1, batch):
            W.interior(ws.x0)[..., :2].copy_(xs[b0:b0 + batch])
            net.forward(ws)
            tt = ts[b0:b0 + batch]
            num += float(((ws.out - tt) ** 2).sum())
            den += float((tt ** 2).sum())
        val = math.sqrt(num / max(den, 1e-30))
    return {"steps": steps, "batch": batch, "train_s": train_s, "ms_per_step": 1e3 * train_s / max(steps, 1),
            "val_rel_l2": val, "loss_history": hist}


def evaluate(net, ne, nprob, seed, tol=1e-8, corr=8.0, width=3.0, device="cuda", log=print, sweeps=(0, 4, 16)):
    """A/B on fresh seeded problems of ne^3 elements (kappa correlation `corr` cells, blobs
    `width` cells wide): PCG (FP32 inner, FP64 refinement) from zero and from the network's
    guess, to the same tolerance.  Times are CUDA-event times of guess + solve."""
    gen = torch.Generator(device=device).manual_seed(seed)
    prob = W.BrickProblem(ne, device=device)
    ws = W.WarmStart(net)
    guess = torch.zeros(prob.n, dtype=torch.float64, device=device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    rows = []
    for k in range(nprob):
        kappa = torch.exp(W.gaussian_random_field(1, ne, corr, gen, device=device))[0]
        y = W.gaussian_blobs(1, ne, width, gen, device=device)[0]
        prob.assemble(kappa.double(), y.double())
        prob.solve(tol=tol)                         # balances the matrix (set-up out of the timing)
        ev[0].record()
        d0 = prob.solve(tol=tol)
        ev[1].record()
        x0 = prob.x.clone()
        row = {"zero_iters": int(d0.num_iter), "zero_ms": ev[0].elapsed_time(ev[1])}
        for sw in sweeps:
            ev[2].record()
            ws.guess(kappa[None], y[None], (ne,) * 3, q=prob.q, out=guess)
            d1 = prob.solve(tol=tol, guess=guess, guess_sweeps=sw)
            ev[3].record()
            torch.cuda.synchronize()
            row.update({f"warm{sw}_iters": int(d1.num_iter), f"warm{sw}_ms": ev[2].elapsed_time(ev[3]),
                        f"guess{sw}_rel_residual": d1.guess_residual / d1.rhs_norm,
                        f"rejected{sw}": bool(d1.guess_rejected),
                        f"diff{sw}": float((prob.x - x0).norm() / x0.norm())})
        row["guess_rel_error"] = float((guess - x0).norm() / x0.norm())
        rows.append(row)
        if log:
            log(json.dumps({"ne": ne, "problem": k, **row}))
    prob.close()
    agg = {k: float(np.mean([r[k] for r in rows])) for k in rows[0]}
    agg["n"] = nprob
    return agg, rows


def _residual(prob, x):
    import ctypes as C
    from . import _lib as L
    l2, lm = C.c_double(), C.c_double()
    L.check(L.lib().rg_residual_norms(prob.mat, C.c_void_p(prob.rhs.data_ptr()), C.c_void_p(x.data_ptr()),
                                      C.byref(l2), C.byref(lm)))
    return l2.value, lm.value


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--rhs-per-kappa", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--gen-time-limit", type=float, default=None)
    ap.add_argument("--train-time-limit", type=float, default=None)
    ap.add_argument("--out", default=W.WEIGHTS_FILE)
    ap.add_argument("--evaluate", metavar="WEIGHTS", default=None,
                    help="only evaluate trained weights: A/B against the zero guess at 64^3 and 128^3")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if a.evaluate:
        net = W.UNet.load(a.evaluate)
        for ne, npb in ((64, 6), (128, 3)):
            agg, _ = evaluate(net, ne, npb, 99 + ne, log=None, sweeps=(0, 4, 8, 16))
            print(json.dumps({"ne": ne, **agg}), flush=True)
        return
    xs, ts, info = generate(a.samples, a.rhs_per_kappa, a.seed, time_limit=a.gen_time_limit)
    print(json.dumps({"data": info}), flush=True)
    net = W.UNet(seed=a.seed)
    res = train(net, xs, ts, a.epochs, a.batch, a.lr, time_limit=a.train_time_limit, seed=a.seed)
    res_s = {k: v for k, v in res.items() if k != "loss_history"}
    print(json.dumps({"train": res_s}), flush=True)
    net.save(a.out, samples=info["samples"], gen_seed=a.seed, steps=res["steps"], batch=a.batch,
             val_rel_l2=res["val_rel_l2"] if res["val_rel_l2"] is not None else -1.0,
             loss_history=np.array(res["loss_history"], dtype=np.float64).reshape(-1, 2))
    print(json.dumps({"saved": a.out}), flush=True)


if __name__ == "__main__":
    main()
