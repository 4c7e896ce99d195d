"""Batched solves of many independent Brick/Rectangle systems with several right hand sides
each (rg_batch_*): one set of launches advances every system, chunks of iterations replay as
CUDA graphs, grid sizes come from the library's autotuner.

    systems = [BrickProblem((32, 48, 64)), BrickProblem((96, 32, 80)), ...]   # assembled
    with BatchSolver([s.mat for s in systems], nrhs=8) as bs:
        diags = bs.solve(rhs_list, x_list, tol=1e-8)

rhs_list[i] / x_list[i] are float64 CUDA tensors of shape (nrhs, n_i) (right hand side k in
row k).  The solve is PCG + Jacobi with FP32 inner iterations and FP64 refinement per right
hand side, stopped by paso's dual-norm test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from . import warmstart as W


# the batched SpMV kernels (rg_batch_info / rg_batch_set_spmv numbering): one row per
# thread, two rows per thread
_SPMV_KERNELS = ("row", "pair")


class BatchSolver:
    def __init__(self, mats, nrhs):
        self.nsys = len(mats)
        self.nrhs = int(nrhs)
        arr = (C.c_void_p * self.nsys)(*[m.value if isinstance(m, C.c_void_p) else m for m in mats])
        self._h = C.c_void_p()
        L.set_stream_from_torch()
        L.check(L.lib().rg_batch_create(arr, self.nsys, self.nrhs, C.byref(self._h)))

    def close(self):
        if self._h:
            L.lib().rg_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            self.close()

    def tune(self):
        L.set_stream_from_torch()
        L.check(L.lib().rg_batch_tune(self._h))
        return self.info()

    def info(self):
        rows, tiles = C.c_int64(), C.c_int64()
        grp, gs, gu, ch, kind = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        us = C.c_double()
        L.check(L.lib().rg_batch_info(self._h, C.byref(rows), C.byref(tiles), C.byref(grp), C.byref(gs),
                                      C.byref(gu), C.byref(ch), C.byref(us), C.byref(kind)))
        return {"rows": rows.value, "tiles": tiles.value, "group": grp.value, "grid_spmv": gs.value,
                "grid_update": gu.value, "chunk": ch.value, "iter_us": us.value,
                "spmv_kernel": _SPMV_KERNELS[kind.value]}

    def set_spmv(self, kernel):
        """Restricts the tuner to one SpMV kernel: None (any) or a name of _SPMV_KERNELS."""
        k = -1 if kernel is None else _SPMV_KERNELS.index(kernel)
        L.check(L.lib().rg_batch_set_spmv(self._h, k))

    def solve(self, rhs, x, tol=1e-8, iter_max=100000, inner_tolerance=1e-2, accept_failure=False):
        """Solves all systems; returns the list of rg_diag (system-major)."""
        lib = L.lib()
        if len(rhs) != self.nsys or len(x) != self.nsys:
            raise ValueError("one right hand side array and one solution array per system")
        for t in list(rhs) + list(x):
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.shape[0] != self.nrhs:
                raise ValueError("arrays must be contiguous float64 CUDA tensors of shape (nrhs, n)")
        o = L.rg_solver_opts()
        lib.rg_solver_opts_default(C.byref(o))
        o.tolerance = tol
        o.iter_max = iter_max
        o.inner_tolerance = inner_tolerance
        o.accept_convergence_failure = int(accept_failure)
        rp = (C.c_void_p * self.nsys)(*[t.data_ptr() for t in rhs])
        xp = (C.c_void_p * self.nsys)(*[t.data_ptr() for t in x])
        diags = (L.rg_diag * (self.nsys * self.nrhs))()
        L.set_stream_from_torch()
        L.check(lib.rg_batch_solve(self._h, rp, xp, C.byref(o), diags))
        return list(diags)


def make_batch(nsys, nrhs, edges=(32, 48, 64, 80, 96), corr_cells=8.0, width_cells=3.0, seed=0,
               device="cuda"):
    """Seeded Brick systems with edge lengths drawn per axis from `edges`, kappa = exp(GRF with
    correlation `corr_cells` cells), u = 0 on the top face, and nrhs right hand sides each from
    4 Gaussian density-anomaly blobs `width_cells` wide.  Returns (systems, rhs list)."""
    gen = torch.Generator(device=device).manual_seed(seed)
    rng = np.random.default_rng(seed)
    systems, rhs = [], []
    for _ in range(nsys):
        shape = tuple(int(v) for v in rng.choice(edges, size=3))
        prob = W.BrickProblem(shape, device=device)
        kappa = torch.exp(W.gaussian_random_field(1, shape, corr_cells, gen, device=device))[0]
        ys = W.gaussian_blobs(nrhs, shape, width_cells, gen, device=device)
        prob.assemble(kappa.double(), ys[0].double())
        b = torch.empty((nrhs, prob.n), dtype=torch.float64, device=device)
        b[0].copy_(prob.rhs)
        for k in range(1, nrhs):
            prob.set_rhs(ys[k].double())
            b[k].copy_(prob.rhs)
        systems.append(prob)
        rhs.append(b)
    return systems, rhs


def main(argv=None):
    """python -m esys_b200.batch [--systems 64] [--nrhs 8] [--seed 0] [--tol 1e-8]: builds a
    seeded batch (make_batch), tunes, solves it twice and prints one JSON line."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="batched Brick solves")
    ap.add_argument("--systems", type=int, default=64)
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tol", type=float, default=1e-8)
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    t0 = time.time()
    systems, rhs = make_batch(a.systems, a.nrhs, seed=a.seed)
    xs = [torch.zeros_like(b) for b in rhs]
    with BatchSolver([s.mat for s in systems], a.nrhs) as bs:
        info = bs.tune()
        bs.solve(rhs, xs, tol=a.tol)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d = bs.solve(rhs, xs, tol=a.tol)
        e1.record()
        torch.cuda.synchronize()
    its = [x.num_iter for x in d]
    print(json.dumps({"systems": a.systems, "nrhs": a.nrhs, "ms": e0.elapsed_time(e1),
                      "setup_s": time.time() - t0, "all_converged": all(x.converged for x in d),
                      "iterations": [min(its), float(np.mean(its)), max(its)], **info}))
    for s in systems:
        s.close()


if __name__ == "__main__":
    main()
