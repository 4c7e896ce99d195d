"""Parity at the benchmark configurations: Brick 64^3 and Brick 128^3 built by the benchmark's
own generator (bench.make_inputs, seed 2026: kappa = exp(Gaussian random field), four Gaussian
blobs for Y, u = 0 on the top face), and instances of the batched workload (bench's
make_batch generator, same seed).  Everything runs through the C-ABI and is compared with the
oracle on the same inputs:

  * CSR pattern: bit-exact;
  * assembled values: |gpu - oracle| <= 1e-13 * max|row| per row; rhs 1e-13 * max|rhs|
    (the GPU gets A per element, as the benchmark passes it; the oracle gets A expanded to the
    Gauss points, the form the reference's DefaultAssembler3D reads);
  * paso PCG in FP64 at tol 1e-10 (CSR and FP64 band layouts): solution within 1e-8
    (relative l2) of the oracle's paso solve at tol 1e-10, iterations within +-1 (the
    reference's own Solver.cpp:46-330 / PCG.cpp:62-367 arithmetic order);
  * textbook FP64 PCG on the band copy and FP32-inner / FP64-refinement PCG at tol 1e-10:
    within 1e-8 of that oracle solution;
  * the benchmark's timed path (learned warm start + FP32 refinement) at the benchmark's
    tolerance 1e-8: its stopping test holds in FP64 and its error against the oracle solution
    is below 1e-6 (measured: ~2e-9 at 128^3);
  * batched instances (FP32 inner / FP64 refinement, all right hand sides of a system in one
    batch) at tol 1e-10 within 1e-8 of the oracle's paso solve of each right hand side.
"""
import numpy as np
import pytest
import torch

import bench
from oracle import oracle as O
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

ASM_TOL = 1e-13
SEED = 2026


def row_scaled_err(ptr, a, b):
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    m = np.zeros(len(ptr) - 1)
    np.maximum.at(m, rows, np.abs(b))
    m = np.maximum(m, 1e-300)
    return float((np.abs(a - b) / m[rows]).max())


class BenchSystem:
    """One benchmark input on the GPU (matrix assembled per element, constrained) and in the
    oracle (values, rhs, and the paso solve at tol 1e-10)."""

    def __init__(self, ne):
        self.ne = ne
        inp = bench.make_inputs(ne, SEED, 8.0 * ne / 128.0)
        self.inp = inp
        nel = ne ** 3
        d = R.Domain(3, (ne, ne, ne))
        self.d = d
        self.keep = []
        A_pe = np.zeros((nel, 3, 3))
        for i in range(3):
            A_pe[:, i, i] = inp["kappa"]
        self.A_pe = A_pe.reshape(-1)
        self.q = R.dev(inp["q"])
        self.m = R.Matrix(d)
        self.rhs = self.assemble(self.m)
        pat = O.pattern(3, (ne, ne, ne))
        A = np.zeros((nel, 8, 3, 3))
        for i in range(3):
            A[:, :, i, i] = inp["kappa"][:, None]
        val, rr = O.assemble(3, (ne, ne, ne), d.dx, pat, A=(O.EXPANDED, A.reshape(-1)), Y=(O.EXPANDED, inp["Y"]))
        del A
        O.insert_constraint(pat, val, rr, inp["q"])
        self.pat, self.val, self.rr = pat, val, rr
        self.ref = O.solve_paso(pat, val.copy(), rr, tol=1e-10)
        assert self.ref.converged

    def assemble(self, m):
        rhs = torch.zeros(self.d.n, dtype=torch.float64, device="cuda")
        R.assemble(m, rhs, self.keep, A=(self.A_pe, R.KINDS["elem"]), Y=(self.inp["Y"], R.KINDS["exp"]))
        R.insert_constraint(m, rhs, self.q)
        return rhs

    def err(self, x):
        return float(np.linalg.norm(x.cpu().numpy() - self.ref.x) / np.linalg.norm(self.ref.x))


_systems = {}


@pytest.fixture(scope="module", params=[64, 128], ids=["brick64", "brick128"])
def bsys(request, cuda):
    ne = request.param
    if ne not in _systems:
        _systems.clear()  # one configuration in memory at a time
        _systems[ne] = BenchSystem(ne)
    return _systems[ne]


def test_pattern_and_values_match_oracle(bsys):
    p, i = bsys.d.pattern()
    assert np.array_equal(p, bsys.pat.ptr)
    assert np.array_equal(i, bsys.pat.idx)
    assert row_scaled_err(bsys.pat.ptr, bsys.m.values(), bsys.val) < ASM_TOL
    rr = bsys.rr
    assert np.abs(bsys.rhs.cpu().numpy() - rr).max() <= ASM_TOL * np.abs(rr).max()


@pytest.mark.parametrize("layout", [L.RG_LAYOUT_CSR, L.RG_LAYOUT_BAND], ids=["csr", "band"])
def test_paso_fp64_solution_matches_oracle(bsys, layout):
    m = R.Matrix(bsys.d)
    rhs = bsys.assemble(m)
    x = torch.zeros(bsys.d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, layout=layout))
    assert st == 0 and dg.converged
    assert bsys.err(x) < 1e-8, bsys.err(x)
    assert abs(int(dg.num_iter) - bsys.ref.num_iter) <= 1, (int(dg.num_iter), bsys.ref.num_iter)


@pytest.mark.parametrize("precision", [L.RG_PREC_FP64, L.RG_PREC_FP32_REFINE], ids=["fp64", "fp32_refine"])
def test_standard_and_mixed_precision_solutions_match_oracle(bsys, precision):
    m = R.Matrix(bsys.d)
    rhs = bsys.assemble(m)
    x = torch.zeros(bsys.d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, mode=L.RG_MODE_STANDARD, precision=precision,
                                       layout=L.RG_LAYOUT_BAND))
    assert st == 0 and dg.converged
    assert dg.residual_norm <= 1e-10 * dg.rhs_norm * (1 + 1e-12)
    assert bsys.err(x) < 1e-8, bsys.err(x)


def test_benchmark_timed_path_matches_oracle(bsys):
    """The benchmark's timed path as bench.py runs it: the network's guess (fields per
    element through rg_ws_element_fields, Chebyshev-smoothed in the solver) and the FP32
    refinement to the benchmark's tolerance."""
    from esys_b200 import warmstart as WS
    ne = bsys.ne
    nel = ne ** 3
    warm = WS.WarmStart(WS.UNet.load(device="cuda"))
    A_d = R.dev(bsys.A_pe)
    Y_d = R.dev(bsys.inp["Y"])
    kap = torch.empty((1, ne, ne, ne), dtype=torch.float32, device="cuda")
    y32 = torch.empty_like(kap)
    L.set_stream_from_torch()
    lib = R.lib()
    L.check(lib.rg_ws_element_fields(R.ptr(A_d), 9, R.ptr(Y_d), 8, nel, R.ptr(kap), R.ptr(y32)))
    assert torch.equal(kap.view(-1).double(), A_d.view(-1, 9)[:, 0].float().double())
    assert torch.allclose(y32.view(-1).double(), Y_d.view(-1, 8).mean(dim=1), rtol=1e-6, atol=1e-7)
    guess = torch.zeros(bsys.d.n, dtype=torch.float64, device="cuda")
    warm.guess(kap, y32, (ne, ne, ne), q=bsys.q, out=guess)
    m = R.Matrix(bsys.d)
    rhs = bsys.assemble(m)
    x = torch.zeros(bsys.d.n, dtype=torch.float64, device="cuda")
    o = R.opts(tolerance=bench.RTOL, mode=L.RG_MODE_STANDARD, precision=L.RG_PREC_FP32_REFINE,
               layout=L.RG_LAYOUT_BAND)
    o.initial_guess = guess.data_ptr()
    o.guess_sweeps = 8
    st, dg = R.solve(m, rhs, x, o)
    assert st == 0 and dg.converged
    assert dg.residual_norm <= bench.RTOL * dg.rhs_norm * (1 + 1e-12)
    assert bsys.err(x) < 1e-6, bsys.err(x)


def test_batched_instances_match_oracle(cuda):
    """The first two systems of the benchmark's batched workload (make_batch reproduces the
    benchmark batch's first systems exactly for the same seed), all 8 right hand sides each,
    solved in one batch at tol 1e-10 against the oracle's paso solves."""
    from esys_b200.batch import BatchSolver, make_batch
    systems, rhs = make_batch(2, 8, seed=SEED)
    xs = [torch.zeros_like(b) for b in rhs]
    with BatchSolver([s.mat for s in systems], 8) as bs:
        diags = bs.solve(rhs, xs, tol=1e-10)
    for i, s in enumerate(systems):
        shape = s.shape
        nel = s.nel
        kappa = s.A[:, 0, 0].cpu().numpy()
        pat = O.pattern(3, shape)
        A = np.zeros((nel, 3, 3))
        for c in range(3):
            A[:, c, c] = kappa
        dx = [1.0 / v for v in shape]
        val, _ = O.assemble(3, shape, dx, pat, A=(O.PER_ELEMENT, A.reshape(-1)))
        q = s.q.cpu().numpy()
        O.insert_constraint(pat, val, np.zeros(pat.n), q)
        for k in range(8):
            assert diags[i * 8 + k].converged
            b = rhs[i][k].cpu().numpy()
            ref = O.solve_paso(pat, val.copy(), b, tol=1e-10)
            assert ref.converged
            err = np.linalg.norm(xs[i][k].cpu().numpy() - ref.x) / np.linalg.norm(ref.x)
            assert err < 1e-8, (i, k, shape, err)
    for s in systems:
        s.close()
