"""GPU parity tests through the C-ABI: the CUDA path against the oracle and against the
reference's own outputs (golden vectors).

Tolerances:
  * pattern: bit-exact;
  * assembled values: |gpu - ref| <= 1e-13 * max|row| per row (rhs: 1e-13 * max|rhs|);
  * solutions: paso mode at tol 1e-10 within 1e-8 relative of the reference solution;
    FP32-inner/FP64-refine within 1e-7 relative at tol 1e-10.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

ASM_TOL = 1e-13


def row_scaled_err(ptr, a, b):
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    m = np.zeros(len(ptr) - 1)
    np.maximum.at(m, rows, np.abs(b))
    m = np.maximum(m, 1e-300)
    return float((np.abs(a - b) / m[rows]).max())


@pytest.mark.parametrize("dim,ne", [(2, (5, 7)), (3, (3, 4, 5)), (2, (200, 200)), (3, (1, 1, 1)),
                                    (3, (64, 48, 33)), (3, (128, 128, 128))])
def test_pattern_bit_exact(cuda, dim, ne):
    d = R.Domain(dim, ne)
    p, i = d.pattern()
    ref = O.pattern(dim, ne)
    assert np.array_equal(p, ref.ptr)
    assert np.array_equal(i, ref.idx)


def _golden_coefs(golden, tag, kname):
    kind = R.KINDS[kname]
    return {k: (golden[f"asm{tag}_{kname}_{k}"], kind) for k in "ABCDXY"}


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kname", ["const", "exp"])
def test_assembly_matches_reference(cuda, golden, dim, kname):
    tag = f"{dim}d"
    ne = tuple(int(v) for v in golden[f"asm{tag}_ne"])
    dx = golden[f"asm{tag}_dx"]
    d = R.Domain(dim, ne, x1=[dx[k] * ne[k] for k in range(dim)])
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, **_golden_coefs(golden, tag, kname))
    val = m.values()
    p, _ = d.pattern()
    assert row_scaled_err(p, val, golden[f"asm{tag}_{kname}_val"]) < ASM_TOL
    ref_rhs = golden[f"asm{tag}_{kname}_rhs"]
    assert np.abs(rhs.cpu().numpy() - ref_rhs).max() <= ASM_TOL * np.abs(ref_rhs).max()


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kname", ["const", "exp"])
def test_reduced_assembly_matches_reference(cuda, golden, dim, kname):
    """rg_assemble_single_reduced against the reference's assemblePDESingleReduced."""
    tag = f"{dim}d"
    ne = tuple(int(v) for v in golden[f"asm{tag}_ne"])
    dx = golden[f"asm{tag}_dx"]
    d = R.Domain(dim, ne, x1=[dx[k] * ne[k] for k in range(dim)])
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    kind = R.KINDS[kname]
    R.assemble_reduced(m, rhs, keep, **{k: (golden[f"red{tag}_{kname}_{k}"], kind) for k in "ABCDXY"})
    p, _ = d.pattern()
    assert row_scaled_err(p, m.values(), golden[f"red{tag}_{kname}_val"]) < ASM_TOL
    ref_rhs = golden[f"red{tag}_{kname}_rhs"]
    assert np.abs(rhs.cpu().numpy() - ref_rhs).max() <= ASM_TOL * np.abs(ref_rhs).max()
    # per-element data is the same as expanded data on ReducedFunction
    if kname == "exp":
        m2 = R.Matrix(d)
        rhs2 = torch.zeros(d.n, dtype=torch.float64, device="cuda")
        R.assemble_reduced(m2, rhs2, keep, **{k: (golden[f"red{tag}_{kname}_{k}"], R.KINDS["elem"])
                                              for k in "ABCDXY"})
        assert np.array_equal(m2.values(), m.values())
        assert torch.equal(rhs2, rhs)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kname", ["const", "exp"])
def test_boundary_assembly_matches_reference(cuda, golden, dim, kname):
    tag = f"{dim}d"
    ne = tuple(int(v) for v in golden[f"asm{tag}_ne"])
    dx = golden[f"asm{tag}_dx"]
    d = R.Domain(dim, ne, x1=[dx[k] * ne[k] for k in range(dim)])
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    kind = R.KINDS[kname]
    R.assemble_boundary(m, rhs, keep, d=(golden[f"bnd{tag}_{kname}_d"], kind),
                        y=(golden[f"bnd{tag}_{kname}_y"], kind))
    rv, rr = golden[f"bnd{tag}_{kname}_val"], golden[f"bnd{tag}_{kname}_rhs"]
    assert np.abs(m.values() - rv).max() <= ASM_TOL * np.abs(rv).max()
    assert np.abs(rhs.cpu().numpy() - rr).max() <= ASM_TOL * np.abs(rr).max()


@pytest.mark.parametrize("dim,ne", [(2, (9, 6)), (3, (6, 5, 7))])
def test_per_element_equals_expanded(cuda, dim, ne):
    """A per-element coefficient is the expanded one with equal values at the Gauss points."""
    rng = np.random.default_rng(5)
    nel = int(np.prod(ne))
    nq = 1 << dim
    Ae = rng.standard_normal((nel, dim * dim))
    De = rng.standard_normal(nel)
    d = R.Domain(dim, ne)
    m1, m2 = R.Matrix(d), R.Matrix(d)
    r1 = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    r2 = torch.zeros_like(r1)
    keep = []
    R.assemble(m1, r1, keep, A=(Ae, R.KINDS["elem"]), D=(De, R.KINDS["elem"]), Y=(De, R.KINDS["elem"]))
    R.assemble(m2, r2, keep, A=(np.repeat(Ae, nq, axis=0), R.KINDS["exp"]),
               D=(np.repeat(De, nq), R.KINDS["exp"]), Y=(np.repeat(De, nq), R.KINDS["exp"]))
    p, _ = d.pattern()
    assert row_scaled_err(p, m1.values(), m2.values()) < ASM_TOL
    assert torch.allclose(r1, r2, rtol=0, atol=ASM_TOL * float(r2.abs().max()))


def test_large_brick_assembly_matches_oracle(cuda):
    """Brick 48x40x32 with expanded isotropic kappa and expanded Y (the benchmark's
    coefficient form) against the oracle."""
    rng = np.random.default_rng(7)
    ne = (48, 40, 32)
    nel = int(np.prod(ne))
    kappa = np.exp(rng.standard_normal(nel))
    A = np.zeros((nel, 8, 3, 3))
    for i in range(3):
        A[:, :, i, i] = kappa[:, None]
    A = A.reshape(-1)
    Y = rng.standard_normal(nel * 8)
    d = R.Domain(3, ne)
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(A, R.KINDS["exp"]), Y=(Y, R.KINDS["exp"]))
    pat = O.pattern(3, ne)
    val, rr = O.assemble(3, ne, d.dx, pat, A=(O.EXPANDED, A), Y=(O.EXPANDED, Y))
    assert row_scaled_err(pat.ptr, m.values(), val) < ASM_TOL
    assert np.abs(rhs.cpu().numpy() - rr).max() <= ASM_TOL * np.abs(rr).max()


def _system(golden, tag):
    ne = tuple(int(v) for v in golden[f"solve{tag}_ne"])
    dim = len(ne)
    d = R.Domain(dim, ne)
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(golden[f"solve{tag}_A"], R.KINDS["exp"]),
               Y=(golden[f"solve{tag}_Y"], R.KINDS["exp"]))
    q = R.dev(golden[f"solve{tag}_q"])
    R.insert_constraint(m, rhs, q)
    return d, m, rhs, keep


@pytest.mark.parametrize("tag", ["2d", "3d"])
def test_constraint_matches_reference(cuda, golden, tag):
    d, m, rhs, _ = _system(golden, tag)
    p, _ = d.pattern()
    assert row_scaled_err(p, m.values(), golden[f"solve{tag}_val"]) < ASM_TOL
    ref = golden[f"solve{tag}_rhs"]
    assert np.abs(rhs.cpu().numpy() - ref).max() <= ASM_TOL * np.abs(ref).max()


def test_constraint_with_values_and_spmv(cuda):
    """rhs -= A u_r with nonzero r, then y = A x on the unbalanced matrix (ypAx)."""
    rng = np.random.default_rng(9)
    ne = (7, 6, 5)
    d = R.Domain(3, ne)
    m = R.Matrix(d)
    nel = int(np.prod(ne))
    A = rng.standard_normal(nel * 8 * 9)
    Y = rng.standard_normal(nel * 8)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(A, R.KINDS["exp"]), Y=(Y, R.KINDS["exp"]))
    q = (rng.random(d.n) < 0.2).astype(float)
    r = rng.standard_normal(d.n)
    R.insert_constraint(m, rhs, R.dev(q), R.dev(r))
    pat = O.pattern(3, ne)
    val, rr = O.assemble(3, ne, d.dx, pat, A=(O.EXPANDED, A), Y=(O.EXPANDED, Y))
    O.insert_constraint(pat, val, rr, q, r)
    gv = m.values()
    assert row_scaled_err(pat.ptr, gv, val) < ASM_TOL
    assert np.abs(rhs.cpu().numpy() - rr).max() <= 1e-12 * np.abs(rr).max()
    x = rng.standard_normal(d.n)
    y0 = rng.standard_normal(d.n)
    y = R.dev(y0)
    L.check(R.lib().rg_spmv(m.h, 2.0, R.ptr(R.dev(x)), -0.5, R.ptr(y)))
    ref = O.spmv(pat, val, x, alpha=2.0, beta=-0.5, y=y0)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("tag", ["2d", "3d"])
def test_paso_solve_matches_reference(cuda, golden, tag):
    d, m, rhs, _ = _system(golden, tag)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10))
    assert st == 0 and dg.converged
    ref = golden[f"solve{tag}_x"]
    err = np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 1e-8
    assert abs(int(dg.num_iter) - int(golden[f"solve{tag}_iter"])) <= 1


@pytest.mark.parametrize("tag", ["2d", "3d"])
@pytest.mark.parametrize("mode,precision,layout", [(L.RG_MODE_STANDARD, L.RG_PREC_FP64, L.RG_LAYOUT_CSR),
                                                   (L.RG_MODE_STANDARD, L.RG_PREC_FP64, L.RG_LAYOUT_BAND),
                                                   (L.RG_MODE_STANDARD, L.RG_PREC_FP32_REFINE, L.RG_LAYOUT_BAND)])
def test_fast_modes_match_reference(cuda, golden, tag, mode, precision, layout):
    d, m, rhs, _ = _system(golden, tag)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, mode=mode, precision=precision, layout=layout))
    assert st == 0 and dg.converged
    ref = golden[f"solve{tag}_x"]
    err = np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < (1e-8 if precision == L.RG_PREC_FP64 else 1e-7)
    # the stopping test is the paso dual-norm test on the FP64 true residual
    assert dg.residual_norm <= 1e-10 * dg.rhs_norm * (1 + 1e-12)


def test_rectangle_200_configuration(cuda, golden):
    """The reference's CPU-runnable case (Rectangle 200x200, Y = 1, u = 0 on y = 0)."""
    d = R.Domain(2, (200, 200))
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(np.eye(2).reshape(-1), R.KINDS["const"]), Y=(np.ones(1), R.KINDS["const"]))
    q = np.zeros(d.n)
    q[:201] = 1.0
    R.insert_constraint(m, rhs, R.dev(q))
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-8))
    assert st == 0
    ref = golden["r200_x"]
    assert np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-8
    assert abs(int(dg.num_iter) - int(golden["r200_iter"])) <= 1


def test_second_solve_reuses_balanced_matrix(cuda, golden):
    d, m, rhs, _ = _system(golden, "3d")
    x1 = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    x2 = torch.zeros_like(x1)
    assert R.solve(m, rhs, x1, R.opts(tolerance=1e-10))[0] == 0
    b = C_int()
    L.check(R.lib().rg_matrix_is_balanced(m.h, R.C.byref(b)))
    assert b.value == 1
    assert R.solve(m, rhs, x2, R.opts(tolerance=1e-10))[0] == 0
    assert torch.equal(x1, x2)
    # values can no longer be changed without a reset (paso balances in place)
    keep = []
    with pytest.raises(ValueError):
        R.assemble(m, None, keep, D=(np.ones(1), R.KINDS["const"]))
    with pytest.raises(ValueError):
        L.check(R.lib().rg_spmv(m.h, 1.0, R.ptr(x1), 0.0, R.ptr(x2)))


def C_int():
    import ctypes
    return ctypes.c_int()


def test_solver_errors_are_reported(cuda, golden):
    d, m, rhs, _ = _system(golden, "2d")
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, _ = R.solve(m, rhs, x, R.opts(tolerance=1e-20))
    assert st == L.RG_INVALID_ARG and "Tolerance" in L.last_error()
    st, _ = R.solve(m, rhs, x, R.opts(iter_max=2))
    assert st == L.RG_MAXITER
    st, dg = R.solve(m, rhs, x, R.opts(iter_max=2, accept_convergence_failure=1))
    assert st == 0 and not dg.converged
    bad = rhs.clone()
    bad[5] = float("nan")
    st, _ = R.solve(m, bad, x, R.opts())
    assert st == L.RG_NAN
    st, dg = R.solve(m, torch.zeros_like(rhs), x, R.opts())
    assert st == 0 and dg.converged and not bool(x.any())
    st, _ = R.solve(m, rhs, x, R.opts(sweeps=2, mode=L.RG_MODE_STANDARD))
    assert st == L.RG_NOT_SUPPORTED
    st, _ = R.solve(m, rhs, x, R.opts(sweeps=2, precision=L.RG_PREC_FP32_REFINE))
    assert st == L.RG_NOT_SUPPORTED


def _residual_norms(m, rhs_t, x_t):
    import ctypes
    l2, lm = ctypes.c_double(), ctypes.c_double()
    L.check(R.lib().rg_residual_norms(m.h, R.ptr(rhs_t), R.ptr(x_t), ctypes.byref(l2), ctypes.byref(lm)))
    return l2.value, lm.value


def test_residual_norms_before_and_after_balancing(cuda, golden):
    """rg_residual_norms measures b - A x of the assembled system, also once a solve has
    balanced the matrix in place."""
    d, m, rhs, _ = _system(golden, "3d")
    ne = tuple(int(v) for v in golden["solve3d_ne"])
    pat = O.pattern(3, ne)
    val = golden["solve3d_val"]
    rng = np.random.default_rng(13)
    x0 = rng.standard_normal(d.n)
    r = golden["solve3d_rhs"] - O.spmv(pat, val, x0)
    l2, lm = _residual_norms(m, rhs, R.dev(x0))
    assert abs(l2 - np.linalg.norm(r)) <= 1e-12 * np.linalg.norm(r)
    assert abs(lm - np.abs(r).max()) <= 1e-12 * np.abs(r).max()
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    assert R.solve(m, rhs, x, R.opts(tolerance=1e-10))[0] == 0
    l2b, lmb = _residual_norms(m, rhs, R.dev(x0))
    assert abs(l2b - l2) <= 1e-12 * l2 and abs(lmb - lm) <= 1e-12 * lm
    # the solution's residual is small relative to the right hand side
    l2s, _ = _residual_norms(m, rhs, x)
    assert l2s <= 1e-8 * np.linalg.norm(golden["solve3d_rhs"])


@pytest.mark.parametrize("tag", ["2d", "3d"])
@pytest.mark.parametrize("sweeps", [2, 3])
def test_jacobi_sweeps_match_reference(cuda, golden, tag, sweeps):
    """paso PCG with the Jacobi smoother of `sweeps` sweeps as preconditioner (the
    reference's Smoother.cpp:161-184, used by PCG.cpp:152 and the initial guess of
    Solver.cpp:181): iterations within one of the reference's, solution within 1e-8."""
    d, m, rhs, _ = _system(golden, tag)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, sweeps=sweeps))
    assert st == 0 and dg.converged
    assert abs(int(dg.num_iter) - int(golden[f"sweep{tag}_{sweeps}_iter"])) <= 1
    ref = golden[f"sweep{tag}_{sweeps}_x"]
    assert np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-8
    # a second solve with one sweep on the same (now balanced) matrix: the captured
    # iterations are rebuilt for the other sweep count
    x1 = torch.zeros_like(x)
    st, dg1 = R.solve(m, rhs, x1, R.opts(tolerance=1e-10))
    assert st == 0 and abs(int(dg1.num_iter) - int(golden[f"solve{tag}_iter"])) <= 1


@pytest.mark.parametrize("tag", ["2d", "3d"])
@pytest.mark.parametrize("sweeps", [1, 2])
def test_paso_band_layout_matches_reference(cuda, golden, tag, sweeps):
    """paso PCG in FP64 with RG_LAYOUT_BAND: the SpMV and the extra Jacobi sweeps read the
    FP64 band copy of the balanced matrix instead of the CSR; iterations within one of the
    reference's, solution within 1e-8.  A following CSR solve on the same matrix rebuilds the
    captured iterations."""
    d, m, rhs, _ = _system(golden, tag)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, sweeps=sweeps, layout=L.RG_LAYOUT_BAND))
    assert st == 0 and dg.converged
    key = f"solve{tag}" if sweeps == 1 else f"sweep{tag}_{sweeps}"
    assert abs(int(dg.num_iter) - int(golden[f"{key}_iter"])) <= 1
    ref = golden[f"{key}_x"]
    assert np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-8
    x1 = torch.zeros_like(x)
    st, dg1 = R.solve(m, rhs, x1, R.opts(tolerance=1e-10, sweeps=sweeps))
    assert st == 0 and abs(int(dg1.num_iter) - int(dg.num_iter)) <= 1
    assert torch.linalg.norm(x1 - x) <= 1e-9 * torch.linalg.norm(x)


@pytest.mark.parametrize("mode", [L.RG_MODE_PASO, L.RG_MODE_STANDARD])
@pytest.mark.parametrize("ne", [(40, 33, 27), (7, 5, 130), (300, 211)])
def test_paso_band_layout_equals_csr(cuda, ne, mode):
    """The FP64 band SpMV (paso and standard PCG) on grids with ragged edge tiles (rows not a
    multiple of 256) and long iteration counts (replayed graphs): the same iterations as the
    CSR SpMV within one (paso) or 0.5 % (textbook CG, whose count over ~900 iterations moves
    with the order in which the 27 products are added) and the same solution to 1e-9."""
    rng = np.random.default_rng(5)
    dim = len(ne)
    nel, nq = int(np.prod(ne)), 2 ** dim
    kappa = np.exp(rng.standard_normal(nel))
    A = np.zeros((nel, nq, dim, dim))
    for i in range(dim):
        A[:, :, i, i] = kappa[:, None]
    Y = rng.standard_normal(nel * nq)
    xs, its = [], []
    for layout in (L.RG_LAYOUT_CSR, L.RG_LAYOUT_BAND):
        d = R.Domain(dim, ne)
        m = R.Matrix(d)
        rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
        keep = []
        R.assemble(m, rhs, keep, A=(A.reshape(-1), R.KINDS["exp"]), Y=(Y, R.KINDS["exp"]))
        q = np.zeros(d.n)
        q[: int(np.prod([v + 1 for v in ne[:-1]]))] = 1.0
        R.insert_constraint(m, rhs, R.dev(q))
        x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
        st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-10, layout=layout, mode=mode))
        assert st == 0 and dg.converged
        xs.append(x)
        its.append(int(dg.num_iter))
    slack = 1 if mode == L.RG_MODE_PASO else max(1, int(0.005 * its[0]))
    assert abs(its[0] - its[1]) <= slack, its
    assert torch.linalg.norm(xs[1] - xs[0]) <= 1e-9 * torch.linalg.norm(xs[0])


def _kappa_problem(d, ne, seed):
    """A = kappa I per element (log-normal kappa), Y random, u = 0 on the first face of the
    last axis, assembled into a new matrix on domain d."""
    rng = np.random.default_rng(seed)
    dim = len(ne)
    nel, nq = int(np.prod(ne)), 2 ** dim
    kappa = np.exp(rng.standard_normal(nel))
    A = np.zeros((nel, nq, dim, dim))
    for i in range(dim):
        A[:, :, i, i] = kappa[:, None]
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(A.reshape(-1), R.KINDS["exp"]), Y=(rng.standard_normal(nel * nq), R.KINDS["exp"]))
    q = np.zeros(d.n)
    q[: int(np.prod([v + 1 for v in ne[:-1]]))] = 1.0
    R.insert_constraint(m, rhs, R.dev(q))
    return m, rhs


def test_band_copies_follow_the_matrix(cuda):
    """Band copies adopted from a destroyed matrix are rewritten before a solve reads them,
    and a matrix whose values change (reset + assemble) gets fresh band copies: CSR, FP64
    band and FP32 band solves of the second matrix all match a fresh matrix's solution."""
    ne = (40, 33, 27)
    d = R.Domain(3, ne)
    m1, b1 = _kappa_problem(d, ne, seed=1)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    assert R.solve(m1, b1, x, R.opts(tolerance=1e-10, layout=L.RG_LAYOUT_BAND))[0] == 0
    assert R.solve(m1, b1, x, R.opts(tolerance=1e-10, precision=L.RG_PREC_FP32_REFINE))[0] == 0
    R.lib().rg_matrix_destroy(m1.h)  # its arrays, band copies included, go to the domain's pool
    m1.h = None
    ref_d = R.Domain(3, ne)
    mr, br = _kappa_problem(ref_d, ne, seed=2)
    xr = torch.zeros(ref_d.n, dtype=torch.float64, device="cuda")
    assert R.solve(mr, br, xr, R.opts(tolerance=1e-10))[0] == 0
    m2, b2 = _kappa_problem(d, ne, seed=2)  # adopts m1's arrays
    for o in (R.opts(tolerance=1e-10), R.opts(tolerance=1e-10, layout=L.RG_LAYOUT_BAND),
              R.opts(tolerance=1e-10, precision=L.RG_PREC_FP32_REFINE)):
        x2 = torch.zeros(d.n, dtype=torch.float64, device="cuda")
        st, dg = R.solve(m2, b2, x2, o)
        assert st == 0 and dg.converged and not dg.fp64_fallback
        assert torch.linalg.norm(x2 - xr) <= 1e-7 * torch.linalg.norm(xr), (o.layout, o.precision)


def test_matrix_keeps_its_domain_and_reuses_storage(cuda, golden):
    """A matrix keeps its domain alive: destroying the domain first (as a garbage collector
    may do) leaves the matrix usable; a matrix created after another on the same domain
    reuses its device arrays and solver vectors and gives the same solution."""
    d, m, rhs, _ = _system(golden, "3d")
    x1 = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    assert R.solve(m, rhs, x1, R.opts(tolerance=1e-10))[0] == 0
    # a second matrix after the first is gone: the domain's spare arrays and workspace
    R.lib().rg_matrix_destroy(m.h)
    m.h = None
    d2, m2, rhs2, _ = _system(golden, "3d")
    x2 = torch.zeros(d2.n, dtype=torch.float64, device="cuda")
    assert R.solve(m2, rhs2, x2, R.opts(tolerance=1e-10))[0] == 0
    assert torch.equal(x1, x2)
    # domain destroyed before its matrix: the matrix still assembles and solves
    dom = R.Domain(3, (4, 3, 5))
    mat = R.Matrix(dom)
    R.lib().rg_domain_destroy(dom.h)
    dom.h = None
    b = torch.zeros(dom.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(mat, b, keep, A=(np.eye(3).reshape(-1), R.KINDS["const"]), D=(np.ones(1), R.KINDS["const"]),
               Y=(np.ones(1), R.KINDS["const"]))  # u = 1
    x = torch.zeros(dom.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(mat, b, x, R.opts(tolerance=1e-10))
    assert st == 0 and float((x - 1.0).abs().max()) < 1e-8
    R.lib().rg_matrix_destroy(mat.h)  # frees the domain as well
    mat.h = None
