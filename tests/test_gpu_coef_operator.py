"""The FP32 inner solve with the operator evaluated from the element coefficients
(RG_LAYOUT_COEF) through the C-ABI, against the oracle's paso solves (paso/src/Solver.cpp:46-330,
PCG.cpp:62-367) of the matrices the reference's assembler builds (DefaultAssembler3D/2D::
assemblePDESingle).

  * representable matrices (A = kappa I per element, constant, per element or expanded with one
    value per element, summed over several assemblies, then insertConstraint): the solve uses
    the coefficient operator (rg_diag.inner_operator = 1), needs no FP64 fallback, and its
    solution at tol 1e-10 is within 1e-8 (relative l2) of the oracle's;
  * anything the record cannot describe (D, an anisotropic or off-diagonal A, face terms,
    nullifyRowsAndCols, an assembly after the constraint): the band copy is used
    (inner_operator = 0) and the solution is as accurate;
  * values changed behind the library's back (through rg_matrix_values' pointer): the FP64
    refinement notices that the FP32 corrections stopped working, finishes in FP64
    (fp64_fallback = 1), and the solution is still the one of the changed matrix.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

COEF = dict(mode=L.RG_MODE_STANDARD, precision=L.RG_PREC_FP32_REFINE, layout=L.RG_LAYOUT_COEF)


def iso_A(kappa, dim, kind):
    nel = len(kappa)
    if kind == "elem":
        A = np.zeros((nel, dim, dim))
        for k in range(dim):
            A[:, k, k] = kappa
    else:  # expanded: the same value at every Gauss point
        A = np.zeros((nel, 2 ** dim, dim, dim))
        for k in range(dim):
            A[:, :, k, k] = kappa[:, None]
    return A.reshape(-1)


class Case:
    """A system assembled on the GPU and by the oracle from the same coefficients."""

    def __init__(self, dim, ne, length=None, seed=0, kinds=("elem",), qmode="face", extra=None):
        rng = np.random.default_rng(seed)
        self.dim, self.ne = dim, ne
        nel = int(np.prod(ne))
        nq = 2 ** dim
        length = length or [1.0] * dim
        self.d = R.Domain(dim, ne, x1=length)
        self.m = R.Matrix(self.d)
        self.rhs = torch.zeros(self.d.n, dtype=torch.float64, device="cuda")
        self.keep = []
        pat = O.pattern(dim, ne)
        val = np.zeros(pat.nnz)
        rr = np.zeros(pat.n)
        for k, kind in enumerate(kinds):
            kappa = np.exp(rng.standard_normal(nel))
            A = iso_A(kappa, dim, kind)
            Y = rng.standard_normal(nel * nq) if k == 0 else None
            coefs = {"A": (A, R.KINDS[kind])}
            ocoefs = {"A": (O.EXPANDED if kind == "exp" else O.PER_ELEMENT, A)}
            if Y is not None:
                coefs["Y"] = (Y, R.KINDS["exp"])
                ocoefs["Y"] = (O.EXPANDED, Y)
            if extra and k == 0:
                for name, arr in extra.items():
                    coefs[name] = (arr, R.KINDS["exp"])
                    ocoefs[name] = (O.EXPANDED, arr)
            R.assemble(self.m, self.rhs, self.keep, **coefs)
            v, r = O.assemble(dim, ne, self.d.dx, pat,
                              **{("C_" if n == "C" else n): c for n, c in ocoefs.items()})
            val += v
            rr += r
        if qmode == "face":
            q = np.zeros(pat.n)
            q[-int(np.prod([e + 1 for e in ne[:-1]])):] = 1.0
        else:
            q = (rng.random(pat.n) < 0.05).astype(float)
        R.insert_constraint(self.m, self.rhs, R.dev(q))
        O.insert_constraint(pat, val, rr, q)
        self.pat, self.val, self.rr = pat, val, rr

    def reference(self):
        ref = O.solve_paso(self.pat, self.val.copy(), self.rr, tol=1e-10)
        assert ref.converged
        return ref.x

    def solve(self, **kw):
        o = R.opts(tolerance=1e-10, **{**COEF, **kw})
        x = torch.zeros(self.d.n, dtype=torch.float64, device="cuda")
        st, dg = R.solve(self.m, self.rhs, x, o)
        return st, dg, x.cpu().numpy()


def rel(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("dim,ne,length,qmode", [
    (3, (40, 33, 27), (1.0, 2.0, 0.5), "face"),   # one khat / state window per plane
    (3, (7, 5, 130), None, "face"),               # thin x-lines
    (3, (300, 10, 10), None, "scatter"),          # long x-lines: one window per stencil column
    (2, (300, 211), (3.0, 1.0), "face"),          # 2D, windows per column
    (2, (120, 90), None, "scatter"),
])
def test_coefficient_operator_solution_matches_oracle(cuda, dim, ne, length, qmode):
    case = Case(dim, ne, length, seed=3, qmode=qmode)
    st, dg, x = case.solve()
    assert st == 0 and dg.converged
    assert dg.inner_operator == 1 and not dg.fp64_fallback
    assert dg.residual_norm <= 1e-10 * dg.rhs_norm * (1 + 1e-12)
    assert rel(x, case.reference()) < 1e-8


def test_expanded_and_summed_assemblies_use_the_coefficients(cuda):
    """A expanded to the Gauss points with one value per element, plus a second assembly of A
    per element: the record sums kappa (the values add)."""
    case = Case(3, (24, 20, 18), seed=4, kinds=("exp", "elem"))
    st, dg, x = case.solve()
    assert st == 0 and dg.converged and dg.inner_operator == 1 and not dg.fp64_fallback
    assert rel(x, case.reference()) < 1e-8


def test_forced_configurations_agree(cuda):
    xs, its = [], []
    for cfg in (0, 1):
        case = Case(3, (40, 30, 20), seed=5)
        L.check(R.lib().rg_solver_set_config(case.m.h, cfg))
        st, dg, x = case.solve()
        assert st == 0 and dg.converged and dg.inner_operator == 1
        c = C.c_int()
        L.check(R.lib().rg_solver_config(case.m.h, C.byref(c), None, None))
        assert c.value == cfg
        xs.append(x)
        its.append(int(dg.num_iter))
    assert rel(xs[0], xs[1]) < 1e-9
    assert abs(its[0] - its[1]) <= 2


@pytest.mark.parametrize("what", ["D", "anisotropic", "offdiag", "face_d", "after_constraint", "nullify"])
def test_values_the_record_cannot_describe_use_the_band_copy(cuda, what):
    rng = np.random.default_rng(6)
    ne = (16, 14, 12)
    nel = int(np.prod(ne))
    extra = None
    if what == "D":
        extra = {"D": np.abs(rng.standard_normal(nel * 8))}
    case = Case(3, ne, seed=6, extra=extra)
    pat, val = case.pat, case.val
    if what in ("anisotropic", "offdiag"):
        A = np.zeros((nel, 3, 3))
        A[:, 0, 0], A[:, 1, 1], A[:, 2, 2] = 1.0, 2.0, 1.0
        if what == "offdiag":
            A[:, 0, 0] = A[:, 1, 1] = 2.0
            A[:, 0, 1] = A[:, 1, 0] = 0.3
        # a fresh matrix with that A and the same constraint
        case.m = R.Matrix(case.d)
        case.rhs = torch.zeros(case.d.n, dtype=torch.float64, device="cuda")
        Y = rng.standard_normal(nel * 8)
        R.assemble(case.m, case.rhs, case.keep, A=(A.reshape(-1), R.KINDS["elem"]), Y=(Y, R.KINDS["exp"]))
        q = np.zeros(pat.n)
        q[-15 * 13:] = 1.0
        R.insert_constraint(case.m, case.rhs, R.dev(q))
        case.val, case.rr = O.assemble(3, ne, case.d.dx, pat, A=(O.PER_ELEMENT, A.reshape(-1)), Y=(O.EXPANDED, Y))
        O.insert_constraint(pat, case.val, case.rr, q)
    elif what == "face_d":
        dface = np.ones(1)
        R.assemble_boundary(case.m, case.rhs, case.keep, d=(dface, R.KINDS["const"]))
        O.assemble_boundary(3, ne, case.d.dx, pat, case.val, case.rr, d=(O.CONSTANT, dface))
    elif what == "after_constraint":
        D = np.full(1, 0.5)
        R.assemble(case.m, case.rhs, case.keep, D=(D, R.KINDS["const"]))
        v, r = O.assemble(3, ne, case.d.dx, pat, D=(O.CONSTANT, D))
        case.val += v
        case.rr += r
    elif what == "nullify":
        mask = np.zeros(pat.n)
        mask[:15] = 1.0
        L.check(R.lib().rg_nullify_rows_and_cols(case.m.h, R.ptr(R.dev(mask)), R.ptr(R.dev(mask)), 1.0))
        rows = np.repeat(np.arange(pat.n), np.diff(pat.ptr))
        hit = (mask[rows] > 0) | (mask[pat.idx] > 0)
        case.val[hit] = np.where(rows[hit] == pat.idx[hit], 1.0, 0.0)
    st, dg, x = case.solve()
    assert st == 0 and dg.converged
    assert dg.inner_operator == 0
    assert rel(x, case.reference()) < 1e-8


def test_reset_starts_a_new_record(cuda):
    case = Case(3, (16, 12, 10), seed=7, extra={"D": np.ones(16 * 12 * 10 * 8)})
    st, dg, _ = case.solve()
    assert dg.inner_operator == 0
    # a reset matrix assembled again from a representable A uses the coefficients
    L.check(R.lib().rg_matrix_reset(case.m.h))
    rng = np.random.default_rng(8)
    nel = 16 * 12 * 10
    kappa = np.exp(rng.standard_normal(nel))
    A = iso_A(kappa, 3, "elem")
    Y = rng.standard_normal(nel * 8)
    case.rhs.zero_()
    R.assemble(case.m, case.rhs, case.keep, A=(A, R.KINDS["elem"]), Y=(Y, R.KINDS["exp"]))
    q = np.zeros(case.pat.n)
    q[-17 * 13:] = 1.0
    R.insert_constraint(case.m, case.rhs, R.dev(q))
    case.val, case.rr = O.assemble(3, (16, 12, 10), case.d.dx, case.pat, A=(O.PER_ELEMENT, A), Y=(O.EXPANDED, Y))
    O.insert_constraint(case.pat, case.val, case.rr, q)
    st, dg, x = case.solve()
    assert st == 0 and dg.inner_operator == 1
    assert rel(x, case.reference()) < 1e-8


def test_values_changed_behind_the_record_stay_correct(cuda):
    """Scaling the values through rg_matrix_values' pointer is invisible to the record: the
    FP32 corrections then come from the old operator, the FP64 residual of the changed matrix
    stops improving, and the solve finishes in FP64 on the changed matrix."""
    case = Case(3, (20, 16, 12), seed=9)
    p = C.c_void_p()
    L.check(R.lib().rg_matrix_values(case.m.h, C.byref(p)))
    torch.cuda.synchronize()
    vals = R._raw(p.value, case.d.nnz)
    vals.mul_(3.0)
    case.val *= 3.0
    st, dg, x = case.solve()
    assert st == 0 and dg.converged
    assert dg.inner_operator == 1 and dg.fp64_fallback == 1
    assert rel(x, case.reference()) < 1e-8


def test_switching_operators_on_one_matrix(cuda):
    """Solves alternating between the coefficient operator and the band copy on one matrix:
    each replays iteration graphs of its own operator (no FP64 fallback, same answer)."""
    case = Case(3, (30, 24, 20), seed=11)
    ref = case.reference()
    for layout in (L.RG_LAYOUT_COEF, L.RG_LAYOUT_BAND, L.RG_LAYOUT_COEF, L.RG_LAYOUT_BAND):
        st, dg, x = case.solve(layout=layout)
        assert st == 0 and dg.converged and not dg.fp64_fallback
        assert dg.inner_operator == (1 if layout == L.RG_LAYOUT_COEF else 0)
        assert rel(x, ref) < 1e-8


def test_fp64_solves_refuse_the_coefficient_layout(cuda):
    case = Case(3, (6, 5, 4), seed=10)
    st, _, _ = case.solve(precision=L.RG_PREC_FP64)
    assert st == L.RG_NOT_SUPPORTED


def test_guess_smoothing_on_the_coefficient_operator(cuda):
    """Chebyshev smoothing of an initial guess (standard mode) runs on the coefficient operator
    when the band copy is not built: the smoothed guess's residual equals the one smoothed on
    the band copy (both FP32 operators, FP64 vectors) to FP32 accuracy, fixed nodes included,
    and both solves meet the tolerance."""
    case = Case(3, (36, 30, 24), seed=12, qmode="scatter")
    rng = np.random.default_rng(13)
    ref = case.reference()
    g = torch.tensor(ref * (1.0 + 0.3 * rng.standard_normal(case.d.n)), device="cuda")
    res = {}
    for layout in (L.RG_LAYOUT_COEF, L.RG_LAYOUT_BAND):
        o = R.opts(tolerance=1e-10, **{**COEF, "layout": layout})
        o.initial_guess = g.data_ptr()
        o.guess_sweeps = 8
        x = torch.zeros(case.d.n, dtype=torch.float64, device="cuda")
        st, dg = R.solve(case.m, case.rhs, x, o)
        assert st == 0 and dg.converged and not dg.fp64_fallback
        assert rel(x.cpu().numpy(), ref) < 1e-8
        res[layout] = dg.guess_residual
    assert abs(res[L.RG_LAYOUT_COEF] - res[L.RG_LAYOUT_BAND]) <= 1e-4 * res[L.RG_LAYOUT_BAND]
