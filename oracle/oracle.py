"""ctypes bindings to the CPU oracle (test infrastructure only).

Two libraries:
  * ``_build/libripley_oracle.so`` - the C restatement in ``ripley_oracle.c``;
  * ``_ref/libripley_ref.so``     - the reference's own DefaultAssembler2D/3D.cpp,
    paso Solver.cpp, PCG.cpp and SparseMatrix_MatrixVector.cpp compiled in place
    (``make -C oracle ref``; present only where the reference tree was available
    when it was built).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module.  The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libripley_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libripley_ref.so")

EMPTY, CONSTANT, EXPANDED, PER_ELEMENT = 0, 1, 2, 3

_lib = None
_ref = None


class _Coef(C.Structure):
    _fields_ = [("p", C.POINTER(C.c_double)), ("kind", C.c_int)]


class _Opts(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("iter_max", C.c_int64), ("sweeps", C.c_int),
                ("verbose", C.c_int)]


class _Diag(C.Structure):
    _fields_ = [("num_iter", C.c_int64), ("num_outer", C.c_int64),
                ("residual_norm", C.c_double), ("converged", C.c_int)]


def build(reference: bool = False) -> None:
    """Compile the oracle (and, when asked and possible, the reference sources)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if reference:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = C.CDLL(ORACLE_SO)
        _lib.ro_pattern_nnz.restype = C.c_int64
        _lib.ro_solve_paso.restype = C.c_int
        _lib.ro_solve_cg.restype = C.c_int
    return _lib


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        _ref.ref_last_error.restype = C.c_char_p
    return _ref


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _i64x3(v):
    v = list(v) + [1] * (3 - len(v))
    return (C.c_int64 * 3)(*v)


def _dx3(v):
    v = list(v) + [1.0] * (3 - len(v))
    return (C.c_double * 3)(*v)


def _coef(c):
    """``c`` is None or a (kind, float64 array) pair."""
    if c is None:
        return _Coef(None, EMPTY), None
    kind, arr = c
    arr = np.ascontiguousarray(arr, dtype=np.float64)
    return _Coef(_dp(arr), kind), arr


@dataclass
class Pattern:
    ptr: np.ndarray
    idx: np.ndarray

    @property
    def n(self):
        return len(self.ptr) - 1

    @property
    def nnz(self):
        return len(self.idx)


def pattern(dim: int, ne) -> Pattern:
    nn = [e + 1 for e in ne]
    L = lib()
    nnz = L.ro_pattern_nnz(dim, _i64x3(nn))
    n = int(np.prod(nn[:dim]))
    ptr = np.zeros(n + 1, np.int32)
    idx = np.zeros(nnz, np.int32)
    L.ro_pattern(dim, _i64x3(nn), _ip(ptr), _ip(idx))
    return Pattern(ptr, idx)


def assemble(dim, ne, dx, pat: Pattern, A=None, B=None, C_=None, D=None, X=None, Y=None,
             use_ref=False, reduced=False):
    """Interior assembly.  Coefficients are (kind, array) pairs or None.  Returns
    (val, rhs).  ``use_ref`` runs the reference's own DefaultAssembler source; ``reduced``
    selects the reduced-order (1-point) assembly of coefficients on ReducedFunction, whose
    expanded data has one value set per element."""
    val = np.zeros(pat.nnz)
    rhs = np.zeros(pat.n)
    coefs = [_coef(c) for c in (A, B, C_, D, X, Y)]
    if use_ref:
        R = ref()
        kinds = (C.c_int * 6)(*[c[0].kind for c in coefs])
        ptrs = (C.POINTER(C.c_double) * 6)(*[c[0].p for c in coefs])
        if any(k == PER_ELEMENT for k in kinds):
            raise ValueError("the reference assembler takes constant or expanded data")
        fn = R.ref_assemble_reduced if reduced else R.ref_assemble
        rc = fn(dim, _i64x3(ne), _dx3(dx), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs), kinds, ptrs)
        if rc:
            raise RuntimeError(R.ref_last_error().decode())
    else:
        fn = lib().ro_assemble_single_reduced if reduced else lib().ro_assemble_single
        fn(dim, _i64x3(ne), _dx3(dx), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs), *[c[0] for c in coefs])
    return val, rhs


def assemble_boundary(dim, ne, dx, pat: Pattern, val, rhs, d=None, y=None, use_ref=False, nb=1, reduced=False):
    """Face terms d, y added into val / rhs (block size nb; ``reduced``: one data point per
    face element, ReducedFunctionOnBoundary)."""
    cd, _kd = _coef(d)
    cy, _ky = _coef(y)
    general = nb != 1 or reduced
    if use_ref:
        R = ref()
        if general:
            rc = R.ref_assemble_boundary_ex(dim, _i64x3(ne), _dx3(dx), int(nb), int(bool(reduced)), _ip(pat.ptr),
                                            _ip(pat.idx), _dp(val), _dp(rhs), cd.kind, cd.p, cy.kind, cy.p)
        else:
            rc = R.ref_assemble_boundary(dim, _i64x3(ne), _dx3(dx), _ip(pat.ptr), _ip(pat.idx),
                                         _dp(val), _dp(rhs), cd.kind, cd.p, cy.kind, cy.p)
        if rc:
            raise RuntimeError(R.ref_last_error().decode())
    elif general:
        lib().ro_assemble_boundary_ex(dim, _i64x3(ne), _dx3(dx), int(nb), int(bool(reduced)), _ip(pat.ptr),
                                      _ip(pat.idx), _dp(val), _dp(rhs), cd, cy)
    else:
        lib().ro_assemble_boundary(dim, _i64x3(ne), _dx3(dx), _ip(pat.ptr), _ip(pat.idx),
                                   _dp(val), _dp(rhs), cd, cy)


def interpolate_nodes(dim, ne, nodal, ncomp=1):
    nodal = np.ascontiguousarray(nodal, dtype=np.float64)
    NE = int(np.prod(ne[:dim]))
    out = np.zeros(NE * (1 << dim) * ncomp)
    lib().ro_interpolate_nodes(dim, _i64x3(ne), _dp(nodal), ncomp, _dp(out))
    return out


def spmv(pat: Pattern, val, x, alpha=1.0, beta=0.0, y=None, use_ref=False):
    y = np.zeros(pat.n) if y is None else np.array(y, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    if use_ref:
        ref().ref_spmv(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), C.c_double(alpha),
                       _dp(x), C.c_double(beta), _dp(y))
    else:
        lib().ro_spmv(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), C.c_double(alpha),
                      _dp(x), C.c_double(beta), _dp(y))
    return y


def insert_constraint(pat: Pattern, val, rhs, q, r=None):
    q = np.ascontiguousarray(q, dtype=np.float64)
    r = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
    lib().ro_insert_constraint(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs),
                               _dp(q), _dp(r))


@dataclass
class SolveResult:
    x: np.ndarray
    status: int
    num_iter: int
    residual_norm: float
    converged: bool
    balance: np.ndarray | None = None
    seconds: float = 0.0


def solve_paso(pat: Pattern, val, b, tol=1e-8, iter_max=100000, sweeps=1, use_ref=False,
               verbose=False) -> SolveResult:
    """paso::Solver PCG+Jacobi.  ``val`` is balanced IN PLACE, as paso does."""
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    x = np.zeros(pat.n)
    if use_ref:
        R = ref()
        it = C.c_int64(0)
        rn = C.c_double(0)
        conv = C.c_int(0)
        sec = C.c_double(0)
        st = R.ref_solve(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(b), _dp(x),
                         C.c_double(tol), C.c_int64(iter_max), sweeps, int(verbose), C.byref(it),
                         C.byref(rn), C.byref(conv), C.byref(sec))
        if st < 0:
            raise RuntimeError(R.ref_last_error().decode())
        return SolveResult(x, st, it.value, rn.value, bool(conv.value), None, sec.value)
    bv = np.zeros(pat.n)
    d = _Diag()
    o = _Opts(tol, iter_max, sweeps, int(verbose))
    st = lib().ro_solve_paso(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(b),
                             _dp(x), _dp(bv), C.byref(o), C.byref(d))
    return SolveResult(x, st, d.num_iter, d.residual_norm, bool(d.converged), bv)


def solve_cg(pat: Pattern, val, b, rtol=1e-10, iter_max=100000, x0=None) -> SolveResult:
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(pat.n) if x0 is None else np.array(x0, dtype=np.float64)
    d = _Diag()
    st = lib().ro_solve_cg(C.c_int64(pat.n), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(b), _dp(x),
                           C.c_double(rtol), C.c_int64(iter_max), C.byref(d))
    return SolveResult(x, st, d.num_iter, d.residual_norm, bool(d.converged))


def set_threads(n: int) -> None:
    if have_ref():
        ref().ref_set_threads(n)


# ---- PDE systems (block size nb = numEq = numComp, 1..3) -----------------------------------
# Block CSR values on the node pattern: val[k nb^2 + ir + nb ic]; vectors u[node nb + comp];
# coefficient data points A (nb, dim, nb, dim), B (nb, dim, nb), C (nb, nb, dim), D (nb, nb),
# X (nb, dim), Y (nb), first index fastest (escript's layout).

def assemble_system(dim, ne, dx, pat: Pattern, nb, A=None, B=None, C_=None, D=None, X=None, Y=None,
                    use_ref=False, reduced=False):
    """assemblePDESystem (``reduced``: assemblePDESystemReduced, one data point per
    element).  Returns (val (nnz nb^2), rhs (n nb))."""
    val = np.zeros(pat.nnz * nb * nb)
    rhs = np.zeros(pat.n * nb)
    coefs = [_coef(c) for c in (A, B, C_, D, X, Y)]
    if use_ref:
        R = ref()
        kinds = (C.c_int * 6)(*[c[0].kind for c in coefs])
        ptrs = (C.POINTER(C.c_double) * 6)(*[c[0].p for c in coefs])
        fn = R.ref_assemble_system_reduced if reduced else R.ref_assemble_system
        rc = fn(dim, _i64x3(ne), _dx3(dx), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs), kinds, ptrs)
        if rc:
            raise RuntimeError(R.ref_last_error().decode())
    else:
        fn = lib().ro_assemble_system_reduced if reduced else lib().ro_assemble_system
        fn(dim, _i64x3(ne), _dx3(dx), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs),
           *[c[0] for c in coefs])
    return val, rhs


def spmv_block(pat: Pattern, nb, val, x, alpha=1.0, beta=0.0, y=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(pat.n * nb) if y is None else np.array(y, dtype=np.float64)
    lib().ro_spmv_block(C.c_int64(pat.n), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), C.c_double(alpha),
                        _dp(x), C.c_double(beta), _dp(y))
    return y


def insert_constraint_block(pat: Pattern, nb, val, rhs, q, r=None):
    q = np.ascontiguousarray(q, dtype=np.float64)
    rr = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
    lib().ro_insert_constraint_block(C.c_int64(pat.n), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(rhs),
                                     _dp(q), _dp(rr) if rr is not None else None)


def solve_paso_block(pat: Pattern, nb, val, b, tol=1e-8, iter_max=100000, use_ref=False, sweeps=1) -> SolveResult:
    """paso::Solver PCG + block Jacobi (``sweeps`` sweeps) on a block CSR matrix; ``val`` is
    balanced IN PLACE."""
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    x = np.zeros(pat.n * nb)
    if use_ref:
        R = ref()
        it = C.c_int64(0)
        rn = C.c_double(0)
        conv = C.c_int(0)
        st = R.ref_solve_block(C.c_int64(pat.n), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(b), _dp(x),
                               C.c_double(tol), C.c_int64(iter_max), int(sweeps), C.byref(it), C.byref(rn),
                               C.byref(conv))
        if st < 0:
            raise RuntimeError(R.ref_last_error().decode())
        return SolveResult(x, st, it.value, rn.value, bool(conv.value))
    bv = np.zeros(pat.n * nb)
    d = _Diag()
    o = _Opts(tol, iter_max, int(sweeps), 0)
    st = lib().ro_solve_paso_block(C.c_int64(pat.n), int(nb), _ip(pat.ptr), _ip(pat.idx), _dp(val), _dp(b),
                                   _dp(x), _dp(bv), C.byref(o), C.byref(d))
    return SolveResult(x, st, d.num_iter, d.residual_norm, bool(d.converged), bv)
