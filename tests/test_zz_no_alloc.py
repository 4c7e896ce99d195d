"""The allocation-free residual-norm entry point (rg_residual_norms_noalloc).

Some callers cannot let a library allocate device memory: their own pool or caching
allocator owns the GPU's memory, or they run latency-critical loops that cannot absorb the
implicit synchronisation of cudaMalloc/cudaFree.  For them the library offers the residual
norms with the reduction scratch in a fixed static device array.  These tests call it
through the C-ABI and compare it with rg_residual_norms, which allocates its scratch with
the matrix:
  * twice in a row on a fresh matrix, before the allocating call has ever run on it (the
    array keeps the previous call's contents, so the second call checks that the state is
    cleared), with the device's free memory unchanged across the calls;
  * on a matrix that a solve has balanced in place (the norms undo the balancing);
  * a PDE system, which it rejects with RG_NOT_SUPPORTED.
The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _norms(fn, m, rhs, x):
    l2, lm = ctypes.c_double(), ctypes.c_double()
    L.check(fn(m.h, R.ptr(rhs), R.ptr(x), ctypes.byref(l2), ctypes.byref(lm)))
    return l2.value, lm.value


def _close(got, ref):
    return abs(got[0] - ref[0]) <= TOL * ref[0] and abs(got[1] - ref[1]) <= TOL * ref[1]


def _scalar_system(ne, seed):
    rng = np.random.default_rng(seed)
    nel = int(np.prod(ne))
    d = R.Domain(3, ne)
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    kappa = np.exp(rng.standard_normal(nel))
    A = np.zeros((nel, 3, 3))
    for i in range(3):
        A[:, i, i] = kappa
    R.assemble(m, rhs, keep, A=(A.reshape(-1), R.KINDS["elem"]), Y=(rng.standard_normal(nel * 8), R.KINDS["exp"]))
    return d, m, rhs, rng


def test_noalloc_residual_norms_match_allocating_entry_point(cuda):
    lib = R.lib()
    # the first call on a device loads the library's kernels for it and looks up the static
    # array's address; it runs on another matrix so that the measured calls below start from
    # a set-up device
    d0, m0, rhs0, _ = _scalar_system((5, 4, 3), 20)
    _norms(lib.rg_residual_norms_noalloc, m0, rhs0, R.dev(np.ones(d0.n)))

    d, m, rhs, rng = _scalar_system((17, 13, 11), 21)
    xs = [R.dev(rng.standard_normal(d.n)) for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got = [_norms(lib.rg_residual_norms_noalloc, m, rhs, x) for x in xs]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "the no-allocation entry point changed free device memory"
    for call, x in enumerate(xs):
        ref = _norms(lib.rg_residual_norms, m, rhs, x)
        assert _close(got[call], ref), (call, got[call], ref)


def test_noalloc_residual_norms_on_a_balanced_matrix(cuda):
    lib = R.lib()
    d, m, rhs, rng = _scalar_system((12, 10, 9), 22)
    q = np.zeros(d.n)
    q[-13 * 11:] = 1.0
    R.insert_constraint(m, rhs, R.dev(q))
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-6))
    assert st == 0 and dg.converged
    b = ctypes.c_int()
    L.check(lib.rg_matrix_is_balanced(m.h, ctypes.byref(b)))
    assert b.value == 1
    for x_t in (x, R.dev(rng.standard_normal(d.n))):
        for _ in range(2):
            got = _norms(lib.rg_residual_norms_noalloc, m, rhs, x_t)
            ref = _norms(lib.rg_residual_norms, m, rhs, x_t)
            assert _close(got, ref), (got, ref)
    # the solution's residual is what the solver reported
    got = _norms(lib.rg_residual_norms_noalloc, m, rhs, x)
    assert got[0] <= 1e-6 * dg.rhs_norm * (1 + 1e-6)


def test_noalloc_residual_norms_reject_pde_systems(cuda):
    d = R.Domain(2, (4, 3))
    m = R.Matrix(d, block_size=2)
    v = torch.zeros(d.n * 2, dtype=torch.float64, device="cuda")
    l2, lm = ctypes.c_double(), ctypes.c_double()
    st = R.lib().rg_residual_norms_noalloc(m.h, R.ptr(v), R.ptr(v), ctypes.byref(l2), ctypes.byref(lm))
    assert st == L.RG_NOT_SUPPORTED
    assert "system" in L.last_error()
