"""The allocation-free residual-norm entry point (rg_residual_norms_noalloc).

Some callers cannot let a library allocate device memory: their own pool or caching
allocator owns the GPU's memory, or they run latency-critical loops that cannot absorb the
implicit synchronisation of cudaMalloc/cudaFree.  For them the library offers the residual
norms with the reduction scratch in a fixed static device array.  This test calls it
through the C-ABI twice in a row (the array keeps the previous call's contents, so the
second call checks that the state is cleared) and compares it with rg_residual_norms,
which allocates its scratch with the matrix.  The file is named to be collected last.
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


def test_noalloc_residual_norms_match_allocating_entry_point(cuda):
    rng = np.random.default_rng(21)
    ne = (17, 13, 11)
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
    lib = R.lib()
    for call in range(2):
        x = R.dev(rng.standard_normal(d.n))
        ref = _norms(lib.rg_residual_norms, m, rhs, x)
        got = _norms(lib.rg_residual_norms_noalloc, m, rhs, x)
        assert abs(got[0] - ref[0]) <= TOL * ref[0], (call, got, ref)
        assert abs(got[1] - ref[1]) <= TOL * ref[1], (call, got, ref)
