"""The mixed-precision configuration at full size: Brick 256^3 (n = 16,974,593, nnz =
454,756,609) from the benchmark's generator (seed 2026, correlation length 16 cells), FP32
inner iterations with FP64 refinement to rtol 1e-10, assembled and solved through the C-ABI
with device buffers, with both inner operators (element coefficients, FP32 band copy).

The oracle's CPU solve of this size takes minutes, so the test checks properties that hold at
any size, against the GPU's FP64 paso solve (which the oracle pins at the benchmark's 64^3 and
128^3 in test_gpu_bench_parity.py):
  * the stopping test holds in FP64: ||b - A x||_2 <= 1e-10 ||b||_2 as the solver reports
    it, and recomputed for the returned x on the FP64 CSR values by rg_residual_norms;
  * the solution agrees with the FP64 paso solve at rtol 1e-11 to 1e-8 relative (l2);
  * the refinement finished in FP32 (no FP64 fallback) on the intended inner operator.
"""
import ctypes as C

import pytest
import torch

import bench
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

NE = 256
TOL = 1e-10


class Big:
    """Coefficients of the 256^3 input on the device and the system built from them."""

    def __init__(self):
        inp = bench.make_inputs(NE, 2026, 16.0)
        nel = NE ** 3
        self.d = R.Domain(3, (NE, NE, NE))
        kap = R.dev(inp["kappa"])
        self.A = torch.zeros((nel, 3, 3), dtype=torch.float64, device="cuda")
        for i in range(3):
            self.A[:, i, i] = kap
        del kap
        self.Y = R.dev(inp["Y"])
        self.q = R.dev(inp["q"])

    def system(self):
        m = R.Matrix(self.d)
        rhs = torch.zeros(self.d.n, dtype=torch.float64, device="cuda")
        cA = L.rg_coef(self.A.data_ptr(), L.RG_COEF_PER_ELEMENT)
        cY = L.rg_coef(self.Y.data_ptr(), L.RG_COEF_EXPANDED)
        e = L.rg_coef(None, 0)
        L.set_stream_from_torch()
        L.check(R.lib().rg_assemble_single(m.h, R.ptr(rhs), C.byref(cA), C.byref(e), C.byref(e), C.byref(e),
                                           C.byref(e), C.byref(cY)))
        R.insert_constraint(m, rhs, self.q)
        return m, rhs


@pytest.fixture(scope="module")
def big(cuda):
    b = Big()
    m, rhs = b.system()
    x = torch.zeros(b.d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=1e-11, layout=L.RG_LAYOUT_BAND))
    assert st == 0 and dg.converged
    b.x64 = x
    del m, rhs
    yield b
    del b.x64


def _residual(m, rhs, x):
    l2, lm = C.c_double(), C.c_double()
    L.check(R.lib().rg_residual_norms(m.h, R.ptr(rhs), R.ptr(x), C.byref(l2), C.byref(lm)))
    return l2.value


@pytest.mark.parametrize("layout,inner", [(L.RG_LAYOUT_COEF, 1), (L.RG_LAYOUT_BAND, 0)], ids=["coef", "band"])
def test_b256_fp32_refinement(big, layout, inner):
    m, rhs = big.system()
    x = torch.zeros(big.d.n, dtype=torch.float64, device="cuda")
    st, dg = R.solve(m, rhs, x, R.opts(tolerance=TOL, mode=L.RG_MODE_STANDARD, precision=L.RG_PREC_FP32_REFINE,
                                       layout=layout))
    assert st == 0 and dg.converged and not dg.fp64_fallback
    assert dg.inner_operator == inner
    assert dg.residual_norm <= TOL * dg.rhs_norm * (1 + 1e-12)
    assert _residual(m, rhs, x) <= TOL * dg.rhs_norm * 1.01
    err = float((x - big.x64).norm() / big.x64.norm())
    assert err < 1e-8, err
