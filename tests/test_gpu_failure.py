"""Failure detection on the GPU without a GPU fault: the bounded waits of the band SpMV
kernels are made to run out (their producer withholds every copy, so nothing is ever in
flight), the solve must return RG_TIMEOUT, and the next solve on the same matrix and domain
must match the oracle, i.e. nothing the interrupted launch left behind (the grid-reduction
counter, the device scalars, the captured iteration graphs) leaks into later work.  The same
hook makes the persistent tcgen05 convolution's waits run out: it must set its device error
flag, free its tensor memory, and the next convolution must be correct.

The paso status mapping the library follows is paso/src/solve.cpp:119-142 (a solver status
becomes an exception); RG_TIMEOUT has no paso counterpart because paso has no device waits.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _problem(ne, seed):
    rng = np.random.default_rng(seed)
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
    q = np.zeros(d.n)
    q[-(ne[0] + 1) * (ne[1] + 1):] = 1.0  # top face
    R.insert_constraint(m, rhs, R.dev(q))
    pat = O.pattern(3, ne)
    val, rr = O.assemble(3, ne, d.dx, pat, A=(O.EXPANDED, A), Y=(O.EXPANDED, Y))
    O.insert_constraint(pat, val, rr, q)
    return d, m, rhs, keep, (pat, val, rr)


@pytest.mark.parametrize("mode,precision,layout,tol", [
    # k_band64_bulk (paso PCG on the FP64 band copy)
    (L.RG_MODE_PASO, L.RG_PREC_FP64, L.RG_LAYOUT_BAND, 1e-8),
    # k_f32_cg on the FP32 band copy, and on the element coefficients
    (L.RG_MODE_STANDARD, L.RG_PREC_FP32_REFINE, L.RG_LAYOUT_BAND, 1e-7),
    (L.RG_MODE_STANDARD, L.RG_PREC_FP32_REFINE, L.RG_LAYOUT_COEF, 1e-7),
])
def test_band_kernel_wait_timeout_is_reported_and_recoverable(cuda, mode, precision, layout, tol):
    d, m, rhs, _keep, (pat, val, rr) = _problem((24, 20, 18), 31)
    ref = O.solve_paso(pat, val.copy(), rr, tol=1e-10)  # balances its copy in place
    assert ref.converged
    o = R.opts(tolerance=1e-10, mode=mode, precision=precision, layout=layout)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    # a normal solve first: the FP32 tuner and the captured iteration graphs exist before the
    # waits are shortened, so the interrupted solve replays graphs captured earlier
    st, dg = R.solve(m, rhs, x, o)
    assert st == 0 and dg.converged
    if layout == L.RG_LAYOUT_COEF:
        assert dg.inner_operator == 1
    first = x.clone()
    lib = R.lib()
    x.fill_(7.0)
    L.check(lib.rg_test_wait_limit(64, 1))
    try:
        st, dg = R.solve(m, rhs, x, o)
    finally:
        L.check(lib.rg_test_wait_limit(0, 0))
    assert st == L.RG_TIMEOUT, (st, L.last_error())
    assert "wait" in L.last_error()
    assert not dg.converged
    # the library, the matrix and its domain stay usable, and nothing from the interrupted
    # launch leaks into the next solve
    x.zero_()
    st, dg = R.solve(m, rhs, x, o)
    assert st == 0 and dg.converged
    err = np.linalg.norm(x.cpu().numpy() - ref.x) / np.linalg.norm(ref.x)
    assert err < tol, err
    assert torch.allclose(x, first, rtol=0, atol=1e-12 * float(first.abs().max()))
    if precision == L.RG_PREC_FP64:
        assert abs(int(dg.num_iter) - ref.num_iter) <= 1
    # an unrelated reduction on the same workspace (the residual norms) is exact as well
    import ctypes
    l2, lm = ctypes.c_double(), ctypes.c_double()
    L.check(lib.rg_residual_norms(m.h, R.ptr(rhs), R.ptr(x), ctypes.byref(l2), ctypes.byref(lm)))
    res = rr - O.spmv(pat, val, x.cpu().numpy())
    assert abs(l2.value - np.linalg.norm(res)) <= 1e-9 * np.linalg.norm(rr)


def test_wait_limit_arguments_are_checked(cuda):
    lib = R.lib()
    assert lib.rg_test_wait_limit(-1, 0) == L.RG_INVALID_ARG
    L.check(lib.rg_test_wait_limit(0, 0))


def test_conv_wait_timeout_sets_error_flag_and_recovers(cuda):
    """The persistent tcgen05 convolution (64^3, 16 -> 16 channels) with its producer withholding
    every copy: the MMA issuer's and the epilogue warps' bounded waits run out (nothing is in
    flight, no UMMA is issued), the kernel releases its tensor memory and sets the device error
    flag; with the limits restored the next convolution matches the fp32 reference."""
    import torch.nn.functional as F
    from esys_b200 import warmstart as W
    torch.manual_seed(1)
    d = 64
    x = W.new_act(1, d, d, d, 16)
    xv = torch.randn(1, d, d, d, 16, device="cuda").to(torch.bfloat16)
    W.interior(x).copy_(xv)
    wt = (torch.randn(27, 16, 16, device="cuda") * 0.05).to(torch.bfloat16).contiguous()
    b = torch.randn(16, device="cuda")
    y = W.new_act(1, d, d, d, 16)
    lib = R.lib()
    err = W.DeviceError()
    L.check(lib.rg_test_wait_limit(64, 1))
    try:
        W.conv3(x, wt, b, y, relu=True, err=err)
        torch.cuda.synchronize()
        with pytest.raises(L.RipleyGPUError):
            err.check()
    finally:
        L.check(lib.rg_test_wait_limit(0, 0))
    ok = W.DeviceError()
    W.conv3(x, wt, b, y, relu=True, err=ok)
    torch.cuda.synchronize()
    ok.check()
    w5 = wt.float().cpu().reshape(3, 3, 3, 16, 16).permute(3, 4, 0, 1, 2)  # (Cout, Cin, kd, kh, kw)
    ref = torch.relu(F.conv3d(xv.float().cpu().permute(0, 4, 1, 2, 3), w5, b.cpu(), padding=1)).permute(0, 2, 3, 4, 1)
    got = W.interior(y).float().cpu()
    assert (got - ref).abs().max().item() <= 2e-2 * ref.abs().max().item()
