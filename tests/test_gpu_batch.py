"""Batched solves (rg_batch_*) against single-system solves of the same systems.

Each right hand side must meet paso's dual-norm test at rtol 1e-8 in the balanced norms the
batch reports, and agree with an FP64 single-system solve to rtol 1e-11 within 1e-6
(relative l2): the distance allowed by the 1e-8 residual tolerance times the conditioning
of these small systems."""
import pytest
import torch

from esys_b200.batch import BatchSolver, make_batch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nrhs", [1, 2, 8])
def test_batch_matches_single_solves(cuda, nrhs):
    systems, rhs = make_batch(5, nrhs, edges=(8, 12, 16, 20), corr_cells=2.0, seed=10 + nrhs)
    xs = [torch.zeros_like(b) for b in rhs]
    with BatchSolver([s.mat for s in systems], nrhs) as bs:
        info = bs.tune()
        assert info["grid_spmv"] > 0 and info["grid_update"] > 0 and 4 <= info["chunk"] <= 64
        diags = bs.solve(rhs, xs, tol=1e-8)
        # a second solve of the same right hand sides gives the same bits
        xs2 = [torch.zeros_like(b) for b in rhs]
        bs.solve(rhs, xs2, tol=1e-8)
    for a, b in zip(xs, xs2):
        assert torch.equal(a, b)
    for i, s in enumerate(systems):
        for k in range(nrhs):
            d = diags[i * nrhs + k]
            assert d.converged
            assert d.residual_norm <= 1e-8 * d.rhs_norm * (1 + 1e-9)
            assert d.num_iter > 0
            s.rhs.copy_(rhs[i][k])
            s.solve(tol=1e-11, fp32=False)
            err = float((xs[i][k] - s.x).norm() / s.x.norm())
            assert err < 1e-6, (i, k, err)
    for s in systems:
        s.close()


def test_batch_uneven_sizes_and_zero_rhs(cuda):
    systems, rhs = make_batch(3, 2, edges=(8, 24), corr_cells=2.0, seed=3)
    rhs[1][1].zero_()      # a zero right hand side converges at once with x = 0
    xs = [torch.full_like(b, 7.0) for b in rhs]
    with BatchSolver([s.mat for s in systems], 2) as bs:
        diags = bs.solve(rhs, xs, tol=1e-8)
    assert not bool(xs[1][1].any())
    assert diags[3].num_iter == 0 and diags[3].converged
    for d in diags:
        assert d.converged
    for s in systems:
        s.close()


def test_batch_rejects_changed_matrices(cuda):
    systems, rhs = make_batch(2, 1, edges=(8,), corr_cells=2.0, seed=4)
    bs = BatchSolver([s.mat for s in systems], 1)
    systems[0].assemble(torch.ones(systems[0].nel, device="cuda", dtype=torch.float64))
    with pytest.raises(ValueError):
        bs.solve(rhs, [torch.zeros_like(b) for b in rhs])
    bs.close()
    for s in systems:
        s.close()


@pytest.mark.parametrize("kernel", ["row", "pair"])
def test_batch_spmv_kernels_agree(cuda, kernel):
    """Both SpMV kernels, pinned through rg_batch_set_spmv, solve the same batch (Bricks of
    edges up to 40, so that some systems span several work units) to solutions within 1e-6
    of each other, each meeting the residual test.  The two kernels sum p.q in different
    orders and FP32 PCG iteration counts move with that (single-tile systems match), so only
    the totals are compared, within 10 %."""
    systems, rhs = make_batch(4, 4, edges=(8, 24, 40), corr_cells=3.0, seed=21)
    out = {}
    for k in ("row", kernel):
        xs = [torch.zeros_like(b) for b in rhs]
        with BatchSolver([s.mat for s in systems], 4) as bs:
            bs.set_spmv(k)
            info = bs.tune()
            assert info["spmv_kernel"] == k
            diags = bs.solve(rhs, xs, tol=1e-8)
        for d in diags:
            assert d.converged and d.residual_norm <= 1e-8 * d.rhs_norm * (1 + 1e-9)
        out[k] = (xs, [int(d.num_iter) for d in diags])
    (x0, it0), (x1, it1) = out["row"], out[kernel]
    for a, b in zip(x0, x1):
        assert float((a - b).norm() / a.norm()) < 1e-6
    assert abs(sum(it1) - sum(it0)) <= 0.1 * sum(it0)
    for s in systems:
        s.close()


def test_batch_set_spmv_rejects_unknown(cuda):
    from esys_b200 import _lib as L
    systems, _ = make_batch(1, 1, edges=(8,), corr_cells=2.0, seed=5)
    with BatchSolver([s.mat for s in systems], 1) as bs:
        with pytest.raises(ValueError):
            L.check(L.lib().rg_batch_set_spmv(bs._h, 2))
    for s in systems:
        s.close()
