"""rg_save_mm, the MatrixMarket writer of the system-matrix plugin (SystemMatrix::saveMM,
paso/src/SystemMatrix.h:70-80, SparseMatrix<double>::saveMM, paso/src/SparseMatrix.cpp:180-240).

The written file is parsed and compared entry by entry, in order, with the oracle's CSR
matrix laid out the way paso writes it: banner, size line (rows, columns, nnz * nb^2),
then per node row its pattern entries, each as its nb x nb block of scalar coordinates
(row-block index outer), 1-based, values with 15 significant digits.  Indices must be
identical; values agree within the assembly tolerance (1e-13 of the row's largest entry)
plus the rounding of the written digits.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import rgcapi as R
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

BANNER = "%%MatrixMarket matrix coordinate real general"


def expected_entries(pat, val, nb):
    nnz = pat.nnz
    node = np.repeat(np.arange(pat.n), np.diff(pat.ptr))
    ir = np.arange(nb)[None, :, None]
    ic = np.arange(nb)[None, None, :]
    rows = node[:, None, None] * nb + ir + 1 + 0 * ic
    cols = pat.idx[:, None, None].astype(np.int64) * nb + ic + 1 + 0 * ir
    vals = val.reshape(nnz, nb, nb).transpose(0, 2, 1)  # val[k nb^2 + ir + nb ic] -> [k, ir, ic]
    return rows.reshape(-1), cols.reshape(-1), vals.reshape(-1)


def read_mm(path):
    with open(path) as f:
        banner = f.readline().rstrip("\n")
        size = [int(v) for v in f.readline().split()]
        data = np.loadtxt(f, ndmin=2)
    return banner, size, data


def check_file(path, pat, val, nb):
    banner, size, data = read_mm(path)
    assert banner == BANNER
    assert size == [pat.n * nb, pat.n * nb, pat.nnz * nb * nb]
    rows, cols, vals = expected_entries(pat, val, nb)
    assert data.shape == (len(rows), 3)
    assert np.array_equal(data[:, 0].astype(np.int64), rows)
    assert np.array_equal(data[:, 1].astype(np.int64), cols)
    # values: the assembly's tolerance against the oracle, 1e-13 of the largest entry of the
    # (scalar) row, plus the rounding of the 15 significant digits written
    rowmax = np.zeros(pat.n * nb)
    np.maximum.at(rowmax, rows - 1, np.abs(vals))
    tol = 1e-13 * rowmax[rows - 1] + 1e-14 * np.abs(vals)
    assert np.all(np.abs(data[:, 2] - vals) <= tol), float((np.abs(data[:, 2] - vals) / rowmax[rows - 1]).max())


def test_save_mm_scalar_matches_oracle(cuda, tmp_path):
    rng = np.random.default_rng(41)
    ne = (3, 4, 5)
    nel = int(np.prod(ne))
    A = rng.standard_normal(nel * 8 * 9)
    D = rng.standard_normal(nel * 8)
    Y = rng.standard_normal(nel * 8)
    d = R.Domain(3, ne)
    m = R.Matrix(d)
    rhs = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble(m, rhs, keep, A=(A, R.KINDS["exp"]), D=(D, R.KINDS["exp"]), Y=(Y, R.KINDS["exp"]))
    q = (rng.random(d.n) < 0.2).astype(float)
    R.insert_constraint(m, rhs, R.dev(q))
    pat = O.pattern(3, ne)
    val, rr = O.assemble(3, ne, d.dx, pat, A=(O.EXPANDED, A), D=(O.EXPANDED, D), Y=(O.EXPANDED, Y))
    O.insert_constraint(pat, val, rr, q)
    path = tmp_path / "scalar.mtx"
    L.check(R.lib().rg_save_mm(m.h, str(path).encode()))
    check_file(path, pat, val, 1)


def test_save_mm_block3_system_matches_oracle(cuda, tmp_path):
    rng = np.random.default_rng(42)
    ne = (3, 4, 5)
    nb = 3
    nel = int(np.prod(ne))
    A = rng.standard_normal(nel * 8 * nb * 3 * nb * 3)
    D = rng.standard_normal(nel * 8 * nb * nb)
    Y = rng.standard_normal(nel * 8 * nb)
    d = R.Domain(3, ne)
    m = R.Matrix(d, block_size=nb)
    rhs = torch.zeros(d.n * nb, dtype=torch.float64, device="cuda")
    keep = []
    R.assemble_system(m, rhs, keep, A=(A, R.KINDS["exp"]), D=(D, R.KINDS["exp"]), Y=(Y, R.KINDS["exp"]))
    pat = O.pattern(3, ne)
    val, _ = O.assemble_system(3, ne, d.dx, pat, nb, A=(O.EXPANDED, A), D=(O.EXPANDED, D), Y=(O.EXPANDED, Y))
    path = tmp_path / "block3.mtx"
    L.check(R.lib().rg_save_mm(m.h, str(path).encode()))
    check_file(path, pat, val, nb)


def test_save_mm_through_linear_pde_and_errors(cuda, tmp_path):
    """LinearPDE.getOperator().saveMM writes the same file; a path that cannot be opened is
    an error (paso: PasoException 'File could not be opened for writing')."""
    from esys_b200.escript import LinearPDE
    from esys_b200.ripley import Rectangle
    dom = Rectangle(4, 3)
    pde = LinearPDE(dom)
    pde.setValue(A=np.eye(2), D=1.0, Y=1.0)
    op = pde.getOperator()
    path = tmp_path / "pde.mtx"
    op.saveMM(str(path))
    pat = O.pattern(2, (4, 3))
    val, _ = O.assemble(2, (4, 3), [0.25, 1.0 / 3.0], pat, A=(O.CONSTANT, np.eye(2).reshape(-1)),
                        D=(O.CONSTANT, np.ones(1)), Y=(O.CONSTANT, np.ones(1)))
    check_file(path, pat, val, 1)
    with pytest.raises(ValueError):
        op.saveMM(str(tmp_path / "no_such_dir" / "x.mtx"))
