"""The element-coefficient operator of the FP32 inner solve (RG_LAYOUT_COEF) on the CPU: the
formula the kernel evaluates per row - the 27 (9 in 2D) coefficients as the Q1 table entry
T[|o|] times the sum of kappa over the elements shared by the node and its neighbour o, read
from the node-indexed array khat (khat[i] = kappa of the element whose upper corner is node i)
- is restated here in numpy and must rebuild the matrix the oracle assembles for A = kappa I per
element (DefaultAssembler3D/2D::assemblePDESingle, ripley/src/DefaultAssembler3D.cpp:152-2226,
DefaultAssembler2D.cpp:151-597), anisotropic spacings included.  The GPU kernel's use of it is
tested against the oracle's solves in tests/test_gpu_coef_operator.py."""
import numpy as np
import pytest

from oracle import oracle as O


def q1_table(dim, dx):
    """T[cls]: the Q1 stiffness entry of two nodes of one box element differing in the axes of
    cls's bits (exact 1D integrals: K = +-1/h, M = h/3 or h/6 per axis)."""
    T = np.zeros(8)
    for cls in range(8):
        k = [(-1.0 if (cls >> a) & 1 else 1.0) / dx[a] for a in range(3)]
        m = [dx[a] / 6.0 if (cls >> a) & 1 else dx[a] / 3.0 for a in range(3)]
        T[cls] = (k[0] * m[1] * m[2] + m[0] * k[1] * m[2] + m[0] * m[1] * k[2]) if dim == 3 else \
            (k[0] * m[1] + m[0] * k[1])
    return T


def khat_array(dim, ne, kappa):
    nn = [e + 1 for e in ne] + [1] * (3 - dim)
    n = int(np.prod(nn[:dim]))
    kh = np.zeros(n + nn[0] * nn[1] + nn[0] + 1024)
    ex = np.arange(int(np.prod(ne)))
    x = ex % ne[0]
    y = (ex // ne[0]) % ne[1]
    z = ex // (ne[0] * ne[1]) if dim == 3 else 0 * ex
    node = (x + 1) + nn[0] * (y + 1) + (nn[0] * nn[1] * (z + 1) if dim == 3 else 0)
    kh[node] += kappa
    return kh, nn, n


def operator_rows(dim, ne, dx, kappa):
    """[(column offset, coefficient of every row)] of the element-coefficient operator (no
    constraint), one entry per stencil point.  On thin grids two stencil points can share a
    column offset (e.g. (0, 1, 0) and (0, -1, 1) when NN1 = 2); the one whose neighbour does
    not exist has coefficient 0, and the kernel, like this function, sums over stencil points."""
    kh, nn, n = khat_array(dim, ne, kappa)
    T = q1_table(dim, dx)
    nk = 8 if dim == 3 else 4
    i = np.arange(n)
    kv = np.zeros((n, 8))
    for j in range(nk):
        a, b, c = j & 1, (j >> 1) & 1, j >> 2
        kv[:, j] = kh[i + a + nn[0] * b + nn[0] * nn[1] * c]
    A = {(-1): [0], 0: [0, 1], 1: [1]}
    out = []
    for oz in ((-1, 0, 1) if dim == 3 else (0,)):
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                K = np.zeros(n)
                for c in (A[oz] if dim == 3 else [0]):
                    for b in A[oy]:
                        for a in A[ox]:
                            K += kv[:, a + 2 * b + 4 * c]
                cls = (ox != 0) + 2 * (oy != 0) + 4 * (oz != 0)
                off = ox + nn[0] * oy + nn[0] * nn[1] * oz
                out.append((off, T[cls] * K))
    return out, n


@pytest.mark.parametrize("dim,ne,length", [(3, (7, 5, 4), (1.0, 2.0, 0.5)), (3, (3, 3, 3), (1.0, 1.0, 1.0)),
                                           (2, (9, 6), (1.0, 3.0)), (3, (12, 1, 2), (2.0, 0.25, 1.0))])
def test_coefficient_operator_rebuilds_the_assembled_matrix(dim, ne, length):
    rng = np.random.default_rng(5)
    nel = int(np.prod(ne))
    kappa = np.exp(rng.standard_normal(nel))
    dx = [length[k] / ne[k] for k in range(dim)] + [1.0] * (3 - dim)
    pat = O.pattern(dim, ne)
    Ape = np.zeros((nel, dim, dim))
    for k in range(dim):
        Ape[:, k, k] = kappa
    val, _ = O.assemble(dim, ne, dx[:dim], pat, A=(O.PER_ELEMENT, Ape.reshape(-1)))
    coeffs, n = operator_rows(dim, ne, dx, kappa)
    # the operator as a dense matrix (small grids), summed over stencil points
    dense = np.zeros((n, n))
    i = np.arange(n)
    for off, c in coeffs:
        j = i + off
        ok = (j >= 0) & (j < n)
        np.add.at(dense, (i[ok], j[ok]), c[ok])
        # a stencil point whose column falls outside the grid has coefficient 0
        assert np.all(c[~ok] == 0.0)
    rows = np.repeat(np.arange(n), np.diff(pat.ptr))
    ref = np.zeros((n, n))
    ref[rows, pat.idx] = val
    scale = np.abs(ref).max(axis=1)
    assert np.max(np.abs(dense - ref) / scale[:, None]) < 1e-13


def test_fixed_nodes_are_flagged_by_the_sign_bit():
    """khat carries the constraint's mask in the sign bit, -0.0 included for nodes that are no
    element's upper corner (the kernel reads it with the bit pattern, not a comparison)."""
    kh = np.zeros(4, dtype=np.float32)
    kh[1] = 2.5
    q = np.array([1.0, 1.0, 0.0, 0.0])
    kh = np.where(q > 0, -np.abs(kh), kh).astype(np.float32)
    bits = kh.view(np.uint32) >> 31
    assert bits.tolist() == [1, 1, 0, 0]
    assert np.abs(kh).tolist() == [0.0, 2.5, 0.0, 0.0]
