"""Generate golden vectors from the reference's own hot-path sources.

Runs the reference's DefaultAssembler2D/3D.cpp and paso Solver.cpp/PCG.cpp/
SparseMatrix_MatrixVector.cpp, compiled in place by ``make -C oracle ref`` into
oracle/_ref/libripley_ref.so, on small seeded inputs and stores inputs and outputs in
tests/golden/golden.npz.  The reference tree is needed only to run this script; the
tests read the committed .npz.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402


def coef_set(rng, dim, nel, kind):
    nq = 1 << dim
    out = {}
    for name, size in (("A", dim * dim), ("B", dim), ("C", dim), ("D", 1), ("X", dim), ("Y", 1)):
        n = size if kind == O.CONSTANT else size * nq * nel
        out[name] = rng.standard_normal(n)
    return out


def top_mask(dim, ne):
    nn = [e + 1 for e in ne]
    n = int(np.prod(nn))
    layer = int(np.prod(nn[: dim - 1]))
    q = np.zeros(n)
    q[(np.arange(n) // layer) == nn[dim - 1] - 1] = 1.0
    return q


def kappa_problem(rng, dim, ne):
    nel = int(np.prod(ne))
    nq = 1 << dim
    kappa = np.exp(rng.standard_normal(nel))
    A = np.zeros((nel, nq, dim, dim))
    for i in range(dim):
        A[:, :, i, i] = kappa[:, None]
    A = A.transpose(0, 1, 3, 2).reshape(-1)  # escript order A[i + d*j]
    Y = rng.standard_normal(nel * nq)
    return A, Y


def main():
    if not O.have_ref():
        O.build(reference=True)
    rng = np.random.default_rng(20261203)
    g = {}
    for dim, ne in ((2, (5, 7)), (3, (3, 4, 5))):
        dx = tuple(0.3 + 0.2 * k for k in range(dim))
        tag = f"{dim}d"
        pat = O.pattern(dim, ne)
        g[f"pat{tag}_ptr"], g[f"pat{tag}_idx"] = pat.ptr, pat.idx
        nel = int(np.prod(ne))
        for kname, kind in (("const", O.CONSTANT), ("exp", O.EXPANDED)):
            cs = coef_set(rng, dim, nel, kind)
            val, rhs = O.assemble(dim, ne, dx, pat, use_ref=True,
                                  **{("C_" if k == "C" else k): (kind, v) for k, v in cs.items()})
            for k, v in cs.items():
                g[f"asm{tag}_{kname}_{k}"] = v
            g[f"asm{tag}_{kname}_val"] = val
            g[f"asm{tag}_{kname}_rhs"] = rhs
            nf = (2 * ne[1] + 2 * ne[0]) if dim == 2 else 2 * (ne[1] * ne[2] + ne[0] * ne[2] + ne[0] * ne[1])
            nqf = 1 << (dim - 1)
            d = rng.standard_normal(1 if kind == O.CONSTANT else nf * nqf)
            y = rng.standard_normal(1 if kind == O.CONSTANT else nf * nqf)
            bval = np.zeros(pat.nnz)
            brhs = np.zeros(pat.n)
            O.assemble_boundary(dim, ne, dx, pat, bval, brhs, d=(kind, d), y=(kind, y), use_ref=True)
            g[f"bnd{tag}_{kname}_d"], g[f"bnd{tag}_{kname}_y"] = d, y
            g[f"bnd{tag}_{kname}_val"], g[f"bnd{tag}_{kname}_rhs"] = bval, brhs
        g[f"asm{tag}_dx"] = np.array(dx)
        g[f"asm{tag}_ne"] = np.array(ne)

    # solves: variable-coefficient Poisson with Dirichlet on the top face, tol 1e-10
    for dim, ne in ((2, (24, 20)), (3, (10, 9, 8))):
        tag = f"{dim}d"
        pat = O.pattern(dim, ne)
        A, Y = kappa_problem(rng, dim, ne)
        dx = [1.0 / e for e in ne]
        val, rhs = O.assemble(dim, ne, dx, pat, A=(O.EXPANDED, A), Y=(O.EXPANDED, Y), use_ref=True)
        q = top_mask(dim, ne)
        O.insert_constraint(pat, val, rhs, q)
        sys_val = val.copy()
        res = O.solve_paso(pat, val, rhs, tol=1e-10, use_ref=True)
        g[f"solve{tag}_ne"] = np.array(ne)
        g[f"solve{tag}_A"], g[f"solve{tag}_Y"], g[f"solve{tag}_q"] = A, Y, q
        g[f"solve{tag}_val"], g[f"solve{tag}_rhs"] = sys_val, rhs
        g[f"solve{tag}_x"] = res.x
        g[f"solve{tag}_iter"] = np.array(res.num_iter)
        g[f"solve{tag}_status"] = np.array(res.status)

    # the reference's CPU-runnable configuration: Rectangle 200x200, A = I, Y = 1,
    # u = 0 on y = 0, PCG + Jacobi rtol 1e-8
    ne = (200, 200)
    pat = O.pattern(2, ne)
    val, rhs = O.assemble(2, ne, (1 / 200, 1 / 200), pat, A=(O.CONSTANT, np.eye(2).reshape(-1)),
                          Y=(O.CONSTANT, np.ones(1)), use_ref=True)
    nn = 201
    q = np.zeros(nn * nn)
    q[:nn] = 1.0  # y == 0 row
    O.insert_constraint(pat, val, rhs, q)
    res = O.solve_paso(pat, val, rhs, tol=1e-8, use_ref=True)
    g["r200_x"] = res.x
    g["r200_iter"] = np.array(res.num_iter)

    out = os.path.join(HERE, "golden.npz")
    # reduced-order interior assembly (coefficients on ReducedFunction, one value set per
    # element), from its own generator so that the cases above keep their values.  (The
    # solution vectors of the solve cases depend on the reference's OpenMP thread count at
    # the 1e-13 level; the committed file keeps those of its first generation.)
    rr = np.random.default_rng(20261204)
    for dim, ne in ((2, (5, 7)), (3, (3, 4, 5))):
        dx = tuple(0.3 + 0.2 * k for k in range(dim))
        tag = f"{dim}d"
        pat = O.pattern(dim, ne)
        nel = int(np.prod(ne))
        for kname, kind in (("const", O.CONSTANT), ("exp", O.EXPANDED)):
            cs = {}
            for name, size in (("A", dim * dim), ("B", dim), ("C", dim), ("D", 1), ("X", dim), ("Y", 1)):
                cs[name] = rr.standard_normal(size if kind == O.CONSTANT else size * nel)
            val, rhs = O.assemble(dim, ne, dx, pat, use_ref=True, reduced=True,
                                  **{("C_" if k == "C" else k): (kind, v) for k, v in cs.items()})
            for k, v in cs.items():
                g[f"red{tag}_{kname}_{k}"] = v
            g[f"red{tag}_{kname}_val"] = val
            g[f"red{tag}_{kname}_rhs"] = rhs

    # PDE systems (block size nb = numEq = numComp): assemblePDESystem for every coefficient
    # with random data, and a Lame elasticity solve clamped on the bottom face
    rs = np.random.default_rng(20261205)
    for dim, ne, nb in ((2, (5, 7), 2), (3, (3, 4, 5), 3)):
        dx = tuple(0.3 + 0.2 * k for k in range(dim))
        tag = f"{dim}d"
        pat = O.pattern(dim, ne)
        nel = int(np.prod(ne))
        nq = 1 << dim
        sizes = {"A": nb * nb * dim * dim, "B": nb * nb * dim, "C": nb * nb * dim, "D": nb * nb, "X": nb * dim,
                 "Y": nb}
        for kname, kind in (("const", O.CONSTANT), ("exp", O.EXPANDED)):
            cs = {k: rs.standard_normal(v if kind == O.CONSTANT else v * nq * nel) for k, v in sizes.items()}
            val, rhs = O.assemble_system(dim, ne, dx, pat, nb, use_ref=True,
                                         **{("C_" if k == "C" else k): (kind, v) for k, v in cs.items()})
            for k, v in cs.items():
                g[f"sys{tag}_{kname}_{k}"] = v
            g[f"sys{tag}_{kname}_val"] = val
            g[f"sys{tag}_{kname}_rhs"] = rhs
        g[f"sys{tag}_nb"] = np.array(nb)
    for dim, ne in ((2, (16, 12)), (3, (5, 4, 6))):
        nb = dim
        tag = f"{dim}d"
        dx = tuple(1.0 / e for e in ne)
        pat = O.pattern(dim, ne)
        nel = int(np.prod(ne))
        nq = 1 << dim
        lam, mu = 1.0, 0.5
        A = np.zeros((dim, dim, dim, dim))
        for k in range(dim):
            for i in range(dim):
                for m in range(dim):
                    for j in range(dim):
                        A[k, i, m, j] = lam * (k == i) * (m == j) + mu * ((k == m) * (i == j) + (k == j) * (i == m))
        A = A.reshape(-1, order="F")
        Y = rs.standard_normal(nb * nq * nel)
        val, rhs = O.assemble_system(dim, ne, dx, pat, nb, A=(O.CONSTANT, A), Y=(O.EXPANDED, Y), use_ref=True)
        nn = [e + 1 for e in ne]
        n = int(np.prod(nn))
        layer = int(np.prod(nn[: dim - 1]))
        q = np.repeat(((np.arange(n) // layer) == 0).astype(np.float64), nb)
        O.insert_constraint_block(pat, nb, val, rhs, q)
        res = O.solve_paso_block(pat, nb, val.copy(), rhs, tol=1e-10, use_ref=True)
        g[f"lame{tag}_ne"] = np.array(ne)
        g[f"lame{tag}_A"], g[f"lame{tag}_Y"], g[f"lame{tag}_q"] = A, Y, q
        g[f"lame{tag}_x"], g[f"lame{tag}_iter"] = res.x, np.array(res.num_iter)

    # face terms of PDE systems and on ReducedFunctionOnBoundary, and the reduced-order
    # system terms: assemblePDEBoundarySystem, assemblePDEBoundarySingleReduced,
    # assemblePDEBoundarySystemReduced, assemblePDESystemReduced
    rb = np.random.default_rng(20261206)
    for dim, ne in ((2, (5, 7)), (3, (3, 4, 5))):
        dx = tuple(0.3 + 0.2 * k for k in range(dim))
        tag = f"{dim}d"
        pat = O.pattern(dim, ne)
        nel = int(np.prod(ne))
        nface = 2 * ne[1] + 2 * ne[0] if dim == 2 else 2 * (ne[1] * ne[2] + ne[0] * ne[2] + ne[0] * ne[1])
        for case, nb, reduced in (("bred", 1, True), ("bsys", dim, False), ("bsysred", dim, True)):
            nq = 1 if reduced else 1 << (dim - 1)
            for kname, kind in (("const", O.CONSTANT), ("exp", O.EXPANDED)):
                cnt = 1 if kind == O.CONSTANT else nface * nq
                d = rb.standard_normal(cnt * nb * nb)
                y = rb.standard_normal(cnt * nb)
                bval = np.zeros(pat.nnz * nb * nb)
                brhs = np.zeros(pat.n * nb)
                O.assemble_boundary(dim, ne, dx, pat, bval, brhs, d=(kind, d), y=(kind, y), use_ref=True, nb=nb,
                                    reduced=reduced)
                g[f"{case}{tag}_{kname}_d"], g[f"{case}{tag}_{kname}_y"] = d, y
                g[f"{case}{tag}_{kname}_val"], g[f"{case}{tag}_{kname}_rhs"] = bval, brhs
        nb = dim
        sizes = {"A": nb * nb * dim * dim, "B": nb * nb * dim, "C": nb * nb * dim, "D": nb * nb, "X": nb * dim,
                 "Y": nb}
        for kname, kind in (("const", O.CONSTANT), ("exp", O.EXPANDED)):
            cs = {k: rb.standard_normal(v if kind == O.CONSTANT else v * nel) for k, v in sizes.items()}
            val, rhs = O.assemble_system(dim, ne, dx, pat, nb, use_ref=True, reduced=True,
                                         **{("C_" if k == "C" else k): (kind, v) for k, v in cs.items()})
            for k, v in cs.items():
                g[f"sysred{tag}_{kname}_{k}"] = v
            g[f"sysred{tag}_{kname}_val"] = val
            g[f"sysred{tag}_{kname}_rhs"] = rhs

    # paso Solver/PCG with Jacobi(sweeps) for sweeps = 2, 3 (Smoother.cpp:100-128) on the
    # solve systems above
    for tag in ("2d", "3d"):
        ne = tuple(int(v) for v in g[f"solve{tag}_ne"])
        pat = O.pattern(len(ne), ne)
        for sw in (2, 3):
            res = O.solve_paso(pat, g[f"solve{tag}_val"].copy(), g[f"solve{tag}_rhs"], tol=1e-10, sweeps=sw,
                               use_ref=True)
            g[f"sweep{tag}_{sw}_x"] = res.x
            g[f"sweep{tag}_{sw}_iter"] = np.array(res.num_iter)

    # the Lame systems with block Jacobi of 2 sweeps
    for dim in (2, 3):
        tag = f"{dim}d"
        ne = tuple(int(v) for v in g[f"lame{tag}_ne"])
        dx = tuple(1.0 / e for e in ne)
        pat = O.pattern(dim, ne)
        val, rhs = O.assemble_system(dim, ne, dx, pat, dim, A=(O.CONSTANT, g[f"lame{tag}_A"]),
                                     Y=(O.EXPANDED, g[f"lame{tag}_Y"]), use_ref=True)
        O.insert_constraint_block(pat, dim, val, rhs, g[f"lame{tag}_q"])
        res = O.solve_paso_block(pat, dim, val, rhs, tol=1e-10, use_ref=True, sweeps=2)
        g[f"lamesw{tag}_x"], g[f"lamesw{tag}_iter"] = res.x, np.array(res.num_iter)

    # arrays already in the committed file keep their values (the solve cases depend on the
    # reference's OpenMP thread count at the 1e-13 level); new keys are added
    if os.path.exists(out):
        with np.load(out) as old:
            kept = {k: old[k] for k in old.files}
        g.update(kept)
    np.savez_compressed(out, **g)
    print(f"wrote {out}: {len(g)} arrays, {os.path.getsize(out) / 1024:.0f} KiB; "
          f"iterations r200={int(g['r200_iter'])} solve2d={int(g['solve2d_iter'])} "
          f"solve3d={int(g['solve3d_iter'])}")


if __name__ == "__main__":
    main()
