"""The reference test suite's known-answer problems, run through the escript-facing API
(esys_b200.escript / esys_b200.ripley) on the GPU.  Each mirrors a reference test:
  test_PCG_JACOBI         escriptcore/test/python/test_linearPDEs.py:1741-1748
  Test_Poisson.test_solve escriptcore/test/python/test_linearPDEs.py:382-407
  SimpleSolve test_single escriptcore/test/python/test_simplesolve.py:125-163,273-282
"""
import numpy as np
import pytest

from esys_b200.escript import (LinearPDE, Poisson, SolverOptions, Solution, ContinuousFunction,
                               Function, Scalar, Data, kronecker, whereZero, Lsup, inner)
from esys_b200 import ripley
from esys_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-8


def check(u, u_ex, tol=TOL):
    return Lsup(u - u_ex) <= tol * Lsup(u_ex)


@pytest.fixture(params=["rect", "brick"])
def domain(request, cuda):
    if request.param == "rect":
        return ripley.Rectangle(12 * 2 - 1, 12 * 2 - 1)
    return ripley.Brick(12 - 1, 12 - 1, 8 - 1)


@pytest.mark.parametrize("precision", [SolverOptions.PRECISION_FP64, SolverOptions.PRECISION_FP32_REFINE])
def test_pcg_jacobi(domain, precision):
    pde = LinearPDE(domain)
    pde.setValue(A=kronecker(domain), D=1.0, Y=1.0)
    so = pde.getSolverOptions()
    so.setSolverMethod(SolverOptions.PCG)
    so.setPreconditioner(SolverOptions.JACOBI)
    so.setPrecision(precision)
    u = pde.getSolution()
    assert check(u, 1.0), "solution is wrong."
    assert so.getDiagnostics("converged")


def test_pcg_jacobi_reduced_coefficients(domain):
    """test_PCG_JACOBI with the coefficients on ReducedFunction (the 1-point rule of
    assemblePDESingleReduced): A_reduced = I, D_reduced = 1, Y_reduced = 1 gives u = 1; mixed
    with full-order coefficients the systems add up."""
    pde = LinearPDE(domain)
    pde.setValue(A_reduced=kronecker(domain), D_reduced=1.0, Y_reduced=1.0)
    u = pde.getSolution()
    assert check(u, 1.0)
    pde2 = LinearPDE(domain)
    pde2.setValue(A=kronecker(domain), D_reduced=1.0, Y=0.5, Y_reduced=0.5)
    assert check(pde2.getSolution(), 1.0)


def test_poisson_quadratic(domain):
    d = domain.getDim()
    cf = ContinuousFunction(domain)
    x = cf.getX()
    u_ex = Scalar(1.0, cf)
    for i in range(d):
        u_ex *= x[i] * (2.0 - x[i])
    msk = Scalar(0.0, cf)
    for i in range(d):
        msk += whereZero(x[i])
    f = Scalar(0, cf)
    for i in range(d):
        f_p = Scalar(1, cf)
        for j in range(d):
            if i == j:
                f_p *= 2.0
            else:
                f_p *= x[j] * (2 - x[j])
        f += f_p
    pde = Poisson(domain)
    pde.setValue(f=f, q=msk)
    u = pde.getSolution()
    # Q1 on these meshes: discretisation error well below 1e-2
    assert check(u, u_ex, 1e-2)


def test_simple_solve_single(domain):
    dim = domain.getDim()
    x = Solution(domain).getX()
    u_ex = 1.0 + 2.0 * x[0] + 3.0 * x[1] + (4.0 * x[2] if dim == 3 else 0.0)
    g_ex = np.array([2.0, 3.0, 4.0][:dim])
    pde = LinearPDE(domain, numEquations=1)
    pde.setValue(r=u_ex, q=whereZero(x[0]), A=kronecker(dim), y=inner(g_ex, domain.getNormal()))
    so = pde.getSolverOptions()
    so.setSolverMethod(SolverOptions.PCG)
    so.setTolerance(1e-8)
    u = pde.getSolution()
    assert Lsup(u - u_ex) < 1e-6 * Lsup(u_ex)


def test_rhs_only_change_reuses_operator(cuda):
    dom = ripley.Brick(10, 8, 6)
    pde = LinearPDE(dom)
    pde.setValue(A=kronecker(3), D=1.0, Y=1.0)
    u1 = pde.getSolution()
    op1 = pde.getOperator()
    pde.setValue(Y=2.0)
    u2 = pde.getSolution()
    assert pde.getOperator() is op1
    assert check(u1, 1.0) and check(u2, 2.0)


def test_unsupported_features_raise(cuda):
    dom = ripley.Rectangle(4, 4)
    with pytest.raises(NotImplementedError):
        LinearPDE(dom, numEquations=4)
    # a non-square PDE can be defined (as in escript) but not solved on the GPU path
    ns = LinearPDE(dom, numEquations=2, numSolutions=3)
    ns.setValue(D=np.ones((2, 3)))
    with pytest.raises(ValueError):
        ns.getSolution()
    pde = LinearPDE(dom)
    with pytest.raises(NotImplementedError):
        pde.setValue(y_contact=1.0)
    with pytest.raises(ValueError):
        pde.setValue(Z=1.0)
    pde.setValue(A=kronecker(2), Y=1.0)
    pde.getSolverOptions().setSolverMethod(SolverOptions.GMRES)
    with pytest.raises(NotImplementedError):
        pde.getSolution()


def test_maxiter_raises_paso_exception(cuda):
    dom = ripley.Rectangle(40, 40)
    pde = LinearPDE(dom)
    x = Solution(dom).getX()
    pde.setValue(A=kronecker(2), Y=1.0, q=whereZero(x[1]))
    pde.getSolverOptions().setIterMax(3)
    with pytest.raises(L.PasoException) as e:
        pde.getSolution()
    assert e.value.status == L.RG_MAXITER


def test_function_space_coordinates(cuda):
    dom = ripley.Brick(3, 2, 2, l0=(1.0, 4.0))
    xq = Function(dom).getX().toNumpy()
    assert xq.shape == (12 * 8, 3)
    g0 = 0.5 - np.sqrt(3) / 6
    assert np.allclose(xq[0], [1.0 + g0, g0 / 2, g0 / 2])
    assert np.allclose(xq[1], [1.0 + 1 - g0, g0 / 2, g0 / 2])
    xn = Solution(dom).getX().toNumpy()
    assert np.allclose(xn[1], [2.0, 0, 0]) and np.allclose(xn[4], [1.0, 0.5, 0])
    # interpolation of a linear field to the Gauss points is exact
    lin = Data(Solution(dom).getX()[0] * 2.0 + Solution(dom).getX()[2], Function(dom))
    assert np.allclose(lin.toNumpy(), 2 * xq[:, 0] + xq[:, 2])


@pytest.mark.parametrize("dim", [2, 3])
def test_lame_system_through_linear_pde(cuda, golden, dim):
    """LinearPDE(numEquations=dim) with A = Lame tensor, Y on Function, u = 0 on the bottom
    face: the reference's solution (paso PCG + block Jacobi) to 1e-8."""
    import torch
    from esys_b200.escript import Vector, Function
    tag = f"{dim}d"
    ne = tuple(int(v) for v in golden[f"lame{tag}_ne"])
    dom = ripley.Rectangle(*ne) if dim == 2 else ripley.Brick(*ne)
    pde = LinearPDE(dom, numEquations=dim)
    assert pde.getNumEquations() == dim and pde.getNumSolutions() == dim
    A = golden[f"lame{tag}_A"].reshape((dim,) * 4, order="F")
    Y = Data._wrap(torch.as_tensor(golden[f"lame{tag}_Y"], device="cuda").reshape(-1, dim), (dim,), Function(dom))
    x = ContinuousFunction(dom).getX()
    q = whereZero(x[dim - 1]) * np.ones(dim)
    pde.setValue(A=A, Y=Y, q=q)
    pde.getSolverOptions().setTolerance(1e-10)
    u = pde.getSolution()
    ref = golden[f"lame{tag}_x"]
    got = u._dev().reshape(-1).cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-8
    assert abs(pde.getSolverOptions().getDiagnostics("num_iter") - int(golden[f"lame{tag}_iter"])) <= 1


def test_system_coupled_known_answer(cuda):
    dom = ripley.Brick(4, 3, 5)
    pde = LinearPDE(dom, numEquations=3)
    A = np.zeros((3, 3, 3, 3))
    for k in range(3):
        for i in range(3):
            A[k, i, k, i] = 1.0
    D = np.array([[2.0, -1.0, 0.0], [-1.0, 2.0, -1.0], [0.0, -1.0, 2.0]])
    pde.setValue(A=A, D=D, Y=D.sum(axis=1))
    u = pde.getSolution()
    assert float((u._dev() - 1.0).abs().max()) < 1e-8


@pytest.mark.parametrize("reduced", [False, True])
def test_robin_boundary_known_answer(domain, reduced):
    """A = I, D = 0, d = y = 2 on the whole boundary (FunctionOnBoundary, or
    ReducedFunctionOnBoundary for d_reduced / y_reduced): n.grad u + d u = y has u = 1."""
    pde = LinearPDE(domain)
    sfx = "_reduced" if reduced else ""
    pde.setValue(A=kronecker(domain), **{"d" + sfx: 2.0, "y" + sfx: 2.0})
    assert check(pde.getSolution(), 1.0)


@pytest.mark.parametrize("reduced", [False, True])
def test_system_boundary_and_reduced_known_answer(cuda, reduced):
    """Lame system with d = I and y = c on the boundary: the constant displacement c
    (zero strain) solves it; then D_reduced = I, Y_reduced = c alone (mass matrix on
    ReducedFunction) gives c too.  Face terms of systems: assemblePDEBoundarySystem
    (d, y) and assemblePDEBoundarySystemReduced (d_reduced, y_reduced)."""
    dom = ripley.Brick(5, 4, 3)
    c = np.array([1.0, -2.0, 0.5])
    lam, mu = 1.0, 0.5
    A = np.zeros((3, 3, 3, 3))
    for k in range(3):
        for i in range(3):
            for m in range(3):
                for j in range(3):
                    A[k, i, m, j] = lam * (k == i) * (m == j) + mu * ((k == m) * (i == j) + (k == j) * (i == m))
    sfx = "_reduced" if reduced else ""
    pde = LinearPDE(dom, numEquations=3)
    pde.setValue(A=A, **{"d" + sfx: np.eye(3), "y" + sfx: c})
    u = pde.getSolution()
    assert float((u._dev() - torch_tensor(c)).abs().max()) < 1e-8
    pde2 = LinearPDE(dom, numEquations=3)
    pde2.setValue(D_reduced=np.eye(3), Y_reduced=c)
    u2 = pde2.getSolution()
    assert float((u2._dev() - torch_tensor(c)).abs().max()) < 1e-8


def torch_tensor(a):
    import torch
    return torch.as_tensor(a, dtype=torch.float64, device="cuda")


def test_reduced_boundary_function_space(cuda):
    from esys_b200.escript import FunctionOnBoundary, ReducedFunctionOnBoundary
    dom = ripley.Brick(3, 2, 2)
    fs = ReducedFunctionOnBoundary(dom)
    assert fs.getTypeCode() == 11 and FunctionOnBoundary(dom).getTypeCode() == 5
    assert fs.getNumDataPointsPerSample() == 1
    xr = fs.getX().toNumpy()
    assert xr.shape == (2 * (2 * 2 + 3 * 2 + 3 * 2), 3)
    # the face centres of face 0 (x = 0), face element (ka, kb) = (0, 0): (0, 0.25, 0.25)
    assert np.allclose(xr[0], [0.0, 0.25, 0.25])
    # a linear field interpolates exactly to the face centres, from the nodes or the Gauss points
    lin = Solution(dom).getX()[0] + 2.0 * Solution(dom).getX()[1]
    assert np.allclose(lin.interpolate(fs).toNumpy(), xr[:, 0] + 2 * xr[:, 1])
    assert np.allclose(lin.interpolate(FunctionOnBoundary(dom)).interpolate(fs).toNumpy(), xr[:, 0] + 2 * xr[:, 1])


def test_jacobi_sweeps_through_solver_options(domain):
    """SolverOptions.setNumSweeps(2): paso's Jacobi smoother with two sweeps as
    preconditioner; the known answer u = 1 of test_PCG_JACOBI, and on a problem with
    Dirichlet data the same solution as with one sweep."""
    pde = LinearPDE(domain)
    pde.setValue(A=kronecker(domain), D=1.0, Y=1.0)
    pde.getSolverOptions().setNumSweeps(2)
    assert check(pde.getSolution(), 1.0)
    x = Solution(domain).getX()
    us = []
    for sw in (1, 2):
        p = LinearPDE(domain)
        p.setValue(A=kronecker(domain), Y=1.0, q=whereZero(x[0]))
        p.getSolverOptions().setNumSweeps(sw)
        p.getSolverOptions().setTolerance(1e-10)
        us.append(p.getSolution())
    assert Lsup(us[1] - us[0]) <= 1e-8 * Lsup(us[0])



def test_matrix_layout_through_solver_options(domain):
    """SolverOptions.setMatrixLayout(LAYOUT_BAND): FP64 solves (paso and standard mode) on
    the FP64 band copy give the known answer u = 1 and, with Dirichlet data, the CSR
    solution; an unknown layout is rejected."""
    pde = LinearPDE(domain)
    pde.setValue(A=kronecker(domain), D=1.0, Y=1.0)
    pde.getSolverOptions().setMatrixLayout(SolverOptions.LAYOUT_BAND)
    assert check(pde.getSolution(), 1.0)
    x = Solution(domain).getX()
    for mode in (SolverOptions.MODE_PASO, SolverOptions.MODE_STANDARD):
        us = []
        for layout in (SolverOptions.LAYOUT_CSR, SolverOptions.LAYOUT_BAND):
            p = LinearPDE(domain)
            p.setValue(A=kronecker(domain), Y=1.0, q=whereZero(x[0]))
            so = p.getSolverOptions()
            so.setSolverMode(mode)
            so.setMatrixLayout(layout)
            so.setTolerance(1e-10)
            us.append(p.getSolution())
        assert Lsup(us[1] - us[0]) <= 1e-8 * Lsup(us[0])
    with pytest.raises(ValueError):
        pde.getSolverOptions().setMatrixLayout(7)


def test_coefficient_layout_through_solver_options(domain):
    """SolverOptions.setMatrixLayout(LAYOUT_COEF) with FP32 refinement: A = I (kronecker) and a
    Dirichlet face evaluate the FP32 operator from the coefficients (diagnostic
    inner_operator = 1) and give the FP64 solution; a D term makes the values not representable
    and the band copy is used (inner_operator = 0), with the same accuracy."""
    x = Solution(domain).getX()
    ref = LinearPDE(domain)
    ref.setValue(A=kronecker(domain), Y=1.0, q=whereZero(x[0]))
    ref.getSolverOptions().setTolerance(1e-10)
    u_ref = ref.getSolution()
    for extra, expect in (({}, 1), ({"D": 0.5}, 0)):
        p = LinearPDE(domain)
        p.setValue(A=kronecker(domain), Y=1.0, q=whereZero(x[0]), **extra)
        so = p.getSolverOptions()
        so.setSolverMode(SolverOptions.MODE_STANDARD)
        so.setPrecision(SolverOptions.PRECISION_FP32_REFINE)
        so.setMatrixLayout(SolverOptions.LAYOUT_COEF)
        so.setTolerance(1e-10)
        u = p.getSolution()
        assert so.getDiagnostics("inner_operator") == expect
        if not extra:
            assert Lsup(u - u_ref) <= 1e-8 * Lsup(u_ref)


# ---- LinearPDE coefficient handling, after escriptcore/test/python/test_linearPDEs.py
# (Test_LinearPDE: test_setCoefficient_*_Scalar / _System, test_reducedOn,
# test_setCoefficient_WithIllegalFunctionSpace, test_resetCoefficient_WithWrongShape)
from esys_b200.escript import (IllegalCoefficient, IllegalCoefficientValue,  # noqa: E402
                               IllegalCoefficientFunctionSpace, UndefinedPDEError, ReducedFunction,
                               FunctionOnBoundary, ReducedFunctionOnBoundary, ReducedSolution, Vector)

_SCALAR = {"A": lambda d: np.ones((d, d)), "B": lambda d: np.ones(d), "C": lambda d: np.ones(d),
           "D": lambda d: 1.0, "X": lambda d: np.ones(d), "Y": lambda d: 1.0, "y": lambda d: 1.0,
           "d": lambda d: 1.0}
_FS = {"A": Function, "B": Function, "C": Function, "D": Function, "X": Function, "Y": Function,
       "y": FunctionOnBoundary, "d": FunctionOnBoundary}
_RHS = ("X", "Y", "y")


@pytest.fixture
def dom2(cuda):
    return ripley.Rectangle(6, 5)


@pytest.mark.parametrize("name", sorted(_SCALAR))
@pytest.mark.parametrize("reduced", [False, True])
def test_set_coefficient_scalar(dom2, name, reduced):
    d = dom2.getDim()
    key = name + ("_reduced" if reduced else "")
    pde = LinearPDE(dom2)
    pde.setValue(**{key: _SCALAR[name](d)})
    c = pde.getCoefficient(key)
    fs = _FS[name](dom2)
    if reduced:
        fs = {Function(dom2): ReducedFunction(dom2),
              FunctionOnBoundary(dom2): ReducedFunctionOnBoundary(dom2)}[fs]
    assert (c.getShape(), c.getFunctionSpace(), pde.getNumSolutions(), pde.getNumEquations()) == \
        (np.shape(_SCALAR[name](d)), fs, 1, 1)
    pde.resetRightHandSideCoefficients()
    assert pde.getCoefficient(key).isEmpty() == (name in _RHS)


@pytest.mark.parametrize("name", ["A", "B", "C", "D", "X", "Y", "d", "y"])
def test_set_coefficient_system_infers_counts(dom2, name):
    """LinearPDE(domain) without counts: the first coefficient's shape sets them."""
    d, N = dom2.getDim(), 3
    shapes = {"A": (N, d, N, d), "B": (N, d, N), "C": (N, N, d), "D": (N, N), "X": (N, d), "Y": (N,),
              "d": (N, N), "y": (N,)}
    pde = LinearPDE(dom2)
    pde.setValue(**{name: np.ones(shapes[name])})
    c = pde.getCoefficient(name)
    assert c.getShape() == shapes[name] and c.getFunctionSpace() == _FS[name](dom2)
    assert pde.getNumEquations() == N
    if name not in ("X", "Y", "y"):
        assert pde.getNumSolutions() == N


def test_counts_from_q_and_r(dom2):
    pde = LinearPDE(dom2, numEquations=3)
    pde.setValue(r=1.0)
    assert pde.getCoefficient("r").getFunctionSpace() == Solution(dom2)
    pde.resetRightHandSideCoefficients()
    assert pde.getCoefficient("r").isEmpty()
    pde2 = LinearPDE(dom2)
    with pytest.raises(UndefinedPDEError):
        pde2.getNumEquations()


def test_reduced_order_on(dom2):
    """test_reducedOn: u = 1 with the solution on ReducedSolution; q goes there too; the
    order cannot change once a coefficient is set."""
    pde = LinearPDE(dom2)
    x = dom2.getX()
    pde.setReducedOrderOn()
    pde.setValue(A=kronecker(dom2), D=x[0], Y=x[0])
    u = pde.getSolution()
    assert u.getFunctionSpace() == ReducedSolution(dom2)
    assert check(u, 1.0)
    with pytest.raises(RuntimeError):
        pde.setReducedOrderOff()
    p2 = LinearPDE(dom2, numEquations=3)
    p2.setReducedOrderOn()
    p2.setValue(q=np.ones(3))
    assert p2.getCoefficient("q").getFunctionSpace() == ReducedSolution(dom2)


def test_coefficient_errors(dom2):
    pde = LinearPDE(dom2)
    with pytest.raises(IllegalCoefficientFunctionSpace):
        pde.setValue(C=Vector(0.0, FunctionOnBoundary(dom2)))
    with pytest.raises(IllegalCoefficient):
        pde.setValue(ROMA=0.0)
    with pytest.raises(IllegalCoefficientValue):
        LinearPDE(dom2, numEquations=2).setValue(C=0.0)
    assert issubclass(IllegalCoefficient, ValueError)


def test_reduced_data_goes_to_full_coefficient(dom2):
    """Data on ReducedFunction given as A interpolates to Function on ripley (a sample's
    value at each of its points); given as A_reduced it stays there; both assemble the
    same operator as the reduced path with the equivalent values."""
    d = dom2.getDim()
    A = Data(np.eye(d), (d, d), ReducedFunction(dom2), expanded=True)
    pde = LinearPDE(dom2)
    pde.setValue(A=A)
    assert pde.getCoefficient("A").getFunctionSpace() == Function(dom2)
    y = Data(2.0, (), ReducedFunctionOnBoundary(dom2), expanded=True)
    pde.setValue(y=y)
    assert pde.getCoefficient("y").getFunctionSpace() == FunctionOnBoundary(dom2)
    assert np.allclose(pde.getCoefficient("y").toNumpy(), 2.0)
