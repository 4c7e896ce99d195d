"""The escript-facing API of the B200 hot path: Data on ripley function spaces,
SolverOptions (SolverBuddy), LinearPDE and Poisson.

This mirrors the reference's Python surface for the path
``LinearPDE(dom); pde.setValue(A=..., D=..., Y=..., q=..., r=...); u = pde.getSolution()``
(escriptcore/py_src/linearPDEs.py:1760-2207) with the same names, argument meaning and
error classes.  Data lives on the GPU as torch float64 tensors; assembly, constraints
and the solve run in libripley_gpu.so.  Single equations and systems of 2 or 3 equations
are provided, with coefficients on Function, ReducedFunction, FunctionOnBoundary and
ReducedFunctionOnBoundary; lumping, contact and Dirac-point coefficients raise
NotImplementedError.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L

EPSILON = float(np.finfo(np.float64).eps)
DEVICE = "cuda"

# ---------------------------------------------------------------------------------------------
# function spaces
# ---------------------------------------------------------------------------------------------

_NODES = ("Solution", "ContinuousFunction", "ReducedSolution", "ReducedContinuousFunction")


class FunctionSpace:
    """A ripley function space: nodes, Gauss points of the elements, element centres or
    Gauss points of the boundary faces."""

    def __init__(self, domain, kind: str):
        self._domain = domain
        self._kind = kind

    # escript API
    def getDomain(self):
        return self._domain

    def getDim(self):
        return self._domain.getDim()

    def getTypeCode(self):
        # ripley's function space codes (ripley/src/Ripley.h:49-59, RipleyDomain.h getXCode)
        return {"Solution": 1, "ReducedSolution": 2, "ContinuousFunction": 3, "Function": 4,
                "ReducedFunction": 10, "FunctionOnBoundary": 5, "ReducedFunctionOnBoundary": 11,
                "ReducedContinuousFunction": 14}[self._kind]

    def __str__(self):
        return f"{self._kind} on {self._domain}"

    __repr__ = __str__

    def __eq__(self, other):
        return (isinstance(other, FunctionSpace) and other._domain is self._domain and
                other.getTypeCode() == self.getTypeCode())

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash((id(self._domain), self.getTypeCode()))

    def _storage(self):
        """Where values live: 'nodes' (DOF = nodes on one rank), 'qp', 'elem', 'face' (the face
        Gauss points) or 'rface' (face centres)."""
        if self._kind in _NODES:
            return "nodes"
        return {"Function": "qp", "ReducedFunction": "elem", "FunctionOnBoundary": "face",
                "ReducedFunctionOnBoundary": "rface"}[self._kind]

    def getNumSamples(self):
        d = self._domain
        return {"nodes": d._n, "qp": d._nel, "elem": d._nel, "face": d._nfaces,
                "rface": d._nfaces}[self._storage()]

    def getNumDataPointsPerSample(self):
        d = self._domain
        return {"nodes": 1, "qp": 1 << d._dim, "elem": 1, "face": 1 << (d._dim - 1), "rface": 1}[self._storage()]

    def _num_points(self):
        return self.getNumSamples() * self.getNumDataPointsPerSample()

    def getX(self):
        return Data._wrap(self._domain._coordinates(self._storage()), (self.getDim(),), self)

    def getSize(self):
        h = min(self._domain._dx[: self.getDim()]) if self._storage() == "nodes" else \
            math.sqrt(sum(v * v for v in self._domain._dx[: self.getDim()]))
        return Scalar(h, self)


def Solution(domain):
    return FunctionSpace(domain, "Solution")


def ReducedSolution(domain):
    return FunctionSpace(domain, "ReducedSolution")


def ContinuousFunction(domain):
    return FunctionSpace(domain, "ContinuousFunction")


def Function(domain):
    return FunctionSpace(domain, "Function")


def ReducedFunction(domain):
    return FunctionSpace(domain, "ReducedFunction")


def FunctionOnBoundary(domain):
    return FunctionSpace(domain, "FunctionOnBoundary")


def ReducedFunctionOnBoundary(domain):
    return FunctionSpace(domain, "ReducedFunctionOnBoundary")


# ---------------------------------------------------------------------------------------------
# Data
# ---------------------------------------------------------------------------------------------

def _flat_index(idx, shape):
    """escript stores a data point column-major (index.h INDEX2(i,j,N) = i + N*j)."""
    if not isinstance(idx, tuple):
        idx = (idx,)
    if len(idx) != len(shape):
        raise IndexError("Data: index rank does not match the data point rank")
    f, stride = 0, 1
    for i, n in zip(idx, shape):
        if not isinstance(i, (int, np.integer)):
            raise IndexError("Data: only integer component indices are supported")
        if i < 0 or i >= n:
            raise IndexError("Data: component index out of range")
        f += int(i) * stride
        stride *= n
    return f


def _np_to_flat(a):
    a = np.asarray(a, dtype=np.float64)
    return a.reshape(-1, order="F"), tuple(a.shape)


class Data:
    """escript::Data restricted to what the hot path needs.

    Storage: ``_t`` is a float64 CUDA tensor of shape (P, ncomp) for expanded data
    (P = samples x data points per sample) or (1, ncomp) for constant data; ncomp is
    the flattened data-point shape in escript's column-major order.
    """

    def __init__(self, value=None, what=None, fs=None, expanded=False):
        # Data(), Data(value, fs), Data(value, shape, fs), Data(other Data, fs)
        self._fs = None
        self._shape = ()
        self._t = None
        if value is None:
            return
        if isinstance(what, FunctionSpace):
            fs, shape = what, None
        else:
            shape = None if what is None else tuple(what)
        if isinstance(value, Data):
            src = value if fs is None else value.interpolate(fs)
            self._fs, self._shape, self._t = src._fs, src._shape, src._t.clone()
            return
        flat, vshape = _np_to_flat(value)
        if shape is not None and vshape == ():
            flat = np.full(int(np.prod(shape)) if shape else 1, float(flat[0]))
            vshape = shape
        elif shape is not None and vshape != shape:
            raise ValueError("Data: value shape does not match the requested shape")
        if fs is None:
            raise ValueError("Data: a function space is required")
        self._fs, self._shape = fs, vshape
        self._t = torch.tensor(flat, dtype=torch.float64, device=DEVICE).reshape(1, -1)
        if expanded:
            self.expand()

    @classmethod
    def _wrap(cls, t, shape, fs):
        d = cls()
        d._fs, d._shape = fs, tuple(shape)
        d._t = t.reshape(t.shape[0], -1)
        return d

    # ---- properties
    def isEmpty(self):
        return self._t is None

    def isConstant(self):
        return self._t is not None and self._t.shape[0] == 1 and self._fs._num_points() != 1

    def isExpanded(self):
        return self._t is not None and not self.isConstant()

    def actsExpanded(self):
        return self.isExpanded()

    def isComplex(self):
        return False

    def getShape(self):
        return self._shape

    def getRank(self):
        return len(self._shape)

    def getDataPointSize(self):
        return int(np.prod(self._shape)) if self._shape else 1

    def getFunctionSpace(self):
        return self._fs

    def getDomain(self):
        return self._fs.getDomain()

    def getNumberOfDataPoints(self):
        return self._fs._num_points()

    def expand(self):
        if self.isConstant():
            self._t = self._t.expand(self._fs._num_points(), -1).contiguous()
        return self

    def copy(self):
        return Data._wrap(self._t.clone(), self._shape, self._fs)

    def toNumpy(self):
        """Values as a numpy array of shape (points, *shape) (C order per point)."""
        t = self._t.expand(self._fs._num_points(), -1) if self.isConstant() else self._t
        a = t.detach().cpu().numpy()
        return a.reshape((a.shape[0],) + tuple(reversed(self._shape))).transpose(
            (0,) + tuple(range(len(self._shape), 0, -1))) if self._shape else a[:, 0]

    def _dev(self, n=None):
        """Contiguous expanded tensor (points, ncomp)."""
        n = self._fs._num_points() if n is None else n
        return self._t.expand(n, -1).contiguous() if self._t.shape[0] == 1 else self._t.contiguous()

    # ---- interpolation
    def interpolate(self, fs):
        src, dst = self._fs._storage(), fs._storage()
        if not _can_interpolate(src, dst):
            raise ValueError(f"interpolate: cannot interpolate from {self._fs} to {fs}")
        if src == dst or self.isConstant():
            # the same points (the node spaces of one rank are one set of nodes) or a constant
            return Data._wrap(self._t.clone(), self._shape, fs)
        dom = self._fs.getDomain()
        if fs.getDomain() is not dom:
            raise ValueError("interpolate: function spaces belong to different domains")
        if (src, dst) in (("elem", "qp"), ("rface", "face")):
            # ReducedElements -> Elements, ReducedFaceElements -> FaceElements: the value of a
            # sample at each of its points (RipleyDomain::probeInterpolationOnDomain allows both)
            q = fs.getNumDataPointsPerSample()
            ncomp = self._t.shape[1]
            out = self._dev()[:, None, :].expand(-1, q, ncomp).reshape(-1, ncomp).contiguous()
            return Data._wrap(out, self._shape, fs)
        if src == "nodes" and dst in ("qp", "elem"):
            ncomp = self._t.shape[1]
            out = torch.empty((fs._num_points(), ncomp), dtype=torch.float64, device=DEVICE)
            nodal = self._dev()
            L.set_stream_from_torch()
            L.check(L.lib().rg_interpolate_nodes(dom._handle, C.c_void_p(nodal.data_ptr()), ncomp,
                                                 C.c_void_p(out.data_ptr()), int(dst == "elem")))
            return Data._wrap(out, self._shape, fs)
        if src == "nodes" and dst == "face":
            return Data._wrap(dom._nodes_to_face(self._dev()), self._shape, fs)
        if src == "nodes" and dst == "rface":
            return Data._wrap(dom._nodes_to_face(self._dev(), reduced=True), self._shape, fs)
        if src == "face" and dst == "rface":
            q = 1 << (dom._dim - 1)
            return Data._wrap(self._dev().reshape(-1, q, self._t.shape[1]).mean(1), self._shape, fs)
        if src == "qp" and dst == "elem":
            q = 1 << dom._dim
            return Data._wrap(self._dev().reshape(-1, q, self._t.shape[1]).mean(1), self._shape, fs)
        raise ValueError(f"interpolate: cannot interpolate from {self._fs} to {fs}")

    # ---- component access
    def __getitem__(self, idx):
        f = _flat_index(idx, self._shape)
        return Data._wrap(self._t[:, f:f + 1].clone(), (), self._fs)

    def __setitem__(self, idx, value):
        f = _flat_index(idx, self._shape)
        if isinstance(value, Data):
            v = value if value._fs == self._fs else value.interpolate(self._fs)
            if v.isExpanded():
                self.expand()
            self._t[:, f:f + 1] = v._t
        else:
            self._t[:, f] = float(value)

    # ---- arithmetic (torch on the device)
    def _binary(self, other, op):
        if isinstance(other, Data):
            a, b = self, other
            if a._fs != b._fs:
                fs = _common_fs(a._fs, b._fs)
                a = a if a._fs == fs else a.interpolate(fs)
                b = b if b._fs == fs else b.interpolate(fs)
            ta, tb = a._t, b._t
            shape = a._shape if a._shape else b._shape
            if a._shape and b._shape and a._shape != b._shape:
                raise ValueError("Data: incompatible shapes")
            return Data._wrap(op(ta, tb), shape, a._fs)
        if isinstance(other, np.ndarray) and other.shape:
            flat, vshape = _np_to_flat(other)
            t = torch.tensor(flat, dtype=torch.float64, device=DEVICE).reshape(1, -1)
            return Data._wrap(op(self._t, t), vshape if not self._shape else self._shape, self._fs)
        return Data._wrap(op(self._t, float(other)), self._shape, self._fs)

    def __add__(self, o):
        return self._binary(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._binary(o, lambda a, b: b + a)

    def __sub__(self, o):
        return self._binary(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._binary(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._binary(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._binary(o, lambda a, b: b * a)

    def __truediv__(self, o):
        return self._binary(o, lambda a, b: a / b)

    def __rtruediv__(self, o):
        return self._binary(o, lambda a, b: b / a)

    def __pow__(self, o):
        return self._binary(o, lambda a, b: a ** b)

    def __neg__(self):
        return Data._wrap(-self._t, self._shape, self._fs)

    def __abs__(self):
        return Data._wrap(self._t.abs(), self._shape, self._fs)

    def __iadd__(self, o):
        r = self + o
        self._fs, self._shape, self._t = r._fs, r._shape, r._t
        return self

    def __isub__(self, o):
        r = self - o
        self._fs, self._shape, self._t = r._fs, r._shape, r._t
        return self

    def __imul__(self, o):
        r = self * o
        self._fs, self._shape, self._t = r._fs, r._shape, r._t
        return self

    def _whereZero(self, tol):
        return Data._wrap((self._t.abs() <= tol).to(torch.float64), self._shape, self._fs)

    def copyWithMask(self, other, mask):
        """Data.copyWithMask: take ``other`` where ``mask`` > 0 (escriptcore/src/Data.cpp:855)."""
        o = other if other._fs == self._fs else other.interpolate(self._fs)
        m = mask if mask._fs == self._fs else mask.interpolate(self._fs)
        self.expand()
        n = self._fs._num_points()
        self._t = torch.where(m._dev(n) > 0, o._dev(n), self._t)

    def __str__(self):
        return f"Data(shape={self._shape}, fs={self._fs}, points={0 if self._t is None else self._t.shape[0]})"

    __repr__ = __str__


def _can_interpolate(src, dst):
    """RipleyDomain::probeInterpolationOnDomain (ripley/src/RipleyDomain.cpp:288-324) by
    storage: nodes go anywhere, element points stay on elements, face points on faces."""
    if src == "nodes":
        return True
    if src in ("qp", "elem"):
        return dst in ("qp", "elem")
    if src in ("face", "rface"):
        return dst in ("face", "rface")
    return src == dst


def _common_fs(a, b):
    order = {"nodes": 0, "qp": 1, "elem": 2, "face": 3, "rface": 4}
    sa, sb = a._storage(), b._storage()
    if sa == sb:
        return a
    if {sa, sb} == {"nodes", "qp"}:
        return a if sa == "qp" else b
    if {sa, sb} == {"nodes", "elem"} or {sa, sb} == {"qp", "elem"}:
        return a if sa == "elem" else b
    if {sa, sb} == {"nodes", "face"}:
        return a if sa == "face" else b
    if {sa, sb} == {"nodes", "rface"} or {sa, sb} == {"face", "rface"}:
        return a if sa == "rface" else b
    raise ValueError(f"cannot combine data on {a} and {b}")


def Scalar(value=0.0, what=None, expanded=False):
    return Data(value, (), what, expanded)


def Vector(value=0.0, what=None, expanded=False):
    return Data(value, (what.getDim(),), what, expanded)


def Tensor(value=0.0, what=None, expanded=False):
    d = what.getDim()
    return Data(value, (d, d), what, expanded)


# ---------------------------------------------------------------------------------------------
# util (escriptcore/py_src/util.py)
# ---------------------------------------------------------------------------------------------

def kronecker(d=3):
    if hasattr(d, "getDim"):
        d = d.getDim()
    return np.eye(int(d))


identityTensor = kronecker


def Lsup(arg):
    if isinstance(arg, Data):
        return float(arg._t.abs().max().item())
    return float(np.max(np.abs(np.asarray(arg))))


def sup(arg):
    if isinstance(arg, Data):
        return float(arg._t.max().item())
    return float(np.max(arg))


def inf(arg):
    if isinstance(arg, Data):
        return float(arg._t.min().item())
    return float(np.min(arg))


def whereZero(arg, tol=None, rtol=math.sqrt(EPSILON)):
    if tol is None:
        if rtol < 0:
            raise ValueError("rtol must be non-negative.")
        tol = Lsup(arg) * rtol
    if isinstance(arg, Data):
        return arg._whereZero(tol)
    if isinstance(arg, np.ndarray):
        return (np.abs(arg) - tol <= 0) * 1.0
    return 1.0 if abs(arg) <= tol else 0.0


def whereNonZero(arg, tol=0.0):
    if isinstance(arg, Data):
        return Data._wrap((arg._t.abs() > tol).to(torch.float64), arg._shape, arg._fs)
    return (np.abs(arg) > tol) * 1.0


def _unary(fn_t, fn_np):
    def f(arg):
        if isinstance(arg, Data):
            return Data._wrap(fn_t(arg._t), arg._shape, arg._fs)
        return fn_np(arg)
    return f


exp = _unary(torch.exp, np.exp)
log = _unary(torch.log, np.log)
sqrt = _unary(torch.sqrt, np.sqrt)
sin = _unary(torch.sin, np.sin)
cos = _unary(torch.cos, np.cos)


def interpolate(arg, where):
    return arg.interpolate(where) if isinstance(arg, Data) else Data(arg, where)


def inner(a, b):
    """Contraction over all indices (util.inner)."""
    if isinstance(a, np.ndarray) and isinstance(b, Data):
        a, b = b, a
    if isinstance(a, Data) and isinstance(b, np.ndarray):
        flat, _ = _np_to_flat(b)
        t = torch.tensor(flat, dtype=torch.float64, device=DEVICE)
        return Data._wrap((a._t * t).sum(1, keepdim=True), (), a._fs)
    if isinstance(a, Data) and isinstance(b, Data):
        p = a * b
        return Data._wrap(p._t.sum(1, keepdim=True), (), p._fs)
    return float(np.sum(np.asarray(a) * np.asarray(b)))


def convertToNumpy(data):
    return data.toNumpy()


# ---------------------------------------------------------------------------------------------
# SolverOptions / SolverBuddy (escriptcore/src/SolverOptions.{h,cpp})
# ---------------------------------------------------------------------------------------------

class SolverOptions:
    """Names and values of escript::SolverOptions (escriptcore/src/SolverOptions.h:82-140)."""
    DEFAULT = 0
    TARGET_CPU, TARGET_GPU = 1, 2
    MKL, PASO, TRILINOS, UMFPACK, MUMPS = 3, 4, 5, 6, 7
    BICGSTAB, CGLS, CGS, CHOLEVSKY, CR, DIRECT, DIRECT_MUMPS, DIRECT_PARDISO, DIRECT_SUPERLU, \
        DIRECT_TRILINOS, GMRES, HRZ_LUMPING, ITERATIVE, LSQR, MINRES, NONLINEAR_GMRES, PCG, \
        PRES20, ROWSUM_LUMPING, TFQMR = range(8, 28)
    AMG, GAUSS_SEIDEL, ILU0, ILUT, JACOBI, NO_PRECONDITIONER, REC_ILU, RILU = range(28, 36)
    # solver modes and precisions of this implementation
    MODE_PASO, MODE_STANDARD = L.RG_MODE_PASO, L.RG_MODE_STANDARD
    PRECISION_FP64, PRECISION_FP32_REFINE = L.RG_PREC_FP64, L.RG_PREC_FP32_REFINE
    LAYOUT_CSR, LAYOUT_BAND, LAYOUT_COEF = L.RG_LAYOUT_CSR, L.RG_LAYOUT_BAND, L.RG_LAYOUT_COEF


class SolverBuddy:
    """Solver configuration and diagnostics; defaults of SolverBuddy::SolverBuddy
    (escriptcore/src/SolverOptions.cpp:40-70)."""

    def __init__(self):
        self.__method = SolverOptions.DEFAULT
        self.__package = SolverOptions.DEFAULT
        self.__preconditioner = SolverOptions.JACOBI
        self.__sweeps = 1
        self.__tolerance = 1e-8
        self.__absolute_tolerance = 0.0
        self.__iter_max = 100000
        self.__verbose = False
        self.__symmetric = False
        self.__accept_failure = False
        self.__mode = SolverOptions.MODE_PASO
        self.__precision = SolverOptions.PRECISION_FP64
        self.__layout = SolverOptions.LAYOUT_CSR
        self.__inner_tolerance = 1e-2
        self.__initial_guess = None
        self.resetDiagnostics(all=True)

    # configuration
    def setSolverMethod(self, method=0):
        self.__method = method

    def getSolverMethod(self):
        return self.__method

    def setPackage(self, package=0):
        self.__package = package

    def getPackage(self):
        return self.__package

    def setPreconditioner(self, preconditioner=SolverOptions.JACOBI):
        self.__preconditioner = preconditioner

    def getPreconditioner(self):
        return self.__preconditioner

    def setNumSweeps(self, sweeps):
        if sweeps < 1:
            raise ValueError("number of sweeps must be positive.")
        self.__sweeps = int(sweeps)

    def getNumSweeps(self):
        return self.__sweeps

    def setTolerance(self, rtol=1e-8):
        if rtol < 0 or rtol > 1:
            raise ValueError("tolerance must be between 0 and 1.")
        self.__tolerance = float(rtol)

    def getTolerance(self):
        return self.__tolerance

    def setAbsoluteTolerance(self, atol=0.0):
        if atol < 0:
            raise ValueError("absolute tolerance must be non-negative.")
        self.__absolute_tolerance = float(atol)

    def getAbsoluteTolerance(self):
        return self.__absolute_tolerance

    def setIterMax(self, iter_max=100000):
        if iter_max < 1:
            raise ValueError("maximum number of iteration steps must be positive.")
        self.__iter_max = int(iter_max)

    def getIterMax(self):
        return self.__iter_max

    def setVerbosity(self, verbose=False):
        self.__verbose = bool(verbose)

    def setVerbosityOn(self):
        self.__verbose = True

    def setVerbosityOff(self):
        self.__verbose = False

    def isVerbose(self):
        return self.__verbose

    def setSymmetry(self, s=False):
        self.__symmetric = bool(s)

    def setSymmetryOn(self):
        self.__symmetric = True

    def setSymmetryOff(self):
        self.__symmetric = False

    def isSymmetric(self):
        return self.__symmetric

    def setAcceptanceConvergenceFailure(self, accept=False):
        self.__accept_failure = bool(accept)

    def acceptConvergenceFailure(self):
        return self.__accept_failure

    # GPU-path extensions
    def setSolverMode(self, mode):
        self.__mode = mode

    def getSolverMode(self):
        return self.__mode

    def setPrecision(self, precision):
        self.__precision = precision

    def getPrecision(self):
        return self.__precision

    def setMatrixLayout(self, layout):
        """LAYOUT_CSR (default: the SpMV of FP64 solves reads the paso CSR values),
        LAYOUT_BAND (FP64 solves of scalar PDEs read an FP64 27-band copy of the balanced
        matrix instead: the same arithmetic with fewer bytes; FP32 refinement uses its FP32
        band copy with either of these two), or LAYOUT_COEF (FP32 refinement only: the FP32
        iterations evaluate the operator from the element coefficients, when the matrix was
        built from A = kappa I per element and a constraint; otherwise the band copy is used,
        diagnostic 'inner_operator').  No reference counterpart."""
        if layout not in (SolverOptions.LAYOUT_CSR, SolverOptions.LAYOUT_BAND, SolverOptions.LAYOUT_COEF):
            raise ValueError("unknown matrix layout %r" % (layout,))
        self.__layout = layout

    def getMatrixLayout(self):
        return self.__layout

    def setInnerTolerance(self, t):
        self.__inner_tolerance = float(t)

    def getInnerTolerance(self):
        return self.__inner_tolerance

    def setInitialGuess(self, u):
        """Start the (standard-mode) solve from ``u`` (Data on Solution) instead of zero."""
        self.__initial_guess = u

    def getInitialGuess(self):
        return self.__initial_guess

    # diagnostics (SolverBuddy::getDiagnostics)
    def resetDiagnostics(self, all=False):
        """SolverBuddy::resetDiagnostics: the cumulative items survive unless all=True."""
        cum = {k: v for k, v in getattr(self, "_SolverBuddy__diag", {}).items() if k.startswith("cum_")}
        self.__diag = {"num_iter": 0, "num_level": 0, "num_inner_iter": 0, "time": 0.0,
                       "set_up_time": 0.0, "net_time": 0.0, "residual_norm": 0.0,
                       "converged": False, "num_outer": 0, "guess_rejected": False,
                       "guess_residual": 0.0, "fp64_fallback": False, "inner_operator": 0}
        if all or not cum:
            cum = {"cum_num_iter": 0, "cum_time": 0.0, "cum_set_up_time": 0.0,
                   "cum_net_time": 0.0, "cum_num_inner_iter": 0}
        self.__diag.update(cum)

    def _updateDiagnostics(self, d: "L.rg_diag"):
        self.__diag.update(num_iter=int(d.num_iter), num_outer=int(d.num_outer),
                           residual_norm=float(d.residual_norm), converged=bool(d.converged),
                           time=float(d.time), set_up_time=float(d.set_up_time),
                           net_time=float(d.net_time), guess_rejected=bool(d.guess_rejected),
                           guess_residual=float(d.guess_residual),
                           fp64_fallback=bool(d.fp64_fallback), inner_operator=int(d.inner_operator))
        self.__diag["cum_num_iter"] += int(d.num_iter)
        self.__diag["cum_time"] += float(d.time)
        self.__diag["cum_set_up_time"] += float(d.set_up_time)
        self.__diag["cum_net_time"] += float(d.net_time)

    def getDiagnostics(self, name):
        if name not in self.__diag:
            raise ValueError(f"unknown diagnostic item {name}")
        return self.__diag[name]

    def hasConverged(self):
        return self.__diag["converged"]

    def _to_c(self) -> "L.rg_solver_opts":
        method = self.__method
        if method not in (SolverOptions.DEFAULT, SolverOptions.PCG, SolverOptions.ITERATIVE):
            raise NotImplementedError("only the PCG solver is available on the GPU path")
        if self.__preconditioner != SolverOptions.JACOBI:
            raise NotImplementedError("only the Jacobi preconditioner is available on the GPU path")
        o = L.rg_solver_opts()
        L.lib().rg_solver_opts_default(C.byref(o))
        o.tolerance = self.__tolerance
        o.iter_max = self.__iter_max
        o.sweeps = self.__sweeps
        o.verbose = int(self.__verbose)
        o.accept_convergence_failure = int(self.__accept_failure)
        o.mode = self.__mode
        o.precision = self.__precision
        o.layout = self.__layout
        o.inner_tolerance = self.__inner_tolerance
        return o

    def __str__(self):
        return (f"SolverOptions(method={self.__method}, preconditioner={self.__preconditioner}, "
                f"tolerance={self.__tolerance}, iter_max={self.__iter_max}, mode={self.__mode}, "
                f"precision={self.__precision})")


# ---------------------------------------------------------------------------------------------
# system matrix (paso::SystemMatrix behind AbstractSystemMatrix)
# ---------------------------------------------------------------------------------------------

class SystemMatrix:
    """Operator returned by LinearPDE.getSystem(): a paso CSR matrix on the GPU."""

    def __init__(self, domain, block_size=1):
        self._domain = domain
        self._nb = int(block_size)
        h = C.c_void_p()
        L.set_stream_from_torch()
        if self._nb == 1:
            L.check(L.lib().rg_matrix_create(domain._handle, C.byref(h)))
        else:
            L.check(L.lib().rg_matrix_create_system(domain._handle, self._nb, C.byref(h)))
        self._handle = h

    def _new_vector(self):
        if self._nb == 1:
            return Scalar(0.0, Solution(self._domain), expanded=True)
        return Data(0.0, (self._nb,), Solution(self._domain), expanded=True)

    def getRowBlockSize(self):
        return self._nb

    def getColumnBlockSize(self):
        return self._nb

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h and L._lib is not None:
            L._lib.rg_matrix_destroy(h)
            self._handle = None

    def isEmpty(self):
        return False

    def resetValues(self, preserveSolverData=False):
        L.check(L.lib().rg_matrix_reset(self._handle))

    def isBalanced(self):
        b = C.c_int()
        L.check(L.lib().rg_matrix_is_balanced(self._handle, C.byref(b)))
        return bool(b.value)

    def values(self):
        """The nnz CSR values as a CUDA tensor view (device memory owned by the matrix)."""
        p = C.c_void_p()
        L.check(L.lib().rg_matrix_values(self._handle, C.byref(p)))
        return _tensor_from_ptr(p.value, self._domain._nnz * self._nb * self._nb, torch.float64)

    def nullifyRowsAndCols(self, row_q, col_q, mdv):
        r = row_q.interpolate(Solution(self._domain)) if row_q._fs._storage() != "nodes" else row_q
        c = col_q.interpolate(Solution(self._domain)) if col_q._fs._storage() != "nodes" else col_q
        rt, ct = r._dev(), c._dev()
        L.set_stream_from_torch()
        L.check(L.lib().rg_nullify_rows_and_cols(self._handle, C.c_void_p(rt.data_ptr()),
                                                 C.c_void_p(ct.data_ptr()), float(mdv)))

    def __mul__(self, u):
        """AbstractSystemMatrix.__mul__ -> vectorMultiply: y = A u."""
        out = self._new_vector()
        x = u._dev(self._domain._n) if u._fs._storage() == "nodes" else None
        if x is None:
            raise ValueError("matrix vector product: function space of input does not match")
        self.ypAx(out, u)
        return out

    def ypAx(self, y, x):
        xt = x._dev(self._domain._n)
        y.expand()
        L.set_stream_from_torch()
        L.check(L.lib().rg_spmv(self._handle, 1.0, C.c_void_p(xt.data_ptr()), 1.0,
                                C.c_void_p(y._t.data_ptr())))

    def solve(self, rhs, options=None):
        options = SolverBuddy() if options is None else options
        out = self._new_vector()
        self.setToSolution(out, rhs, options)
        return out

    def setToSolution(self, out, rhs, options):
        """AbstractSystemMatrix::setToSolution -> paso solve (paso/src/SystemMatrix.h:614-641)."""
        options.resetDiagnostics()
        o = options._to_c()
        b = rhs._dev(self._domain._n)
        out.expand()
        x0 = options.getInitialGuess()
        keep = None
        if x0 is not None:
            if o.mode == L.RG_MODE_PASO and o.precision == L.RG_PREC_FP64:
                o.mode = L.RG_MODE_STANDARD
            keep = x0._dev(self._domain._n)
            o.initial_guess = keep.data_ptr()
        d = L.rg_diag()
        L.set_stream_from_torch()
        st = L.lib().rg_solve(self._handle, C.c_void_p(b.data_ptr()), C.c_void_p(out._t.data_ptr()),
                              C.byref(o), C.byref(d))
        options._updateDiagnostics(d)
        L.check(st)

    def residualNorms(self, rhs, u):
        """(||rhs - A u||_2, ||rhs - A u||_inf) of the assembled system."""
        b = rhs._dev(self._domain._n)
        x = u._dev(self._domain._n)
        l2, lm = C.c_double(), C.c_double()
        L.set_stream_from_torch()
        L.check(L.lib().rg_residual_norms(self._handle, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                          C.byref(l2), C.byref(lm)))
        return l2.value, lm.value

    def saveMM(self, filename):
        L.check(L.lib().rg_save_mm(self._handle, str(filename).encode()))


def _tensor_from_ptr(ptr, count, dtype):
    """Non-owning torch view of device memory owned by the library."""
    typestr = {torch.float64: "<f8", torch.float32: "<f4", torch.int32: "<i4"}[dtype]

    class _View:
        __cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr,
                                    "data": (int(ptr), False), "version": 3, "stream": None}

    return torch.as_tensor(_View(), device=DEVICE)


# ---------------------------------------------------------------------------------------------
# LinearPDE / Poisson (escriptcore/py_src/linearPDEs.py)
# ---------------------------------------------------------------------------------------------

class IllegalCoefficient(ValueError):
    """An unknown coefficient name (linearPDEs.py:56)."""


class IllegalCoefficientValue(ValueError):
    """A coefficient value of the wrong shape (linearPDEs.py:63)."""


class IllegalCoefficientFunctionSpace(ValueError):
    """A coefficient on a function space that cannot be interpolated to the one the PDE
    needs (linearPDEs.py:69)."""


class UndefinedPDEError(ValueError):
    """The number of equations or solutions cannot be determined yet (linearPDEs.py:75)."""


# index pattern of each coefficient: E = equation, S = solution component, D = space
# dimension; E (S) is dropped when the PDE has one equation (solution component)
_PATTERN = {"A": "EDSD", "B": "EDS", "C": "ESD", "D": "ES", "X": "ED", "Y": "E", "d": "ES", "y": "E",
            "q": "S", "r": "S"}


def _pattern_of(name):
    return _PATTERN[name[:-len("_reduced")] if name.endswith("_reduced") else name]


def _shape_for(pattern, dim, ne, ns):
    out = []
    for t in pattern:
        if t == "E":
            if ne > 1:
                out.append(ne)
        elif t == "S":
            if ns > 1:
                out.append(ns)
        else:
            out.append(dim)
    return tuple(out)


def _estimate_counts(pattern, dim, shape):
    """(numEquations, numSolutions) a coefficient of this shape implies (None where the
    coefficient says nothing about it), or None if no counts fit: the largest counts whose
    shape matches, as PDECoef.estimateNumEquationsAndNumSolutions does."""
    shape = tuple(shape)
    top = (max(shape) if shape else 0) + 1
    es = list(range(1, top + 1)) if "E" in pattern else [None]
    us = list(range(1, top + 1)) if "S" in pattern else [None]
    for e, u in sorted(((e, u) for e in es for u in us), key=lambda c: -((c[0] or 0) + (c[1] or 0))):
        if _shape_for(pattern, dim, e or 1, u or 1) == shape:
            return e, u
    return None


_INTERIOR = ("A", "B", "C", "D", "X", "Y")
_REDUCED = ("A_reduced", "B_reduced", "C_reduced", "D_reduced", "X_reduced", "Y_reduced")
_BOUNDARY = ("d", "y")
_BOUNDARY_REDUCED = ("d_reduced", "y_reduced")
_CONSTRAINT = ("q", "r")
_UNSUPPORTED = ("d_contact", "y_contact", "d_contact_reduced", "y_contact_reduced", "d_dirac", "y_dirac")
_ALL = _INTERIOR + _REDUCED + _BOUNDARY + _BOUNDARY_REDUCED + _CONSTRAINT


class LinearPDE:
    """-(A_ij u_,j + B_i u)_,i + C_j u_,j + D u = -X_i,i + Y, with n_i(A_ij u_,j + B_i u)
    + d u = n_i X_i + y on the boundary and u = r where q > 0 (single equation)."""

    def __init__(self, domain, numEquations=None, numSolutions=None, isComplex=False, debug=False):
        if isComplex:
            raise NotImplementedError("complex PDEs are not part of the GPU path")
        self._ne = None if numEquations is None else int(numEquations)
        self._ns = None if numSolutions is None else int(numSolutions)
        if max(self._ne or 0, self._ns or 0) > 3:
            raise NotImplementedError("PDE systems of more than 3 equations are not part of the GPU path")
        self._domain = domain
        self._coef = {}
        self._options = SolverBuddy()
        self._operator = None
        self._rhs = None
        self._operator_valid = False
        self._rhs_valid = False
        self._solution = None
        self._debug = debug
        self._symmetric = False
        self._reduce_sol = False
        self._reduce_eq = False

    # ---- escript API
    def getDomain(self):
        return self._domain

    def getDim(self):
        return self._domain.getDim()

    def getNumEquations(self):
        """The number of equations; the number of solutions when only that is known."""
        if self._ne is None:
            if self._ns is None:
                raise UndefinedPDEError("Number of equations is undefined. Please specify argument numEquations.")
            self._ne = self._ns
        return self._ne

    def getNumSolutions(self):
        """The number of solution components; the number of equations when only that is known."""
        if self._ns is None:
            if self._ne is None:
                raise UndefinedPDEError("Number of solution is undefined. Please specify argument numSolutions.")
            self._ns = self._ne
        return self._ns

    @property
    def _nb(self):
        """Block size of the operator: the GPU path solves square systems of 1..3 equations."""
        ne, ns = self.getNumEquations(), self.getNumSolutions()
        if ne != ns:
            raise ValueError("number of equations and number of solutions don't match")
        if ne > 3:
            raise NotImplementedError("PDE systems of more than 3 equations are not part of the GPU path")
        return ne

    def getSolverOptions(self):
        return self._options

    def setSolverOptions(self, options=None):
        self._options = SolverBuddy() if options is None else options

    def setSymmetryOn(self):
        self._symmetric = True
        self._options.setSymmetryOn()

    def setSymmetryOff(self):
        self._symmetric = False

    def isSymmetric(self):
        return self._symmetric

    # reduced order (linearPDEs.py:854-960).  On ripley the reduced solution space has the same
    # nodes (Q1 has no lower order, RipleyDomain::newSystemMatrix accepts both), so only the
    # function spaces of the solution, q and r change.
    def _set_reduced(self, sol=None, eq=None):
        if (sol is not None and sol != self._reduce_sol) or (eq is not None and eq != self._reduce_eq):
            if self._coef:
                raise RuntimeError("order cannot be altered after coefficients have been defined.")
            if sol is not None:
                self._reduce_sol = sol
            if eq is not None:
                self._reduce_eq = eq
            self._operator_valid = self._rhs_valid = False
            self._solution = None

    def setReducedOrderOn(self):
        self._set_reduced(True, True)

    def setReducedOrderOff(self):
        self._set_reduced(False, False)

    def setReducedOrderTo(self, flag=False):
        self._set_reduced(bool(flag), bool(flag))

    def setReducedOrderForSolutionOn(self):
        self._set_reduced(sol=True)

    def setReducedOrderForSolutionOff(self):
        self._set_reduced(sol=False)

    def setReducedOrderForSolutionTo(self, flag=False):
        self._set_reduced(sol=bool(flag))

    def setReducedOrderForEquationOn(self):
        self._set_reduced(eq=True)

    def setReducedOrderForEquationOff(self):
        self._set_reduced(eq=False)

    def setReducedOrderForEquationTo(self, flag=False):
        self._set_reduced(eq=bool(flag))

    def reduceSolutionOrder(self):
        return self._reduce_sol

    def reduceEquationOrder(self):
        return self._reduce_eq

    def getFunctionSpaceForEquation(self):
        return ReducedSolution(self._domain) if self._reduce_eq else Solution(self._domain)

    def getFunctionSpaceForSolution(self):
        return ReducedSolution(self._domain) if self._reduce_sol else Solution(self._domain)

    def hasCoefficient(self, name):
        return name in _ALL or name in _UNSUPPORTED

    def getFunctionSpaceForCoefficient(self, name):
        if name in _INTERIOR:
            return Function(self._domain)
        if name in _REDUCED:
            return ReducedFunction(self._domain)
        if name in _BOUNDARY:
            return FunctionOnBoundary(self._domain)
        if name in _BOUNDARY_REDUCED:
            return ReducedFunctionOnBoundary(self._domain)
        if name in _CONSTRAINT:
            return self.getFunctionSpaceForSolution()
        raise IllegalCoefficient(f"illegal coefficient {name} requested for general PDE.")

    def getShapeOfCoefficient(self, name):
        if name not in _ALL:
            raise IllegalCoefficient(f"illegal coefficient {name} requested for general PDE.")
        return _shape_for(_pattern_of(name), self.getDim(), self.getNumEquations(), self.getNumSolutions())

    def _shape_of(self, name):
        return self.getShapeOfCoefficient(name)

    def createSolution(self):
        ns = self.getNumSolutions()
        fs = self.getFunctionSpaceForSolution()
        if ns == 1:
            return Scalar(0.0, fs, expanded=True)
        return Data(0.0, (ns,), fs, expanded=True)

    def createRightHandSide(self):
        ne = self.getNumEquations()
        fs = self.getFunctionSpaceForEquation()
        if ne == 1:
            return Scalar(0.0, fs, expanded=True)
        return Data(0.0, (ne,), fs, expanded=True)

    def getCoefficient(self, name):
        if name in self._coef:
            return self._coef[name]
        if self.hasCoefficient(name):
            return Data()
        raise IllegalCoefficient(f"illegal coefficient {name} requested for general PDE.")

    def _coef_data(self, name, value):
        """The coefficient as Data on its function space with its shape; raises
        IllegalCoefficientFunctionSpace / IllegalCoefficientValue."""
        fs = self.getFunctionSpaceForCoefficient(name)
        shape = self.getShapeOfCoefficient(name)
        if isinstance(value, Data):
            try:
                dat = value.interpolate(fs)
            except ValueError as e:
                raise IllegalCoefficientFunctionSpace(f"{value.getFunctionSpace()} cannot be interpolated to {fs}: "
                                                      f"{e}") from None
        else:
            a = np.asarray(value, dtype=np.float64)
            if a.shape != shape:
                raise IllegalCoefficientValue(f"Coefficient {name}: expected shape {shape}, got {a.shape}")
            dat = Data(a, shape, fs)
        if dat._shape != shape:
            raise IllegalCoefficientValue(f"Coefficient {name}: expected shape {shape}, got {dat._shape}")
        return dat

    def setValue(self, **coefficients):
        """LinearProblem.setValue (linearPDEs.py:1392-1449 / 2114-2207): unknown names raise
        IllegalCoefficient; the numbers of equations and solutions, when not given, come from
        the first coefficients' shapes; a value on a function space that cannot be
        interpolated to the coefficient's goes to the reduced coefficient of the same name
        where there is one."""
        for name in coefficients:
            if not self.hasCoefficient(name):
                raise IllegalCoefficient(f"Attempt to set unknown coefficient {name}")
        for name, value in coefficients.items():
            if name in _UNSUPPORTED and not (value is None or (isinstance(value, Data) and value.isEmpty())):
                raise NotImplementedError(f"coefficient {name} is not part of the GPU path")

        def empty(v):
            return v is None or (isinstance(v, Data) and v.isEmpty())

        if self._ne is None or self._ns is None:
            for name, value in sorted(coefficients.items()):
                if empty(value) or name in _UNSUPPORTED:
                    continue
                shape = value.getShape() if isinstance(value, Data) else np.asarray(value).shape
                est = _estimate_counts(_pattern_of(name), self.getDim(), shape)
                if est is None:
                    raise IllegalCoefficientValue(f"Illegal shape {shape} of coefficient {name}")
                if self._ne is None and est[0] is not None:
                    self._ne = est[0]
                if self._ns is None and est[1] is not None:
                    self._ns = est[1]
        self.getNumEquations()
        self.getNumSolutions()
        for name, value in coefficients.items():
            if name in _UNSUPPORTED:
                continue
            target = name
            if empty(value):
                self._coef.pop(name, None)
            else:
                try:
                    dat = self._coef_data(name, value)
                except IllegalCoefficientFunctionSpace:
                    red = name + "_reduced"
                    if red in _ALL and red not in coefficients:
                        dat = self._coef_data(red, value)
                        target = red
                    else:
                        raise
                self._coef[target] = dat
            self._altered(target)
        self._solution = None

    def _altered(self, name):
        if name in ("A", "B", "C", "D", "d", "A_reduced", "B_reduced", "C_reduced", "D_reduced", "d_reduced"):
            self._operator_valid = False
        if name in ("X", "Y", "y", "r", "X_reduced", "Y_reduced", "y_reduced"):
            self._rhs_valid = False
        if name == "q":
            self._operator_valid = False
            self._rhs_valid = False

    def resetRightHandSideCoefficients(self):
        """Removes the coefficients that define the right hand side (X, Y, y, their reduced
        forms and r)."""
        for name in ("X", "Y", "y", "X_reduced", "Y_reduced", "y_reduced", "r"):
            if self._coef.pop(name, None) is not None:
                self._altered(name)
        self._solution = None

    def resetAllCoefficients(self):
        self._coef.clear()
        self._operator_valid = self._rhs_valid = False
        self._solution = None

    def _coef_c(self, name, keep):
        """rg_coef for a coefficient; keeps the device tensor alive in ``keep``."""
        d = self._coef.get(name)
        if d is None:
            return L.rg_coef(None, L.RG_COEF_EMPTY)
        t = d._t.contiguous()
        keep.append(t)
        kind = L.RG_COEF_CONSTANT if d.isConstant() else L.RG_COEF_EXPANDED
        return L.rg_coef(t.data_ptr(), kind)

    def getSystem(self):
        """Build operator and right hand side (linearPDEs.py:1881-2082, non-lumped branch):
        interior terms (Function and ReducedFunction), face terms (FunctionOnBoundary and
        ReducedFunctionOnBoundary), then the constraint.  A right hand side rebuilt alone
        assembles only X, Y, y (and their reduced forms) into the existing operator."""
        if self._operator_valid and self._rhs_valid:
            return self._operator, self._rhs
        keep = []
        lib = L.lib()
        empty = L.rg_coef(None, L.RG_COEF_EMPTY)
        rhs_only = self._operator_valid
        if not rhs_only:
            self._operator = SystemMatrix(self._domain, self._nb)
        self._rhs = self.createRightHandSide()
        h = self._operator._handle
        rp = C.c_void_p(self._rhs._t.data_ptr())
        L.set_stream_from_torch()

        def names(group):
            return [(n if (not rhs_only or n[0] in "XYy") else None) for n in group]

        def coefs(group):
            return [self._coef_c(n, keep) if n else empty for n in names(group)]

        L.check(lib.rg_assemble_system(h, rp, *[C.byref(c) for c in coefs(_INTERIOR)]))
        if any(n and n in self._coef for n in names(_REDUCED)):
            L.check(lib.rg_assemble_system_reduced(h, rp, *[C.byref(c) for c in coefs(_REDUCED)]))
        if any(n and n in self._coef for n in names(_BOUNDARY)):
            bd = coefs(_BOUNDARY)
            L.check(lib.rg_assemble_boundary(h, rp, C.byref(bd[0]), C.byref(bd[1])))
        if any(n and n in self._coef for n in names(_BOUNDARY_REDUCED)):
            bd = coefs(_BOUNDARY_REDUCED)
            L.check(lib.rg_assemble_boundary_reduced(h, rp, C.byref(bd[0]), C.byref(bd[1])))
        self._insert_constraint(rhs_only=rhs_only)
        torch.cuda.current_stream().synchronize()
        self._operator_valid = True
        self._rhs_valid = True
        return self._operator, self._rhs

    def _insert_constraint(self, rhs_only):
        """LinearPDE.insertConstraint (linearPDEs.py:2084-2112)."""
        q = self._coef.get("q")
        if q is None:
            return
        r = self._coef.get("r")
        qt = q._dev(self._domain._n)
        rt = r._dev(self._domain._n) if r is not None else None
        L.set_stream_from_torch()
        L.check(L.lib().rg_insert_constraint(self._operator._handle, C.c_void_p(self._rhs._t.data_ptr()),
                                             C.c_void_p(qt.data_ptr()),
                                             C.c_void_p(rt.data_ptr()) if rt is not None else None,
                                             int(rhs_only)))
        torch.cuda.current_stream().synchronize()

    def getOperator(self):
        return self.getSystem()[0]

    def getRightHandSide(self):
        return self.getSystem()[1]

    def getSolution(self):
        """LinearPDE.getSolution (linearPDEs.py:1861-1879)."""
        if self._solution is None:
            mat, f = self.getSystem()
            u = mat.solve(f, self._options)
            fs = self.getFunctionSpaceForSolution()
            self._solution = u if u.getFunctionSpace() == fs else u.interpolate(fs)
        return self._solution

    def getResidualNorms(self, u=None):
        """l2 and max norms of the residual rhs - A u of the current system
        (LinearPDE.getResidual measured in paso's stopping norms)."""
        mat, f = self.getSystem()
        return mat.residualNorms(f, self.getSolution() if u is None else u)

    def isUsingLumping(self):
        return False


class Poisson(LinearPDE):
    """-grad(grad u) = f with u = 0 where q > 0 (linearPDEs.py:2285-2340)."""

    def __init__(self, domain, debug=False):
        super().__init__(domain, debug=debug)
        super().setValue(A=kronecker(domain.getDim()))

    def setValue(self, **coefficients):
        out = {}
        for k, v in coefficients.items():
            if k == "f":
                out["Y"] = v
            elif k == "q":
                out["q"] = v
            else:
                raise ValueError(f"illegal coefficient {k} requested for Poisson equation.")
        super().setValue(**out)
