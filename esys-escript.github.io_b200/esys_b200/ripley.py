"""ripley Rectangle / Brick domains on one GPU (ripley/src/ripleycpp.cpp:151-238, 521-546).

A domain owns the device CSR pattern of paso's system matrix (built by
rg_domain_create) and supplies the coordinates of its function spaces.  Node, DOF and
element numbering follow ripley on one rank: node id = k0 + NN0*k1 (+ NN0*NN1*k2),
element id likewise over NE, faces ordered left, right, bottom, top (, front, back).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L
from .escript import (Data, DEVICE, Function, FunctionOnBoundary, Solution, ContinuousFunction,
                      ReducedFunction)

_G = (0.5 - math.sqrt(3.0) / 6.0, 0.5 + math.sqrt(3.0) / 6.0)


def _range_arg(l, name):
    if isinstance(l, (tuple, list)):
        if len(l) != 2:
            raise ValueError(f"Argument {name} must be a float or 2-tuple")
        return float(l[0]), float(l[1])
    return 0.0, float(l)


class RipleyDomain:
    def __init__(self, dim, ne, ranges):
        self._dim = dim
        self._ne = [int(v) for v in ne] + [1] * (3 - dim)
        if any(v <= 0 for v in self._ne):
            raise ValueError("Number of elements in each spatial dimension must be positive")
        self._x0 = [r[0] for r in ranges] + [0.0] * (3 - dim)
        self._x1 = [r[1] for r in ranges] + [1.0] * (3 - dim)
        self._nn = [v + 1 for v in self._ne[:dim]] + [1] * (3 - dim)
        self._dx = [(self._x1[k] - self._x0[k]) / self._ne[k] for k in range(dim)] + [1.0] * (3 - dim)
        h = C.c_void_p()
        ne_c = (C.c_int64 * 3)(*self._ne)
        x0_c = (C.c_double * 3)(*self._x0)
        x1_c = (C.c_double * 3)(*self._x1)
        L.set_stream_from_torch()
        L.check(L.lib().rg_domain_create(dim, ne_c, x0_c, x1_c, C.byref(h)))
        self._handle = h
        n, nnz = C.c_int64(), C.c_int64()
        L.check(L.lib().rg_domain_info(h, C.byref(n), C.byref(nnz), None, None, None))
        self._n, self._nnz = n.value, nnz.value
        self._nel = int(np.prod(self._ne[:dim]))
        if dim == 2:
            self._face_counts = [self._ne[1], self._ne[1], self._ne[0], self._ne[0]]
        else:
            self._face_counts = [self._ne[1] * self._ne[2]] * 2 + [self._ne[0] * self._ne[2]] * 2 + \
                                [self._ne[0] * self._ne[1]] * 2
        self._nfaces = int(sum(self._face_counts))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h and L._lib is not None:
            L._lib.rg_domain_destroy(h)
            self._handle = None

    # ---- escript Domain API
    def getDim(self):
        return self._dim

    def getMPISize(self):
        return 1

    def getMPIRank(self):
        return 0

    def getNumDataPointsGlobal(self):
        return self._n

    def getX(self):
        return ContinuousFunction(self).getX()

    def getNormal(self):
        fs = FunctionOnBoundary(self)
        nq = 1 << (self._dim - 1)
        parts = []
        for face, cnt in enumerate(self._face_counts):
            v = torch.zeros(self._dim, dtype=torch.float64, device=DEVICE)
            v[face // 2] = 1.0 if face % 2 else -1.0
            parts.append(v.expand(cnt * nq, -1))
        return Data._wrap(torch.cat(parts).contiguous(), (self._dim,), fs)

    def getSize(self):
        return Function(self).getSize()

    def getGridParameters(self):
        return (tuple(self._x0[: self._dim]), tuple(self._dx[: self._dim]), tuple(self._nn[: self._dim]))

    def getNumElements(self):
        return self._nel

    def getNumNodes(self):
        return self._n

    def createAssembler(self, typename="DefaultAssembler", options=None):
        """Brick::createAssembler (ripley/src/Brick.cpp:3972-3997): only the default assembler."""
        if typename != "DefaultAssembler":
            raise ValueError(f"unknown assembler {typename} (only DefaultAssembler is on the GPU path)")
        return "DefaultAssembler"

    def pattern(self):
        """Host copy of the CSR pattern (ptr, idx) as int32 numpy arrays."""
        ptr = np.zeros(self._n + 1, np.int32)
        idx = np.zeros(self._nnz, np.int32)
        L.check(L.lib().rg_pattern_to_host(self._handle, ptr.ctypes.data_as(C.c_void_p),
                                           idx.ctypes.data_as(C.c_void_p)))
        return ptr, idx

    def __str__(self):
        name = "Brick" if self._dim == 3 else "Rectangle"
        return f"{name}({', '.join(str(v) for v in self._ne[: self._dim])})"

    __repr__ = __str__

    # ---- coordinates
    def _axis(self, k, where):
        """1D coordinates along axis k at nodes or at element Gauss points."""
        if where == "nodes":
            return self._x0[k] + self._dx[k] * torch.arange(self._nn[k], dtype=torch.float64, device=DEVICE)
        e = torch.arange(self._ne[k], dtype=torch.float64, device=DEVICE)
        g = torch.tensor(_G, dtype=torch.float64, device=DEVICE)
        return self._x0[k] + self._dx[k] * (e[:, None] + g[None, :])  # (NE, 2)

    def _coordinates(self, storage):
        d = self._dim
        if storage == "nodes":
            axes = [self._axis(k, "nodes") for k in range(d)]
            grids = torch.meshgrid(*reversed(axes), indexing="ij")  # slowest axis first
            return torch.stack([g.reshape(-1) for g in reversed(grids)], 1)
        if storage == "elem":
            axes = [self._x0[k] + self._dx[k] * (0.5 + torch.arange(self._ne[k], dtype=torch.float64,
                                                                     device=DEVICE)) for k in range(d)]
            grids = torch.meshgrid(*reversed(axes), indexing="ij")
            return torch.stack([g.reshape(-1) for g in reversed(grids)], 1)
        if storage == "qp":
            # point (e, q): element e = k0 + NE0 k1 (+ NE0 NE1 k2), q = q0 + 2 q1 (+ 4 q2)
            ax = [self._axis(k, "qp") for k in range(d)]  # each (NE_k, 2)
            if d == 2:
                x = ax[0][None, :, None, :].expand(self._ne[1], -1, 2, -1)  # (k1,k0,q1,q0)
                y = ax[1][:, None, :, None].expand(-1, self._ne[0], -1, 2)
                return torch.stack([x.reshape(-1), y.reshape(-1)], 1)
            x = ax[0][None, None, :, None, None, :].expand(self._ne[2], self._ne[1], -1, 2, 2, -1)
            y = ax[1][None, :, None, None, :, None].expand(self._ne[2], -1, self._ne[0], 2, -1, 2)
            z = ax[2][:, None, None, :, None, None].expand(-1, self._ne[1], self._ne[0], -1, 2, 2)
            return torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1)
        if storage == "face":
            return torch.cat([self._face_points(f) for f in range(2 * d)])
        if storage == "rface":
            return torch.cat([self._face_points(f, reduced=True) for f in range(2 * d)])
        raise ValueError(storage)

    def _face_axes(self, face):
        ax = face // 2
        return ax, [a for a in range(self._dim) if a != ax]

    def _face_points(self, face, reduced=False):
        """Gauss points of face ``face``: (face element (lower in-face axis fastest), q); with
        ``reduced`` the face element centres."""
        ax, fa = self._face_axes(face)
        side = face % 2
        g = torch.tensor((0.5,) if reduced else _G, dtype=torch.float64, device=DEVICE)
        nq = g.numel()
        c_fixed = self._x0[ax] + (self._x1[ax] - self._x0[ax]) * side
        cols = {}
        if self._dim == 2:
            a = fa[0]
            pa = self._x0[a] + self._dx[a] * (torch.arange(self._ne[a], dtype=torch.float64,
                                                          device=DEVICE)[:, None] + g[None, :])
            cols[a] = pa.reshape(-1)
            cols[ax] = torch.full_like(cols[a], c_fixed)
        else:
            a, b = fa
            pa = self._x0[a] + self._dx[a] * (torch.arange(self._ne[a], dtype=torch.float64, device=DEVICE)[:, None] + g[None, :])
            pb = self._x0[b] + self._dx[b] * (torch.arange(self._ne[b], dtype=torch.float64, device=DEVICE)[:, None] + g[None, :])
            # index order: (kb, ka, qb, qa)
            A = pa[None, :, None, :].expand(self._ne[b], -1, nq, -1)
            B = pb[:, None, :, None].expand(-1, self._ne[a], -1, nq)
            cols[a] = A.reshape(-1)
            cols[b] = B.reshape(-1)
            cols[ax] = torch.full_like(cols[a], c_fixed)
        return torch.stack([cols[k] for k in range(self._dim)], 1)

    def _nodes_to_face(self, nodal, reduced=False):
        """Interpolate nodal values (n, ncomp) to the face Gauss points (``reduced``: to the
        face element centres)."""
        ncomp = nodal.shape[1]
        d = self._dim
        grid = nodal.reshape(tuple(reversed(self._nn[:d])) + (ncomp,))  # (.., NN1, NN0, c)
        g = torch.tensor((0.5,) if reduced else _G, dtype=torch.float64, device=DEVICE)
        out = []
        for face in range(2 * d):
            ax, fa = self._face_axes(face)
            side = face % 2
            sl = [slice(None)] * d
            sl[d - 1 - ax] = self._nn[ax] - 1 if side else 0
            plane = grid[tuple(sl)]  # remaining axes in reversed order
            if d == 2:
                v = plane  # (NN_a, c)
                lo, hi = v[:-1], v[1:]
                vals = lo[:, None, :] * (1 - g)[None, :, None] + hi[:, None, :] * g[None, :, None]
                out.append(vals.reshape(-1, ncomp))
            else:
                v = plane  # (NN_b, NN_a, c)
                v00, v10 = v[:-1, :-1], v[:-1, 1:]
                v01, v11 = v[1:, :-1], v[1:, 1:]
                ga = g[None, None, None, :, None]
                gb = g[None, None, :, None, None]
                vals = (v00[:, :, None, None, :] * (1 - ga) * (1 - gb) + v10[:, :, None, None, :] * ga * (1 - gb)
                        + v01[:, :, None, None, :] * (1 - ga) * gb + v11[:, :, None, None, :] * ga * gb)
                out.append(vals.reshape(-1, ncomp))
        return torch.cat(out)


def Rectangle(n0, n1, l0=1.0, l1=1.0, d0=-1, d1=-1, diracPoints=(), diracTags=(),
              escriptworld=None, **kwargs):
    """Rectangle with n0 x n1 elements over [0,l0] x [0,l1] (or coordinate ranges)."""
    if diracPoints:
        raise NotImplementedError("dirac points are not part of the GPU path")
    return RipleyDomain(2, (int(n0), int(n1)), (_range_arg(l0, "l0"), _range_arg(l1, "l1")))


def Brick(n0, n1, n2, l0=1.0, l1=1.0, l2=1.0, d0=-1, d1=-1, d2=-1, diracPoints=(), diracTags=(),
          escriptworld=None, **kwargs):
    """Brick with n0 x n1 x n2 elements over [0,l0] x [0,l1] x [0,l2] (or coordinate ranges)."""
    if diracPoints:
        raise NotImplementedError("dirac points are not part of the GPU path")
    return RipleyDomain(3, (int(n0), int(n1), int(n2)),
                        (_range_arg(l0, "l0"), _range_arg(l1, "l1"), _range_arg(l2, "l2")))
