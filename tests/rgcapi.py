"""Thin test helpers that drive libripley_gpu.so through its C-ABI with device buffers
held in torch tensors (no Python API layer in between)."""
import ctypes as C

import numpy as np
import torch

from esys_b200 import _lib as L


def lib():
    return L.lib()


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Domain:
    def __init__(self, dim, ne, x1=None):
        ne3 = list(ne) + [1] * (3 - dim)
        x1 = list(x1) if x1 is not None else [1.0] * dim
        self.dim, self.ne = dim, tuple(ne)
        self.h = C.c_void_p()
        L.set_stream_from_torch()
        L.check(lib().rg_domain_create(dim, (C.c_int64 * 3)(*ne3), (C.c_double * 3)(0, 0, 0),
                                       (C.c_double * 3)(*(x1 + [1.0] * (3 - dim))), C.byref(self.h)))
        n, nnz = C.c_int64(), C.c_int64()
        dx = (C.c_double * 3)()
        L.check(lib().rg_domain_info(self.h, C.byref(n), C.byref(nnz), None, None, dx))
        self.n, self.nnz = n.value, nnz.value
        self.dx = tuple(dx[:dim])

    def pattern(self):
        p = np.zeros(self.n + 1, np.int32)
        i = np.zeros(self.nnz, np.int32)
        L.check(lib().rg_pattern_to_host(self.h, p.ctypes.data_as(C.c_void_p), i.ctypes.data_as(C.c_void_p)))
        return p, i

    def __del__(self):
        if getattr(self, "h", None):
            lib().rg_domain_destroy(self.h)
            self.h = None


class Matrix:
    def __init__(self, dom, block_size=1):
        self.dom = dom
        self.nb = block_size
        self.h = C.c_void_p()
        if block_size == 1:
            L.check(lib().rg_matrix_create(dom.h, C.byref(self.h)))
        else:
            L.check(lib().rg_matrix_create_system(dom.h, block_size, C.byref(self.h)))

    def values(self):
        p = C.c_void_p()
        L.check(lib().rg_matrix_values(self.h, C.byref(p)))
        torch.cuda.synchronize()
        return _raw(p.value, self.dom.nnz * self.nb * self.nb).clone().cpu().numpy()

    def __del__(self):
        if getattr(self, "h", None):
            lib().rg_matrix_destroy(self.h)
            self.h = None


def _raw(p, count, typestr="<f8"):
    class V:
        __cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr,
                                    "data": (int(p), False), "version": 3, "stream": None}
    return torch.as_tensor(V(), device="cuda")


KINDS = {"const": L.RG_COEF_CONSTANT, "exp": L.RG_COEF_EXPANDED, "elem": L.RG_COEF_PER_ELEMENT}


def coef(arr, kind, keep):
    if arr is None:
        return L.rg_coef(None, L.RG_COEF_EMPTY)
    t = dev(arr)
    keep.append(t)
    return L.rg_coef(t.data_ptr(), kind)


def assemble(mat, rhs_t, keep, **coefs):
    """coefs: name -> (array, kind) for A,B,C,D,X,Y."""
    cs = [coef(*coefs[k], keep) if k in coefs else L.rg_coef(None, 0) for k in "ABCDXY"]
    L.set_stream_from_torch()
    L.check(lib().rg_assemble_single(mat.h if mat else None, ptr(rhs_t), *[C.byref(c) for c in cs]))


def assemble_system(mat, rhs_t, keep, **coefs):
    """coefs: name -> (array, kind) for A,B,C,D,X,Y of a PDE system."""
    cs = [coef(*coefs[k], keep) if k in coefs else L.rg_coef(None, 0) for k in "ABCDXY"]
    L.set_stream_from_torch()
    L.check(lib().rg_assemble_system(mat.h, ptr(rhs_t), *[C.byref(c) for c in cs]))


def assemble_reduced(mat, rhs_t, keep, **coefs):
    """coefs: name -> (array, kind) for A,B,C,D,X,Y on ReducedFunction."""
    cs = [coef(*coefs[k], keep) if k in coefs else L.rg_coef(None, 0) for k in "ABCDXY"]
    L.set_stream_from_torch()
    L.check(lib().rg_assemble_single_reduced(mat.h if mat else None, ptr(rhs_t), *[C.byref(c) for c in cs]))


def assemble_system_reduced(mat, rhs_t, keep, **coefs):
    """coefs: name -> (array, kind) for A,B,C,D,X,Y of a PDE system on ReducedFunction."""
    cs = [coef(*coefs[k], keep) if k in coefs else L.rg_coef(None, 0) for k in "ABCDXY"]
    L.set_stream_from_torch()
    L.check(lib().rg_assemble_system_reduced(mat.h, ptr(rhs_t), *[C.byref(c) for c in cs]))


def assemble_boundary(mat, rhs_t, keep, d=None, y=None, reduced=False):
    dc = coef(*d, keep) if d else L.rg_coef(None, 0)
    yc = coef(*y, keep) if y else L.rg_coef(None, 0)
    L.set_stream_from_torch()
    fn = lib().rg_assemble_boundary_reduced if reduced else lib().rg_assemble_boundary
    L.check(fn(mat.h, ptr(rhs_t), C.byref(dc), C.byref(yc)))


def insert_constraint(mat, rhs_t, q_t, r_t=None, rhs_only=0):
    L.set_stream_from_torch()
    L.check(lib().rg_insert_constraint(mat.h, ptr(rhs_t), ptr(q_t), ptr(r_t), rhs_only))


def opts(**kw):
    o = L.rg_solver_opts()
    lib().rg_solver_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def solve(mat, rhs_t, x_t, o=None):
    d = L.rg_diag()
    o = o or opts()
    L.set_stream_from_torch()
    st = lib().rg_solve(mat.h, ptr(rhs_t), ptr(x_t), C.byref(o), C.byref(d))
    return st, d
