"""CPU tests of the boundary: the C-ABI library loads without a GPU, exports every
symbol include/ripley_gpu.h declares, and the host-side API logic (options, argument
checks) behaves like the reference's."""
import ctypes as C
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "ripley_gpu.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from esys_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # the Python binding covers exactly the header's functions
    assert sorted(_lib.exported_symbols()) == names


def test_version_and_error_buffer_without_gpu():
    from esys_b200 import _lib
    lib = _lib.lib()
    assert lib.rg_version() >= 100
    buf = C.create_string_buffer(8)
    assert lib.rg_last_error(buf, 8) == 0
    assert lib.rg_last_error(None, 0) == _lib.RG_INVALID_ARG


def test_invalid_domain_arguments_rejected_before_any_device_work():
    from esys_b200 import _lib
    lib = _lib.lib()
    h = C.c_void_p()
    ne = (C.c_int64 * 3)(0, 4, 4)
    x0 = (C.c_double * 3)(0, 0, 0)
    x1 = (C.c_double * 3)(1, 1, 1)
    assert lib.rg_domain_create(3, ne, x0, x1, C.byref(h)) == _lib.RG_INVALID_ARG
    assert "positive" in _lib.last_error()
    ne = (C.c_int64 * 3)(4, 4, 4)
    assert lib.rg_domain_create(4, ne, x0, x1, C.byref(h)) == _lib.RG_INVALID_ARG
    big = (C.c_int64 * 3)(2000, 2000, 2000)
    assert lib.rg_domain_create(3, big, x0, x1, C.byref(h)) == _lib.RG_INVALID_ARG
    assert "overflow" in _lib.last_error()
    assert lib.rg_solve(None, None, None, None, None) == _lib.RG_INVALID_ARG


def test_solver_options_defaults_and_validation():
    from esys_b200.escript import SolverBuddy, SolverOptions
    so = SolverBuddy()
    # SolverBuddy::SolverBuddy defaults (escriptcore/src/SolverOptions.cpp:40-70)
    assert so.getTolerance() == 1e-8
    assert so.getIterMax() == 100000
    assert so.getNumSweeps() == 1
    assert so.getPreconditioner() == SolverOptions.JACOBI
    assert so.getSolverMethod() == SolverOptions.DEFAULT
    with pytest.raises(ValueError):
        so.setTolerance(-1.0)
    with pytest.raises(ValueError):
        so.setIterMax(0)
    so.setSolverMethod(SolverOptions.PCG)
    o = so._to_c()
    assert o.method == 10 and o.preconditioner == 20 and o.tolerance == 1e-8
    so.setSolverMethod(SolverOptions.GMRES)
    with pytest.raises(NotImplementedError):
        so._to_c()
    so.setSolverMethod(SolverOptions.PCG)
    so.setPreconditioner(SolverOptions.ILU0)
    with pytest.raises(NotImplementedError):
        so._to_c()


def test_status_mapping_to_reference_exceptions():
    from esys_b200 import _lib
    with pytest.raises(ValueError):
        _lib.check(_lib.RG_INVALID_ARG)
    with pytest.raises(_lib.PasoException) as e:
        _lib.check(_lib.RG_MAXITER)
    assert e.value.status == _lib.RG_MAXITER
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.RG_NOT_SUPPORTED)
    with pytest.raises(_lib.RipleyGPUError):
        _lib.check(_lib.RG_CUDA_ERROR)
