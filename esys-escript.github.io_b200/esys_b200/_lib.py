"""ctypes binding of libripley_gpu.so, the sm_100a C-ABI library (include/ripley_gpu.h).

The shared library is built in-tree by ``make -C esys-escript.github.io_b200`` and lives
next to this file.  There is no fallback: if the library or a GPU is missing, every
compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libripley_gpu.so")

# status codes (include/ripley_gpu.h)
RG_OK, RG_INVALID_ARG, RG_CUDA_ERROR, RG_MAXITER, RG_BREAKDOWN, RG_NAN, RG_TIMEOUT, \
    RG_DIVERGENCE, RG_NOT_SUPPORTED = range(9)

RG_COEF_EMPTY, RG_COEF_CONSTANT, RG_COEF_EXPANDED, RG_COEF_PER_ELEMENT = range(4)
RG_METHOD_PCG = 10
RG_PRECOND_JACOBI = 20
RG_MODE_PASO, RG_MODE_STANDARD = 0, 1
RG_PREC_FP64, RG_PREC_FP32_REFINE = 0, 1
RG_LAYOUT_CSR, RG_LAYOUT_BAND, RG_LAYOUT_COEF = 0, 1, 2


class PasoException(RuntimeError):
    """Solver failure, raised where paso raises PasoException (paso/src/solve.cpp:119-142)."""

    def __init__(self, msg, status):
        super().__init__(msg)
        self.status = status


class RipleyGPUError(RuntimeError):
    """A CUDA error inside the library."""


class rg_coef(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("kind", C.c_int)]


class rg_solver_opts(C.Structure):
    _fields_ = [("method", C.c_int), ("preconditioner", C.c_int), ("tolerance", C.c_double),
                ("iter_max", C.c_int64), ("sweeps", C.c_int), ("verbose", C.c_int),
                ("accept_convergence_failure", C.c_int), ("mode", C.c_int),
                ("precision", C.c_int), ("layout", C.c_int), ("inner_tolerance", C.c_double),
                ("initial_guess", C.c_void_p), ("guess_sweeps", C.c_int)]


class rg_act(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("n", C.c_int), ("d", C.c_int), ("h", C.c_int), ("w", C.c_int),
                ("c", C.c_int)]


class rg_diag(C.Structure):
    _fields_ = [("num_iter", C.c_int64), ("num_outer", C.c_int64),
                ("residual_norm", C.c_double), ("residual_max", C.c_double),
                ("rhs_norm", C.c_double), ("converged", C.c_int), ("time", C.c_double),
                ("set_up_time", C.c_double), ("net_time", C.c_double),
                ("guess_residual", C.c_double), ("guess_rejected", C.c_int), ("fp64_fallback", C.c_int),
                ("inner_operator", C.c_int)]


_lib = None

# name -> (restype, argtypes); every function returns int status unless noted
_SIGNATURES = {
    "rg_version": (C.c_int, []),
    "rg_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "rg_set_stream": (C.c_int, [C.c_void_p]),
    "rg_domain_create": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    "rg_domain_destroy": (C.c_int, [C.c_void_p]),
    "rg_domain_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_double)]),
    "rg_pattern": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                             C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "rg_pattern_to_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "rg_matrix_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "rg_matrix_destroy": (C.c_int, [C.c_void_p]),
    "rg_matrix_reset": (C.c_int, [C.c_void_p]),
    "rg_matrix_values": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "rg_matrix_is_balanced": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "rg_matrix_balance_vector": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "rg_assemble_single": (C.c_int, [C.c_void_p, C.c_void_p] + [C.POINTER(rg_coef)] * 6),
    "rg_assemble_boundary": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(rg_coef),
                                       C.POINTER(rg_coef)]),
    "rg_assemble_boundary_reduced": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(rg_coef),
                                               C.POINTER(rg_coef)]),
    "rg_assemble_single_reduced": (C.c_int, [C.c_void_p, C.c_void_p] + [C.POINTER(rg_coef)] * 6),
    "rg_assemble_system": (C.c_int, [C.c_void_p, C.c_void_p] + [C.POINTER(rg_coef)] * 6),
    "rg_matrix_create_system": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "rg_assemble_system_reduced": (C.c_int, [C.c_void_p, C.c_void_p] + [C.POINTER(rg_coef)] * 6),
    "rg_matrix_create_system": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "rg_matrix_block_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "rg_insert_constraint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "rg_nullify_rows_and_cols": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "rg_spmv": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p]),
    "rg_interpolate_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "rg_save_mm": (C.c_int, [C.c_void_p, C.c_char_p]),
    "rg_residual_norms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]),
    "rg_solver_set_config": (C.c_int, [C.c_void_p, C.c_int]),
    "rg_test_wait_limit": (C.c_int, [C.c_int, C.c_int]),
    "rg_residual_norms_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
    "rg_solver_opts_default": (None, [C.POINTER(rg_solver_opts)]),
    "rg_solver_config": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "rg_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(rg_solver_opts),
                           C.POINTER(rg_diag)]),
    "rg_ws_conv3": (C.c_int, [C.POINTER(rg_act), C.c_void_p, C.c_void_p, C.POINTER(rg_act), C.c_int,
                              C.POINTER(rg_act), C.c_void_p]),
    "rg_ws_conv3_wgrad": (C.c_int, [C.POINTER(rg_act), C.POINTER(rg_act), C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                    C.c_void_p]),
    "rg_ws_avgpool": (C.c_int, [C.POINTER(rg_act), C.POINTER(rg_act)]),
    "rg_ws_avgpool_bwd": (C.c_int, [C.POINTER(rg_act), C.POINTER(rg_act), C.POINTER(rg_act), C.c_int, C.POINTER(rg_act)]),
    "rg_ws_upcat": (C.c_int, [C.POINTER(rg_act), C.POINTER(rg_act), C.POINTER(rg_act)]),
    "rg_ws_upcat_bwd": (C.c_int, [C.POINTER(rg_act), C.POINTER(rg_act), C.POINTER(rg_act)]),
    "rg_ws_head": (C.c_int, [C.POINTER(rg_act), C.c_void_p, C.c_void_p, C.c_void_p]),
    "rg_ws_head_bwd_x": (C.c_int, [C.POINTER(rg_act), C.c_void_p, C.c_void_p, C.POINTER(rg_act)]),
    "rg_ws_colsum": (C.c_int, [C.POINTER(rg_act), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "rg_ws_mse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p]),
    "rg_ws_h1_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rg_ws_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float,
                             C.c_float, C.c_float, C.c_float, C.c_int]),
    "rg_ws_weights_bf16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "rg_ws_field_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_void_p,
                                    C.c_void_p]),
    "rg_ws_pack_input": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(rg_act), C.c_void_p]),
    "rg_ws_element_fields": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int64, C.c_void_p,
                                       C.c_void_p]),
    "rg_ws_nodes_to_cells": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_void_p]),
    "rg_ws_cells_to_nodes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                       C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "rg_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "rg_batch_destroy": (C.c_int, [C.c_void_p]),
    "rg_batch_tune": (C.c_int, [C.c_void_p]),
    "rg_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "rg_batch_set_spmv": (C.c_int, [C.c_void_p, C.c_int]),
    "rg_batch_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(rg_solver_opts),
                                 C.c_void_p]),
    "rg_timers_enable": (C.c_int, [C.c_int]),
    "rg_timers_reset": (C.c_int, []),
    "rg_timers_count": (C.c_int, []),
    "rg_timer_name": (C.c_char_p, [C.c_int]),
    "rg_timers_read": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_double)]),
}


def exported_symbols():
    """Names the header declares and this binding expects the library to export."""
    return sorted(_SIGNATURES)


def lib():
    """Load the library (once).  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RipleyGPUError(
                f"{LIB_PATH} is missing; build it with `make -C {os.path.dirname(HERE)}`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().rg_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Map a status to the reference's exception classes."""
    if status == RG_OK:
        return
    msg = last_error() or what
    if status == RG_INVALID_ARG:
        raise ValueError(msg)
    if status == RG_CUDA_ERROR:
        raise RipleyGPUError(msg)
    if status == RG_NOT_SUPPORTED:
        raise NotImplementedError(msg)
    raise PasoException(msg, status)


def timers():
    """{kind name: (launches, timed launches, total ms)} of the library's kernels."""
    out = {}
    lb = lib()
    for k in range(lb.rg_timers_count()):
        n, t, ms = C.c_int64(), C.c_int64(), C.c_double()
        lb.rg_timers_read(k, C.byref(n), C.byref(t), C.byref(ms))
        out[lb.rg_timer_name(k).decode()] = (n.value, t.value, ms.value)
    return out


def set_stream_from_torch() -> None:
    """Order library work after the torch work already queued on torch's current stream."""
    import torch
    lib().rg_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
