"""B200 implementation of esys-escript's ripley Q1 assembly + paso PCG/Jacobi path.

    from esys_b200.ripley import Brick, Rectangle
    from esys_b200.escript import LinearPDE, Function, Solution, whereZero, kronecker

mirrors ``from esys.ripley import Brick`` / ``from esys.escript import ...`` for that
path.  All numerical work runs in libripley_gpu.so (sm_100a); see include/ripley_gpu.h.
"""
from . import _lib  # noqa: F401

__all__ = ["escript", "ripley"]
