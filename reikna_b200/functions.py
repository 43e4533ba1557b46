"""Element functions for transformation code, by the names reikna's code uses.

reikna's transformations call arithmetic helpers that grunnur renders as device
functions for the operand types (``grunnur.functions.mul``, ``div``, ``conj``,
``polar_unit``, ``exp``, ``norm``, ``add``, ``cast``; used through ``render_kwds``,
e.g. reikna/transformations.py:60-140).  Here each returns an object whose text is
the name of a generic device function (overloaded for float / double and their
complex pairs) compiled with every run-time kernel, so ``${mul}(a, b)`` in a
template works the same way.
"""

from __future__ import annotations


class _Function:
    def __init__(self, name: str):
        self.name = name

    def __str__(self):
        return self.name

    def __repr__(self):
        return f"<device function {self.name}>"


def mul(*in_dtypes, out_dtype=None):
    """``a * b`` of real or complex operands."""
    return _Function("rkf::mul")


def div(in_dtype1=None, in_dtype2=None, out_dtype=None):
    """``a / b`` of real or complex operands."""
    return _Function("rkf::div")


def add(*in_dtypes, out_dtype=None):
    """``a + b`` of real or complex operands."""
    return _Function("rkf::add")


def conj(dtype=None):
    """Complex conjugate."""
    return _Function("rkf::conj")


def norm(dtype=None):
    """``|z|^2``."""
    return _Function("rkf::norm")


def polar_unit(dtype=None):
    """``exp(i theta)`` of a real angle."""
    return _Function("rkf::polar_unit")


def exp(dtype=None):
    """Exponential of a real or complex value."""
    return _Function("rkf::exp")


def cast(out_dtype, in_dtype=None):
    """Conversion to ``out_dtype`` (real to complex with a zero imaginary part,
    complex to real keeps the real part)."""
    from .fft.user import ctype

    return _Function(f"rkf::cast<{ctype(out_dtype)}>")
