"""Shared checks, following reikna's tests/helpers.py conventions."""

from __future__ import annotations

import math

import numpy

# reikna's FFT test tolerances (tests/test_fft/test_fft.py:148-170, 204-207)
FFT_ATOL = 2e-5
FFT_RTOL = 1e-3


def rel_l2(a, b) -> float:
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    den = numpy.linalg.norm(b.ravel())
    return float(numpy.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def fft_bound(dtype, n_total: int) -> float:
    """Stated rel-L2 bound vs the FP64 oracle: 2e-6 log2 N (c64), 1e-14 log2 N (c128)."""
    lg = max(1.0, math.log2(max(2, n_total)))
    return (2e-6 if numpy.dtype(dtype) == numpy.complex64 else 1e-14) * lg


def uniform_array(rng, shape, dtype):
    """reikna's get_test_array for complex dtypes: uniform [0, 1) real and imaginary parts."""
    shape = (shape,) if isinstance(shape, int) else tuple(shape)
    return (rng.uniform(0, 1, shape) + 1j * rng.uniform(0, 1, shape)).astype(dtype)


def normal_array(rng, shape, dtype):
    shape = (shape,) if isinstance(shape, int) else tuple(shape)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def diff_is_negligible(m, m_ref, atol, rtol) -> bool:
    return bool(numpy.isclose(m, m_ref, atol=atol, rtol=rtol).all())
