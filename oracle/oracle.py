"""Python access to the CPU oracle (test infrastructure only).

``liboracle.so`` is the C restatement of reikna's FFT algorithm (see
``reikna_fft_oracle.c``).  This module builds it on demand with ``make`` and exposes:

* ``fft(x, axes, inverse)`` -- reikna-semantics FFT on the CPU (complex64 in FP32,
  complex128 in FP64 arithmetic), OpenMP over lines;
* ``radix_array``, ``global_radix_info``, ``kweights``, ``kernel_chain`` -- the
  planner restatement, pinned against golden fixtures of reikna's own planner;
* ``rfft_half``, ``irfft_half``, ``aprfft``, ``iaprfft`` -- the real and antiperiodic
  transforms of reikna's specialised-FFT example, over the oracle FFT;
* ``numpy_ref`` -- the FP64 numpy reference reikna's tests compare against.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from pathlib import Path

import numpy

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None
_lock = threading.Lock()


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or any(
        p.stat().st_mtime > LIB.stat().st_mtime for p in (HERE / "reikna_fft_oracle.c", HERE / "rko_body.h")
    ):
        env = dict(os.environ)
        env.pop("CC", None)
        res = subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], capture_output=True, text=True, env=env)
        if res.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                build()
                L = ctypes.CDLL(str(LIB))
                i64p = ctypes.POINTER(ctypes.c_int64)
                ip = ctypes.POINTER(ctypes.c_int)
                L.rko_radix_array.argtypes = [ctypes.c_int, ctypes.c_int, ip]
                L.rko_global_radix_info.argtypes = [ctypes.c_int64, ip, ip, ip]
                L.rko_kweights.argtypes = [
                    ctypes.c_int64,
                    ctypes.c_int64,
                    ctypes.POINTER(ctypes.c_double),
                    ctypes.POINTER(ctypes.c_double),
                ]
                L.rko_plan_create.argtypes = [ctypes.c_int, i64p, ctypes.c_int, ip, ctypes.c_int64]
                L.rko_plan_create.restype = ctypes.c_void_p
                L.rko_plan_destroy.argtypes = [ctypes.c_void_p]
                L.rko_plan_nkernels.argtypes = [ctypes.c_void_p]
                L.rko_plan_kernel.argtypes = [ctypes.c_void_p, ctypes.c_int, i64p]
                L.rko_exec_c64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
                L.rko_exec_c128.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
                for name in ("rko_exec_c64_shift", "rko_exec_c128_shift"):
                    getattr(L, name).argtypes = [
                        ctypes.c_void_p,
                        ctypes.c_void_p,
                        ctypes.c_void_p,
                        ctypes.c_int,
                        ctypes.c_int,
                        ctypes.POINTER(ctypes.c_int),
                        ctypes.c_double,
                    ]
                _lib = L
    return _lib


def radix_array(size: int, use_max_radix: bool = False) -> list[int]:
    out = (ctypes.c_int * 32)()
    n = lib().rko_radix_array(size, int(use_max_radix), out)
    if n < 0:
        raise ValueError("size must be a power of 2")
    return list(out[:n])


def global_radix_info(size: int) -> tuple[list[int], list[int], list[int]]:
    r, r1, r2 = (ctypes.c_int * 32)(), (ctypes.c_int * 32)(), (ctypes.c_int * 32)()
    n = lib().rko_global_radix_info(size, r, r1, r2)
    if n < 0:
        raise ValueError("size must be a power of 2")
    return list(r[:n]), list(r1[:n]), list(r2[:n])


def kweights(size_real: int, size_bound: int) -> numpy.ndarray:
    a = numpy.zeros(2 * size_bound, numpy.float64)
    b = numpy.zeros(2 * size_bound, numpy.float64)
    lib().rko_kweights(
        size_real, size_bound, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), b.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    )
    return numpy.vstack([a[0::2] + 1j * a[1::2], b[0::2] + 1j * b[1::2]])


class Plan:
    def __init__(self, shape, axes=None, local_limit: int = 1024):
        shape = tuple(int(s) for s in shape)
        axes = tuple(range(len(shape))) if axes is None else tuple(int(a) for a in axes)
        self.shape, self.axes = shape, axes
        sh = (ctypes.c_int64 * len(shape))(*shape)
        ax = (ctypes.c_int * max(1, len(axes)))(*axes)
        self._h = lib().rko_plan_create(len(shape), sh, len(axes), ax, local_limit)
        if not self._h:
            raise ValueError("oracle planning failed")

    def chain(self) -> list[dict]:
        out = []
        info = (ctypes.c_int64 * 64)()
        for i in range(lib().rko_plan_nkernels(self._h)):
            n = lib().rko_plan_kernel(self._h, i, info)
            v = list(info[:n])
            nr = v[9]
            out.append(
                dict(
                    kind="local" if v[0] == 0 else "global",
                    axis=v[1],
                    fft_size=v[2],
                    fft_size_real=v[3],
                    reverse_direction=bool(v[4]),
                    pad_in=bool(v[5]),
                    takes_kweights=bool(v[6]),
                    unpad_out=bool(v[7]),
                    pass_num=v[8],
                    radix=v[10 : 10 + nr],
                    radix1=v[10 + nr],
                    radix2=v[11 + nr],
                )
            )
        return out

    def __call__(self, x: numpy.ndarray, inverse: bool = False, threads: int | None = None) -> numpy.ndarray:
        x = numpy.ascontiguousarray(x)
        if x.shape != self.shape:
            raise ValueError("shape mismatch")
        out = numpy.empty_like(x)
        nt = threads or os.cpu_count() or 1
        if x.dtype == numpy.complex64:
            rc = lib().rko_exec_c64(self._h, x.ctypes.data, out.ctypes.data, int(inverse), nt)
        elif x.dtype == numpy.complex128:
            rc = lib().rko_exec_c128(self._h, x.ctypes.data, out.ctypes.data, int(inverse), nt)
        else:
            raise TypeError("oracle FFT needs complex64 or complex128")
        if rc != 0:
            raise MemoryError("oracle execution failed")
        return out

    def shifted(self, x: numpy.ndarray, scale: float = 1.0, inverse: bool = False, threads: int | None = None,
                out: numpy.ndarray | None = None) -> numpy.ndarray:
        """FFT with a fused output fftshift over all axes and a scale (reikna output transformation)."""
        x = numpy.ascontiguousarray(x)
        out = numpy.empty_like(x) if out is None else out
        sh = (ctypes.c_int * len(self.shape))(*[n // 2 for n in self.shape])
        nt = threads or os.cpu_count() or 1
        fn = lib().rko_exec_c64_shift if x.dtype == numpy.complex64 else lib().rko_exec_c128_shift
        if fn(self._h, x.ctypes.data, out.ctypes.data, int(inverse), nt, sh, float(scale)) != 0:
            raise MemoryError("oracle execution failed")
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().rko_plan_destroy(h)
            self._h = None


def fft(x: numpy.ndarray, axes=None, inverse: bool = False, threads: int | None = None) -> numpy.ndarray:
    """reikna-semantics FFT of ``x`` over ``axes`` on the CPU."""
    return Plan(x.shape, axes)(x, inverse=inverse, threads=threads)


def kernel_chain(shape, axes=None, local_limit: int = 1024) -> list[dict]:
    return Plan(shape, axes, local_limit).chain()


def _complex_of(x: numpy.ndarray):
    return numpy.complex64 if x.dtype in (numpy.float32, numpy.complex64) else numpy.complex128


def rfft_half(x: numpy.ndarray, threads: int | None = None) -> numpy.ndarray:
    """Spectrum of real signals along the last axis through the half-length complex FFT
    (examples/demo_specialized_fft.py:58-79; the RFFT computation :175-241 and the
    ``prepare_rfft_output`` kernel of demo_specialized_fft.mako:1-33).  The half-length
    FFT is the oracle's reikna-semantics FFT in the input's precision; the A/B step
    runs in FP64."""
    x = numpy.asarray(x)
    n = x.shape[-1]
    h = n // 2
    z = (x[..., 0::2] + 1j * x[..., 1::2]).astype(_complex_of(x))
    zf = fft(z, axes=(z.ndim - 1,), threads=threads).astype(numpy.complex128)
    w = numpy.exp(-2j * numpy.pi * numpy.arange(h) / n)
    a, b = 0.5 * (1 - 1j * w), 0.5 * (1 + 1j * w)
    zrev = numpy.roll(zf[..., ::-1], 1, axis=-1)  # Z[(h - k) mod h]
    out = numpy.empty(x.shape[:-1] + (h + 1,), numpy.complex128)
    out[..., :h] = zf * a + numpy.conj(zrev) * b
    out[..., h] = zf[..., 0].real - zf[..., 0].imag
    return out


def irfft_half(xf: numpy.ndarray, threads: int | None = None) -> numpy.ndarray:
    """Real signals from their half spectra along the last axis through the half-length
    inverse FFT (examples/demo_specialized_fft.py:82-101; the IRFFT computation
    :244-331, ``prepare_irfft_input`` of demo_specialized_fft.mako:36-62): the
    imaginary parts of the first and last bins are ignored, as numpy's irfft does."""
    xf = numpy.array(xf, numpy.complex128)
    h = xf.shape[-1] - 1
    n = 2 * h
    xf[..., 0] = xf[..., 0].real
    xf[..., -1] = xf[..., -1].real
    w = numpy.exp(-2j * numpy.pi * numpy.arange(h) / n)
    a, b = numpy.conj(0.5 * (1 - 1j * w)), numpy.conj(0.5 * (1 + 1j * w))
    zf = xf[..., :-1] * a + numpy.conj(xf[..., h:0:-1]) * b
    z = fft(zf, axes=(zf.ndim - 1,), inverse=True, threads=threads)
    out = numpy.empty(xf.shape[:-1] + (n,), numpy.float64)
    out[..., 0::2] = z.real
    out[..., 1::2] = z.imag
    return out


def aprfft(x: numpy.ndarray, threads: int | None = None) -> numpy.ndarray:
    """Odd harmonics of real antiperiodic signals (x[k] = -x[N/2 + k]) from their first
    halves x (..., N/2) -> (..., N/4) (examples/demo_specialized_fft.py:104-121 and the
    APRFFT computation :379-453): y = x * 4 sin(2 pi n / N), Y = rfft(y), Y *= -i,
    Y[0] = Y[0] / 2 + 2 sum(x cos(2 pi n / N)), F = cumsum(Y[:-1])."""
    x = numpy.asarray(x)
    size = x.shape[-1] * 2
    n = numpy.arange(size // 2)
    y = x.astype(numpy.float64) * (4 * numpy.sin(2 * numpy.pi * n / size))
    yf = rfft_half(y.astype(x.dtype), threads=threads)
    re1 = 2 * numpy.sum(x.astype(numpy.float64) * numpy.cos(2 * numpy.pi * n / size), axis=-1)
    yf = yf * -1j
    yf[..., 0] = yf[..., 0] / 2 + re1
    return numpy.cumsum(yf[..., :-1], axis=-1)


def iaprfft(xf: numpy.ndarray, threads: int | None = None) -> numpy.ndarray:
    """First halves (..., N/2) of real antiperiodic signals from their N/4 odd harmonics
    (examples/demo_specialized_fft.py:124-141 and the IAPRFFT computation :456-581):
    Y[1:-1] = i (F[1:] - F[:-1]), Y[0] = -2 Im F[0], Y[-1] = 2 Im F[-1], y = irfft(Y),
    x[n] = y[n] / (4 sin(2 pi n / N)) for n >= 1, x[0] = sum(Re F) / (N / 2)."""
    xf = numpy.asarray(xf, numpy.complex128)
    q = xf.shape[-1]
    size = 4 * q
    yf = numpy.empty(xf.shape[:-1] + (q + 1,), numpy.complex128)
    yf[..., 1:-1] = 1j * (xf[..., 1:] - xf[..., :-1])
    yf[..., 0] = -2 * xf[..., 0].imag
    yf[..., -1] = 2 * xf[..., -1].imag
    y = irfft_half(yf, threads=threads)
    out = numpy.empty(xf.shape[:-1] + (size // 2,), numpy.float64)
    out[..., 1:] = y[..., 1:] / 4 / numpy.sin(2 * numpy.pi * numpy.arange(1, size // 2) / size)
    out[..., 0] = xf.real.sum(axis=-1) / (size / 2)
    return out


def numpy_ref(x: numpy.ndarray, axes=None, inverse: bool = False) -> numpy.ndarray:
    """FP64 reference: numpy.fft.fftn / ifftn in complex128."""
    x = numpy.asarray(x, numpy.complex128)
    axes = tuple(range(x.ndim)) if axes is None else tuple(axes)
    return numpy.fft.ifftn(x, axes=axes) if inverse else numpy.fft.fftn(x, axes=axes)


def rel_l2(a: numpy.ndarray, b: numpy.ndarray) -> float:
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    den = numpy.linalg.norm(b.ravel())
    return float(numpy.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
