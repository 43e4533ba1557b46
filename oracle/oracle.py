"""Python access to the CPU oracle (test infrastructure only).

``liboracle.so`` is the C restatement of reikna's FFT algorithm (see
``reikna_fft_oracle.c``).  This module builds it on demand with ``make`` and exposes:

* ``fft(x, axes, inverse)`` -- reikna-semantics FFT on the CPU (complex64 in FP32,
  complex128 in FP64 arithmetic), OpenMP over lines;
* ``radix_array``, ``global_radix_info``, ``kweights``, ``kernel_chain`` -- the
  planner restatement, pinned against golden fixtures of reikna's own planner;
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
