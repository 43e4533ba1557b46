"""Run-time compilation of pass kernels with NVRTC (for transformations given as code).

reikna compiles every kernel from source when a computation is compiled
(reikna/core/computation.py:521-579, through grunnur); this library ships its kernels
prebuilt and compiles at run time only the passes that must call a transformation
written as source code.  The NVRTC library is loaded through ctypes from the CUDA
installation or from the ``nvidia-cuda-nvrtc`` wheel next to PyTorch; compiled cubins
are cached on disk (``RK_RTC_CACHE``, default ``~/.cache/reikna_b200/rtc``) keyed by a
hash of the source and options.
"""

from __future__ import annotations

import ctypes
import glob
import hashlib
import os
from pathlib import Path

from . import build as _build

_nvrtc = None

ARCH = "sm_100a"


class CompileError(RuntimeError):
    pass


def _candidates():
    env = os.environ.get("RK_NVRTC")
    if env:
        yield env
    try:
        import nvidia.cuda_nvrtc as m

        for base in list(getattr(m, "__path__", [])):
            yield from sorted(glob.glob(os.path.join(base, "lib", "libnvrtc.so*")), reverse=True)
    except ImportError:
        pass
    for base in ("/usr/local/cuda/lib64", "/usr/local/cuda/lib", "/usr/lib/x86_64-linux-gnu"):
        yield from sorted(glob.glob(os.path.join(base, "libnvrtc.so*")), reverse=True)
    yield "libnvrtc.so.12"
    yield "libnvrtc.so"


def nvrtc():
    """The loaded NVRTC library (ctypes)."""
    global _nvrtc
    if _nvrtc is not None:
        return _nvrtc
    last = None
    for path in _candidates():
        if "builtins" in os.path.basename(path):
            continue
        try:
            lib = ctypes.CDLL(path)
            lib.nvrtcCreateProgram.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_char_p,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            lib.nvrtcCompileProgram.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
            lib.nvrtcGetProgramLogSize.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]
            lib.nvrtcGetProgramLog.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
            lib.nvrtcGetCUBINSize.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]
            lib.nvrtcGetCUBIN.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
            lib.nvrtcDestroyProgram.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
            lib.nvrtcGetErrorString.restype = ctypes.c_char_p
            _nvrtc = lib
            return lib
        except OSError as e:
            last = e
    raise CompileError(f"NVRTC is not available: {last}")


# NVRTC has no C library headers: the few fixed-width types the kernel headers use
PRELUDE = """
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef unsigned long long uintptr_t;
"""


def _cache_dir() -> Path:
    p = os.environ.get("RK_RTC_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "reikna_b200" / "rtc"


def compile_cubin(source: str, name: str = "kernel.cu", options=(), keep: bool = False) -> bytes:
    """Compile ``source`` for sm_100a; returns the cubin.  ``keep`` writes the source
    next to the cached cubin (reikna's ``keep``)."""
    opts = [f"-arch={ARCH}", "-std=c++17", "-default-device",
            f"-I{_build.CSRC}", f"-I{_build.INCLUDE}", *options]
    key = hashlib.sha256((PRELUDE + source + "\0" + "\0".join(opts)).encode()).hexdigest()[:32]
    cache = _cache_dir()
    path = cache / f"{key}.cubin"
    if path.exists():
        return path.read_bytes()
    lib = nvrtc()
    prog = ctypes.c_void_p()
    src = (PRELUDE + source).encode()
    rc = lib.nvrtcCreateProgram(ctypes.byref(prog), src, name.encode(), 0, None, None)
    if rc:
        raise CompileError(f"nvrtcCreateProgram: {lib.nvrtcGetErrorString(rc).decode()}")
    try:
        arr = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        n = ctypes.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
        log = ctypes.create_string_buffer(n.value)
        lib.nvrtcGetProgramLog(prog, log)
        if rc:
            raise CompileError(f"run-time compilation failed ({lib.nvrtcGetErrorString(rc).decode()}):\n"
                               f"{log.value.decode(errors='replace')}")
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        lib.nvrtcGetCUBIN(prog, buf)
        cubin = buf.raw
    finally:
        lib.nvrtcDestroyProgram(ctypes.byref(prog))
    try:
        cache.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_bytes(cubin)
        tmp.replace(path)
        if keep:
            path.with_suffix(".cu").write_text(source)
    except OSError:
        pass
    return cubin
