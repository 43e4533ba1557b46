"""ctypes binding of the C ABI declared in ``include/reikna_b200.h``.

The shared library is built in-tree by :mod:`reikna_b200.build`.  There is no CPU
fallback: if the library cannot be loaded, every entry point raises.
"""

from __future__ import annotations

import ctypes
import json
import os
import threading
from pathlib import Path

MAXD = 8

OK = 0
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_NOMEM = -4
ERR_DEVICE = -5

FMT_C64 = 1
FMT_C128 = 2
FMT_F32 = 3
FMT_F64 = 4
FMT_F32_PAIR = 5
FMT_F64_PAIR = 6
FMT_I32 = 7
FMT_CONST = 9
FMT_IGNORE = 10
FMT_USER = 11

POST_NONE = 0
POST_NORM = 1

WIN_NONE = 0
WIN_HANN = 1

FLAG_NO_PLANE = 1
FLAG_NO_BLUE1 = 2
FLAG_SPLIT_TC = 4
FLAG_PLANE_WIDE = 8
FLAG_NO_TMA = 16
FLAG_PAIR = 32
FLAG_REAL_POST = 64
FLAG_REAL_PRE = 128
FLAG_ANTIPERIODIC = 256
FLAG_NO_HALF = 512
FLAG_R16 = 1024
FLAG_BATCHABLE = 2048
FLAG_BLUE_PAIR = 4096  # fused 8192-point Bluestein lines on a two-CTA cluster a line (tuning)

EXPORTED = (
    "rk_edge_init",
    "rk_fft_plan_create",
    "rk_fft_execute",
    "rk_fft_execute_user",
    "rk_fft_plan_pass_info",
    "rk_fft_plan_set_pass_kernel",
    "rk_fft_plan_destroy",
    "rk_fft_plan_device_bytes",
    "rk_fft_plan_describe",
    "rk_fft_plan_launches",
    "rk_fftshift_execute",
    "rk_last_error",
    "rk_version",
    "rk_abi_sizes",
    "rk_fft_profile",
    "rk_fft_profile_read",
    "rk_device_status",
    "rk_set_wait_limit",
    "rk_get_wait_limit",
    "rk_stream_check",
    "rk_selftest_stalled_wait",
    "rk_fft1d_c64_noalloc",
    "rk_batch_create",
    "rk_batch_execute",
    "rk_batch_destroy",
    "rk_batch_info",
    "rk_fft_plan_tc_passes",
    "rk_transpose_execute",
    "rk_rfft_twiddles",
    "rk_rfft_post",
    "rk_irfft_pre",
    "rk_aprfft_twiddles",
    "rk_aprfft_twiddle",
    "rk_aprfft_post",
    "rk_iaprfft_pre",
)

I64A = ctypes.c_int64 * MAXD
I32A = ctypes.c_int32 * MAXD


class Edge(ctypes.Structure):
    _fields_ = [
        ("format", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("shape", I64A),
        ("strides", I64A),
        ("offset", ctypes.c_int64),
        ("strides2", I64A),
        ("offset2", ctypes.c_int64),
        ("shift", I32A),
        ("scale_re", ctypes.c_double),
        ("scale_im", ctypes.c_double),
        ("scale_slot", ctypes.c_int32),
        ("scale_div_slot", ctypes.c_int32),
        ("post", ctypes.c_int32),
        ("post_param", ctypes.c_double),
        ("window", ctypes.c_int32),
        ("window_axis", ctypes.c_int32),
        ("window_len", ctypes.c_int64),
        ("conj", ctypes.c_int32),
        ("add_slot", ctypes.c_int32),
        ("add_re", ctypes.c_double),
        ("add_im", ctypes.c_double),
        ("post_slot", ctypes.c_int32),
    ]


class FftDesc(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("shape", I64A),
        ("naxes", ctypes.c_int32),
        ("axes", I32A),
        ("flags", ctypes.c_int32),
        ("input", Edge),
        ("output", Edge),
    ]


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (status {code})")
        self.code = code


_lib = None
_lock = threading.Lock()


def library_path() -> Path:
    env = os.environ.get("REIKNA_B200_LIB")
    if env:
        return Path(env)
    return Path(__file__).resolve().parent / "_lib" / "libreikna_b200.so"


def lib() -> ctypes.CDLL:
    """Load the shared library (once); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not path.exists():
            raise ImportError(
                f"reikna_b200 native library not found at {path}; "
                "build it with `python -m reikna_b200.build` (there is no CPU fallback)"
            )
        L = ctypes.CDLL(str(path))
        vp = ctypes.c_void_p
        L.rk_edge_init.argtypes = [ctypes.POINTER(Edge), ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
        L.rk_fft_plan_create.argtypes = [ctypes.POINTER(FftDesc), ctypes.POINTER(vp)]
        L.rk_fft_execute.argtypes = [
            vp,
            ctypes.POINTER(vp),
            ctypes.c_int32,
            ctypes.POINTER(vp),
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.POINTER(ctypes.c_double),
            ctypes.c_int32,
            vp,
        ]
        L.rk_fft_plan_destroy.argtypes = [vp]
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.rk_fft_execute_user.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int32, ctypes.POINTER(vp), ctypes.c_int32,
                                          ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.c_int32, u64p,
                                          ctypes.c_int32, u64p, ctypes.c_int32, vp]
        L.rk_fft_plan_pass_info.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int64)]
        L.rk_fft_plan_set_pass_kernel.argtypes = [vp, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int64, ctypes.c_char_p]
        L.rk_fft_plan_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.rk_fft_plan_describe.argtypes = [
            ctypes.POINTER(FftDesc),
            ctypes.c_char_p,
            ctypes.c_int64,
            ctypes.POINTER(ctypes.c_int64),
        ]
        L.rk_fft_plan_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.rk_fft_plan_tc_passes.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.rk_transpose_execute.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, vp]
        L.rk_rfft_twiddles.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, vp]
        L.rk_rfft_post.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, vp]
        L.rk_irfft_pre.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, vp]
        L.rk_aprfft_twiddles.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, vp]
        L.rk_aprfft_twiddle.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, vp]
        L.rk_aprfft_post.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, vp]
        L.rk_iaprfft_pre.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, vp]
        L.rk_fftshift_execute.argtypes = [
            vp,
            vp,
            ctypes.c_int32,
            ctypes.c_int32,
            ctypes.POINTER(ctypes.c_int64),
            ctypes.c_int32,
            ctypes.POINTER(ctypes.c_int32),
            ctypes.c_int32,
            vp,
            vp,
        ]
        L.rk_abi_sizes.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        L.rk_fft_profile.argtypes = [vp, ctypes.c_int32]
        L.rk_device_status.argtypes = [ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
        L.rk_set_wait_limit.argtypes = [ctypes.c_int64]
        L.rk_get_wait_limit.argtypes = [ctypes.POINTER(ctypes.c_int64)]
        L.rk_stream_check.argtypes = [vp]
        L.rk_selftest_stalled_wait.argtypes = [vp]
        L.rk_fft1d_c64_noalloc.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, vp]
        L.rk_fft_profile_read.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
        i32p, i64p = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)
        L.rk_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ctypes.POINTER(vp)]
        L.rk_batch_execute.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), i32p, ctypes.POINTER(vp), i32p, vp]
        L.rk_batch_destroy.argtypes = [vp]
        L.rk_batch_info.argtypes = [vp, i64p, i32p, i32p]
        L.rk_last_error.restype = ctypes.c_char_p
        L.rk_version.restype = ctypes.c_char_p
        for name in EXPORTED:
            if name not in ("rk_last_error", "rk_version"):
                getattr(L, name).restype = ctypes.c_int
        eb, db = ctypes.c_int64(0), ctypes.c_int64(0)
        L.rk_abi_sizes(ctypes.byref(eb), ctypes.byref(db))
        if eb.value != ctypes.sizeof(Edge) or db.value != ctypes.sizeof(FftDesc):
            raise ImportError(
                f"ABI mismatch: C sizes edge={eb.value} desc={db.value}, "
                f"ctypes sizes edge={ctypes.sizeof(Edge)} desc={ctypes.sizeof(FftDesc)}"
            )
        _lib = L
        return L


def check(code: int) -> None:
    if code != OK:
        msg = lib().rk_last_error().decode(errors="replace")
        if code == ERR_INVALID:
            raise ValueError(msg)
        if code == ERR_UNSUPPORTED:
            raise NotImplementedError(msg)
        raise NativeError(code, msg)


def edge(fmt: int, shape: tuple[int, ...]) -> Edge:
    e = Edge()
    arr = (ctypes.c_int64 * len(shape))(*shape)
    check(lib().rk_edge_init(ctypes.byref(e), fmt, len(shape), arr))
    return e


def desc(dtype_fmt: int, shape: tuple[int, ...], axes: tuple[int, ...], flags: int = 0) -> FftDesc:
    d = FftDesc()
    d.dtype = dtype_fmt
    d.ndim = len(shape)
    for i, s in enumerate(shape):
        d.shape[i] = s
    d.naxes = len(axes)
    for i, a in enumerate(axes):
        d.axes[i] = a
    d.flags = flags
    d.input = edge(dtype_fmt, shape)
    d.output = edge(dtype_fmt, shape)
    return d


def describe(d: FftDesc) -> dict:
    """Planner output (kernel chain) as a dict; needs no GPU."""
    need = ctypes.c_int64(0)
    check(lib().rk_fft_plan_describe(ctypes.byref(d), None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(int(need.value))
    check(lib().rk_fft_plan_describe(ctypes.byref(d), buf, need.value, ctypes.byref(need)))
    return json.loads(buf.value.decode())


class Plan:
    """Owns an ``rk_fft_plan``; executes it on device pointers."""

    def __init__(self, d: FftDesc):
        self.desc = d
        h = ctypes.c_void_p()
        check(lib().rk_fft_plan_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        n = ctypes.c_int32(0)
        check(lib().rk_fft_plan_launches(h, ctypes.byref(n)))
        self.launches = int(n.value)

    @property
    def tc_passes(self) -> int:
        """Passes running on the tensor cores (split-precision mode)."""
        n = ctypes.c_int32(0)
        check(lib().rk_fft_plan_tc_passes(self._h, ctypes.byref(n)))
        return int(n.value)

    @property
    def device_bytes(self) -> int:
        b = ctypes.c_int64(0)
        check(lib().rk_fft_plan_device_bytes(self._h, ctypes.byref(b)))
        return int(b.value)

    def execute(self, outs, ins, inverse: int = 0, scalars=(), stream: int = 0) -> None:
        # the pointer arrays are kept per plan and refilled (the call path's host cost)
        arrs = self.__dict__.get("_arrs")
        if arrs is None or len(arrs[0]) != len(outs) or len(arrs[1]) != len(ins):
            arrs = self._arrs = ((ctypes.c_void_p * max(1, len(outs)))(), (ctypes.c_void_p * max(1, len(ins)))())
        outs_a, ins_a = arrs
        for i, v in enumerate(outs):
            outs_a[i] = v
        for i, v in enumerate(ins):
            ins_a[i] = v
        sc = None
        if scalars:
            flat = []
            for s in scalars:
                c = complex(s)
                flat += [c.real, c.imag]
            sc = (ctypes.c_double * len(flat))(*flat)
        rc = lib().rk_fft_execute(self._h, outs_a, len(outs), ins_a, len(ins), int(inverse), sc, len(scalars),
                                  stream)
        if rc:
            check(rc)

    def execute_user(self, outs, ins, inverse: int = 0, scalars=(), user_in=(), user_out=(), stream: int = 0) -> None:
        """``execute`` with the words handed to run-time compiled edge code."""
        outs_a = (ctypes.c_void_p * max(1, len(outs)))(*outs)
        ins_a = (ctypes.c_void_p * max(1, len(ins)))(*ins)
        flat = []
        for s in scalars:
            c = complex(s)
            flat += [c.real, c.imag]
        sc = (ctypes.c_double * max(1, len(flat)))(*flat) if flat else None
        ui = (ctypes.c_uint64 * max(1, len(user_in)))(*user_in)
        uo = (ctypes.c_uint64 * max(1, len(user_out)))(*user_out)
        check(lib().rk_fft_execute_user(self._h, outs_a, len(outs), ins_a, len(ins), int(inverse), sc, len(scalars),
                                        ui, len(user_in), uo, len(user_out), ctypes.c_void_p(stream)))

    def pass_info(self) -> list[dict]:
        """Launch shape of every pass (kind, L, mode, variant, complex128, threads, user
        bits, lines per CTA, shared memory bytes)."""
        out = []
        for i in range(self.launches_total):
            info = (ctypes.c_int32 * 8)()
            smem = ctypes.c_int64(0)
            check(lib().rk_fft_plan_pass_info(self._h, i, info, ctypes.byref(smem)))
            keys = ("kind", "L", "mode", "var", "dbl", "nt", "user", "nl")
            out.append(dict(zip(keys, list(info)), smem=int(smem.value)))
        return out

    @property
    def launches_total(self) -> int:
        return len(self.describe()["passes"])

    def set_pass_kernel(self, index: int, cubin: bytes, name: str) -> None:
        check(lib().rk_fft_plan_set_pass_kernel(self._h, int(index), cubin, len(cubin), name.encode()))

    def profile(self, max_calls: int) -> None:
        """Record per-pass CUDA events for the next ``max_calls`` executions."""
        check(lib().rk_fft_profile(self._h, int(max_calls)))

    def profile_read(self) -> tuple[list[float], int]:
        """(summed ms per pass, number of recorded executions); synchronises."""
        ms = (ctypes.c_double * max(1, self.launches))()
        calls = ctypes.c_int32(0)
        check(lib().rk_fft_profile_read(self._h, ms, self.launches, ctypes.byref(calls)))
        return list(ms[: self.launches]), int(calls.value)

    def describe(self) -> dict:
        return describe(self.desc)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().rk_fft_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def device_status(clear: bool = False) -> int:
    """Device status word of the current device (nonzero: a kernel gave up a bounded
    wait or met a task it has no code for); synchronises the device."""
    v = ctypes.c_int32(0)
    check(lib().rk_device_status(ctypes.byref(v), int(bool(clear))))
    return int(v.value)


STATUS_TIMEOUT = 1
STATUS_BAD_VARIANT = 2


def set_wait_limit(cycles: int) -> None:
    """Limit, in SM clock cycles, of the kernels' bounded waits on the current device."""
    check(lib().rk_set_wait_limit(int(cycles)))


def wait_limit() -> int:
    v = ctypes.c_int64(0)
    check(lib().rk_get_wait_limit(ctypes.byref(v)))
    return int(v.value)


def stream_check(stream: int = 0) -> None:
    """Synchronise ``stream``; raise :class:`NativeError` (``ERR_DEVICE``) if the device
    status word is set (a bounded wait ran out)."""
    check(lib().rk_stream_check(ctypes.c_void_p(stream)))


class Batch:
    """Owns an ``rk_batch``: several plans run by one persistent kernel launch."""

    def __init__(self, plans):
        self.plans = list(plans)  # the batch points into the plans: keep them alive
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = ctypes.c_void_p()
        check(lib().rk_batch_create(arr, len(self.plans), ctypes.byref(h)))
        self._h = h

    def info(self) -> dict:
        nt, npass, grid = ctypes.c_int64(0), ctypes.c_int32(0), ctypes.c_int32(0)
        check(lib().rk_batch_info(self._h, ctypes.byref(nt), ctypes.byref(npass), ctypes.byref(grid)))
        return {"tasks": int(nt.value), "passes": int(npass.value), "grid": int(grid.value)}

    def execute(self, calls, stream: int = 0) -> None:
        """``calls[i] = (outs, ins, inverse, scalars)`` for member i."""
        n = len(self.plans)
        if len(calls) != n:
            raise ValueError(f"batch has {n} members, got {len(calls)} calls")
        keep = []
        outs_a = (ctypes.c_void_p * n)()
        ins_a = (ctypes.c_void_p * n)()
        inv_a = (ctypes.c_int32 * n)()
        sc_a = (ctypes.c_void_p * n)()
        nsc_a = (ctypes.c_int32 * n)()
        for i, (outs, ins, inverse, scalars) in enumerate(calls):
            o = (ctypes.c_void_p * len(outs))(*outs)
            s = (ctypes.c_void_p * len(ins))(*ins)
            flat = []
            for v in scalars:
                c = complex(v)
                flat += [c.real, c.imag]
            d = (ctypes.c_double * max(1, len(flat)))(*flat)
            keep += [o, s, d]
            outs_a[i] = ctypes.cast(o, ctypes.c_void_p)
            ins_a[i] = ctypes.cast(s, ctypes.c_void_p)
            inv_a[i] = int(inverse)
            sc_a[i] = ctypes.cast(d, ctypes.c_void_p)
            nsc_a[i] = len(scalars)
        check(lib().rk_batch_execute(self._h, outs_a, ins_a, inv_a, sc_a, nsc_a, ctypes.c_void_p(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().rk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def fftshift_execute(out_ptr, in_ptr, elem_bytes, shape, axes, inverse, scratch_ptr, stream) -> None:
    sh = (ctypes.c_int64 * len(shape))(*shape)
    ax = (ctypes.c_int32 * max(1, len(axes)))(*axes)
    check(
        lib().rk_fftshift_execute(
            ctypes.c_void_p(out_ptr),
            ctypes.c_void_p(in_ptr),
            elem_bytes,
            len(shape),
            sh,
            len(axes),
            ax,
            int(inverse),
            ctypes.c_void_p(scratch_ptr or 0),
            ctypes.c_void_p(stream),
        )
    )
