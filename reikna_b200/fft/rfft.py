"""Half-length real transforms of reikna's specialised-FFT example
(examples/demo_specialized_fft.py:175-624) as computations: ``RFFT`` / ``IRFFT`` and
the antiperiodic ``APRFFT`` / ``IAPRFFT``.

``RFFT(arr_t, dont_store_last=False)``: real (..., N) -> complex (..., N/2 + 1) (or
N/2 without the last bin), like ``numpy.fft.rfft`` along the last axis.
``IRFFT(arr_t)``: complex (..., H + 1) -> real (..., 2H), like ``numpy.fft.irfft``.
``APRFFT(arr_t)``: real (..., N/2), the first half of a signal with
x[n + N/2] = -x[n] -> its N/4 odd harmonics.  ``IAPRFFT(arr_t)``: the inverse.
Signatures ``(output:o, input:i)``.

As in the reference, the real array is read by a complex FFT of half its length as
interleaved (re, im) pairs.  When that half length is a power of two (8 to 8192
points for float32, 4096 for float64) each transform is one pass: the step between
the real signal's spectrum and the pairs' spectrum runs inside the FFT's last store
(forward: the planner's half-length route for RFFT, which reads any view of the real
array; ``RK_FLAG_REAL_POST`` for APRFFT) or first load (inverse,
``RK_FLAG_REAL_PRE``), with the antiperiodic twiddles on the other side
(``RK_FLAG_ANTIPERIODIC``): one read of the input and one write of the output.  Other lengths run the FFT plan between
element-wise kernels (``csrc/rk_rfft.cu``).
"""

from __future__ import annotations

import numpy

from .. import _native as N
from ..core.computation import Computation, array_pointer
from ..core.signature import Annotation, ArrayMetadata, Parameter, Type
from .fft import FFT


def _meta(arr_t):
    return Type(arr_t).as_array_metadata() if not isinstance(arr_t, ArrayMetadata) else arr_t


def _contiguous(meta) -> bool:
    return tuple(meta.strides) == tuple(ArrayMetadata(tuple(meta.shape), meta.dtype).strides)


def _complex_for(dt):
    return numpy.dtype(numpy.complex64 if numpy.dtype(dt) == numpy.float32 else numpy.complex128)


def _real_for(dt):
    return numpy.dtype(numpy.float32 if numpy.dtype(dt) == numpy.complex64 else numpy.float64)


def _torch_dtype(dt):
    import torch

    return torch.complex64 if numpy.dtype(dt) == numpy.complex64 else torch.complex128


class _Half:
    """The half-length complex FFT, its table and the intermediate buffer (the
    multi-kernel route, for half lengths no one-pass plan covers)."""

    def __init__(self, device, batch_shape, half, cdtype, antiperiodic: bool = False):
        import torch

        self.fmt = N.FMT_C64 if cdtype == numpy.complex64 else N.FMT_C128
        self.esz = numpy.dtype(cdtype).itemsize
        self.half = half
        self.batch = int(numpy.prod(batch_shape)) if batch_shape else 1
        shape = tuple(batch_shape) + (half,)
        comp = FFT(ArrayMetadata(shape, cdtype), axes=(len(shape) - 1,))
        self.cc = comp.compile(device)
        self.plan = self.cc._runner.plan
        with torch.cuda.device(device):
            entries = 2 * half if antiperiodic else half + 1
            self.table = torch.empty(entries, dtype=_torch_dtype(cdtype), device=device)
            self.temp = torch.empty(shape, dtype=_torch_dtype(cdtype), device=device)
            stream = torch.cuda.current_stream(device).cuda_stream
            make = N.lib().rk_aprfft_twiddles if antiperiodic else N.lib().rk_rfft_twiddles
            N.check(make(self.table.data_ptr(), self.fmt, half, stream))
            torch.cuda.current_stream(device).synchronize()

    def aligned(self, ptr: int) -> int:
        if ptr % self.esz:
            raise ValueError("the real array must start on a boundary of its complex pair type")
        return ptr


def _fused_plan(device, batch_shape, half, cdt, flags: int, in_len: int, out_len: int):
    """One-pass plan (RK_FLAG_REAL_POST / RK_FLAG_REAL_PRE) of the half-length FFT over
    the last axis with input and output edges of ``in_len`` / ``out_len`` complex
    elements a row, or None when the half length has no such plan."""
    import torch

    fmt = N.FMT_C64 if numpy.dtype(cdt) == numpy.complex64 else N.FMT_C128
    shape = tuple(batch_shape) + (half,)
    d = N.desc(fmt, shape, (len(shape) - 1,), flags)
    d.input = N.edge(fmt, tuple(batch_shape) + (in_len,))
    d.output = N.edge(fmt, tuple(batch_shape) + (out_len,))
    try:
        with torch.cuda.device(device):
            return N.Plan(d)
    except NotImplementedError:
        return None


def _half_route_plan(device, meta, bins: int):
    """The planner's half-length route for a real (..., N) input and (..., bins)
    complex output: the real array is read as sample pairs with scalar loads where a
    line is not aligned to the pair type, so any view works.  None when N / 2 is not
    a length that route covers in one pass."""
    import torch

    cdt = _complex_for(meta.dtype)
    fmt = N.FMT_C64 if cdt == numpy.complex64 else N.FMT_C128
    rfmt = N.FMT_F32 if cdt == numpy.complex64 else N.FMT_F64
    shape = tuple(meta.shape)
    d = N.desc(fmt, shape, (len(shape) - 1,))
    d.input = N.edge(rfmt, shape)
    d.output = N.edge(fmt, shape[:-1] + (bins,))
    try:
        if N.describe(d)["passes"][0]["note"] != "half":
            return None
        with torch.cuda.device(device):
            return N.Plan(d)
    except NotImplementedError:
        return None


def _edges(comp, name):
    leaves = [p.name for p in comp._tr_tree.get_leaf_parameters()]
    if leaves != ["output", "input"]:
        raise NotImplementedError(f"transformations connected to {name} are not fused")
    ann = {p.name: p.annotation for p in comp._tr_tree.get_leaf_parameters()}
    if not (_contiguous(ann["input"].as_array_metadata()) and _contiguous(ann["output"].as_array_metadata())):
        raise NotImplementedError(f"{name} works on C-contiguous arrays")
    return ann


def _fused_runner(fused, ann, esz: int, inverse: int, real_side: str):
    def run(stream: int, args):
        out = array_pointer(args["output"], ann["output"])
        inp = array_pointer(args["input"], ann["input"])
        if (inp if real_side == "input" else out) % esz:
            raise ValueError("the real array must start on a boundary of its complex pair type")
        fused.execute([out], [inp], inverse=inverse, stream=stream)

    run.launches = fused.launches
    run.plan = fused
    return run


class RFFT(Computation):
    """Spectrum of real signals along the last axis through a half-length complex FFT."""

    def __init__(self, arr_t, *, dont_store_last: bool = False):
        meta = _meta(arr_t)
        if meta.dtype not in (numpy.dtype(numpy.float32), numpy.dtype(numpy.float64)):
            raise ValueError("RFFT expects a real float32 or float64 array")
        n = meta.shape[-1]
        if n % 2:
            raise ValueError("RFFT expects an even length along the last axis")
        self._dont_store_last = dont_store_last
        out = ArrayMetadata(tuple(meta.shape[:-1]) + (n // 2 + (0 if dont_store_last else 1),), _complex_for(meta.dtype))
        self._meta = meta
        Computation.__init__(self, [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))])

    def _build_runner(self, device, **_ignored):
        ann = _edges(self, "RFFT")
        meta = self._meta
        store_last = 0 if self._dont_store_last else 1
        half, cdt = meta.shape[-1] // 2, _complex_for(meta.dtype)
        route = _half_route_plan(device, meta, half + store_last)
        if route is not None:
            def run(stream: int, args):
                out = array_pointer(args["output"], ann["output"])
                inp = array_pointer(args["input"], ann["input"])
                route.execute([out], [inp], inverse=0, stream=stream)

            run.launches = route.launches
            run.plan = route
            return run
        h = _Half(device, meta.shape[:-1], half, cdt)

        def runner(stream: int, args):
            out = array_pointer(args["output"], ann["output"])
            inp = h.aligned(array_pointer(args["input"], ann["input"]))
            h.plan.execute([h.temp.data_ptr()], [inp], inverse=0, stream=stream)
            N.check(N.lib().rk_rfft_post(out, h.temp.data_ptr(), h.table.data_ptr(), h.fmt, h.half, h.batch,
                                         store_last, stream))

        runner.launches = h.plan.launches + 1
        runner.half = h
        return runner


class IRFFT(Computation):
    """Real signals from their half spectra along the last axis (numpy.fft.irfft)."""

    def __init__(self, arr_t):
        meta = _meta(arr_t)
        if meta.dtype not in (numpy.dtype(numpy.complex64), numpy.dtype(numpy.complex128)):
            raise ValueError("IRFFT expects a complex64 or complex128 array")
        if meta.shape[-1] < 2:
            raise ValueError("IRFFT expects at least two bins along the last axis")
        out = ArrayMetadata(tuple(meta.shape[:-1]) + ((meta.shape[-1] - 1) * 2,), _real_for(meta.dtype))
        self._meta = meta
        Computation.__init__(self, [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))])

    def _build_runner(self, device, **_ignored):
        ann = _edges(self, "IRFFT")
        meta = self._meta
        half = meta.shape[-1] - 1
        fused = _fused_plan(device, meta.shape[:-1], half, meta.dtype, N.FLAG_REAL_PRE, half + 1, half)
        if fused is not None:
            return _fused_runner(fused, ann, meta.dtype.itemsize, 1, "output")
        h = _Half(device, meta.shape[:-1], half, meta.dtype)

        def runner(stream: int, args):
            out = h.aligned(array_pointer(args["output"], ann["output"]))
            inp = array_pointer(args["input"], ann["input"])
            N.check(N.lib().rk_irfft_pre(h.temp.data_ptr(), inp, h.table.data_ptr(), h.fmt, h.half, h.batch, stream))
            h.plan.execute([out], [h.temp.data_ptr()], inverse=1, stream=stream)

        runner.launches = h.plan.launches + 1
        runner.half = h
        return runner


class APRFFT(Computation):
    """Odd harmonics of real antiperiodic signals (x[n + N/2] = -x[n]) from their first
    halves: real (..., N/2) -> complex (..., N/4), ``numpy.fft.rfft(full)[1::2]``
    (examples/demo_specialized_fft.py:379-453).

    With L = N/4 a power of two (8 to 8192 for float32, 4096 for float64) this is one
    pass: the pairs (x[2m], x[2m+1]) times W_N/2^m on the first load, FFT_L, and
    F[k] = C[k] (1 - i w_k) + conj(C[L - 1 - k]) (1 + i w_k), w_k = exp(-i pi
    (2k + 1) / 2L), on the last store.  The reference gets F from an RFFT of the
    sine-weighted signal, a cumulative sum over the bins and a cosine-weighted
    reduction; both are the same linear map of x."""

    def __init__(self, arr_t):
        meta = _meta(arr_t)
        if meta.dtype not in (numpy.dtype(numpy.float32), numpy.dtype(numpy.float64)):
            raise ValueError("APRFFT expects a real float32 or float64 array")
        n = meta.shape[-1]
        if n % 2 or n < 2:
            raise ValueError("APRFFT expects an even length along the last axis")
        out = ArrayMetadata(tuple(meta.shape[:-1]) + (n // 2,), _complex_for(meta.dtype))
        self._meta = meta
        Computation.__init__(self, [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))])

    def _build_runner(self, device, **_ignored):
        ann = _edges(self, "APRFFT")
        meta = self._meta
        half, cdt = meta.shape[-1] // 2, _complex_for(meta.dtype)
        flags = N.FLAG_REAL_POST | N.FLAG_ANTIPERIODIC
        fused = _fused_plan(device, meta.shape[:-1], half, cdt, flags, half, half)
        if fused is not None:
            return _fused_runner(fused, ann, cdt.itemsize, 0, "input")
        h = _Half(device, meta.shape[:-1], half, cdt, antiperiodic=True)
        lib = N.lib()

        def runner(stream: int, args):
            out = array_pointer(args["output"], ann["output"])
            inp = h.aligned(array_pointer(args["input"], ann["input"]))
            t = h.temp.data_ptr()
            N.check(lib.rk_aprfft_twiddle(t, inp, h.table.data_ptr(), h.fmt, h.half, h.batch, 0, stream))
            h.plan.execute([t], [t], inverse=0, stream=stream)
            N.check(lib.rk_aprfft_post(out, t, h.table.data_ptr(), h.fmt, h.half, h.batch, stream))

        runner.launches = h.plan.launches + 2
        runner.half = h
        return runner


class IAPRFFT(Computation):
    """First halves of real antiperiodic signals from their odd harmonics: complex
    (..., N/4) -> real (..., N/2), ``numpy.fft.irfft(spectrum)[:N/2]`` with the even
    harmonics zero (examples/demo_specialized_fft.py:456-581).  The inverse of
    ``APRFFT``: C[k] = (F[k] conj(1 - i w_k) + conj(F[L - 1 - k]) conj(1 + i w_k)) / 4
    on the first load, the inverse FFT_L, and the pairs c[m] W_N/2^-m on the last store
    (one pass under the same length limits as ``APRFFT``)."""

    def __init__(self, arr_t):
        meta = _meta(arr_t)
        if meta.dtype not in (numpy.dtype(numpy.complex64), numpy.dtype(numpy.complex128)):
            raise ValueError("IAPRFFT expects a complex64 or complex128 array")
        out = ArrayMetadata(tuple(meta.shape[:-1]) + (meta.shape[-1] * 2,), _real_for(meta.dtype))
        self._meta = meta
        Computation.__init__(self, [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))])

    def _build_runner(self, device, **_ignored):
        ann = _edges(self, "IAPRFFT")
        meta = self._meta
        half = meta.shape[-1]
        flags = N.FLAG_REAL_PRE | N.FLAG_ANTIPERIODIC
        fused = _fused_plan(device, meta.shape[:-1], half, meta.dtype, flags, half, half)
        if fused is not None:
            return _fused_runner(fused, ann, meta.dtype.itemsize, 1, "output")
        h = _Half(device, meta.shape[:-1], half, meta.dtype, antiperiodic=True)
        lib = N.lib()

        def runner(stream: int, args):
            out = h.aligned(array_pointer(args["output"], ann["output"]))
            inp = array_pointer(args["input"], ann["input"])
            t = h.temp.data_ptr()
            N.check(lib.rk_iaprfft_pre(t, inp, h.table.data_ptr(), h.fmt, h.half, h.batch, stream))
            h.plan.execute([out], [t], inverse=1, stream=stream)
            N.check(lib.rk_aprfft_twiddle(out, out, h.table.data_ptr(), h.fmt, h.half, h.batch, 1, stream))

        runner.launches = h.plan.launches + 2
        runner.half = h
        return runner
