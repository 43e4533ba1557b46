"""Half-length real transforms: ``RFFT`` and ``IRFFT`` of reikna's specialised-FFT
example (examples/demo_specialized_fft.py:175-331), as computations.

When N/2 is a power of two the half-length FFT is a single pass (up to 8192 points
for float32 input, 4096 for float64) and the spectrum step runs inside its store
(``RK_FLAG_REAL_POST``): one read of the signal and one write of the spectrum.

``RFFT(arr_t, dont_store_last=False)``: real (..., N) -> complex (..., N/2 + 1)
(or N/2 without the last bin), signature ``(output:o, input:i)``, like
``numpy.fft.rfft`` along the last axis.  ``IRFFT(arr_t)``: complex (..., H + 1) ->
real (..., 2H), like ``numpy.fft.irfft``.  As in the reference, the real array is
read by a complex FFT of half the length as interleaved (re, im) pairs, and one
element-wise kernel forms the spectrum of the real signal from it (RFFT) or
prepares the half-length spectrum for the inverse (IRFFT); see
``csrc/rk_rfft.cu``.
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
    """The half-length complex FFT, its W^k table and the intermediate buffer."""

    def __init__(self, device, batch_shape, half, cdtype):
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
            self.table = torch.empty(half + 1, dtype=_torch_dtype(cdtype), device=device)
            self.temp = torch.empty(shape, dtype=_torch_dtype(cdtype), device=device)
            stream = torch.cuda.current_stream(device).cuda_stream
            N.check(N.lib().rk_rfft_twiddles(self.table.data_ptr(), self.fmt, half, stream))
            torch.cuda.current_stream(device).synchronize()

    def aligned(self, ptr: int) -> int:
        if ptr % self.esz:
            raise ValueError("the real array must start on a boundary of its complex pair type")
        return ptr


def _fused_plan(device, meta, store_last: int):
    """One-pass plan (RK_FLAG_REAL_POST) when the half length allows it, else None."""
    import torch

    half = meta.shape[-1] // 2
    cdt = _complex_for(meta.dtype)
    fmt = N.FMT_C64 if cdt == numpy.complex64 else N.FMT_C128
    shape = tuple(meta.shape[:-1]) + (half,)
    d = N.desc(fmt, shape, (len(shape) - 1,), N.FLAG_REAL_POST)
    d.output = N.edge(fmt, tuple(meta.shape[:-1]) + (half + store_last,))
    try:
        with torch.cuda.device(device):
            return N.Plan(d)
    except NotImplementedError:
        return None


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
        leaves = [p.name for p in self._tr_tree.get_leaf_parameters()]
        if leaves != ["output", "input"]:
            raise NotImplementedError("transformations connected to RFFT are not fused")
        ann = {p.name: p.annotation for p in self._tr_tree.get_leaf_parameters()}
        if not (_contiguous(ann["input"].as_array_metadata()) and _contiguous(ann["output"].as_array_metadata())):
            raise NotImplementedError("RFFT works on C-contiguous arrays")
        meta = self._meta
        store_last = 0 if self._dont_store_last else 1
        fused = _fused_plan(device, meta, store_last)
        if fused is not None:
            esz = numpy.dtype(_complex_for(meta.dtype)).itemsize

            def fused_runner(stream: int, args):
                out = array_pointer(args["output"], ann["output"])
                inp = array_pointer(args["input"], ann["input"])
                if inp % esz:
                    raise ValueError("the real array must start on a boundary of its complex pair type")
                fused.execute([out], [inp], inverse=0, stream=stream)

            fused_runner.launches = fused.launches
            fused_runner.plan = fused
            return fused_runner
        h = _Half(device, meta.shape[:-1], meta.shape[-1] // 2, _complex_for(meta.dtype))

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
        leaves = [p.name for p in self._tr_tree.get_leaf_parameters()]
        if leaves != ["output", "input"]:
            raise NotImplementedError("transformations connected to IRFFT are not fused")
        ann = {p.name: p.annotation for p in self._tr_tree.get_leaf_parameters()}
        if not (_contiguous(ann["input"].as_array_metadata()) and _contiguous(ann["output"].as_array_metadata())):
            raise NotImplementedError("IRFFT works on C-contiguous arrays")
        meta = self._meta
        h = _Half(device, meta.shape[:-1], meta.shape[-1] - 1, meta.dtype)

        def runner(stream: int, args):
            out = h.aligned(array_pointer(args["output"], ann["output"]))
            inp = array_pointer(args["input"], ann["input"])
            N.check(N.lib().rk_irfft_pre(h.temp.data_ptr(), inp, h.table.data_ptr(), h.fmt, h.half, h.batch, stream))
            h.plan.execute([out], [h.temp.data_ptr()], inverse=1, stream=stream)

        runner.launches = h.plan.launches + 1
        runner.half = h
        return runner
