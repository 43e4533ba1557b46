"""Built-in transformations.

Same names, parameter names and signatures as ``reikna.transformations``
(reikna/transformations.py:11-347), plus the transformations that reikna's examples
define for the FFT hot path: ``fftshift`` (examples/demo_fftshift_transformation.py:24),
``real_to_complex`` (examples/demo_real_to_complex_fft.py:20), and the spectrogram
pieces ``rolling_frame``, ``hanning_window`` and ``crop_frequencies``
(examples/demo_specgram.py:97-193).  Each carries an ``op`` descriptor that the FFT
planner fuses into its first load or last store; every one of them can be connected
to an FFT's input or output (the ones that make sense on that side).
"""

from __future__ import annotations

import numpy

from .core.signature import Annotation, ArrayMetadata, Parameter, Type
from .core.transformation import Transformation


def _meta(arr_t) -> ArrayMetadata:
    return Type(arr_t).as_array_metadata() if not isinstance(arr_t, ArrayMetadata) else arr_t


def real_for(dtype) -> numpy.dtype:
    return numpy.dtype({numpy.dtype(numpy.complex64): numpy.float32, numpy.dtype(numpy.complex128): numpy.float64}.get(
        numpy.dtype(dtype), dtype))


def complex_for(dtype) -> numpy.dtype:
    return numpy.dtype({numpy.dtype(numpy.float32): numpy.complex64, numpy.dtype(numpy.float64): numpy.complex128}.get(
        numpy.dtype(dtype), dtype))


def _contig(shape, dtype) -> ArrayMetadata:
    return ArrayMetadata(shape, dtype)


def copy(arr_t, out_arr_t=None) -> Transformation:
    """Identity (1 output, 1 input): ``output = input``; strides may differ."""
    inp = _meta(arr_t)
    out = _meta(out_arr_t) if out_arr_t is not None else inp
    if out.shape != inp.shape or out.dtype != inp.dtype:
        raise ValueError("Input and output arrays must have the same shape and data type")
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(inp, "i"))],
        op={"kind": "copy"},
    )


def cast(arr_t, dtype) -> Transformation:
    """Typecast (1 output, 1 input): ``output = cast[dtype](input)``."""
    inp = _meta(arr_t)
    out = inp.with_(dtype=dtype)
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(inp, "i"))],
        op={"kind": "cast"},
    )


def _scale_trf(arr_t, param_dtype=None, const=None, div=False) -> Transformation:
    inp = _meta(arr_t)
    params = [Parameter("output", Annotation(inp, "o")), Parameter("input", Annotation(inp, "i"))]
    if param_dtype is not None:
        params.append(Parameter("param", Annotation(numpy.dtype(param_dtype))))
        return Transformation(params, op={"kind": "scale", "param": "param", "div": div})
    c = complex(const)
    if div:
        c = 1.0 / c
    return Transformation(params, op={"kind": "scale", "const": c})


def mul_param(arr_t, param_dtype) -> Transformation:
    """Scaling by a runtime scalar (1 output, 1 input, 1 scalar): ``output = input * param``."""
    return _scale_trf(arr_t, param_dtype=param_dtype)


def mul_const(arr_t, param) -> Transformation:
    """Scaling by a constant (1 output, 1 input): ``output = input * param``."""
    return _scale_trf(arr_t, const=param)


def div_param(arr_t, param_dtype) -> Transformation:
    """Division by a runtime scalar: ``output = input / param``."""
    return _scale_trf(arr_t, param_dtype=param_dtype, div=True)


def div_const(arr_t, param) -> Transformation:
    """Division by a constant: ``output = input / param``."""
    return _scale_trf(arr_t, const=param, div=True)


def add_param(arr_t, param_dtype) -> Transformation:
    """Addition of a runtime scalar (1 output, 1 input, 1 scalar): ``output = input + param``."""
    inp = _meta(arr_t)
    return Transformation(
        [
            Parameter("output", Annotation(inp, "o")),
            Parameter("input", Annotation(inp, "i")),
            Parameter("param", Annotation(numpy.dtype(param_dtype))),
        ],
        op={"kind": "add", "param": "param"},
    )


def add_const(arr_t, param) -> Transformation:
    """Addition of a constant (1 output, 1 input): ``output = input + param``."""
    inp = _meta(arr_t)
    return Transformation(
        [Parameter("output", Annotation(inp, "o")), Parameter("input", Annotation(inp, "i"))],
        op={"kind": "add", "const": complex(param)},
    )


def split_complex(input_arr_t) -> Transformation:
    """Complex input to two real outputs: ``real = Re(input), imag = Im(input)``."""
    inp = _meta(input_arr_t)
    out = _contig(inp.shape, real_for(inp.dtype))
    return Transformation(
        [
            Parameter("real", Annotation(out, "o")),
            Parameter("imag", Annotation(out, "o")),
            Parameter("input", Annotation(inp, "i")),
        ],
        op={"kind": "split"},
    )


def combine_complex(output_arr_t) -> Transformation:
    """Two real inputs to a complex output: ``output = real + 1j * imag``."""
    out = _meta(output_arr_t)
    inp = _contig(out.shape, real_for(out.dtype))
    return Transformation(
        [
            Parameter("output", Annotation(out, "o")),
            Parameter("real", Annotation(inp, "i")),
            Parameter("imag", Annotation(inp, "i")),
        ],
        op={"kind": "combine"},
    )


def norm_const(arr_t, order) -> Transformation:
    """``output = abs(input) ** order`` (1 output, 1 input)."""
    inp = _meta(arr_t)
    out_dtype = real_for(inp.dtype)
    return Transformation(
        [
            Parameter("output", Annotation(_contig(inp.shape, out_dtype), "o")),
            Parameter("input", Annotation(inp, "i")),
        ],
        op={"kind": "norm", "order": float(order)},
    )


def norm_param(arr_t) -> Transformation:
    """``output = abs(input) ** order`` with a runtime ``order`` (1 output, 1 input, 1 scalar)."""
    inp = _meta(arr_t)
    out_dtype = real_for(inp.dtype)
    return Transformation(
        [
            Parameter("output", Annotation(_contig(inp.shape, out_dtype), "o")),
            Parameter("input", Annotation(inp, "i")),
            Parameter("order", Annotation(out_dtype)),
        ],
        op={"kind": "norm_param"},
    )


def ignore(arr_t) -> Transformation:
    """Ignores the output it is attached to."""
    return Transformation([Parameter("input", Annotation(_meta(arr_t), "i"))], op={"kind": "ignore"})


def broadcast_const(arr_t, val) -> Transformation:
    """Broadcasts a constant to the array output (1 output)."""
    inp = _meta(arr_t)
    v = numpy.asarray(val, inp.dtype)
    if v.shape != ():
        raise ValueError("The constant must be a scalar")
    return Transformation([Parameter("output", Annotation(inp, "o"))], op={"kind": "const", "value": complex(v.item())})


def broadcast_param(arr_t) -> Transformation:
    """Broadcasts a runtime scalar ``param`` to the array output (1 output, 1 scalar)."""
    inp = _meta(arr_t)
    return Transformation(
        [Parameter("output", Annotation(inp, "o")), Parameter("param", Annotation(inp.dtype))],
        op={"kind": "const_param"},
    )


def copy_broadcasted(arr_t, out_arr_t=None) -> Transformation:
    """Identity with numpy-style broadcasting of the input (input-only)."""
    inp = _meta(arr_t)
    out = _meta(out_arr_t) if out_arr_t is not None else inp
    if out.dtype != inp.dtype:
        raise ValueError("Input and output arrays must have the same data type")
    if len(inp.shape) > len(out.shape) or any(
        not (a == 1 or a == b) for a, b in zip(reversed(inp.shape), reversed(out.shape))
    ):
        raise ValueError("Input is not broadcastable to output")
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(inp, "i"))],
        connectors=["output"],
        op={"kind": "broadcast"},
    )


# --- transformations from reikna's FFT examples ---------------------------------


def fftshift(arr_t, axes=None, *, inverse: bool = False) -> Transformation:
    """``output = numpy.fft.fftshift(input, axes)`` as an output transformation
    (``ifftshift`` with ``inverse=True``).  Repositions elements: the FFT routes
    in-place calls through a private copy of the input."""
    meta = _meta(arr_t)
    nd = len(meta.shape)
    ax = tuple(range(nd)) if axes is None else tuple(sorted(a % nd for a in axes))
    return Transformation(
        [Parameter("output", Annotation(meta, "o")), Parameter("input", Annotation(meta, "i"))],
        connectors=["input"],
        op={"kind": "shift", "axes": ax, "inverse": bool(inverse)},
    )


def real_to_complex(arr_t) -> Transformation:
    """Real array to complex with zero imaginary part (input transformation)."""
    meta = _meta(arr_t)
    out = _contig(meta.shape, complex_for(meta.dtype))
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))],
        op={"kind": "real_to_complex"},
    )


def rolling_frame(arr_t, fft_size: int, noverlap: int, pad_to: int | None = None) -> Transformation:
    """1-D signal to overlapping frames (frame_num, pad_to or fft_size), zero padded."""
    meta = _meta(arr_t)
    if len(meta.shape) != 1:
        raise ValueError("rolling_frame expects a 1-D array")
    step = fft_size - noverlap
    frame_num = (meta.shape[0] - noverlap) // step
    frame_size = fft_size if pad_to is None else pad_to
    out = _contig((frame_num, frame_size), meta.dtype)
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))],
        connectors=["output"],
        op={"kind": "frame", "step": step, "fft_size": fft_size},
    )


def hanning_window(arr_t, fft_size: int) -> Transformation:
    """Multiplies rows by the von Hann window 0.5 (1 - cos(2 pi n / (fft_size - 1)))."""
    meta = _meta(arr_t)
    return Transformation(
        [Parameter("output", Annotation(meta, "o")), Parameter("input", Annotation(meta, "i"))],
        op={"kind": "window", "window": "hann", "size": int(fft_size)},
    )


def transpose_2d(arr_t) -> Transformation:
    """``output = input.T`` for a 2-D array (output transformation).  On an FFT output
    it is fused into the last pass' store (no separate transpose kernel, unlike the
    ``Transpose`` step that ends reikna's spectrogram example, demo_specgram.py:268)."""
    meta = _meta(arr_t)
    if len(meta.shape) != 2:
        raise ValueError("transpose_2d expects a 2-D array")
    out = _contig((meta.shape[1], meta.shape[0]), meta.dtype)
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))],
        connectors=["input"],
        op={"kind": "transpose"},
    )


def crop_frequencies(arr_t) -> Transformation:
    """Keeps the first cols // 2 + 1 columns of a 2-D array (output transformation)."""
    meta = _meta(arr_t)
    out = _contig((meta.shape[0], meta.shape[1] // 2 + 1), meta.dtype)
    return Transformation(
        [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(meta, "i"))],
        connectors=["input"],
        op={"kind": "crop"},
    )
