"""Transformations written as code (reikna's Transformation(parameters, code, ...),
reikna/core/transformation.py:42-120) on FFT edges: rendered from reikna's template
syntax, compiled at run time into the first / last pass, and checked against the
built-in transformations and numpy.

The fftshift below is written in the snippet form the reference's fftshift example
uses (an output transformation that writes each element to its shifted index with
``store_idx``), in this project's own words."""

import numpy
import pytest

from helpers import fft_bound, rel_l2

from reikna_b200 import transformations as tr
from reikna_b200.core import Annotation, ArrayMetadata, Parameter, Transformation
from reikna_b200.fft import FFT

SHIFT_CODE = """
<% nd = len(output.shape) %>
%for d in range(nd):
VSIZE_T j${d} = ${idxs[d]};
%if d in axes:
j${d} += ${output.shape[d] // 2};
if (j${d} >= ${output.shape[d]}) j${d} -= ${output.shape[d]};
%endif
%endfor
${output.ctype} v = ${input.load_same};
${output.store_idx}(${", ".join("j%d" % d for d in range(nd))}, v);
"""


def code_fftshift(meta, axes=None):
    axes = tuple(range(len(meta.shape)) if axes is None else sorted(axes))
    return Transformation(
        [Parameter("output", Annotation(meta, "o")), Parameter("input", Annotation(meta, "i"))],
        SHIFT_CODE, connectors=["input"], render_kwds=dict(axes=axes))


# input side: x * w[column] * gain, with w a 1-D array read by load_idx
SCALE_CODE = """
${output.store_same}(rkf::mul(rkf::mul(${input.load_same}, ${window.load_idx}(${idxs[-1]})), ${gain}));
"""


def code_window(meta, wmeta):
    return Transformation(
        [Parameter("output", Annotation(meta, "o")), Parameter("input", Annotation(meta, "i")),
         Parameter("window", Annotation(wmeta, "i")), Parameter("gain", Annotation(numpy.float32))],
        SCALE_CODE)


def _shift_fft(meta, axes=None):
    fft = FFT(meta, axes=axes)
    sh = code_fftshift(meta)
    fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
    return fft


def test_code_edge_descriptor_and_source_compile():
    """No GPU: the edge becomes a run-time compiled edge and its kernel source
    compiles with NVRTC for sm_100a."""
    from reikna_b200 import _native as N
    from reikna_b200 import _rtc
    from reikna_b200.fft.user import kernel_source

    meta = ArrayMetadata((64, 48), numpy.complex64)
    fft = _shift_fft(meta)
    d, ispec, ospec, *_ = fft.native_descriptor()
    assert d.output.format == N.FMT_USER and ospec.kind == "user" and d.input.format == N.FMT_C64
    assert [p for p in fft.signature.parameters] == ["shifted", "input", "inverse"]
    edge = fft._user_edges["output"]
    src = kernel_source([edge], "float", 64, 0, 0, 256)
    assert "RK_USER_STORE" in src and "j1 += 24" in src
    try:
        cubin = _rtc.compile_cubin(src)
    except _rtc.CompileError as e:
        if "not available" in str(e):
            pytest.skip("NVRTC missing")
        raise
    assert len(cubin) > 1000


def test_template_renderer_control_lines():
    from reikna_b200.core.template import render

    out = render("<% n = 3 %>\n%for i in range(n):\n${i}\n%endfor\n## dropped\n%if n > 2:\nbig\n%else:\nsmall\n%endif\n")
    assert out.split() == ["0", "1", "2", "big"]


@pytest.mark.gpu
@pytest.mark.parametrize("shape,axes", [((256, 256, 256), None), ((64, 48), None), ((33, 100), (1,)),
                                        ((1000, 1000), None), ((7, 9, 11), (0, 2))])
def test_code_fftshift_matches_builtin_and_numpy(shape, axes):
    import torch

    rng = numpy.random.default_rng(sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64)
    t = torch.from_numpy(x).cuda()
    ax = tuple(range(len(shape))) if axes is None else axes
    fft = FFT(t, axes=ax)
    sh = code_fftshift(t, axes=ax)
    fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
    out = torch.empty_like(t)
    fft.compile()(None, out, t)
    ref_b = torch.empty_like(t)
    fb = FFT(t, axes=ax)
    bsh = tr.fftshift(t, axes=ax)
    fb.parameter.output.connect(bsh, bsh.input, shifted=bsh.output)
    fb.compile()(None, ref_b, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fftshift(numpy.fft.fftn(x.astype(numpy.complex128), axes=ax), axes=ax)
    n = int(numpy.prod([shape[a] for a in ax]))
    got = out.cpu().numpy()
    assert rel_l2(got, ref) < fft_bound(numpy.complex64, n)
    assert rel_l2(got, ref_b.cpu().numpy()) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [numpy.complex64, numpy.complex128])
@pytest.mark.parametrize("inverse", [0, 1])
def test_code_input_transformation_with_array_and_scalar(dtype, inverse):
    import torch

    rng = numpy.random.default_rng(3)
    shape = (40, 512)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    rdt = numpy.float32 if dtype == numpy.complex64 else numpy.float64
    w = rng.uniform(0.5, 1.5, shape[1]).astype(rdt)
    t = torch.from_numpy(x).cuda()
    fft = FFT(t, axes=(1,))
    trf = code_window(ArrayMetadata(shape, dtype), ArrayMetadata((shape[1],), rdt))
    fft.parameter.input.connect(trf, trf.output, raw=trf.input, window=trf.window, gain=trf.gain)
    # a built-in transformation after the code one on the same chain
    sc = tr.mul_const(t, 0.5)
    fft.parameter.raw.connect(sc, sc.output, raw2=sc.input)
    out = torch.empty_like(t)
    fft.compile()(None, out, t, torch.from_numpy(w).cuda(), 3.0, inverse)
    torch.cuda.synchronize()
    f = numpy.fft.ifft if inverse else numpy.fft.fft
    ref = f(x.astype(numpy.complex128) * 0.5 * w * 3.0, axis=1)
    bound = fft_bound(dtype, shape[1])
    assert rel_l2(out.cpu().numpy(), ref) < bound
