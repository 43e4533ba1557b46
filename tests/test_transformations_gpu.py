"""The built-in transformations that fold into the FFT's edges as an additive term, a
runtime norm order, a constant input, an ignored output or a broadcast input
(reikna/transformations.py:48-347: add_const, add_param, norm_param, broadcast_const,
broadcast_param, ignore, copy_broadcasted), on the GPU against numpy in FP64."""

import numpy
import pytest

from helpers import fft_bound, rel_l2

pytestmark = pytest.mark.gpu


def _c(rng, shape, dtype=numpy.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def _t(x):
    import torch

    return torch.from_numpy(numpy.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("shape,axes", [((64, 1024), (1,)), ((8, 256, 256), None), ((40, 3001), (1,)),
                                        ((3, 2**16), (1,)), ((16, 16, 128), (0, 1))])
@pytest.mark.parametrize("inverse", [0, 1])
def test_add_and_mul_constants_on_both_edges(shape, axes, inverse):
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(sum(shape) + inverse)
    x = _c(rng, shape)
    t = _t(x)
    fft = FFT(t, axes=axes)
    a_in = tr.add_const(t, 0.5 - 0.25j)
    m_in = tr.mul_const(t, 2.0)
    # input: fft_in = 2 (x + (0.5 - 0.25i))
    fft.parameter.input.connect(m_in, m_in.output, x1=m_in.input)
    fft.parameter.x1.connect(a_in, a_in.output, x=a_in.input)
    a_out = tr.add_const(t, 1.0 + 3.0j)
    m_out = tr.mul_const(t, -0.5j)
    # output: leaf = -0.5i (y + (1 + 3i))
    fft.parameter.output.connect(a_out, a_out.input, y1=a_out.output)
    fft.parameter.y1.connect(m_out, m_out.input, y=m_out.output)
    out = torch.empty_like(t)
    fft.compile()(None, out, t, inverse)
    torch.cuda.synchronize()
    ax = tuple(range(len(shape))) if axes is None else axes
    f = numpy.fft.ifftn if inverse else numpy.fft.fftn
    ref = -0.5j * (f(2 * (x.astype(numpy.complex128) + (0.5 - 0.25j)), axes=ax) + (1 + 3j))
    n = int(numpy.prod([shape[a] for a in ax]))
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


def test_runtime_scalars_add_and_mul():
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(3)
    x = _c(rng, (32, 512))
    t = _t(x)
    fft = FFT(t, axes=(1,))
    mp = tr.mul_param(t, numpy.complex64)
    ap = tr.add_param(t, numpy.complex64)
    dp = tr.div_param(t, numpy.float32)
    ap2 = tr.add_param(t, numpy.float32)
    fft.parameter.input.connect(mp, mp.output, x1=mp.input, p=mp.param)
    fft.parameter.x1.connect(ap, ap.output, x=ap.input, q=ap.param)
    fft.parameter.output.connect(dp, dp.input, y1=dp.output, d=dp.param)
    fft.parameter.y1.connect(ap2, ap2.input, y=ap2.output, r=ap2.param)
    cc = fft.compile()
    for p, q, d, r in ((2j, 0.5 + 1j, 4.0, -1.0), (1 - 1j, 0.0, 0.5, 2.5)):
        out = torch.empty_like(t)
        cc(None, y=out, x=t, p=p, q=q, d=d, r=r)
        torch.cuda.synchronize()
        ref = numpy.fft.fft(p * (x.astype(numpy.complex128) + q), axis=1) / d + r
        assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 512)


@pytest.mark.parametrize("order", [1.0, 1.5, 2.0])
def test_norm_param(order):
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(4)
    x = _c(rng, (16, 2048))
    t = _t(x)
    fft = FFT(t, axes=(1,))
    npm = tr.norm_param(t)
    fft.parameter.output.connect(npm, npm.input, mag=npm.output, order=npm.order)
    mag = torch.empty(x.shape, dtype=torch.float32, device="cuda")
    fft.compile()(None, mag=mag, input=t, order=order)
    torch.cuda.synchronize()
    ref = numpy.abs(numpy.fft.fft(x.astype(numpy.complex128), axis=1)) ** order
    assert rel_l2(mag.cpu().numpy(), ref) < order * fft_bound(numpy.complex64, 2048)


@pytest.mark.parametrize("shape", [(8, 1024), (4, 64, 64), (6, 3001)])
def test_constant_input_const_and_param(shape):
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    meta = numpy.zeros(shape, numpy.complex64)
    out = torch.empty(shape, dtype=torch.complex64, device="cuda")
    for kind in ("const", "param"):
        fft = FFT(meta, axes=tuple(range(1, len(shape))))
        val = 0.75 - 2.0j
        if kind == "const":
            bc = tr.broadcast_const(meta, val)
            fft.parameter.input.connect(bc, bc.output)
            fft.compile()(None, out)
        else:
            bc = tr.broadcast_param(meta)
            fft.parameter.input.connect(bc, bc.output, value=bc.param)
            fft.compile()(None, out, val)
        torch.cuda.synchronize()
        ref = numpy.fft.fftn(numpy.full(shape, val, numpy.complex128), axes=tuple(range(1, len(shape))))
        got = out.cpu().numpy()
        assert numpy.abs(got - ref).max() < 1e-5 * numpy.abs(ref).max(), kind


def test_real_and_constant_imaginary_parts():
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(5)
    xr = rng.uniform(-1, 1, (16, 1000)).astype(numpy.float32)
    meta = numpy.zeros(xr.shape, numpy.complex64)
    fft = FFT(meta, axes=(1,))
    cc = tr.combine_complex(meta)
    im = tr.broadcast_const(cc.parameter.imag, 0.5)
    fft.parameter.input.connect(cc, cc.output, re=cc.real, im=cc.imag)
    fft.parameter.im.connect(im, im.output)
    out = torch.empty(xr.shape, dtype=torch.complex64, device="cuda")
    fft.compile()(None, out, _t(xr))
    torch.cuda.synchronize()
    ref = numpy.fft.fft(xr.astype(numpy.float64) + 0.5j, axis=1)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 1000)


def test_ignored_output_runs():
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(6)
    t = _t(_c(rng, (64, 4096)))
    before = t.clone()
    fft = FFT(t, axes=(1,))
    ig = tr.ignore(t)
    fft.parameter.output.connect(ig, ig.input)
    assert [p.name for p in fft.signature.parameters.values()] == ["input", "inverse"]
    fft.compile()(None, t)
    N.stream_check(torch.cuda.current_stream().cuda_stream)
    assert torch.equal(t, before)


@pytest.mark.parametrize("row_shape,shape,axes", [((256,), (32, 256), (0, 1)), ((1, 64), (16, 64), (1,)),
                                                  ((20, 1), (20, 30), (0, 1))])
def test_copy_broadcasted_input(row_shape, shape, axes):
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(7)
    row = _c(rng, row_shape)
    meta = numpy.zeros(shape, numpy.complex64)
    fft = FFT(meta, axes=axes)
    cb = tr.copy_broadcasted(row, meta)
    fft.parameter.input.connect(cb, cb.output, row=cb.input)
    out = torch.empty(shape, dtype=torch.complex64, device="cuda")
    fft.compile()(None, out, _t(row))
    torch.cuda.synchronize()
    ref = numpy.fft.fftn(numpy.broadcast_to(row.astype(numpy.complex128), shape), axes=axes)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, int(numpy.prod([shape[a] for a in axes])))
