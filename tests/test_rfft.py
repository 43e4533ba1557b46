"""Half-length RFFT / IRFFT (reikna examples/demo_specialized_fft.py) against numpy.

The example's own check is atol = rtol = 1e-4 against numpy's rfft / irfft
(demo_specialized_fft.py:627-662); the tests also hold the complex64 rel-L2 bound.
"""

import numpy
import pytest

from helpers import fft_bound, rel_l2


def test_rfft_signatures_and_errors():
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import IRFFT, RFFT

    r = RFFT(ArrayMetadata((8, 100), numpy.float32))
    assert tuple(r.parameter.output.shape) == (8, 51) and r.parameter.output.dtype == numpy.complex64
    r = RFFT(ArrayMetadata((100,), numpy.float64), dont_store_last=True)
    assert tuple(r.parameter.output.shape) == (50,) and r.parameter.output.dtype == numpy.complex128
    i = IRFFT(ArrayMetadata((8, 51), numpy.complex64))
    assert tuple(i.parameter.output.shape) == (8, 100) and i.parameter.output.dtype == numpy.float32
    with pytest.raises(ValueError):
        RFFT(ArrayMetadata((8, 101), numpy.float32))
    with pytest.raises(ValueError):
        RFFT(ArrayMetadata((8, 100), numpy.complex64))
    with pytest.raises(ValueError):
        IRFFT(ArrayMetadata((8, 100), numpy.float32))


@pytest.mark.gpu
@pytest.mark.parametrize(
    "shape,dtype",
    [((64, 4096), numpy.float32), ((1000, 1000), numpy.float32), ((3, 16384), numpy.float64), ((5, 3000), numpy.float32),
     ((2,), numpy.float32), ((7, 2, 256), numpy.float32)],
)
def test_rfft_and_irfft(shape, dtype):
    import torch

    from reikna_b200.fft import IRFFT, RFFT

    rng = numpy.random.default_rng(61)
    x = rng.uniform(-1, 1, shape).astype(dtype)
    t = torch.from_numpy(x).cuda()
    cdt = torch.complex64 if dtype == numpy.float32 else torch.complex128
    ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
    n = shape[-1]
    spec = torch.empty(shape[:-1] + (n // 2 + 1,), dtype=cdt, device="cuda")
    RFFT(t).compile()(None, spec, t)
    back = torch.empty_like(t)
    IRFFT(spec).compile()(None, back, spec)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64), axis=-1)
    got = spec.cpu().numpy()
    assert rel_l2(got, ref) < fft_bound(ctype, n)
    assert numpy.allclose(got, ref, atol=1e-4 * max(1.0, numpy.abs(ref).max()), rtol=1e-4)
    y = back.cpu().numpy()
    assert rel_l2(y, x.astype(numpy.float64)) < 2 * fft_bound(ctype, n)
    assert numpy.allclose(y, numpy.fft.irfft(ref, n=n, axis=-1), atol=1e-4, rtol=1e-4)


@pytest.mark.gpu
def test_rfft_without_last_bin_and_irfft_ignores_imaginary_edges():
    import torch

    from reikna_b200.fft import IRFFT, RFFT

    rng = numpy.random.default_rng(62)
    x = rng.standard_normal((16, 512)).astype(numpy.float32)
    t = torch.from_numpy(x).cuda()
    spec = torch.empty((16, 256), dtype=torch.complex64, device="cuda")
    RFFT(t, dont_store_last=True).compile()(None, spec, t)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64))[:, :256]
    assert rel_l2(spec.cpu().numpy(), ref) < fft_bound(numpy.complex64, 512)
    full = numpy.fft.rfft(x.astype(numpy.float64)).astype(numpy.complex64)
    full[:, 0] += 3j
    full[:, -1] -= 2j
    s = torch.from_numpy(full).cuda()
    out = torch.empty((16, 512), dtype=torch.float32, device="cuda")
    IRFFT(s).compile()(None, out, s)
    torch.cuda.synchronize()
    assert numpy.allclose(out.cpu().numpy(), numpy.fft.irfft(full.astype(numpy.complex128)), atol=1e-4, rtol=1e-4)


def test_real_post_flag_plans_one_pass():
    from reikna_b200 import _native as N

    d = N.desc(N.FMT_C64, (64, 512), (1,), N.FLAG_REAL_POST)
    d.output = N.edge(N.FMT_C64, (64, 513))
    plan = N.describe(d)
    assert len(plan["passes"]) == 1 and plan["passes"][0]["var"] == 3
    d = N.desc(N.FMT_C64, (64, 500), (1,), N.FLAG_REAL_POST)
    with pytest.raises(NotImplementedError):
        N.describe(d)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dtype", [((16384, 1024), numpy.float32), ((4, 16384), numpy.float32), ((3, 8192), numpy.float64)])
def test_fused_rfft_is_one_launch(shape, dtype):
    import torch

    from reikna_b200.fft import RFFT

    rng = numpy.random.default_rng(63)
    x = rng.uniform(-1, 1, shape).astype(dtype)
    t = torch.from_numpy(x).cuda()
    cdt = torch.complex64 if dtype == numpy.float32 else torch.complex128
    for last in (False, True):
        n = shape[-1]
        spec = torch.empty(shape[:-1] + (n // 2 + (0 if last else 1),), dtype=cdt, device="cuda")
        c = RFFT(t, dont_store_last=last).compile()
        assert c.launches == 1
        c(None, spec, t)
        torch.cuda.synchronize()
        ref = numpy.fft.rfft(x.astype(numpy.float64))[..., : spec.shape[-1]]
        ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
        assert rel_l2(spec.cpu().numpy(), ref) < fft_bound(ctype, n)
