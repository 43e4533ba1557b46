"""Fused Bluestein pass on a two-CTA cluster a line (RK_FLAG_BLUE_PAIR, 8192-point
padded complex64 lines) against numpy FP64 and against the default one-CTA pass.

Every length here pads to M = 8192: with the flag the plan runs one Bluestein pass in
which CTA r of a cluster owns the padded spectrum's bins 2j + r and the two halves of
the output are combined through distributed shared memory.
"""

import numpy
import pytest

from helpers import fft_bound, normal_array, rel_l2

pytestmark = pytest.mark.gpu

PAIR = 4096  # RK_FLAG_BLUE_PAIR


def _compile(t, flags=PAIR, fft=None):
    from reikna_b200.fft import FFT

    comp = fft if fft is not None else FFT(t, axes=(t.ndim - 1,))
    return comp, comp.compile(flags=flags)


def _notes(comp, flags):
    return [p["note"] for p in comp.describe(flags)["passes"]]


@pytest.mark.parametrize("n", [2049, 3001, 4001, 4095])
@pytest.mark.parametrize("rows", [1, 5, 37])
def test_pair_matches_fp64_and_one_cta(n, rows):
    import torch

    from reikna_b200 import _native as N

    x = normal_array(numpy.random.default_rng(n + rows), (rows, n), numpy.complex64)
    t = torch.from_numpy(x).cuda()
    assert N.FLAG_BLUE_PAIR == PAIR
    comp, c2 = _compile(t)
    assert _notes(comp, PAIR) == ["bluestein-pair"]
    assert _notes(comp, 0) == ["bluestein-fused"]
    assert _notes(comp, PAIR | N.FLAG_BATCHABLE) == ["bluestein-fused"]
    _, c1 = _compile(t, 0)
    xr = x.astype(numpy.complex128)
    for inverse in (0, 1):
        y2, y1 = torch.empty_like(t), torch.empty_like(t)
        c2(None, y2, t, inverse)
        c1(None, y1, t, inverse)
        torch.cuda.synchronize()
        ref = numpy.fft.ifft(xr, axis=1) if inverse else numpy.fft.fft(xr, axis=1)
        e2, e1 = rel_l2(y2.cpu().numpy(), ref), rel_l2(y1.cpu().numpy(), ref)
        assert e2 < fft_bound(numpy.complex64, n), (inverse, e2)
        # same algorithm split differently: the same accuracy class as one CTA a line
        assert e2 < 2 * e1 + 1e-7, (inverse, e2, e1)


def test_pair_in_place_and_offset_view():
    import torch

    rows, n = 9, 3001
    x = normal_array(numpy.random.default_rng(80), (rows, n), numpy.complex64)
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    t = torch.from_numpy(x).cuda()
    _, c = _compile(t)
    c(None, t, t)
    torch.cuda.synchronize()
    assert rel_l2(t.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)
    # a view starting one element into its allocation
    base = torch.zeros(rows * n + 1, dtype=torch.complex64, device="cuda")
    view = base[1:].view(rows, n)
    view.copy_(torch.from_numpy(x))
    out = torch.empty_like(view)
    _, c = _compile(view)
    c(None, out, view)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


def test_pair_with_scale_transformations():
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rows, n = 6, 3001
    x = normal_array(numpy.random.default_rng(81), (rows, n), numpy.complex64)
    t = torch.from_numpy(x).cuda()
    fft = FFT(t, axes=(1,))
    si = tr.mul_const(t, 2.0 + 1.0j)
    so = tr.mul_const(t, 0.25 - 0.5j)
    fft.parameter.input.connect(si, si.output, raw=si.input)
    fft.parameter.output.connect(so, so.input, scaled=so.output)
    assert _notes(fft, PAIR) == ["bluestein-pair"]
    out = torch.empty_like(t)
    fft.compile(flags=PAIR)(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fft(x.astype(numpy.complex128) * (2.0 + 1.0j), axis=1) * (0.25 - 0.5j)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


def test_pair_device_status_clean():
    import torch

    from reikna_b200 import _native as N

    x = normal_array(numpy.random.default_rng(82), (1000, 3001), numpy.complex64)
    t = torch.from_numpy(x).cuda()
    _, c = _compile(t)
    out = torch.empty_like(t)
    for _ in range(3):
        c(None, out, t)
    torch.cuda.synchronize()
    assert N.device_status(clear=True) == 0
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 3001)
