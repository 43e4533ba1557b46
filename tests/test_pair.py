"""Row and column passes of a plane in one plane-ordered persistent launch
(RK_FLAG_PAIR): same results as the two passes launched separately."""

import numpy
import pytest

from helpers import fft_bound, normal_array, rel_l2


def test_pair_plan_notes():
    from reikna_b200 import _native as N

    d = N.describe(N.desc(N.FMT_C64, (256, 256, 256), (0, 1, 2), N.FLAG_PAIR))
    assert [p["note"] for p in d["passes"]][:2] == ["pair-rows", "pair-cols"]
    d = N.describe(N.desc(N.FMT_C64, (256, 256, 256), (0, 1, 2)))
    assert d["passes"][0]["note"] == "plane"


@pytest.mark.gpu
@pytest.mark.parametrize("shape,axes", [((256, 256, 256), (0, 1, 2)), ((6, 128, 128), (1, 2)), ((3, 256, 256), (1, 2))])
def test_pair_matches_separate_passes(shape, axes):
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(41)
    x = normal_array(rng, shape, numpy.complex64)
    t = torch.from_numpy(x).cuda()
    outs = []
    for flags in (N.FLAG_PAIR, N.FLAG_NO_PLANE | N.FLAG_NO_TMA):
        c = FFT(t, axes=axes).compile(flags=flags)
        # the pair runs as one launch: its second pass records an empty interval
        c._runner.plan.profile(1)
        c(None, torch.empty_like(t), t)
        ms, _ = c._runner.plan.profile_read()
        c._runner.plan.profile(0)
        if flags == N.FLAG_PAIR:
            assert ms[0] > 0 and ms[1] < 0.1 * ms[0]
        for inverse in (0, 1):
            o = torch.empty_like(t)
            c(None, o, t, inverse)
            outs.append(o)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[2]) and torch.equal(outs[1], outs[3])
    n = int(numpy.prod([shape[a] for a in axes]))
    ref = numpy.fft.fftn(x.astype(numpy.complex128), axes=axes)
    assert rel_l2(outs[0].cpu().numpy(), ref) < fft_bound(numpy.complex64, n)
    assert N.device_status(clear=True) == 0


@pytest.mark.gpu
def test_pair_with_fftshift_and_scale_in_place():
    import torch

    from reikna_b200 import _native as N
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(42)
    x = normal_array(rng, (64, 256, 256), numpy.complex64)
    t = torch.from_numpy(x).cuda()
    fft = FFT(t)
    sh = tr.fftshift(t)
    sc = tr.mul_const(t, 1.0 / x.size)
    fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
    fft.parameter.shifted.connect(sc, sc.input, result=sc.output)
    c = fft.compile(flags=N.FLAG_PAIR)
    out = torch.empty_like(t)
    c(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fftshift(numpy.fft.fftn(x.astype(numpy.complex128))) / x.size
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, x.size)
    t2 = t.clone()
    c2 = FFT(t2).compile(flags=N.FLAG_PAIR)
    c2(None, t2, t2)
    torch.cuda.synchronize()
    assert rel_l2(t2.cpu().numpy(), numpy.fft.fftn(x.astype(numpy.complex128))) < fft_bound(numpy.complex64, x.size)
