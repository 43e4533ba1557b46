"""Kernel-shape autotuner: candidate plans follow the computation's passes, every
candidate gives the same transform, and the tuned callable is correct."""

import numpy
import pytest

from helpers import fft_bound, rel_l2

from reikna_b200 import _native as N
from reikna_b200 import autotune
from reikna_b200.core import ArrayMetadata
from reikna_b200.fft import FFT


def test_candidates_follow_the_plan():
    c3d = autotune.candidates(FFT(ArrayMetadata((64, 256, 256), numpy.complex64)))
    assert c3d[0] == 0 and N.FLAG_NO_PLANE in c3d and N.FLAG_PLANE_WIDE in c3d and N.FLAG_PAIR in c3d
    cb = autotune.candidates(FFT(ArrayMetadata((100, 3001), numpy.complex64), axes=(1,)))
    assert N.FLAG_NO_BLUE1 in cb and N.FLAG_R16 in cb and N.FLAG_NO_PLANE not in cb
    c1 = autotune.candidates(FFT(ArrayMetadata((64, 1024), numpy.complex64), axes=(1,)), allow_split=True)
    assert N.FLAG_SPLIT_TC in c1
    assert N.FLAG_SPLIT_TC not in autotune.candidates(FFT(ArrayMetadata((64, 1024), numpy.complex64), axes=(1,)))


def test_r16_plan_is_a_different_kernel_shape():
    f = FFT(ArrayMetadata((10, 3001), numpy.complex64), axes=(1,))
    assert f.describe(0)["passes"][0]["var"] == 1
    assert f.describe(N.FLAG_R16)["passes"][0]["var"] == 17


@pytest.mark.gpu
@pytest.mark.parametrize("shape,axes", [((1000, 3001), (1,)), ((32, 256, 256), None), ((64, 4096), (1,))])
def test_every_candidate_and_the_tuned_plan_agree(shape, axes, tmp_path, monkeypatch):
    import torch

    monkeypatch.setenv("RK_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    rng = numpy.random.default_rng(sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64)
    t = torch.from_numpy(x).cuda()
    comp = FFT(t, axes=axes)
    ax = tuple(range(len(shape))) if axes is None else axes
    ref = numpy.fft.fftn(x.astype(numpy.complex128), axes=ax)
    n = int(numpy.prod([shape[a] for a in ax]))
    for flags in autotune.candidates(comp):
        out = torch.empty_like(t)
        comp.compile(flags=flags)(None, out, t)
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n), flags
    out = torch.empty_like(t)
    cc = autotune.compile_tuned(comp, (out, t), reps=5)
    assert not cc.tuning["cached"] and len(cc.tuning["tried"]) == len(autotune.candidates(comp))
    cc(None, out, t)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)
    assert autotune.tune(comp, (out, t))["cached"]
