"""Spectrogram fused into one FFT pass, frame-major and bins-by-frames (transposed
store), against numpy (examples/demo_specgram.py restated without matplotlib)."""

import numpy
import pytest


def _reference(sig, nfft, hop):
    nf = (len(sig) - (nfft - hop)) // hop
    idx = numpy.arange(nf)[:, None] * hop + numpy.arange(nfft)[None, :]
    w = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(nfft) / (nfft - 1)))
    return numpy.abs(numpy.fft.rfft(sig.astype(numpy.float64)[idx] * w, axis=1))


def test_transposed_spectrogram_plans_a_lane_fastest_store():
    from reikna_b200.spectrogram import spectrogram

    # bins-by-frames: the same half-length pass, storing lane-fastest (variant 5); the
    # full-length route stores lane-fastest with variant 2
    d = spectrogram(2**14, 256, 64, transposed=True).describe()
    assert len(d["passes"]) == 1 and d["passes"][0]["var"] == 5 and d["passes"][0]["note"] == "half"
    d = spectrogram(2**14, 256, 64, transposed=True).describe(flags=2**9)
    assert len(d["passes"]) == 1 and d["passes"][0]["var"] == 2
    # frame-major: the half-length transform of the windowed sample pairs with the
    # real-spectrum step and the magnitude in its store
    d = spectrogram(2**14, 256, 64).describe()
    p = d["passes"]
    assert len(p) == 1 and p[0]["note"] == "half" and p[0]["var"] == 6 and p[0]["L"] == 128


def test_transpose_2d_shape_and_errors():
    from reikna_b200 import transformations as tr
    from reikna_b200.core import ArrayMetadata

    t = tr.transpose_2d(ArrayMetadata((3, 5), numpy.float32))
    assert tuple(t.parameter.output.shape) == (5, 3)
    with pytest.raises(ValueError):
        tr.transpose_2d(ArrayMetadata((3, 5, 2), numpy.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("length,nfft,hop", [(2**16, 1024, 256), (2**22, 1024, 256), (10000, 256, 100), (5000, 64, 16), (2**15, 2048, 512)])
@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("flags", [0, 2**9])
def test_spectrogram(length, nfft, hop, transposed, flags):
    import torch

    from reikna_b200.spectrogram import frames, spectrogram

    rng = numpy.random.default_rng(9)
    t = numpy.arange(length)
    sig = rng.standard_normal(length)
    for _ in range(8):
        sig += rng.uniform(0.1, 2) * numpy.sin(2 * numpy.pi * rng.uniform(0, 0.5) * t + rng.uniform(0, 2 * numpy.pi))
    sig = sig.astype(numpy.float32)
    comp = spectrogram(length, nfft, hop, transposed=transposed)
    nf = frames(length, nfft, hop)
    shape = (nfft // 2 + 1, nf) if transposed else (nf, nfft // 2 + 1)
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    comp.compile(flags=flags)(None, out, torch.from_numpy(sig).cuda())
    torch.cuda.synchronize()
    ref = _reference(sig, nfft, hop)
    if transposed:
        ref = ref.T
    got = out.cpu().numpy()
    assert numpy.allclose(got, ref, atol=1e-4 * ref.max(), rtol=1e-4)
