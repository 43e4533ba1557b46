"""Computations composed of other computations (reikna's ComputationPlan,
reikna/core/computation.py:346-640): a user-written two-stage spectrogram — the
fused FFT into a temporary, then ``Transpose`` — as in the reference's spectrogram
example (examples/demo_specgram.py:196-268), against the one-pass transposed
spectrogram of this library."""

import numpy
import pytest

from reikna_b200 import transformations as tr
from reikna_b200.algorithms import Transpose
from reikna_b200.core import Annotation, ArrayMetadata, Computation, Parameter
from reikna_b200.fft import FFT


class TwoStageSpectrogram(Computation):
    """Spectrogram as the reference example builds it: FFT with framing, window,
    magnitude and crop transformations into a temporary, then a transpose."""

    def __init__(self, signal_len, nfft, hop):
        frame = tr.rolling_frame(ArrayMetadata((signal_len,), numpy.float32), nfft, nfft - hop, None)
        shape = frame.parameter.output.shape
        fft_arr = ArrayMetadata(shape, numpy.complex64)
        real_arr = ArrayMetadata(shape, numpy.float32)
        win = tr.hanning_window(real_arr, nfft)
        zero = tr.broadcast_const(real_arr, 0)
        to_c = tr.combine_complex(fft_arr)
        amp = tr.norm_const(fft_arr, 1)
        crop = tr.crop_frequencies(amp.parameter.output)
        fft = FFT(fft_arr, axes=(1,))
        fft.parameter.input.connect(to_c, to_c.parameter.output, input_real=to_c.parameter.real,
                                    input_imag=to_c.parameter.imag)
        fft.parameter.input_imag.connect(zero, zero.parameter.output)
        fft.parameter.input_real.connect(win, win.parameter.output, unwindowed_input=win.parameter.input)
        fft.parameter.unwindowed_input.connect(frame, frame.parameter.output, flat_input=frame.parameter.input)
        fft.parameter.output.connect(amp, amp.parameter.input, amplitude=amp.parameter.output)
        fft.parameter.amplitude.connect(crop, crop.parameter.input, cropped_amplitude=crop.parameter.output)
        self._fft = fft
        self._transpose = Transpose(fft.parameter.cropped_amplitude)
        Computation.__init__(self, [
            Parameter("output", Annotation(self._transpose.parameter.output, "o")),
            Parameter("input", Annotation(fft.parameter.flat_input, "i")),
        ])

    def _build_plan(self, plan_factory, device_params, args):
        plan = plan_factory()
        temp = plan.temp_array_like(self._fft.parameter.cropped_amplitude)
        plan.computation_call(self._fft, temp, args.input)
        plan.computation_call(self._transpose, args.output, temp)
        return plan


def test_nested_signature():
    c = TwoStageSpectrogram(8192, 256, 64)
    assert list(c.signature.parameters) == ["output", "input"]
    assert c.parameter.output.shape == (129, (8192 - 192) // 64)


class ScaledTwice(Computation):
    """A plan with a persistent scalar argument and two nested calls on one temporary."""

    def __init__(self, arr):
        self._fft = FFT(arr)
        Computation.__init__(self, [Parameter("output", Annotation(arr, "o")),
                                    Parameter("input", Annotation(arr, "i"))])

    def _build_plan(self, plan_factory, device_params, args):
        plan = plan_factory()
        temp = plan.temp_array_like(args.output)
        plan.computation_call(self._fft, temp, args.input, 0)
        plan.computation_call(self._fft, args.output, temp, 1)
        return plan


@pytest.mark.gpu
def test_kernel_call_is_refused():
    class K(Computation):
        def __init__(self):
            Computation.__init__(self, [Parameter("output", Annotation(ArrayMetadata((4,), numpy.float32), "o"))])

        def _build_plan(self, plan_factory, device_params, args):
            plan = plan_factory()
            plan.kernel_call(None, [args.output], (4,))
            return plan

    import torch

    if not torch.cuda.is_available():
        pytest.skip("compiling needs a device")
    with pytest.raises(NotImplementedError):
        K().compile()


@pytest.mark.gpu
@pytest.mark.parametrize("n,nfft,hop", [(2**16, 256, 64), (2**22, 1024, 256)])
def test_two_stage_matches_fused_transposed(n, nfft, hop):
    import torch

    from reikna_b200.spectrogram import spectrogram

    rng = numpy.random.default_rng(n)
    sig = rng.standard_normal(n).astype(numpy.float32)
    x = torch.from_numpy(sig).cuda()
    two = TwoStageSpectrogram(n, nfft, hop).compile()
    one = spectrogram(n, nfft, hop, transposed=True).compile()
    a = torch.empty(two.parameter.output.shape, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    two(None, a, x)
    one(None, b, x)
    torch.cuda.synchronize()
    assert two.launches == 2 and one.launches == 1
    ga, gb = a.cpu().numpy(), b.cpu().numpy()
    assert numpy.linalg.norm(ga - gb) / numpy.linalg.norm(gb) < 2e-6 * numpy.log2(nfft)
    # and both against numpy in FP64
    nf = gb.shape[1]
    idx = numpy.arange(nf)[:, None] * hop + numpy.arange(nfft)[None, :]
    w = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(nfft) / (nfft - 1)))
    ref = numpy.abs(numpy.fft.rfft(sig.astype(numpy.float64)[idx] * w, axis=1)).T
    assert numpy.linalg.norm(ga - ref) / numpy.linalg.norm(ref) < 2e-6 * numpy.log2(nfft)


@pytest.mark.gpu
def test_round_trip_through_a_temporary():
    import torch

    rng = numpy.random.default_rng(1)
    x = (rng.standard_normal((64, 256)) + 1j * rng.standard_normal((64, 256))).astype(numpy.complex64)
    t = torch.from_numpy(x).cuda()
    c = ScaledTwice(t).compile()
    out = torch.empty_like(t)
    c(None, out, t)
    torch.cuda.synchronize()
    assert numpy.abs(out.cpu().numpy() - x).max() < 1e-5
