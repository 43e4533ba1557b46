"""Spectrogram of a real signal as one fused FFT computation.

Follows the reference's spectrogram example (examples/demo_specgram.py:97-268): frames
of ``nfft`` samples every ``hop`` samples (``rolling_frame``), a von Hann window
(``hanning_window``), zero imaginary part (``combine_complex`` + ``broadcast_const``),
an FFT along the frame axis, the magnitude (``norm_const(1)``) and the first
``nfft // 2 + 1`` bins (``crop_frequencies``).  Every step is a transformation on the
FFT's input or output, so the whole chain runs inside the FFT's first and last pass:
the signal is read once and the float32 magnitudes are written once.  The
reference's example ends with a separate ``Transpose`` kernel to get the
bins-by-frames picture; here ``transposed=True`` connects ``transpose_2d`` to the
output, which the last pass applies as it stores (lane-fastest through shared
memory), so the (nfft // 2 + 1, frames) result costs no extra pass.
"""

from __future__ import annotations

import numpy

from . import transformations as tr
from .core import ArrayMetadata
from .fft import FFT


def spectrogram(signal_len: int, nfft: int = 1024, hop: int = 256, transposed: bool = False) -> FFT:
    """Computation ``(cropped: float32 (frames, nfft//2+1), flat_input: float32 (signal_len,))``,
    or with ``transposed`` ``(picture: float32 (nfft//2+1, frames), flat_input)``."""
    if nfft < 2 or hop < 1 or signal_len < nfft:
        raise ValueError("need nfft >= 2, hop >= 1 and a signal at least one frame long")
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
    fft.parameter.input.connect(to_c, to_c.parameter.output, input_real=to_c.parameter.real, input_imag=to_c.parameter.imag)
    fft.parameter.input_imag.connect(zero, zero.parameter.output)
    fft.parameter.input_real.connect(win, win.parameter.output, unwindowed_input=win.parameter.input)
    fft.parameter.unwindowed_input.connect(frame, frame.parameter.output, flat_input=frame.parameter.input)
    fft.parameter.output.connect(amp, amp.parameter.input, amplitude=amp.parameter.output)
    fft.parameter.amplitude.connect(crop, crop.parameter.input, cropped=crop.parameter.output)
    if transposed:
        tp = tr.transpose_2d(crop.parameter.output)
        fft.parameter.cropped.connect(tp, tp.parameter.input, picture=tp.parameter.output)
    return fft


def frames(signal_len: int, nfft: int = 1024, hop: int = 256) -> int:
    """Number of whole frames ``rolling_frame`` takes from a signal."""
    return (signal_len - (nfft - hop)) // hop
