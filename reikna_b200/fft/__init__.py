from .fft import FFT
from .fftshift import FFTShift
from .rfft import IRFFT, RFFT

__all__ = ["FFT", "FFTShift", "RFFT", "IRFFT"]
