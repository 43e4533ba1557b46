from .fft import FFT
from .fftshift import FFTShift

__all__ = ["FFT", "FFTShift"]
