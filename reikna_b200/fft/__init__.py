from .fft import FFT
from .fftshift import FFTShift
from .rfft import APRFFT, IAPRFFT, IRFFT, RFFT

__all__ = ["FFT", "FFTShift", "RFFT", "IRFFT", "APRFFT", "IAPRFFT"]
