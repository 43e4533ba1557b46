"""Array algorithms next to the FFT: ``Transpose`` (reikna/algorithms/transpose.py)."""

from .transpose import Transpose

__all__ = ["Transpose"]
