"""Integer helpers with the semantics of ``reikna.helpers`` (reikna/helpers.py:87-208)."""

from __future__ import annotations

from collections.abc import Iterable


def product(seq: Iterable[int]) -> int:
    """Product of the elements of ``seq`` (1 for an empty sequence)."""
    result = 1
    for x in seq:
        result *= x
    return result


def min_blocks(length: int, block: int) -> int:
    """Minimum number of blocks of size ``block`` that cover ``length`` elements."""
    return (length - 1) // block + 1


def log2(num: int) -> int:
    """Integer base-2 logarithm, rounded down."""
    return max(int(num).bit_length() - 1, 0)


def bounding_power_of_2(num: int) -> int:
    """Smallest power of two that is >= ``num``."""
    if num <= 1:
        return 1
    return 1 << (int(num) - 1).bit_length()


def wrap_in_tuple(seq_or_elem) -> tuple[int, ...]:
    if seq_or_elem is None:
        return ()
    if isinstance(seq_or_elem, int):
        return (seq_or_elem,)
    return tuple(seq_or_elem)


def normalize_axes(ndim: int, axes) -> tuple[int, ...]:
    """Tuple of non-negative axes (``None`` means all axes)."""
    if axes is None:
        return tuple(range(ndim))
    axes = wrap_in_tuple(axes)
    axes = tuple(a if a >= 0 else ndim + a for a in axes)
    if any(a < 0 or a >= ndim for a in axes):
        raise IndexError("Array index out of range")
    return axes
