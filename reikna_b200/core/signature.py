"""Parameter types of computations and transformations.

Mirrors the public surface of ``reikna.core.signature`` (reikna/core/signature.py:37-327):
``Type``, ``Annotation`` (roles ``'i'``, ``'o'``, ``'io'``, ``'s'``), ``Parameter`` and
``Signature.bind_with_defaults``.  Array metadata (``ArrayMetadata``) replaces
grunnur's: shape, dtype, byte strides and byte offset, built from numpy arrays,
torch tensors or anything with ``shape``/``dtype``.
"""

from __future__ import annotations

import inspect
from collections.abc import Mapping, Sequence
from typing import Any

import numpy

_TORCH_TO_NUMPY = None


def _torch_dtype_map():
    global _TORCH_TO_NUMPY
    if _TORCH_TO_NUMPY is None:
        try:
            import torch

            _TORCH_TO_NUMPY = {
                torch.complex64: numpy.dtype(numpy.complex64),
                torch.complex128: numpy.dtype(numpy.complex128),
                torch.float32: numpy.dtype(numpy.float32),
                torch.float64: numpy.dtype(numpy.float64),
                torch.int32: numpy.dtype(numpy.int32),
                torch.int64: numpy.dtype(numpy.int64),
                torch.int8: numpy.dtype(numpy.int8),
                torch.uint8: numpy.dtype(numpy.uint8),
                torch.int16: numpy.dtype(numpy.int16),
                torch.float16: numpy.dtype(numpy.float16),
                torch.bool: numpy.dtype(numpy.bool_),
            }
        except ImportError:  # pragma: no cover
            _TORCH_TO_NUMPY = {}
    return _TORCH_TO_NUMPY


def as_numpy_dtype(dtype) -> numpy.dtype:
    m = _torch_dtype_map()
    if dtype in m:
        return m[dtype]
    return numpy.dtype(dtype)


def _is_torch_tensor(obj) -> bool:
    return type(obj).__module__.startswith("torch") and hasattr(obj, "data_ptr")


class ArrayMetadata:
    """Shape, dtype, strides (bytes) and first element offset (bytes) of an array."""

    def __init__(self, shape, dtype, strides=None, first_element_offset: int = 0, buffer_size=None):
        if isinstance(shape, int):
            shape = (shape,)
        self.shape = tuple(int(s) for s in shape)
        self.dtype = as_numpy_dtype(dtype)
        if strides is None:
            st = []
            acc = self.dtype.itemsize
            for s in reversed(self.shape):
                st.append(acc)
                acc *= s
            strides = tuple(reversed(st))
        self.strides = tuple(int(s) for s in strides)
        self.first_element_offset = int(first_element_offset)
        self.buffer_size = buffer_size

    @classmethod
    def from_arraylike(cls, arr) -> ArrayMetadata:
        if isinstance(arr, ArrayMetadata):
            return arr
        if hasattr(arr, "as_array_metadata"):
            return arr.as_array_metadata()
        if _is_torch_tensor(arr):
            dt = as_numpy_dtype(arr.dtype)
            return cls(tuple(arr.shape), dt, tuple(s * dt.itemsize for s in arr.stride()), 0)
        strides = getattr(arr, "strides", None)
        offset = getattr(arr, "offset", 0) or 0
        return cls(tuple(arr.shape), arr.dtype, strides, offset)

    def with_(self, **kwds) -> ArrayMetadata:
        shape = kwds.get("shape", self.shape)
        dtype = kwds.get("dtype", self.dtype)
        same_layout = "shape" not in kwds and "dtype" not in kwds
        strides = kwds.get("strides", self.strides if same_layout else None)
        return ArrayMetadata(shape, dtype, strides, kwds.get("first_element_offset", 0))

    def as_array_metadata(self) -> ArrayMetadata:
        return self

    def __eq__(self, other):
        return (
            isinstance(other, ArrayMetadata)
            and self.shape == other.shape
            and self.dtype == other.dtype
            and self.strides == other.strides
            and self.first_element_offset == other.first_element_offset
        )

    def __hash__(self):
        return hash((self.shape, self.dtype, self.strides, self.first_element_offset))

    def __repr__(self):
        return f"ArrayMetadata(shape={self.shape}, dtype={self.dtype}, strides={self.strides})"


def _result_type(val) -> numpy.dtype:
    if isinstance(val, bool):
        return numpy.dtype(numpy.bool_)
    if isinstance(val, int):
        return numpy.dtype(numpy.int64 if abs(val) >= 2**31 else numpy.int32)
    if isinstance(val, float):
        return numpy.dtype(numpy.float64)
    if isinstance(val, complex):
        return numpy.dtype(numpy.complex128)
    return numpy.asarray(val).dtype


class Type:
    """An array type (shape, dtype, strides, offset) or, degenerately, a scalar dtype."""

    def __init__(self, metadata):
        if isinstance(metadata, Type):
            self._metadata = metadata._metadata
        elif isinstance(metadata, ArrayMetadata):
            self._metadata = metadata
        elif (
            hasattr(metadata, "shape")
            and hasattr(metadata, "dtype")
            and not isinstance(metadata, (numpy.dtype, type))
        ):
            self._metadata = ArrayMetadata.from_arraylike(metadata)
        else:
            self._metadata = as_numpy_dtype(metadata)

    def as_array_metadata(self) -> ArrayMetadata:
        if isinstance(self._metadata, ArrayMetadata):
            return self._metadata
        raise ValueError("This is a scalar type")

    array_metadata = property(as_array_metadata)

    @property
    def dtype(self) -> numpy.dtype:
        return self._metadata.dtype if isinstance(self._metadata, ArrayMetadata) else self._metadata

    @property
    def shape(self) -> tuple[int, ...]:
        return self.as_array_metadata().shape

    @property
    def strides(self) -> tuple[int, ...]:
        return self.as_array_metadata().strides

    @property
    def offset(self) -> int:
        return self.as_array_metadata().first_element_offset

    def is_scalar(self) -> bool:
        return isinstance(self._metadata, numpy.dtype)

    def is_array(self) -> bool:
        return not self.is_scalar()

    def __eq__(self, other):
        return isinstance(other, Type) and self._metadata == other._metadata

    def __hash__(self):
        return hash((Type, self._metadata))

    def compatible_with(self, other: Type) -> bool:
        if self.is_scalar() or other.is_scalar():
            return self.is_scalar() and other.is_scalar() and self._metadata == other._metadata
        a, b = self._metadata, other._metadata
        if a.dtype != b.dtype:
            return False
        n = min(len(a.shape), len(b.shape))
        if a.shape[len(a.shape) - n :] != b.shape[len(b.shape) - n :]:
            return False
        if a.strides[len(a.strides) - n :] != b.strides[len(b.strides) - n :]:
            return False
        if any(s != 1 for s in a.shape[: len(a.shape) - n]) or any(s != 1 for s in b.shape[: len(b.shape) - n]):
            return False
        return a.first_element_offset == b.first_element_offset

    def with_dtype(self, dtype) -> Type:
        if self.is_array():
            return Type(self._metadata.with_(dtype=dtype))
        return Type(dtype)

    @classmethod
    def from_value(cls, val) -> Type:
        if isinstance(val, Type):
            return cls(val)
        if isinstance(val, numpy.dtype) or (isinstance(val, type) and issubclass(val, numpy.generic)):
            return cls(numpy.dtype(val))
        if hasattr(val, "shape") and hasattr(val, "dtype"):
            return cls(ArrayMetadata.from_arraylike(val))
        return cls(_result_type(val))

    def cast_scalar(self, val):
        if not self.is_scalar():
            raise ValueError("Can only cast scalars to a scalar type, this is an array")
        return numpy.asarray(val, dtype=self.dtype).flat[0]

    def __repr__(self):
        return f"Type({self._metadata})"


class Annotation(Type):
    """Computation parameter annotation with a role: ``'i'``, ``'o'``, ``'io'`` or ``'s'``."""

    def __init__(self, type_, role: str | None = None, *, constant: bool = False):
        super().__init__(type_)
        if role is None:
            role = "s" if self.is_scalar() else ("i" if constant else "io")
        if role not in ("i", "o", "io", "s"):
            raise ValueError(f"Invalid role: {role}")
        self.role = role
        self.constant = constant
        if role == "s":
            if not self.is_scalar():
                raise ValueError("Only scalars can have the scalar role")
            self.input = False
            self.output = False
        else:
            if self.is_scalar():
                raise ValueError("Scalars cannot have input or output role")
            self.input = "i" in role
            self.output = "o" in role

    def can_be_argument_for(self, annotation: Annotation) -> bool:
        if not self.compatible_with(annotation):
            return False
        return self.role == annotation.role or (self.role == "io" and annotation.is_array())

    def _as_type(self) -> Type:
        return Type(self)

    def __repr__(self):
        return f"Annotation({self._metadata}, role={self.role}{', constant' if self.constant else ''})"


class Parameter(inspect.Parameter):
    """A named, annotated computation parameter (scalars may have defaults)."""

    def __init__(self, name: str, annotation: Annotation, default: Any = inspect.Parameter.empty):
        if default is not inspect.Parameter.empty:
            if annotation.is_array():
                raise ValueError("Array parameters cannot have default values")
            default = annotation.cast_scalar(default)
        inspect.Parameter.__init__(
            self, name, inspect.Parameter.POSITIONAL_OR_KEYWORD, default=default, annotation=annotation
        )

    def rename(self, new_name: str) -> Parameter:
        return Parameter(new_name, self.annotation, default=self.default)


class Signature(inspect.Signature):
    """Ordered parameters of a computation."""

    def __init__(self, parameters: Sequence[Parameter]):
        inspect.Signature.__init__(self, parameters)

    def bind_with_defaults(self, args: tuple, kwds: Mapping[str, Any], *, cast: bool = False):
        bound = self.bind(*args, **kwds)
        for param in self.parameters.values():
            if param.name not in bound.arguments:
                bound.arguments[param.name] = param.default
            elif cast and param.annotation.is_scalar():
                bound.arguments[param.name] = param.annotation.cast_scalar(bound.arguments[param.name])
        return bound
