"""Computation base class and compiled callables.

Mirrors ``reikna.core.computation`` (reikna/core/computation.py:115-801): a
``Computation`` has a signature of root parameters, ``parameter.<name>.connect(...)``
attaches transformations (returning the computation), and ``compile(device)``
returns a callable taking ``(stream, *args, **kwds)`` bound by signature.

Execution model here: ``compile`` builds native plans (C ABI, sm_100a kernels) and
the callable enqueues them asynchronously on a CUDA stream (``None`` = the current
torch stream), like reikna's queue-ordered kernel calls.
"""

from __future__ import annotations

import weakref
from collections.abc import Callable, Iterable
from typing import Any

import numpy

from .signature import Parameter, Signature, Type, as_numpy_dtype
from .transformation import Transformation, TransformationParameter, TransformationTree


def _check_external_name(name: str) -> None:
    if name.startswith("_"):
        raise ValueError("External parameter name cannot start with the underscore.")


class ComputationParameter(Type):
    """A typed computation parameter; ``connect`` is a shortcut for ``Computation.connect``."""

    def __init__(self, computation, name: str, type_: Type):
        super().__init__(type_)
        self._computation = weakref.ref(computation)
        self._name = name

    def belongs_to(self, comp) -> bool:
        return self._computation() is comp

    def connect(self, _trf: Transformation, _tr_connector, **tr_from_comp) -> Computation:
        return self._computation().connect(self._name, _trf, _tr_connector, **tr_from_comp)

    def __str__(self):
        return self._name


class ParameterContainer:
    def __init__(self, parent, parameters: Iterable[Parameter]):
        self._param_objs = {p.name: ComputationParameter(parent, p.name, p.annotation) for p in parameters}

    def __getattr__(self, name: str) -> ComputationParameter:
        try:
            return self._param_objs[name]
        except KeyError as exc:
            raise AttributeError(name) from exc


class Computation:
    """Base class of computations (see ``reikna.core.Computation``)."""

    def __init__(self, root_parameters: Iterable[Parameter]):
        root_parameters = list(root_parameters)
        for p in root_parameters:
            _check_external_name(p.name)
        self._original_parameters = root_parameters
        self._tr_tree = TransformationTree(root_parameters)
        self._update_attributes()

    def _update_attributes(self) -> None:
        leaves = self._tr_tree.get_leaf_parameters()
        self.signature = Signature(leaves)
        self.parameter = ParameterContainer(self, leaves)

    def connect(self, _comp_connector, _trf: Transformation, _tr_connector, **tr_from_comp) -> Computation:
        """Attach transformation ``_trf`` to parameter ``_comp_connector`` (see reikna)."""
        if isinstance(_comp_connector, ComputationParameter) and not _comp_connector.belongs_to(self):
            raise ValueError("The connection target must belong to this computation.")
        param_name = str(_comp_connector)
        if param_name in tr_from_comp:
            raise ValueError(
                "Parameter '" + param_name + "' cannot be supplied "
                "both as the main connector and one of the child connections"
            )
        tr_from_comp[param_name] = _tr_connector
        comp_from_tr = {}
        for comp_name, tr_conn in tr_from_comp.items():
            _check_external_name(comp_name)
            if isinstance(tr_conn, TransformationParameter) and not tr_conn.belongs_to(_trf):
                raise ValueError("The transformation parameter must belong to the provided transformation")
            comp_from_tr[str(tr_conn)] = comp_name
        self._tr_tree.connect(param_name, _trf, comp_from_tr)
        self._update_attributes()
        return self

    def compile(self, device=None, **kwds) -> ComputationCallable:
        """Plan and build the native kernels on ``device`` (torch device, index or None)."""
        import torch

        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        elif isinstance(device, int):
            device = torch.device("cuda", device)
        elif not isinstance(device, torch.device):
            device = torch.device(device)
        if device.type != "cuda":
            raise ValueError("reikna_b200 computations run on CUDA devices only")
        with torch.cuda.device(device):
            runner = self._build_runner(device, **kwds)
        return ComputationCallable(device, self._tr_tree.get_leaf_parameters(), runner)

    def _build_runner(self, device, **kwds) -> Callable:
        raise NotImplementedError


def stream_handle(stream) -> int:
    """cudaStream_t of ``stream``: None (current torch stream), torch stream or int."""
    import torch

    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    if hasattr(stream, "handle"):
        return int(stream.handle)
    raise TypeError(f"cannot interpret {stream!r} as a CUDA stream")


def array_pointer(arr, annotation) -> int:
    """Device pointer of a CUDA array argument after checking it against its annotation."""
    if not (hasattr(arr, "data_ptr") and hasattr(arr, "is_cuda")):
        raise TypeError(f"expected a CUDA tensor, got {type(arr).__name__}")
    if not arr.is_cuda:
        raise ValueError("array arguments must live on a CUDA device")
    dt = as_numpy_dtype(arr.dtype)
    if dt != annotation.dtype:
        raise ValueError(f"dtype mismatch: got {dt}, expected {annotation.dtype}")
    if tuple(arr.shape) != tuple(annotation.shape):
        raise ValueError(f"shape mismatch: got {tuple(arr.shape)}, expected {tuple(annotation.shape)}")
    strides = tuple(s * dt.itemsize for s in arr.stride())
    for s, e, n in zip(strides, annotation.strides, annotation.shape):
        if n > 1 and s != e:
            raise ValueError(f"stride mismatch: got {strides}, expected {annotation.strides}")
    return int(arr.data_ptr())


class ComputationCallable:
    """A compiled computation: ``callable(stream, *args, **kwds)``; asynchronous."""

    def __init__(self, device, parameters, runner):
        self.device = device
        self.signature = Signature(parameters)
        self.parameter = ParameterContainer(self, parameters)
        self._runner = runner

    def __call__(self, stream, *args, **kwds):
        bound = self.signature.bind_with_defaults(args, kwds, cast=True)
        return self._runner(stream_handle(stream), bound.arguments)

    @property
    def launches(self) -> int:
        return getattr(self._runner, "launches", 0)


def scalar_value(v) -> complex:
    return complex(numpy.asarray(v).item())
