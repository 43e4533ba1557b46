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

import inspect
import weakref
from collections.abc import Callable, Iterable
from typing import Any

import numpy

from .signature import Annotation, Parameter, Signature, Type, as_numpy_dtype
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

    def compile(self, device=None, compiler_options=(), *, fast_math: bool = False, keep: bool = False,
                **kwds) -> ComputationCallable:
        """Plan and build the native kernels on ``device`` (torch device, index or None).

        ``compiler_options``, ``fast_math`` and ``keep`` are reikna's compile options
        (reikna/core/computation.py:259-287); they apply to the kernels this library
        compiles at run time (user transformations), the prebuilt ones ignore them.
        Other keywords (``flags``) go to the native planner."""
        import torch

        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        elif isinstance(device, int):
            device = torch.device("cuda", device)
        elif not isinstance(device, torch.device):
            device = torch.device(device)
        if device.type != "cuda":
            raise ValueError("reikna_b200 computations run on CUDA devices only")
        self._compile_options = {"compiler_options": list(compiler_options), "fast_math": bool(fast_math),
                                 "keep": bool(keep)}
        with torch.cuda.device(device):
            if type(self)._build_plan is not Computation._build_plan:
                return self._compile_plan(device, **kwds)
            runner = self._build_runner(device, **kwds)
        return ComputationCallable(device, self._tr_tree.get_leaf_parameters(), runner)

    def _build_runner(self, device, **kwds) -> Callable:
        raise NotImplementedError

    # -- computations composed of other computations (reikna's ComputationPlan) ------
    def _build_plan(self, plan_factory, device_params, args) -> ComputationPlan:
        """Derived classes that compose other computations override this (see
        reikna/core/computation.py:289-308): record temporaries and nested computation
        calls on ``plan_factory()`` and return the plan."""
        raise NotImplementedError

    def _compile_plan(self, device, **kwds) -> ComputationCallable:
        for name, node in self._tr_tree.nodes.items():
            if node.input_ntr is not None or node.output_ntr is not None:
                if name in {p.name for p in self._original_parameters}:
                    raise NotImplementedError(
                        "transformations connected to a computation built from nested calls; connect them to "
                        "the nested computations instead")
        args = KernelArguments({p.name: KernelArgument(p.name, p.annotation) for p in self._original_parameters})
        plan = self._build_plan(lambda: ComputationPlan(self, device, kwds), DeviceParameters(device), args)
        if not isinstance(plan, ComputationPlan):
            raise TypeError("_build_plan() must return the plan it was given")
        return plan.finalize()


def _current_raw_stream() -> int:
    import torch

    get = getattr(torch._C, "_cuda_getCurrentRawStream", None)
    if get is not None:
        return int(get(torch.cuda.current_device()))
    return torch.cuda.current_stream().cuda_stream


def stream_handle(stream) -> int:
    """cudaStream_t of ``stream``: None (current torch stream), torch stream or int."""
    if stream is None:
        return _current_raw_stream()
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    if hasattr(stream, "handle"):
        return int(stream.handle)
    raise TypeError(f"cannot interpret {stream!r} as a CUDA stream")


class ArrayCheck:
    """The expected torch dtype, shape and element strides of an array parameter, for
    a cheap per-call check (``array_pointer`` gives the detailed error otherwise)."""

    def __init__(self, annotation):
        from .signature import _torch_dtype_map

        self.annotation = annotation
        inv = {v: k for k, v in _torch_dtype_map().items()}
        self.tdtype = inv.get(numpy.dtype(annotation.dtype))
        self.shape = tuple(annotation.shape)
        isz = numpy.dtype(annotation.dtype).itemsize
        self.strides = tuple(st // isz for st in annotation.strides)

    def __call__(self, arr) -> int:
        try:
            if arr.is_cuda and arr.dtype == self.tdtype and arr.shape == self.shape and arr.stride() == self.strides:
                return arr.data_ptr()
        except AttributeError:
            pass
        return array_pointer(arr, self.annotation)


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
        # positional calls bind without inspect.Signature.bind (per-call host cost)
        params = list(self.signature.parameters.values())
        self._names = [p.name for p in params]
        self._defaults = [p.default for p in params]
        self._scalar_dt = [p.annotation.dtype if p.annotation.is_scalar() else None for p in params]
        self._required = sum(1 for p in params if p.default is inspect.Parameter.empty)

    def _bind_positional(self, args) -> dict | None:
        n = len(args)
        if n < self._required or n > len(self._names):
            return None
        out = {}
        for i, name in enumerate(self._names):
            if i < n:
                v = args[i]
                dt = self._scalar_dt[i]
                if dt is not None:
                    v = numpy.asarray(v, dtype=dt).flat[0]
                out[name] = v
            else:
                d = self._defaults[i]
                if d is inspect.Parameter.empty:
                    return None
                out[name] = d
        return out

    def __call__(self, stream, *args, **kwds):
        bound = None if kwds else self._bind_positional(args)
        if bound is None:
            bound = self.signature.bind_with_defaults(args, kwds, cast=True).arguments
        return self._runner(stream_handle(stream), bound)

    @property
    def launches(self) -> int:
        return getattr(self._runner, "launches", 0)


def scalar_value(v) -> complex:
    return complex(numpy.asarray(v).item())


# ---- nested computations ---------------------------------------------------------------


class DeviceParameters:
    """What ``_build_plan`` learns about the device (grunnur's DeviceParameters
    subset that host-side planning uses)."""

    def __init__(self, device):
        import torch

        pr = torch.cuda.get_device_properties(device)
        self.device = device
        self.api_id = "cuda"
        self.warp_size = 32
        self.max_total_local_size = 1024
        self.local_mem_size = 227 * 1024
        self.compute_units = pr.multi_processor_count
        self.type = "gpu"


class KernelArgument(Type):
    """A value a plan passes to a nested call: a root parameter of the computation,
    a temporary, a persistent array or a persistent scalar."""

    def __init__(self, name: str, type_):
        super().__init__(type_)
        self.name = name

    def __repr__(self):
        return f"KernelArgument({self.name})"


class KernelArguments:
    def __init__(self, args):
        self._args = dict(args)

    def all(self):
        return self._args.values()

    def __getattr__(self, name: str) -> KernelArgument:
        try:
            return self._args[name]
        except KeyError as exc:
            raise AttributeError(name) from exc


class ComputationPlan:
    """Recorder of a composed computation (reikna/core/computation.py:346-640):
    temporaries, persistent and constant arrays, and nested computation calls, run
    in order on the caller's stream.  Each nested computation is compiled for the
    device when it is recorded; a temporary is allocated once when the plan is
    finalized and lives as long as the compiled callable."""

    def __init__(self, owner: Computation, device, kwds):
        self._owner = owner
        self._device = device
        self._kwds = dict(kwds)
        self._annotations = {p.name: p.annotation for p in owner._original_parameters}
        self._temps: dict[str, Annotation] = {}
        self._values: dict[str, Any] = {}
        self._calls: list[tuple[ComputationCallable, list[str]]] = []
        self._ids = {"temp": 0, "value": 0}

    def _new(self, kind: str) -> str:
        self._ids[kind] += 1
        return f"_{kind}{self._ids[kind]}"

    def temp_array(self, shape, dtype, strides=None, offset: int = 0, nbytes=None) -> KernelArgument:
        from .signature import ArrayMetadata

        shape = (shape,) if isinstance(shape, int) else tuple(shape)
        meta = ArrayMetadata(shape, dtype, strides=strides, first_element_offset=offset, buffer_size=nbytes)
        name = self._new("temp")
        ann = Annotation(meta, "io")
        self._annotations[name] = ann
        self._temps[name] = ann
        return KernelArgument(name, ann)

    def temp_array_like(self, arr) -> KernelArgument:
        from .signature import ArrayMetadata

        meta = arr.as_array_metadata() if hasattr(arr, "as_array_metadata") else ArrayMetadata.from_arraylike(arr)
        return self.temp_array(meta.shape, meta.dtype, strides=meta.strides, offset=meta.first_element_offset,
                               nbytes=meta.buffer_size)

    def persistent_array(self, arr) -> KernelArgument:
        import torch

        from .signature import ArrayMetadata

        t = torch.as_tensor(numpy.ascontiguousarray(arr)).to(self._device)
        name = self._new("value")
        ann = Annotation(ArrayMetadata.from_arraylike(t), "i")
        self._annotations[name] = ann
        self._values[name] = t
        return KernelArgument(name, ann)

    constant_array = persistent_array

    def _scalar(self, annotation, value) -> KernelArgument:
        name = self._new("value")
        ann = Annotation(annotation.dtype)
        self._annotations[name] = ann
        self._values[name] = annotation.cast_scalar(value)
        return KernelArgument(name, ann)

    def computation_call(self, computation: Computation, *args, **kwds) -> None:
        """Add a call of ``computation`` with ``args``: plan arguments, or scalars
        (kept as persistent values)."""
        sig = computation.signature
        bound = sig.bind_with_defaults(args, kwds, cast=False)
        names = []
        for arg, param in zip(bound.args, sig.parameters.values()):
            if not isinstance(arg, KernelArgument):
                if param.annotation.is_array():
                    raise ValueError("Ad hoc arguments are only allowed for scalar parameters")
                arg = self._scalar(param.annotation, arg)
            ann = self._annotations.get(arg.name)
            if ann is None:
                raise ValueError(f"'{arg.name}' is not an argument of this plan")
            if not ann.can_be_argument_for(param.annotation):
                raise ValueError(f"Got {ann} for '{param.name}', expected {param.annotation}")
            names.append(arg.name)
        opts = getattr(self._owner, "_compile_options", {})
        cc = computation.compile(self._device, opts.get("compiler_options", ()), fast_math=opts.get("fast_math", False),
                                 keep=opts.get("keep", False), **self._kwds)
        self._calls.append((cc, names))

    def kernel_call(self, template_def, args, global_size, local_size=None, render_kwds=None,
                    kernel_name="_kernel_func"):
        raise NotImplementedError(
            "kernel_call: this library runs prebuilt sm_100a kernels; compose computations with computation_call")

    def finalize(self) -> ComputationCallable:
        import torch

        internal = dict(self._values)
        for name, ann in self._temps.items():
            meta = ann.as_array_metadata()
            isz = meta.dtype.itemsize
            span = meta.first_element_offset + sum((n - 1) * st for n, st in zip(meta.shape, meta.strides)) + isz
            nbytes = max(meta.buffer_size or 0, span)
            buf = torch.empty(nbytes, dtype=torch.uint8, device=self._device)
            from .signature import _torch_dtype_map

            tdt = {v: k for k, v in _torch_dtype_map().items()}[numpy.dtype(meta.dtype)]
            internal[name] = torch.as_strided(buf.view(tdt), meta.shape, [st // isz for st in meta.strides],
                                              meta.first_element_offset // isz)
        calls = self._calls

        def runner(stream: int, args):
            vals = dict(internal)
            vals.update(args)
            ext = torch.cuda.ExternalStream(stream) if stream else None
            for cc, names in calls:
                cc(ext, *[vals[n] for n in names])

        runner.launches = sum(cc.launches for cc, _ in calls)
        runner.internal = internal
        return ComputationCallable(self._device, self._owner._tr_tree.get_leaf_parameters(), runner)
