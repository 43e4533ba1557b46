"""Transformations and the transformation tree of a computation.

Same public contract as ``reikna.core.transformation`` (reikna/core/transformation.py:42-553):
a ``Transformation`` is an element-wise map between arrays with parameters of roles
``'i'``/``'o'``/``'s'``; connecting one to a computation parameter rewrites the
computation signature depth-first, keeping the order of parameters at each
branching level (reikna/core/computation.py:177-188).

Difference by design: reikna transformations carry Mako/C snippets that are inlined
into every kernel.  Here the built-in transformations carry an operation descriptor
(``op``) that the FFT planner folds into the first-load / last-store stage of its
CUDA passes.  A transformation built from a code string alone has no descriptor and
cannot be compiled into a plan (``compile`` raises ``NotImplementedError``).
"""

from __future__ import annotations

import weakref
from collections.abc import Callable, Iterable, Mapping, Sequence
from typing import Any

from .signature import Annotation, Parameter, Signature, Type


class TransformationParameter(Type):
    """A typed transformation parameter; usable wherever array metadata is needed."""

    def __init__(self, trf: Transformation, name: str, type_: Type):
        super().__init__(type_)
        self._trf = weakref.ref(trf)
        self._name = name

    def belongs_to(self, trf: Transformation) -> bool:
        return self._trf() is trf

    def __str__(self):
        return self._name


class _ParamContainer:
    def __init__(self, parent, parameters: Iterable[Parameter]):
        self._param_objs = {p.name: TransformationParameter(parent, p.name, p.annotation) for p in parameters}

    def __getattr__(self, name: str) -> TransformationParameter:
        try:
            return self._param_objs[name]
        except KeyError as exc:
            raise AttributeError(name) from exc


class Transformation:
    """An element-wise transformation of arrays.

    :param parameters: list of :py:class:`Parameter`; ``'io'`` roles are not allowed.
    :param code: optional source text (kept for reference; not compiled).
    :param render_kwds: kept with the code.
    :param connectors: parameter names usable as connection points (default: arrays).
    :param op: operation descriptor understood by the FFT planner.
    """

    def __init__(
        self,
        parameters: Sequence[Parameter],
        code: str | None = None,
        render_kwds: Mapping[str, Any] | None = None,
        connectors: Sequence[str] | None = None,
        op: Mapping[str, Any] | None = None,
    ):
        for param in parameters:
            if param.annotation.input and param.annotation.output:
                raise ValueError(f"Transformation cannot have 'io' parameters ('{param.name}')")
        self.signature = Signature(parameters)
        for param in self.signature.parameters.values():
            setattr(self, param.name, TransformationParameter(self, param.name, param.annotation))
        self.parameter = _ParamContainer(self, parameters)
        self.connectors = (
            list(connectors) if connectors is not None else [p.name for p in parameters if p.annotation.is_array()]
        )
        self.code = code
        self.render_kwds = dict(render_kwds or {})
        self.op = dict(op) if op is not None else None


class Node:
    """A node of the transformation tree: at most one input and one output transformation."""

    def __init__(self, input_ntr=None, output_ntr=None):
        self.input_ntr = input_ntr
        self.output_ntr = output_ntr

    def connect(self, ntr: NodeTransformation) -> Node:
        if ntr.output:
            return Node(input_ntr=self.input_ntr, output_ntr=ntr)
        return Node(input_ntr=ntr, output_ntr=self.output_ntr)

    def get_child_names(self) -> tuple[list[str], list[str]]:
        def names(ntr):
            return ([], []) if ntr is None else ntr.get_child_names()

        ob, oa = names(self.output_ntr)
        ib, ia = names(self.input_ntr)
        if self.output_ntr is None and self.input_ntr is None:
            return [], []
        if self.output_ntr is None:
            return ib, ia
        if self.input_ntr is None:
            return ob, oa
        return ob + oa, ib + ia

    def get_connections(self) -> list[NodeTransformation]:
        return [n for n in (self.output_ntr, self.input_ntr) if n is not None]


class NodeTransformation:
    """An edge of the tree: a transformation attached to node ``connector_node_name``."""

    def __init__(self, connector_node_name: str, trf: Transformation, node_from_tr: Mapping[str, str]):
        self.trf = trf
        self.connector_node_name = connector_node_name
        self.node_from_tr = dict(node_from_tr)
        given = set(self.node_from_tr)
        available = set(trf.signature.parameters)
        if given != available:
            raise ValueError(
                f"Supplied transformation names {sorted(given)} "
                f"do not fully coincide with the existing ones: {sorted(available)}"
            )
        tr_conn = [t for t, n in self.node_from_tr.items() if n == connector_node_name]
        if len(tr_conn) != 1:
            raise ValueError("There should be only one transformation parameter corresponding to the connector node")
        self.tr_connector = tr_conn[0]
        # an output transformation consumes the node (its connector is one of its inputs)
        self.output = trf.signature.parameters[self.tr_connector].annotation.input

    def get_child_names(self) -> tuple[list[str], list[str]]:
        names = [self.node_from_tr[p] for p in self.trf.signature.parameters]
        i = names.index(self.connector_node_name)
        return names[:i], names[i + 1 :]

    def translate_node_names(self, translator: Callable[[str], str]) -> NodeTransformation:
        return NodeTransformation(
            translator(self.connector_node_name),
            self.trf,
            {t: translator(n) for t, n in self.node_from_tr.items()},
        )


class TransformationTree:
    """The tree of transformations attached to a computation's root parameters."""

    def __init__(self, root_parameters: Iterable[Parameter]):
        self.root_names: list[str] = []
        self.root_parameters: dict[str, Parameter] = {}
        self.nodes: dict[str, Node] = {}
        self.leaf_parameters: dict[str, Parameter] = {}
        for param in root_parameters:
            self.root_names.append(param.name)
            if param.name in self.root_parameters and param != self.root_parameters[param.name]:
                old = self.root_parameters[param.name]
                if old.annotation._as_type() != param.annotation._as_type():
                    raise ValueError(f"Type mismatch for two parameters with name `{param.name}`")
                if old.default != param.default:
                    raise ValueError(f"Default value mismatch for two parameters with name `{param.name}`")
                merged = Parameter(param.name, Annotation(param.annotation, "io"), default=param.default)
                self.root_parameters[param.name] = merged
                self.leaf_parameters[param.name] = merged
            else:
                self.nodes[param.name] = Node()
                self.root_parameters[param.name] = param
                self.leaf_parameters[param.name] = param

    def _subtree_names(self, names: Sequence[str], ignore: set, visited: set, leaves_only: bool) -> list[str]:
        result: list[str] = []
        for i, name in enumerate(names):
            if name in ignore or name in visited:
                continue
            visited.add(name)
            ignore_children = set(names[i + 1 :])
            before, after = self.nodes[name].get_child_names()
            sub_before = self._subtree_names(before, ignore_children, visited, leaves_only)
            sub_after = self._subtree_names(after, ignore_children, visited, leaves_only)
            if not leaves_only:
                result.append(name)
            result += sub_before
            if leaves_only and name in self.leaf_parameters:
                result.append(name)
            result += sub_after
        return result

    def get_subtree_names(self, root_names: Sequence[str] | None = None, *, leaves_only: bool = False) -> list[str]:
        if root_names is None:
            root_names = self.root_names
        return self._subtree_names(list(root_names), set(), set(), leaves_only)

    def get_root_parameters(self) -> list[Parameter]:
        return [self.root_parameters[n] for n in self.root_names]

    def get_leaf_parameters(self, root_names: Sequence[str] | None = None) -> list[Parameter]:
        return [self.leaf_parameters[n] for n in self.get_subtree_names(root_names, leaves_only=True)]

    def _connect(self, ntr: NodeTransformation) -> None:
        for tr_param in ntr.trf.signature.parameters.values():
            node_name = ntr.node_from_tr[tr_param.name]
            if node_name == ntr.connector_node_name:
                ann = self.leaf_parameters[node_name].annotation
                if ann.input and ann.output:
                    self.leaf_parameters[node_name] = Parameter(node_name, Annotation(ann, "i" if ntr.output else "o"))
                else:
                    del self.leaf_parameters[node_name]
            elif node_name in self.leaf_parameters and self.leaf_parameters[node_name].annotation.is_array():
                ann = self.leaf_parameters[node_name].annotation
                if (ann.input and ntr.output) or (ann.output and not ntr.output):
                    self.leaf_parameters[node_name] = Parameter(node_name, Annotation(ann, "io"))
            else:
                self.leaf_parameters[node_name] = tr_param.rename(node_name)
            if node_name not in self.nodes:
                self.nodes[node_name] = Node()
        self.nodes[ntr.connector_node_name] = self.nodes[ntr.connector_node_name].connect(ntr)

    def connect(self, comp_connector: str, trf: Transformation, comp_from_tr: Mapping[str, str]) -> None:
        ntr = NodeTransformation(comp_connector, trf, comp_from_tr)
        for tr_name, node_name in comp_from_tr.items():
            if node_name not in self.leaf_parameters:
                if node_name == comp_connector:
                    raise ValueError("Parameter '" + node_name + "' is not a part of the signature")
                if node_name in self.nodes:
                    raise ValueError("Parameter '" + node_name + "' is hidden by transformations")
                continue
            node_ann = self.leaf_parameters[node_name].annotation
            tr_ann = trf.signature.parameters[tr_name].annotation
            if tr_ann._as_type() != node_ann._as_type():
                raise ValueError(
                    "Incompatible types of the transformation parameter "
                    f"'{tr_name}' ({tr_ann}) and the node '{node_name}' ({node_ann})"
                )
            if not tr_ann.is_array():
                continue
            if node_name == comp_connector:
                if ntr.output and not node_ann.output:
                    raise ValueError("'" + node_name + "' is not an output node")
                if not ntr.output and not node_ann.input:
                    raise ValueError("'" + node_name + "' is not an input node")
            elif ntr.output and node_ann.output:
                raise ValueError(
                    f"Cannot connect transformation parameter '{tr_name}' to an existing output node '{node_name}'"
                )
        self._connect(ntr)

    def connections(self):
        for name in self.get_subtree_names(leaves_only=False):
            yield from self.nodes[name].get_connections()
