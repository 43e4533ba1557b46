"""Fold the transformations attached to an FFT's ``input``/``output`` into edge ops.

reikna inlines transformation snippets into the first kernel's loads and the last
kernel's stores (reikna/core/transformation.py:460-518,
reikna/core/transformation_modules.py:260-318).  Here the chain of built-in
transformations hanging off the root parameter is reduced to one ``rk_edge``: user
array layout (strides, offset, bounds), element format, index remap (fftshift),
complex scale (constants and runtime scalars), window, and a norm post-op.  The
native kernels apply that edge on the first load / last store of the plan.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy

from .. import _native as N
from ..core.signature import ArrayMetadata


@dataclass
class EdgeSpec:
    ndim: int
    arrays: list[str] = field(default_factory=list)          # leaf names (1, or 2 for pairs)
    metas: list[ArrayMetadata] = field(default_factory=list)
    kind: str = "complex"                                     # complex | real | pair
    shape: list[int] = field(default_factory=list)            # user extent along each FFT dim
    strides: list[int] = field(default_factory=list)          # element strides per FFT dim
    strides2: list[int] = field(default_factory=list)
    shift: list[int] = field(default_factory=list)
    scale: complex = 1.0 + 0j
    scale_params: list[tuple[str, bool]] = field(default_factory=list)
    window: tuple[int, int] | None = None                     # (axis, length)
    norm: float | None = None
    frame: tuple[int, int] | None = None                      # (step, fft_size)
    crop: tuple[int, ...] | None = None

    def fmt(self) -> int:
        dt = self.metas[0].dtype
        if self.kind == "complex":
            return N.FMT_C64 if dt == numpy.complex64 else N.FMT_C128
        if self.kind == "real":
            return N.FMT_F32 if dt == numpy.float32 else N.FMT_F64
        return N.FMT_F32_PAIR if dt == numpy.float32 else N.FMT_F64_PAIR


def _elem_strides(meta: ArrayMetadata) -> list[int]:
    isz = meta.dtype.itemsize
    out = []
    for s in meta.strides:
        if s % isz:
            raise ValueError("array strides must be multiples of the element size")
        out.append(s // isz)
    return out


def _op(ntr):
    op = ntr.trf.op
    if op is None:
        raise NotImplementedError(
            "transformations defined only by source code cannot be fused into the native FFT passes; "
            "use the built-in transformations of reikna_b200.transformations"
        )
    return op


def _check_supported(kind: str) -> None:
    if kind in ("add", "norm_param", "const_param", "broadcast", "ignore"):
        raise NotImplementedError(f"transformation '{kind}' cannot be fused into the FFT passes")


def fold_input(tree, root: str, fft_shape: tuple[int, ...]) -> EdgeSpec:
    nd = len(fft_shape)
    spec = EdgeSpec(ndim=nd, shape=list(fft_shape), shift=[0] * nd)

    def leaf(name: str):
        param = tree.leaf_parameters[name]
        if not param.annotation.is_array():
            raise ValueError(f"'{name}' must be an array")
        return name, param.annotation.as_array_metadata()

    def walk_real(node: str):
        """Follow a real-valued branch (inside combine / real_to_complex)."""
        ntr = tree.nodes[node].input_ntr
        if ntr is None:
            return leaf(node)
        op = _op(ntr)
        k = op["kind"]
        _check_supported(k)
        if k in ("copy", "cast"):
            return walk_real(ntr.node_from_tr["input"])
        if k == "scale":
            _apply_scale(op, ntr)
            return walk_real(ntr.node_from_tr["input"])
        if k == "window":
            spec.window = (nd - 1, op["size"])
            return walk_real(ntr.node_from_tr["input"])
        if k == "frame":
            if spec.frame is not None:
                raise NotImplementedError("nested framing")
            spec.frame = (op["step"], op["fft_size"])
            return walk_real(ntr.node_from_tr["input"])
        if k == "const":
            return ("const", op["value"])
        raise NotImplementedError(f"transformation '{k}' on a real input branch")

    def _apply_scale(op, ntr):
        if "const" in op:
            spec.scale *= op["const"]
        else:
            spec.scale_params.append((ntr.node_from_tr[op["param"]], op["div"]))

    def walk(node: str):
        ntr = tree.nodes[node].input_ntr
        if ntr is None:
            name, meta = leaf(node)
            spec.arrays = [name]
            spec.metas = [meta]
            spec.kind = "complex"
            return
        op = _op(ntr)
        k = op["kind"]
        _check_supported(k)
        if k in ("copy", "cast"):
            return walk(ntr.node_from_tr["input"])
        if k == "scale":
            _apply_scale(op, ntr)
            return walk(ntr.node_from_tr["input"])
        if k == "window":
            spec.window = (nd - 1, op["size"])
            return walk(ntr.node_from_tr["input"])
        if k == "real_to_complex":
            r = walk_real(ntr.node_from_tr["input"])
            if r[0] == "const":
                raise NotImplementedError("constant FFT input")
            spec.arrays, spec.metas, spec.kind = [r[0]], [r[1]], "real"
            return
        if k == "combine":
            re = walk_real(ntr.node_from_tr["real"])
            im = walk_real(ntr.node_from_tr["imag"])
            if im[0] == "const":
                if im[1] != 0:
                    raise NotImplementedError("combine_complex with a non-zero constant imaginary part")
                if re[0] == "const":
                    raise NotImplementedError("constant FFT input")
                spec.arrays, spec.metas, spec.kind = [re[0]], [re[1]], "real"
                return
            if re[0] == "const":
                raise NotImplementedError("combine_complex with a constant real part")
            spec.arrays, spec.metas, spec.kind = [re[0], im[0]], [re[1], im[1]], "pair"
            return
        raise NotImplementedError(f"transformation '{k}' on the FFT input")

    walk(root)
    meta = spec.metas[0]
    if spec.frame is not None:
        step, fsize = spec.frame
        if len(meta.shape) != 1 or nd != 2:
            raise NotImplementedError("framing expects a 1-D signal and a 2-D FFT array")
        s = _elem_strides(meta)[0]
        spec.strides = [step * s, s]
        spec.shape = [fft_shape[0], min(fsize, fft_shape[1])]
    else:
        if len(meta.shape) != nd:
            raise ValueError("input array rank differs from the FFT array rank")
        spec.strides = _elem_strides(meta)
        spec.shape = list(meta.shape)
    if spec.kind == "pair":
        if spec.metas[1].shape != meta.shape:
            raise ValueError("real and imaginary arrays differ in shape")
        spec.strides2 = _elem_strides(spec.metas[1])
        if spec.strides2 != spec.strides:
            raise NotImplementedError("real and imaginary arrays must share strides")
    return spec


def fold_output(tree, root: str, fft_shape: tuple[int, ...]) -> EdgeSpec:
    nd = len(fft_shape)
    spec = EdgeSpec(ndim=nd, shape=list(fft_shape), shift=[0] * nd)
    state = {"real": False, "transposed": False}

    def leaf(name: str):
        param = tree.leaf_parameters[name]
        if not param.annotation.is_array():
            raise ValueError(f"'{name}' must be an array")
        return name, param.annotation.as_array_metadata()

    def walk(node: str):
        ntr = tree.nodes[node].output_ntr
        if ntr is None:
            name, meta = leaf(node)
            spec.arrays, spec.metas = [name], [meta]
            spec.kind = "real" if state["real"] else "complex"
            return
        op = _op(ntr)
        k = op["kind"]
        _check_supported(k)
        if k in ("copy", "cast"):
            return walk(ntr.node_from_tr["output"])
        if k == "scale":
            if state["real"]:
                raise NotImplementedError("scaling after a norm transformation")
            if "const" in op:
                spec.scale *= op["const"]
            else:
                spec.scale_params.append((ntr.node_from_tr[op["param"]], op["div"]))
            return walk(ntr.node_from_tr["output"])
        if k == "transpose":
            if nd != 2:
                raise NotImplementedError("transpose_2d expects a 2-D FFT array")
            state["transposed"] = not state["transposed"]
            return walk(ntr.node_from_tr["output"])
        if state["transposed"] and k in ("shift", "crop"):
            raise NotImplementedError(f"transformation '{k}' after transpose_2d")
        if k == "shift":
            for a in op["axes"]:
                n = fft_shape[a]
                s = (n + 1) // 2 if op["inverse"] else n // 2
                spec.shift[a] = (spec.shift[a] + s) % n
            return walk(ntr.node_from_tr["output"])
        if k == "crop":
            if nd != 2:
                raise NotImplementedError("crop_frequencies expects a 2-D FFT array")
            spec.crop = (fft_shape[0], fft_shape[1] // 2 + 1)
            return walk(ntr.node_from_tr["output"])
        if k == "norm":
            if state["real"]:
                raise NotImplementedError("repeated norm")
            state["real"] = True
            spec.norm = op["order"]
            return walk(ntr.node_from_tr["output"])
        if k == "split":
            if state["real"]:
                raise NotImplementedError("split_complex after a norm")
            r = leaf(ntr.node_from_tr["real"])
            i = leaf(ntr.node_from_tr["imag"])
            for nm in (ntr.node_from_tr["real"], ntr.node_from_tr["imag"]):
                if tree.nodes[nm].output_ntr is not None:
                    raise NotImplementedError("transformations after split_complex")
            spec.arrays, spec.metas, spec.kind = [r[0], i[0]], [r[1], i[1]], "pair"
            return
        raise NotImplementedError(f"transformation '{k}' on the FFT output")

    walk(root)
    meta = spec.metas[0]
    if len(meta.shape) != nd:
        raise ValueError("output array rank differs from the FFT array rank")
    spec.strides = _elem_strides(meta)
    spec.shape = list(meta.shape)
    if state["transposed"]:
        # FFT element (i, j) lands at user element (j, i)
        spec.strides = spec.strides[::-1]
        spec.shape = spec.shape[::-1]
    if spec.crop is not None:
        spec.shape = [min(a, b) for a, b in zip(spec.shape, spec.crop)]
    if spec.kind == "pair":
        spec.strides2 = _elem_strides(spec.metas[1])
        if state["transposed"]:
            spec.strides2 = spec.strides2[::-1]
        if spec.strides2 != spec.strides:
            raise NotImplementedError("real and imaginary arrays must share strides")
    return spec


def edge_struct(spec: EdgeSpec, slots: dict[str, int]) -> N.Edge:
    e = N.Edge()
    e.format = spec.fmt()
    e.ndim = spec.ndim
    for i in range(spec.ndim):
        e.shape[i] = spec.shape[i]
        e.strides[i] = spec.strides[i]
        e.strides2[i] = spec.strides2[i] if spec.strides2 else spec.strides[i]
        e.shift[i] = spec.shift[i]
    isz = spec.metas[0].dtype.itemsize
    e.offset = spec.metas[0].first_element_offset // isz
    e.offset2 = spec.metas[1].first_element_offset // isz if len(spec.metas) > 1 else 0
    e.scale_re = spec.scale.real
    e.scale_im = spec.scale.imag
    e.scale_slot = -1
    e.scale_div_slot = -1
    mul = [p for p, d in spec.scale_params if not d]
    div = [p for p, d in spec.scale_params if d]
    if len(mul) > 1 or len(div) > 1:
        raise NotImplementedError("more than one runtime scale parameter per side")
    if mul:
        e.scale_slot = slots[mul[0]]
    if div:
        e.scale_div_slot = slots[div[0]]
    e.post = N.POST_NORM if spec.norm is not None else N.POST_NONE
    e.post_param = spec.norm if spec.norm is not None else 2.0
    if spec.window is not None:
        e.window = N.WIN_HANN
        e.window_axis = spec.window[0]
        e.window_len = spec.window[1]
    return e
