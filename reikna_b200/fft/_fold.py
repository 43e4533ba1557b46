"""Fold the transformations attached to an FFT's ``input``/``output`` into edge ops.

reikna inlines transformation snippets into the first kernel's loads and the last
kernel's stores (reikna/core/transformation.py:460-518,
reikna/core/transformation_modules.py:260-318).  Here the chain of built-in
transformations hanging off the root parameter is reduced to one ``rk_edge``: user
array layout (strides, offset, bounds, broadcasting), element format, index remap
(fftshift, transpose, crop), an affine value map ``scale * value + add`` built from
constants and runtime scalars, a window, and a norm post-op (constant or runtime
order).  The native kernels apply that edge on the first load / last store of the
plan.  Transformations defined by source code instead of a built-in descriptor are
compiled into those passes by :mod:`reikna_b200.fft.user`.

Every element-wise op of reikna's built-in set (reikna/transformations.py:11-347) is
an affine map of the element (copy, cast, mul/div/add by a constant or a scalar
parameter), a norm (norm_const / norm_param), a constant source (broadcast_const /
broadcast_param), a broadcasting copy (copy_broadcasted) or a sink (ignore).  A chain
of affine maps composes into one affine map whose coefficients are monomials (and a
sum of monomials for the additive term) in the runtime scalars; when a coefficient
involves a runtime scalar its value is computed per call and handed to the native
call in an extra scalar slot.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy

from .. import _native as N
from ..core.signature import ArrayMetadata


# ---- monomials in the runtime scalars ------------------------------------------------


@dataclass(frozen=True)
class Mono:
    """``const * prod(param ** power)`` over named runtime scalars."""

    const: complex = 1.0 + 0j
    params: tuple = ()   # ((name, +1 | -1), ...)

    def __mul__(self, other: "Mono") -> "Mono":
        return Mono(self.const * other.const, self.params + other.params)

    def value(self, vals: dict) -> complex:
        v = complex(self.const)
        for name, power in self.params:
            v = v * vals[name] if power > 0 else v / vals[name]
        return v

    @property
    def is_const(self) -> bool:
        return not self.params


def _sum_value(terms, vals) -> complex:
    return sum((t.value(vals) for t in terms), 0j)


@dataclass
class Affine:
    """``mul * value + sum(add)``."""

    mul: Mono = field(default_factory=Mono)
    add: list = field(default_factory=list)

    # the transformation v -> m v + c applied after this map (output side)
    def then(self, m: Mono, c: list) -> "Affine":
        return Affine(m * self.mul, [m * t for t in self.add] + list(c))

    # this map applied after v -> m v + c (input side: the walk goes from the FFT
    # toward the leaf, each step exposing the transformation that feeds the current one)
    def after(self, m: Mono, c: list) -> "Affine":
        return Affine(self.mul * m, [self.mul * t for t in c] + list(self.add))


def _op_affine(op, ntr) -> tuple[Mono, list]:
    """(m, c) of a scale or add descriptor: v -> m v + c."""
    if op["kind"] == "scale":
        if "const" in op:
            return Mono(complex(op["const"])), []
        name = ntr.node_from_tr[op["param"]]
        return Mono(1.0, ((name, -1 if op["div"] else 1),)), []
    if "const" in op:
        return Mono(), [Mono(complex(op["const"]))]
    return Mono(), [Mono(1.0, ((ntr.node_from_tr[op["param"]], 1),))]


# ---- edge specifications ---------------------------------------------------------------


@dataclass
class EdgeSpec:
    ndim: int
    arrays: list[str] = field(default_factory=list)          # leaf names (1, or 2 for pairs)
    metas: list[ArrayMetadata] = field(default_factory=list)
    kind: str = "complex"                                     # complex | real | pair | const | ignore
    shape: list[int] = field(default_factory=list)            # user extent along each FFT dim
    strides: list[int] = field(default_factory=list)          # element strides per FFT dim
    strides2: list[int] = field(default_factory=list)
    shift: list[int] = field(default_factory=list)
    affine: Affine = field(default_factory=Affine)
    window: tuple[int, int] | None = None                     # (axis, length)
    norm: float | None = None
    norm_param: str | None = None
    frame: tuple[int, int] | None = None                      # (step, fft_size)
    crop: tuple[int, ...] | None = None
    broadcast: bool = False
    dtype: object = None                                      # FFT dtype (formats of array-less edges)

    @property
    def scale(self) -> complex:
        """The constant multiplier (1 when runtime scalars are involved)."""
        return self.affine.mul.const if self.affine.mul.is_const else 1.0 + 0j

    def fmt(self) -> int:
        if self.kind == "user":
            return N.FMT_USER
        if self.kind == "const":
            return N.FMT_CONST
        if self.kind == "ignore":
            return N.FMT_IGNORE
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


class UserTransformationError(NotImplementedError):
    """A transformation defined by source code (no built-in descriptor) on an edge that
    the built-in folding cannot express; the FFT compiles such edges separately."""

    def __init__(self, trf):
        super().__init__("transformation defined by source code")
        self.trf = trf


def _op(ntr):
    op = ntr.trf.op
    if op is None:
        raise UserTransformationError(ntr.trf)
    return op


def _leaf(tree, name: str):
    param = tree.leaf_parameters[name]
    if not param.annotation.is_array():
        raise ValueError(f"'{name}' must be an array")
    return name, param.annotation.as_array_metadata()


def _kind_of(meta: ArrayMetadata) -> str:
    return "complex" if numpy.dtype(meta.dtype).kind == "c" else "real"


def fold_input(tree, root: str, fft_shape: tuple[int, ...], fft_dtype=None) -> EdgeSpec:
    nd = len(fft_shape)
    spec = EdgeSpec(ndim=nd, shape=list(fft_shape), shift=[0] * nd, dtype=fft_dtype)
    state = {"window": False}

    def step(k, op, ntr, aff: Affine) -> Affine:
        if k in ("scale", "add"):
            if k == "add" and state["window"]:
                raise NotImplementedError("an addition inside a window transformation")
            m, c = _op_affine(op, ntr)
            return aff.after(m, c)
        return aff

    def walk_branch(node: str, aff: Affine):
        """Follow one value branch toward its leaf: returns ("array", name, meta, aff)
        or ("const", Mono-list, aff) for a constant source."""
        ntr = tree.nodes[node].input_ntr
        if ntr is None:
            name, meta = _leaf(tree, node)
            return ("array", name, meta, aff)
        op = _op(ntr)
        k = op["kind"]
        if k in ("copy", "cast"):
            return walk_branch(ntr.node_from_tr["input"], aff)
        if k in ("scale", "add"):
            return walk_branch(ntr.node_from_tr["input"], step(k, op, ntr, aff))
        if k == "window":
            spec.window = (nd - 1, op["size"])
            state["window"] = True
            return walk_branch(ntr.node_from_tr["input"], aff)
        if k == "frame":
            if spec.frame is not None:
                raise NotImplementedError("nested framing")
            spec.frame = (op["step"], op["fft_size"])
            return walk_branch(ntr.node_from_tr["input"], aff)
        if k == "broadcast":
            spec.broadcast = True
            return walk_branch(ntr.node_from_tr["input"], aff)
        if k == "const":
            return ("const", [Mono(complex(op["value"]))], aff)
        if k == "const_param":
            return ("const", [Mono(1.0, ((ntr.node_from_tr["param"], 1),))], aff)
        if k == "real_to_complex":
            r = walk_branch(ntr.node_from_tr["input"], Affine())
            return _complex_of(r, None, aff)
        if k == "combine":
            re = walk_branch(ntr.node_from_tr["real"], Affine())
            im = walk_branch(ntr.node_from_tr["imag"], Affine())
            return _complex_of(re, im, aff)
        raise NotImplementedError(f"transformation '{k}' on the FFT input")

    def _complex_of(re, im, aff: Affine):
        """A complex value re + i im from two real branches (im None: zero)."""
        i_unit = Mono(1j)
        if im is None:
            im = ("const", [], Affine())
        if re[0] == "const" and im[0] == "const":
            terms = [re[2].mul * t for t in re[1]] + re[2].add + [i_unit * re2 for re2 in
                                                                  [im[2].mul * t for t in im[1]] + im[2].add]
            return ("const", terms, aff)
        if im[0] == "const":
            # re array: value = m_re x + c_re + i (const)
            ra = re[3]
            c = ra.add + [i_unit * (im[2].mul * t) for t in im[1]] + [i_unit * t for t in im[2].add]
            return ("real", re[1], re[2], aff.after(ra.mul, c))
        if re[0] == "const":
            ia = im[3]
            c = [re[2].mul * t for t in re[1]] + re[2].add + [i_unit * t for t in ia.add]
            return ("real_im", im[1], im[2], aff.after(i_unit * ia.mul, c))
        ra, ia = re[3], im[3]
        if ra.mul != ia.mul:
            raise NotImplementedError("combine_complex with differently scaled real and imaginary parts")
        c = ra.add + [i_unit * t for t in ia.add]
        return ("pair", (re[1], im[1]), (re[2], im[2]), aff.after(ra.mul, c))

    res = walk_branch(root, Affine())
    kind = res[0]
    if kind == "const":
        spec.kind = "const"
        spec.affine = Affine(Mono(), [res[2].mul * t for t in res[1]] + res[2].add)
        spec.arrays, spec.metas = [], []
        spec.strides = [0] * nd
        spec.shape = list(fft_shape)
        return spec
    if kind == "array":
        _, name, meta, aff = res
        spec.arrays, spec.metas, spec.kind = [name], [meta], _kind_of(meta)
    elif kind in ("real", "real_im"):
        _, name, meta, aff = res
        spec.arrays, spec.metas, spec.kind = [name], [meta], "real"
    else:
        _, names, metas, aff = res
        spec.arrays, spec.metas, spec.kind = list(names), list(metas), "pair"
    spec.affine = aff
    meta = spec.metas[0]
    if spec.frame is not None:
        step_, fsize = spec.frame
        if len(meta.shape) != 1 or nd != 2:
            raise NotImplementedError("framing expects a 1-D signal and a 2-D FFT array")
        s = _elem_strides(meta)[0]
        spec.strides = [step_ * s, s]
        spec.shape = [fft_shape[0], min(fsize, fft_shape[1])]
    elif spec.broadcast:
        spec.strides, spec.shape = _broadcast_layout(meta, fft_shape)
    else:
        if len(meta.shape) != nd:
            raise ValueError("input array rank differs from the FFT array rank")
        spec.strides = _elem_strides(meta)
        spec.shape = list(meta.shape)
    if spec.kind == "pair":
        if spec.metas[1].shape != meta.shape:
            raise ValueError("real and imaginary arrays differ in shape")
        spec.strides2 = _elem_strides(spec.metas[1]) if not spec.broadcast else \
            _broadcast_layout(spec.metas[1], fft_shape)[0]
        if spec.strides2 != spec.strides:
            raise NotImplementedError("real and imaginary arrays must share strides")
    return spec


def _broadcast_layout(meta: ArrayMetadata, fft_shape) -> tuple[list[int], list[int]]:
    """Strides and extents that read ``meta`` broadcast (numpy rules) to ``fft_shape``:
    stride 0 along every broadcast dimension."""
    nd = len(fft_shape)
    src = list(meta.shape)
    st = _elem_strides(meta)
    if len(src) > nd:
        raise ValueError("input is not broadcastable to the FFT shape")
    src = [1] * (nd - len(src)) + src
    st = [0] * (nd - len(st)) + st
    strides = []
    for n_src, s, n in zip(src, st, fft_shape):
        if n_src == n:
            strides.append(s)
        elif n_src == 1:
            strides.append(0)
        else:
            raise ValueError("input is not broadcastable to the FFT shape")
    return strides, list(fft_shape)


def fold_output(tree, root: str, fft_shape: tuple[int, ...], fft_dtype=None) -> EdgeSpec:
    nd = len(fft_shape)
    spec = EdgeSpec(ndim=nd, shape=list(fft_shape), shift=[0] * nd, dtype=fft_dtype)
    state = {"real": False, "transposed": False, "aff": Affine()}

    def walk(node: str):
        ntr = tree.nodes[node].output_ntr
        if ntr is None:
            name, meta = _leaf(tree, node)
            spec.arrays, spec.metas = [name], [meta]
            spec.kind = "real" if state["real"] else "complex"
            return
        op = _op(ntr)
        k = op["kind"]
        if k in ("copy", "cast"):
            return walk(ntr.node_from_tr["output"])
        if k in ("scale", "add"):
            if state["real"]:
                raise NotImplementedError(f"transformation '{k}' after a norm transformation")
            m, c = _op_affine(op, ntr)
            state["aff"] = state["aff"].then(m, c)
            return walk(ntr.node_from_tr["output"])
        if k == "ignore":
            spec.kind = "ignore"
            spec.arrays, spec.metas = [], []
            return
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
        if k in ("norm", "norm_param"):
            if state["real"]:
                raise NotImplementedError("repeated norm")
            state["real"] = True
            if k == "norm":
                spec.norm = op["order"]
            else:
                spec.norm = 2.0
                spec.norm_param = ntr.node_from_tr["order"]
            return walk(ntr.node_from_tr["output"])
        if k == "split":
            if state["real"]:
                raise NotImplementedError("split_complex after a norm")
            r = _leaf(tree, ntr.node_from_tr["real"])
            i = _leaf(tree, ntr.node_from_tr["imag"])
            for nm in (ntr.node_from_tr["real"], ntr.node_from_tr["imag"]):
                if tree.nodes[nm].output_ntr is not None:
                    raise NotImplementedError("transformations after split_complex")
            spec.arrays, spec.metas, spec.kind = [r[0], i[0]], [r[1], i[1]], "pair"
            return
        raise NotImplementedError(f"transformation '{k}' on the FFT output")

    walk(root)
    spec.affine = state["aff"]
    if spec.kind == "ignore":
        spec.strides = [0] * nd
        return spec
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


def edge_struct(spec: EdgeSpec, slots: dict[str, int], synth=None) -> N.Edge:
    """The ``rk_edge`` of ``spec``.  ``slots``: runtime scalar name -> slot index;
    ``synth(fn)``: reserves an extra slot whose value ``fn(values)`` is computed per
    call (coefficients that involve runtime scalars)."""
    e = N.Edge()
    e.format = spec.fmt()
    e.ndim = spec.ndim
    for i in range(spec.ndim):
        e.shape[i] = spec.shape[i]
        e.strides[i] = spec.strides[i]
        e.strides2[i] = spec.strides2[i] if spec.strides2 else spec.strides[i]
        e.shift[i] = spec.shift[i]
    if spec.metas:
        isz = spec.metas[0].dtype.itemsize
        e.offset = spec.metas[0].first_element_offset // isz
        e.offset2 = spec.metas[1].first_element_offset // isz if len(spec.metas) > 1 else 0
    aff = spec.affine
    e.scale_slot = e.scale_div_slot = e.add_slot = e.post_slot = -1
    e.scale_re, e.scale_im = 1.0, 0.0
    if aff.mul.is_const:
        e.scale_re, e.scale_im = aff.mul.const.real, aff.mul.const.imag
    elif len(aff.mul.params) == 1:
        name, power = aff.mul.params[0]
        e.scale_re, e.scale_im = aff.mul.const.real, aff.mul.const.imag
        if power > 0:
            e.scale_slot = slots[name]
        else:
            e.scale_div_slot = slots[name]
    else:
        if synth is None:
            raise NotImplementedError("more than one runtime scale parameter per side")
        mul = aff.mul
        e.scale_slot = synth(lambda vals, m=mul: m.value(vals))
    e.add_re = e.add_im = 0.0
    if aff.add:
        if all(t.is_const for t in aff.add):
            c = sum((t.const for t in aff.add), 0j)
            e.add_re, e.add_im = c.real, c.imag
        else:
            if synth is None:
                raise NotImplementedError("runtime additive terms need per-call slots")
            terms = list(aff.add)
            e.add_slot = synth(lambda vals, ts=terms: _sum_value(ts, vals))
    e.post = N.POST_NORM if spec.norm is not None else N.POST_NONE
    e.post_param = spec.norm if spec.norm is not None else 2.0
    if spec.norm_param is not None:
        e.post_slot = slots[spec.norm_param]
    if spec.window is not None:
        e.window = N.WIN_HANN
        e.window_axis = spec.window[0]
        e.window_len = spec.window[1]
    return e


def native_edges(ispec: EdgeSpec, ospec: EdgeSpec, scalar_names: list[str]):
    """Both edges plus the per-call scalar list builder: the runtime scalars in
    signature order, then the values of the slots the edges reserved."""
    slots = {n: i for i, n in enumerate(scalar_names)}
    extra = []

    def synth(fn):
        extra.append(fn)
        return len(scalar_names) + len(extra) - 1

    ein = edge_struct(ispec, slots, synth)
    eout = edge_struct(ospec, slots, synth)

    def scalars(values: dict) -> list[complex]:
        base = [values[n] for n in scalar_names]
        return base + [f(values) for f in extra]

    return ein, eout, scalars


def user_spec(fft_shape) -> EdgeSpec:
    """The native side of an edge served by run-time compiled code: the element's
    flat C-order index in the FFT array is all the code needs."""
    nd = len(fft_shape)
    strides, st = [0] * nd, 1
    for i in range(nd - 1, -1, -1):
        strides[i] = st
        st *= fft_shape[i]
    return EdgeSpec(ndim=nd, kind="user", shape=list(fft_shape), strides=strides, shift=[0] * nd)
