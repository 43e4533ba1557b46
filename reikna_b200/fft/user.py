"""Transformations given as source code, compiled into the FFT's first or last pass.

reikna inlines a transformation's code into the kernels that read or write the
connected parameter (reikna/core/transformation.py:460-518,
reikna/core/transformation_modules.py:19-318): an input transformation computes the
element the kernel loads (``${output.store_same}(value)`` sets it, ``${input.load_same}``
/ ``${input.load_idx}(i, ...)`` read its own inputs), an output transformation consumes
the element the kernel stores (``${input.load_same}`` is that element,
``${output.store_same}(v)`` / ``${output.store_idx}(i, ..., v)`` write it on).  The code is
a template in reikna's syntax (``${...}``, ``<% %>``, ``% for`` / ``% if`` lines,
rendered by :mod:`reikna_b200.core.template`) with the same names: the parameter
objects, ``idxs`` (the element's index variables), ``VSIZE_T``, and the
transformation's ``render_kwds``.

Here the chain of transformations on an FFT edge becomes a set of device functions
(one per tree node) plus ``rk_user_load`` / ``rk_user_store``, which the kernel's
edge path calls with the element's flat index.  For every pass that touches the
edge, the pass kernel is compiled at run time with those functions
(:mod:`reikna_b200._rtc`) and installed in the native plan
(``rk_fft_plan_set_pass_kernel``); the arrays and scalars the code reads arrive per
call as up to eight 64-bit words per edge (``rk_fft_execute_user``).  Built-in
element-wise transformations (copy, cast, scale, add) may be mixed into such a chain.
"""

from __future__ import annotations

import struct

import numpy

from ..core.template import render

MAX_WORDS = 8

_CTYPES = {
    numpy.dtype(numpy.complex64): "float2",
    numpy.dtype(numpy.complex128): "double2",
    numpy.dtype(numpy.float32): "float",
    numpy.dtype(numpy.float64): "double",
    numpy.dtype(numpy.int32): "int",
    numpy.dtype(numpy.uint32): "unsigned int",
    numpy.dtype(numpy.int64): "long long",
    numpy.dtype(numpy.uint64): "unsigned long long",
}


def ctype(dtype) -> str:
    dt = numpy.dtype(dtype)
    if dt not in _CTYPES:
        raise NotImplementedError(f"no device type for {dt}")
    return _CTYPES[dt]


# generic element helpers the generated code (and user code, through
# reikna_b200.cluda.functions) uses; overloads cover real and complex operands
HELPERS = r"""
namespace rkf {
__device__ __forceinline__ float2 cv2(float x) { return make_float2(x, 0.f); }
__device__ __forceinline__ float2 cv2(double x) { return make_float2((float)x, 0.f); }
__device__ __forceinline__ float2 cv2(float2 x) { return x; }
__device__ __forceinline__ float2 cv2(double2 x) { return make_float2((float)x.x, (float)x.y); }
__device__ __forceinline__ double2 cvd2(float x) { return make_double2(x, 0.0); }
__device__ __forceinline__ double2 cvd2(double x) { return make_double2(x, 0.0); }
__device__ __forceinline__ double2 cvd2(float2 x) { return make_double2(x.x, x.y); }
__device__ __forceinline__ double2 cvd2(double2 x) { return x; }
template <typename To> struct Cvt;
template <> struct Cvt<float2> { template <typename F> static __device__ float2 f(F x) { return cv2(x); } };
template <> struct Cvt<double2> { template <typename F> static __device__ double2 f(F x) { return cvd2(x); } };
template <> struct Cvt<float> {
    static __device__ float f(float x) { return x; }
    static __device__ float f(double x) { return (float)x; }
    static __device__ float f(float2 x) { return x.x; }
    static __device__ float f(double2 x) { return (float)x.x; }
};
template <> struct Cvt<double> {
    static __device__ double f(float x) { return x; }
    static __device__ double f(double x) { return x; }
    static __device__ double f(float2 x) { return x.x; }
    static __device__ double f(double2 x) { return x.x; }
};
template <typename To, typename F> __device__ __forceinline__ To cast(F x) { return Cvt<To>::f(x); }

__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ double mul(double a, double b) { return a * b; }
__device__ __forceinline__ float2 mul(float2 a, float b) { return make_float2(a.x * b, a.y * b); }
__device__ __forceinline__ float2 mul(float a, float2 b) { return make_float2(a * b.x, a * b.y); }
__device__ __forceinline__ double2 mul(double2 a, double b) { return make_double2(a.x * b, a.y * b); }
__device__ __forceinline__ double2 mul(double a, double2 b) { return make_double2(a * b.x, a * b.y); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 mul(double2 a, float2 b) { return mul(a, cvd2(b)); }
__device__ __forceinline__ double2 mul(float2 a, double2 b) { return mul(cvd2(a), b); }
__device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float conj(float a) { return a; }
__device__ __forceinline__ double conj(double a) { return a; }
__device__ __forceinline__ float norm(float2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double norm(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ float norm(float a) { return a * a; }
__device__ __forceinline__ double norm(double a) { return a * a; }
__device__ __forceinline__ float inv(float a) { return 1.f / a; }
__device__ __forceinline__ double inv(double a) { return 1.0 / a; }
__device__ __forceinline__ float2 inv(float2 a) { const float n = norm(a); return make_float2(a.x / n, -a.y / n); }
__device__ __forceinline__ double2 inv(double2 a) { const double n = norm(a); return make_double2(a.x / n, -a.y / n); }
template <typename A, typename B> __device__ __forceinline__ auto div(A a, B b) { return mul(a, inv(b)); }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 add(float2 a, float b) { return make_float2(a.x + b, a.y); }
__device__ __forceinline__ float2 add(float a, float2 b) { return make_float2(a + b.x, b.y); }
__device__ __forceinline__ double2 add(double2 a, double b) { return make_double2(a.x + b, a.y); }
__device__ __forceinline__ double2 add(double a, double2 b) { return make_double2(a + b.x, b.y); }
__device__ __forceinline__ float2 polar_unit(float t) { float s, c; sincosf(t, &s, &c); return make_float2(c, s); }
__device__ __forceinline__ double2 polar_unit(double t) { double s, c; sincos(t, &s, &c); return make_double2(c, s); }
__device__ __forceinline__ float2 exp(float2 a) { const float e = expf(a.x); float s, c; sincosf(a.y, &s, &c); return make_float2(e * c, e * s); }
__device__ __forceinline__ double2 exp(double2 a) { const double e = ::exp(a.x); double s, c; sincos(a.y, &s, &c); return make_double2(e * c, e * s); }
__device__ __forceinline__ float exp(float a) { return expf(a); }
__device__ __forceinline__ double exp(double a) { return ::exp(a); }
}  // namespace rkf
"""


def _c_const(value, dtype) -> str:
    dt = numpy.dtype(dtype)
    v = complex(value)
    if dt.kind == "c":
        mk = "make_float2" if dt == numpy.complex64 else "make_double2"
        return f"{mk}({v.real!r}, {v.imag!r})"
    if dt.kind == "f":
        return f"({ctype(dt)})({v.real!r})"
    return f"({ctype(dt)})({int(v.real)})"


class _Param:
    """What a template sees for one transformation parameter (reikna's
    KernelParameter: ``ctype``, ``dtype``, ``shape``, ``strides``, ``load_same`` /
    ``store_same`` / ``load_idx`` / ``store_idx``)."""

    def __init__(self, annotation, **kw):
        self.annotation = annotation
        self.dtype = annotation.dtype
        self.ctype = ctype(annotation.dtype)
        if annotation.is_array():
            self.shape = annotation.shape
            self.strides = annotation.strides
            self.offset = annotation.offset
        self._str = kw.pop("value", None)
        self.__dict__.update(kw)

    def __str__(self):
        if self._str is None:
            raise ValueError("an array parameter has no value in transformation code; use load/store")
        return self._str


class EdgeCode:
    """Device code of one FFT edge whose chain holds a transformation given as code."""

    def __init__(self, tree, root: str, side: str, fft_meta):
        self.tree = tree
        self.root = root
        self.side = side                       # "input" or "output"
        self.shape = tuple(fft_meta.shape)
        self.fft_dtype = numpy.dtype(fft_meta.dtype)
        self.nd = len(self.shape)
        self.idx = self._idx(self.nd)
        self.leaves = []                       # (name, annotation, kind: array | scalar)
        self._leaf_pos = {}
        self.functions = []
        self.words = 0
        self._emit(root)
        if self.words > MAX_WORDS:
            raise NotImplementedError(f"transformation code on one FFT edge may use at most {MAX_WORDS} words of "
                                      f"arrays and scalars, this one needs {self.words}")

    # -- leaves ------------------------------------------------------------------------
    def _leaf(self, name: str) -> int:
        if name in self._leaf_pos:
            return self._leaf_pos[name]
        ann = self.tree.leaf_parameters[name].annotation
        kind = "array" if ann.is_array() else "scalar"
        self._leaf_pos[name] = len(self.leaves)
        nwords = 2 if (kind == "scalar" and numpy.dtype(ann.dtype) == numpy.complex128) else 1
        self.leaves.append((name, ann, kind, self.words, nwords))
        self.words += nwords
        return self._leaf_pos[name]

    def _leaf_ref(self, name: str) -> str:
        return f"L.l{self._leaf(name)}"

    # -- code generation ---------------------------------------------------------------
    # every node function takes the indices of its own array (a node of another rank,
    # e.g. a 1-D window read with load_idx, has its own index list)
    @staticmethod
    def _idx(nd: int) -> list[str]:
        return [f"_idx{i}" for i in range(nd)]

    def _sig(self, nd: int) -> str:
        return ", ".join(f"VSIZE_T {i}" for i in self._idx(nd))

    def _args(self, nd: int) -> str:
        return ", ".join(self._idx(nd))

    def _flat(self, ann) -> str:
        isz = ann.dtype.itemsize
        terms = [f"({i}) * ({st // isz})" for i, st in zip(self._idx(len(ann.shape)), ann.strides)]
        return " + ".join(terms + [str(ann.offset // isz)])

    def _ann(self, node: str):
        """Annotation of a node: its leaf parameter, or the transformation parameter
        connected to it."""
        if node in self.tree.leaf_parameters:
            return self.tree.leaf_parameters[node].annotation
        n = self.tree.nodes[node]
        ntr = n.input_ntr if self.side == "input" else n.output_ntr
        return ntr.trf.signature.parameters[ntr.tr_connector].annotation

    def _emit(self, node: str) -> str:
        """Emit the function of ``node``; returns its name."""
        fname = f"node_{len(self.functions)}"
        self.functions.append(None)  # reserve the slot (children get later numbers)
        slot = len(self.functions) - 1
        n = self.tree.nodes[node]
        ntr = n.input_ntr if self.side == "input" else n.output_ntr
        ann = self._ann(node)
        ct = ctype(ann.dtype)
        nd = len(ann.shape)
        sig, args = self._sig(nd), self._args(nd)
        if ntr is None:
            # a leaf array of the computation
            lr = self._leaf_ref(node)
            if self.side == "input":
                body = f"__device__ __forceinline__ {ct} {fname}(const Leaves& L, {sig}) {{\n" \
                       f"    return {lr}[{self._flat(ann)}];\n}}\n"
            else:
                body = f"__device__ __forceinline__ void {fname}(const Leaves& L, {sig}, {ct} _val) {{\n" \
                       f"    {lr}[{self._flat(ann)}] = _val;\n}}\n"
            self.functions[slot] = body
            return fname
        trf = ntr.trf
        params = trf.signature.parameters
        ns = {"idxs": self._idx(nd), "VSIZE_T": "VSIZE_T"}
        pre = []
        for pname, p in params.items():
            child = ntr.node_from_tr[pname]
            pann = p.annotation
            if pname == ntr.tr_connector:
                if self.side == "input":
                    ns[pname] = _Param(pann, store_same="_val =")
                else:
                    ns[pname] = _Param(pann, load_same="_val")
                continue
            if not pann.is_array():
                ns[pname] = _Param(pann, value=self._leaf_ref(child))
                continue
            cf = self._emit(child)
            cct = ctype(pann.dtype)
            cnd = len(pann.shape)
            csig, cargs = self._sig(cnd), self._args(cnd)
            # load_same / store_same use this node's own indices (same rank only)
            same = args if cnd == nd else None
            if self.side == "input":
                lam = f"IN_{cf}"
                pre.append(f"    auto {lam} = [&]({csig}) {{ return {cf}(L, {cargs}); }};")
                ns[pname] = _Param(pann, load_same=f"{cf}(L, {same})" if same is not None else None, load_idx=lam)
            else:
                lam, lam_s = f"OUT_{cf}", f"OUTS_{cf}"
                pre.append(f"    auto {lam} = [&]({csig}, {cct} _v) {{ {cf}(L, {cargs}, _v); }};")
                if same is not None:
                    pre.append(f"    auto {lam_s} = [&]({cct} _v) {{ {cf}(L, {same}, _v); }};")
                ns[pname] = _Param(pann, store_same=lam_s if same is not None else None, store_idx=lam)
        if trf.code is not None:
            ns.update(trf.render_kwds)
            code = render(trf.code, **ns)
        else:
            code = self._builtin(trf, ntr, ns)
        if self.side == "input":
            head = f"__device__ __forceinline__ {ct} {fname}(const Leaves& L, {sig}) {{\n    {ct} _val;\n"
            tail = "    return _val;\n}\n"
        else:
            head = f"__device__ __forceinline__ void {fname}(const Leaves& L, {sig}, {ct} _val) {{\n"
            tail = "}\n"
        self.functions[slot] = head + "\n".join(pre) + "\n" + code + "\n" + tail
        return fname

    def _builtin(self, trf, ntr, ns) -> str:
        """Code for a built-in element-wise transformation inside a code chain."""
        op = trf.op or {}
        k = op.get("kind")
        if self.side == "input":
            src = ns["input"].load_same
            out_t = ns["output"].ctype
            if k in ("copy", "cast"):
                return f"    _val = rkf::cast<{out_t}>({src});"
            if k == "scale":
                c = ns["param"]._str if "param" in op else _c_const(op["const"], trf.signature.parameters["output"].annotation.dtype)
                f = "rkf::div" if op.get("div") and "param" in op else "rkf::mul"
                return f"    _val = rkf::cast<{out_t}>({f}({src}, {c}));"
            if k == "add":
                c = ns["param"]._str if "param" in op else _c_const(op["const"], trf.signature.parameters["output"].annotation.dtype)
                return f"    _val = rkf::cast<{out_t}>(rkf::add({src}, {c}));"
        else:
            out = ns["output"]
            out_t = out.ctype
            if k in ("copy", "cast"):
                return f"    {out.store_same}(rkf::cast<{out_t}>(_val));"
            if k == "scale":
                c = ns["param"]._str if "param" in op else _c_const(op["const"], trf.signature.parameters["output"].annotation.dtype)
                f = "rkf::div" if op.get("div") and "param" in op else "rkf::mul"
                return f"    {out.store_same}(rkf::cast<{out_t}>({f}(_val, {c})));"
            if k == "add":
                c = ns["param"]._str if "param" in op else _c_const(op["const"], trf.signature.parameters["output"].annotation.dtype)
                return f"    {out.store_same}(rkf::cast<{out_t}>(rkf::add(_val, {c})));"
        raise NotImplementedError(
            f"built-in transformation '{k}' in a chain with transformation code (only copy, cast, scale and add mix)")

    # -- module ------------------------------------------------------------------------
    def module(self) -> str:
        """The device functions and the load / store entry the kernel calls."""
        ns = f"rkusr_{self.side}"
        fields = []
        unpack = []
        for i, (name, ann, kind, w, nw) in enumerate(self.leaves):
            ct = ctype(ann.dtype)
            if kind == "array":
                fields.append(f"    {ct}* l{i};")
                unpack.append(f"    L.l{i} = reinterpret_cast<{ct}*>(s.user[{w}]);")
            else:
                fields.append(f"    {ct} l{i};")
                if nw == 2:
                    unpack.append(f"    L.l{i} = make_double2(__longlong_as_double((long long)s.user[{w}]), "
                                  f"__longlong_as_double((long long)s.user[{w + 1}]));")
                else:
                    unpack.append(f"    {{ {ct} t; memcpy(&t, &s.user[{w}], sizeof(t)); L.l{i} = t; }}")
        decomp = []
        for d in range(self.nd - 1, 0, -1):
            decomp.append(f"    const VSIZE_T {self.idx[d]} = flat % {self.shape[d]}; flat /= {self.shape[d]};")
        decomp.append(f"    const VSIZE_T {self.idx[0]} = flat;")
        root_fn = "node_0"
        fct = ctype(self.fft_dtype)
        body = [f"namespace {ns} {{", "typedef long long VSIZE_T;", "struct Leaves {", *fields, "};"]
        # functions are emitted children first so that each is declared before use
        body += list(reversed(self.functions))
        body.append("}  // namespace " + ns)
        if self.side == "input":
            body += [
                "template <typename T> __device__ __forceinline__ rk::cplx<T> rk_user_load(const rk::Side& s, long long flat) {",
                f"    using namespace {ns};",
                "    Leaves L;",
                *unpack,
                *decomp,
                f"    const {fct} v = {root_fn}(L, {self._args(self.nd)});",
                "    return rk::cmk<rk::cplx<T>>((T)v.x, (T)v.y);",
                "}",
                "#define RK_USER_LOAD rk_user_load",
            ]
        else:
            body += [
                "template <typename T> __device__ __forceinline__ void rk_user_store(const rk::Side& s, long long flat, rk::cplx<T> v) {",
                f"    using namespace {ns};",
                "    Leaves L;",
                *unpack,
                *decomp,
                f"    {fct} w; w.x = v.x; w.y = v.y;",
                f"    {root_fn}(L, {self._args(self.nd)}, w);",
                "}",
                "#define RK_USER_STORE rk_user_store",
            ]
        return "\n".join(body)

    def words_of(self, args, array_pointer) -> list[int]:
        """The 64-bit words of one call: array pointers and scalar bit patterns."""
        out = [0] * self.words
        for name, ann, kind, w, nw in self.leaves:
            v = args[name]
            if kind == "array":
                out[w] = array_pointer(v, ann)
                continue
            x = numpy.asarray(v).astype(ann.dtype)
            raw = x.tobytes()
            if nw == 2:
                out[w], out[w + 1] = struct.unpack("<QQ", raw)
            else:
                out[w] = int.from_bytes(raw.ljust(8, b"\0"), "little")
        return out


def kernel_source(edges, T: str, L: int, mode: int, var: int, nt: int) -> str:
    """Source of one pass kernel calling the edges' code."""
    mods = "\n".join(e.module() for e in edges)
    return f"""
#include "rk_dft.cuh"
#include "rk_params.h"
{HELPERS}
{mods}
#include "rk_kernels.cuh"
extern "C" __global__ void __launch_bounds__({nt}) rk_user_pass(const rk::PassParams p) {{
    extern __shared__ __align__(16) unsigned char rk_smem[];
    rk::line_body<{T}, {L}, {mode}, {var}>(p, blockIdx.x, rk_smem, threadIdx.x);
}}
"""
