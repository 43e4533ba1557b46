"""``FFT`` computation: drop-in for ``reikna.fft.FFT`` (reikna/fft/fft.py:595-756).

Same constructor ``FFT(arr_t, axes=None)``, same signature
``(output:o, input:i, inverse:s int32 = 0)``, same semantics: the forward transform
uses exp(-2 pi i n k / N), the inverse is normalised so that IFFT(FFT(x)) = x, output
may alias input, transformations connected to ``input``/``output`` run inside the
first and last pass.  Planning and the kernels are native (``include/reikna_b200.h``).
"""

from __future__ import annotations

import numpy

from .. import _native as N
from ..core.computation import ArrayCheck, Computation, array_pointer, scalar_value
from ..core.signature import Annotation, ArrayMetadata, Parameter, Type
from ._fold import UserTransformationError, fold_input, fold_output, native_edges, user_spec


def _is_complex(dtype) -> bool:
    return numpy.dtype(dtype).kind == "c"


class FFT(Computation):
    """Fast Fourier Transform over ``axes`` of an array of ``arr_t``'s type.

    :param arr_t: array-like (torch tensor, numpy array, ``ArrayMetadata``, ``Type``).
    :param axes: axes to transform (default: all); negative values count from the end.
    """

    def __init__(self, arr_t, axes=None):
        meta = Type(arr_t).as_array_metadata() if not isinstance(arr_t, ArrayMetadata) else arr_t
        if not _is_complex(meta.dtype):
            raise ValueError("FFT computation requires array of a complex dtype")
        Computation.__init__(
            self,
            [
                Parameter("output", Annotation(meta, "o")),
                Parameter("input", Annotation(meta, "i")),
                Parameter("inverse", Annotation(numpy.int32), default=0),
            ],
        )
        nd = len(meta.shape)
        axes = tuple(range(nd)) if axes is None else tuple(int(a) for a in axes)
        axes = tuple(a + nd if a < 0 else a for a in axes)
        if any(a < 0 or a >= nd for a in axes) or len(set(axes)) != len(axes):
            raise ValueError(f"invalid axes {axes} for a {nd}-dimensional array")
        self._axes = axes
        self._meta = meta

    def native_descriptor(self, flags: int = 0):
        """The ``rk_fft_desc`` this computation compiles to, and its argument layout."""
        meta = self._meta
        tree = self._tr_tree
        shape = tuple(meta.shape)
        self._user_edges = {}
        try:
            ispec = fold_input(tree, "input", shape, meta.dtype)
        except UserTransformationError:
            from .user import EdgeCode

            self._user_edges["input"] = EdgeCode(tree, "input", "input", meta)
            ispec = user_spec(shape)
        try:
            ospec = fold_output(tree, "output", shape, meta.dtype)
        except UserTransformationError:
            from .user import EdgeCode

            self._user_edges["output"] = EdgeCode(tree, "output", "output", meta)
            ospec = user_spec(shape)
        leaves = tree.get_leaf_parameters()
        scalar_names = [p.name for p in leaves if p.annotation.is_scalar() and p.name != "inverse"]
        ein, eout, scalars = native_edges(ispec, ospec, scalar_names)
        d = N.FftDesc()
        d.dtype = N.FMT_C64 if meta.dtype == numpy.complex64 else N.FMT_C128
        d.ndim = len(shape)
        for i, s in enumerate(shape):
            d.shape[i] = s
        d.naxes = len(self._axes)
        for i, a in enumerate(self._axes):
            d.axes[i] = a
        d.flags = flags
        d.input = ein
        d.output = eout
        return d, ispec, ospec, scalar_names, scalars

    def describe(self, flags: int = 0) -> dict:
        """Kernel chain the native planner builds for this computation (no GPU needed)."""
        d, *_ = self.native_descriptor(flags)
        return N.describe(d)

    def _build_runner(self, device, flags: int = 0, **_ignored):
        d, ispec, ospec, scalar_names, scalar_list = self.native_descriptor(flags)
        plan = N.Plan(d)
        ann = {p.name: p.annotation for p in self._tr_tree.get_leaf_parameters()}
        user = dict(self._user_edges)
        if user:
            self._install_user_kernels(plan, user)

        checks = {n: ArrayCheck(ann[n]) for n in list(ospec.arrays) + list(ispec.arrays)}
        out_checks = [(n, checks[n]) for n in ospec.arrays]
        in_checks = [(n, checks[n]) for n in ispec.arrays]

        def bind(args):
            """(output pointers, input pointers, inverse, scalars) of one call."""
            outs = [c(args[n]) for n, c in out_checks]
            ins = [c(args[n]) for n, c in in_checks]
            scalars = scalar_list({n: scalar_value(args[n]) for n in scalar_names}) if scalar_names else \
                scalar_list({})
            return outs, ins, int(args["inverse"]), scalars

        if user:
            uin, uout = user.get("input"), user.get("output")

            def runner(stream: int, args):
                outs, ins, inverse, scalars = bind(args)
                wi = uin.words_of(args, array_pointer) if uin else []
                wo = uout.words_of(args, array_pointer) if uout else []
                plan.execute_user(outs, ins, inverse=inverse, scalars=scalars, user_in=wi, user_out=wo, stream=stream)
        else:

            def runner(stream: int, args):
                outs, ins, inverse, scalars = bind(args)
                plan.execute(outs, ins, inverse=inverse, scalars=scalars, stream=stream)

        runner.launches = plan.launches
        runner.plan = plan
        runner.bind = bind
        runner.flags = flags
        return runner

    def _install_user_kernels(self, plan, user) -> None:
        """Compile, for every pass that reads or writes an edge given as code, its
        kernel with that code, and install it in the plan."""
        from .. import _rtc
        from .user import kernel_source

        opts = getattr(self, "_compile_options", {})
        options = list(opts.get("compiler_options", ()))
        if opts.get("fast_math"):
            options.append("-use_fast_math")
        for i, info in enumerate(plan.pass_info()):
            if not info["user"]:
                continue
            edges = ([user["input"]] if info["user"] & 1 else []) + ([user["output"]] if info["user"] & 2 else [])
            src = kernel_source(edges, "double" if info["dbl"] else "float", info["L"], info["mode"], info["var"],
                                info["nt"])
            cubin = _rtc.compile_cubin(src, f"rk_user_pass{i}.cu", options, keep=opts.get("keep", False))
            plan.set_pass_kernel(i, cubin, "rk_user_pass")
