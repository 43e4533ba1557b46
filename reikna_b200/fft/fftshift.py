"""``FFTShift`` computation: drop-in for ``reikna.fft.FFTShift`` (reikna/fft/fftshift.py:14-110).

Signature ``(output:o, input:i, inverse:s int32 = 0)``; ``inverse = 1`` gives
``numpy.fft.ifftshift``.  Output may alias input.  Transformations connected to the
parameters are supported when they are a plain scale (``mul_param``/``mul_const``):
the shift then runs through a one-pass native FFT plan with no transformed axes and
an index remap on the output edge.
"""

from __future__ import annotations

import numpy

from .. import _native as N
from ..core.computation import Computation, array_pointer
from ..core.signature import Annotation, ArrayMetadata, Parameter, Type


class FFTShift(Computation):
    def __init__(self, arr_t, axes=None):
        meta = Type(arr_t).as_array_metadata() if not isinstance(arr_t, ArrayMetadata) else arr_t
        Computation.__init__(
            self,
            [
                Parameter("output", Annotation(meta, "o")),
                Parameter("input", Annotation(meta, "i")),
                Parameter("inverse", Annotation(numpy.int32), default=0),
            ],
        )
        nd = len(meta.shape)
        axes = tuple(range(nd)) if axes is None else tuple(int(a) % nd for a in axes)
        self._axes = axes
        self._meta = meta

    def _build_runner(self, device, **_ignored):
        meta = self._meta
        tree = self._tr_tree
        leaves = tree.get_leaf_parameters()
        plain = all(tree.nodes[n].input_ntr is None and tree.nodes[n].output_ntr is None for n in ("input", "output"))
        shape = tuple(meta.shape)
        isz = meta.dtype.itemsize
        contiguous = ArrayMetadata(shape, meta.dtype).strides == meta.strides
        moved = 1
        for a in self._axes:
            moved *= shape[a]
        if plain and contiguous and isz in (4, 8, 16):
            import torch

            all_even = all(shape[a] % 2 == 0 for a in self._axes)
            scratch = {}

            def runner(stream: int, args):
                out = array_pointer(args["output"], tree.leaf_parameters["output"].annotation)
                inp = array_pointer(args["input"], tree.leaf_parameters["input"].annotation)
                sp = 0
                if out == inp and not all_even:
                    if "buf" not in scratch:
                        scratch["buf"] = torch.empty(max(1, meta.strides[0] * shape[0] if shape else isz),
                                                     dtype=torch.uint8, device=device)
                    sp = scratch["buf"].data_ptr()
                N.fftshift_execute(out, inp, isz, shape, self._axes, int(args["inverse"]), sp, stream)

            runner.launches = 1
            return runner

        # general route: a native plan with no transformed axes and an output remap
        from ..fft._fold import fold_input, fold_output, native_edges

        if not numpy.dtype(meta.dtype).kind == "c":
            raise NotImplementedError("FFTShift with transformations supports complex arrays only")
        ispec = fold_input(tree, "input", shape, meta.dtype)
        ospec = fold_output(tree, "output", shape, meta.dtype)
        scalar_names = [p.name for p in leaves if p.annotation.is_scalar() and p.name != "inverse"]
        ein, eout, scalar_list = native_edges(ispec, ospec, scalar_names)
        plans = {}
        ann = {p.name: p.annotation for p in leaves}

        def make(inverse: int):
            d = N.FftDesc()
            d.dtype = N.FMT_C64 if meta.dtype == numpy.complex64 else N.FMT_C128
            d.ndim = len(shape)
            for i, s in enumerate(shape):
                d.shape[i] = s
            d.naxes = 0
            d.input = ein
            o = N.Edge.from_buffer_copy(eout)
            for a in self._axes:
                n = shape[a]
                s = (n + 1) // 2 if inverse else n // 2
                o.shift[a] = (o.shift[a] + s) % n
            d.output = o
            return N.Plan(d)

        def runner(stream: int, args):
            inv = int(args["inverse"]) != 0
            if inv not in plans:
                plans[inv] = make(inv)
            outs = [array_pointer(args[n], ann[n]) for n in ospec.arrays]
            ins = [array_pointer(args[n], ann[n]) for n in ispec.arrays]
            scalars = scalar_list({n: complex(numpy.asarray(args[n]).item()) for n in scalar_names})
            plans[inv].execute(outs, ins, inverse=0, scalars=scalars, stream=stream)

        runner.launches = 1
        return runner
