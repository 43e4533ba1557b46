"""``Transpose`` computation: drop-in for ``reikna.algorithms.Transpose``
(reikna/algorithms/transpose.py:99-244).

Same constructor ``Transpose(arr_t, output_arr_t=None, axes=None,
block_width_override=None)``, signature ``(output:o, input:i)`` and errors.  An axis
permutation is realised, as in the reference, by a shortest sequence of moves that
swap a block of axes [b, c) with all trailing axes [c, n); each move is one batched
2-D transpose (``rk_transpose_execute``, 32 x 32 shared-memory tiles), with
intermediates held by the compiled callable.
"""

from __future__ import annotations

import collections

import numpy

from .. import _native as N
from ..core.computation import Computation, array_pointer
from ..core.signature import Annotation, ArrayMetadata, Parameter, Type


def transpose_shape(shape, axes):
    return tuple(shape[i] for i in axes)


def _move(order, b, c):
    """Swap the axis block [b, c) with the trailing block [c, n)."""
    return order[:b] + order[c:] + order[b:c]


def moves(n: int, axes) -> list[tuple[int, int]]:
    """Shortest list of (b, c) moves turning axis order 0..n-1 into ``axes`` (breadth
    first over permutations; n is at most 8)."""
    start, target = tuple(range(n)), tuple(axes)
    if start == target:
        return []
    prev = {start: None}
    queue = collections.deque([start])
    while queue:
        cur = queue.popleft()
        for b in range(n - 1):
            for c in range(b + 1, n):
                nxt = _move(cur, b, c)
                if nxt in prev:
                    continue
                prev[nxt] = (cur, (b, c))
                if nxt == target:
                    path = []
                    node = nxt
                    while prev[node] is not None:
                        node, mv = prev[node]
                        path.append(mv)
                    return path[::-1]
                queue.append(nxt)
    raise ValueError(f"cannot reach axis order {axes}")  # unreachable for permutations


def transposes(shape, axes):
    """(batch, height, width) element counts of each batched 2-D transpose."""
    shape = tuple(shape)
    out = []
    for b, c in moves(len(shape), axes):
        out.append((int(numpy.prod(shape[:b])), int(numpy.prod(shape[b:c])), int(numpy.prod(shape[c:]))))
        shape = _move(shape, b, c)
    return out


class Transpose(Computation):
    """Changes the order of axes of an array, like ``numpy.transpose``.

    :param arr_t: array-like describing the input.
    :param output_arr_t: array-like describing the output (default: the permuted
        shape, same dtype).
    :param axes: new axis order (default: reversed).
    :param block_width_override: accepted for compatibility; the tile size is fixed.
    """

    def __init__(self, arr_t, output_arr_t=None, axes=None, block_width_override=None):
        self._block_width_override = block_width_override
        inp = Type(arr_t).as_array_metadata() if not isinstance(arr_t, ArrayMetadata) else arr_t
        all_axes = range(len(inp.shape))
        if axes is None:
            axes = tuple(reversed(all_axes))
        else:
            axes = tuple(axes)
            if set(axes) != set(all_axes):
                raise ValueError("All transpose axes must be distinct")
        self._axes = axes
        out_shape = transpose_shape(inp.shape, axes)
        if output_arr_t is not None:
            out = Type(output_arr_t).as_array_metadata() if not isinstance(output_arr_t, ArrayMetadata) else output_arr_t
        else:
            out = ArrayMetadata(out_shape, inp.dtype)
        if tuple(out.shape) != tuple(out_shape):
            raise ValueError(f"Expected output array shape: {out_shape}, got {tuple(out.shape)}")
        if out.dtype != inp.dtype:
            raise ValueError("Input and output array must have the same dtype")
        self._in = inp
        self._out = out
        Computation.__init__(
            self, [Parameter("output", Annotation(out, "o")), Parameter("input", Annotation(inp, "i"))]
        )

    def _build_runner(self, device, **_ignored):
        import torch

        leaves = [p.name for p in self._tr_tree.get_leaf_parameters()]
        if leaves != ["output", "input"]:
            raise NotImplementedError("transformations connected to Transpose are not fused")
        for meta in (self._in, self._out):
            c = ArrayMetadata(tuple(meta.shape), meta.dtype)
            if tuple(meta.strides) != tuple(c.strides):
                raise NotImplementedError("Transpose works on C-contiguous arrays")
        esz = numpy.dtype(self._in.dtype).itemsize
        if esz not in (1, 2, 4, 8, 16):
            raise NotImplementedError(f"element size {esz} is not supported")
        ops = transposes(self._in.shape, self._axes)
        n = int(numpy.prod(self._in.shape))
        # intermediates: at most two, used alternately
        temps = [torch.empty(max(n, 1) * esz, dtype=torch.uint8, device=device) for _ in range(min(2, max(0, len(ops) - 1)))]
        ann = {p.name: p.annotation for p in self._tr_tree.get_leaf_parameters()}

        def runner(stream: int, args):
            dst_final = array_pointer(args["output"], ann["output"])
            src = array_pointer(args["input"], ann["input"])
            if not ops:
                # identity permutation: a plain device copy on the stream
                ctx = torch.cuda.stream(torch.cuda.ExternalStream(stream)) if stream else torch.cuda.stream(None)
                with ctx:
                    args["output"].copy_(args["input"])
                return
            for k, (b, h, w) in enumerate(ops):
                dst = dst_final if k == len(ops) - 1 else temps[k % 2].data_ptr()
                N.check(N.lib().rk_transpose_execute(dst, src, esz, b, h, w, stream))
                src = dst

        runner.launches = max(1, len(ops))
        runner.temps = temps
        return runner
