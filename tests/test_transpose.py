"""Transpose computation (reikna/algorithms/transpose.py): exact against numpy."""

import numpy
import pytest


def _apply_moves(x, axes):
    from reikna_b200.algorithms.transpose import transposes

    y = x.copy()
    for b, h, w in transposes(x.shape, axes):
        y = y.reshape(b, h, w).transpose(0, 2, 1).copy()
    return y.reshape(numpy.transpose(x, axes).shape)


@pytest.mark.parametrize(
    "shape,axes",
    [((4, 5), (1, 0)), ((4, 5, 6), (2, 1, 0)), ((4, 5, 6), (0, 2, 1)), ((2, 3, 4, 5), (1, 0, 3, 2)),
     ((2, 3, 4, 5), (3, 1, 2, 0)), ((3, 4, 5), (0, 1, 2))],
)
def test_move_sequences_realise_the_permutation(shape, axes):
    x = numpy.arange(int(numpy.prod(shape))).reshape(shape)
    assert numpy.array_equal(_apply_moves(x, axes), numpy.transpose(x, axes))


def test_errors_follow_the_reference():
    from reikna_b200.algorithms import Transpose
    from reikna_b200.core import ArrayMetadata

    a = ArrayMetadata((4, 5), numpy.float32)
    with pytest.raises(ValueError, match="distinct"):
        Transpose(a, axes=(0, 0))
    with pytest.raises(ValueError, match="Expected output array shape"):
        Transpose(a, output_arr_t=ArrayMetadata((4, 5), numpy.float32))
    with pytest.raises(ValueError, match="same dtype"):
        Transpose(a, output_arr_t=ArrayMetadata((5, 4), numpy.float64))
    t = Transpose(a)
    assert [p.name for p in t.signature.parameters.values()] == ["output", "input"]


@pytest.mark.gpu
@pytest.mark.parametrize(
    "shape,axes,dtype",
    [
        ((33, 65), None, numpy.float32),
        ((1000, 501), None, numpy.complex64),
        ((4, 5, 6), (2, 1, 0), numpy.complex64),
        ((2, 3, 40, 50), (1, 0, 3, 2), numpy.complex128),
        ((7, 300, 9), (0, 2, 1), numpy.uint8),
        ((64, 64, 64), (1, 2, 0), numpy.float64),
        ((3, 4), (0, 1), numpy.float32),
    ],
)
def test_transpose_exact(shape, axes, dtype):
    import torch

    from reikna_b200.algorithms import Transpose

    rng = numpy.random.default_rng(51)
    if numpy.dtype(dtype).kind == "c":
        x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    elif numpy.dtype(dtype).kind == "u":
        x = rng.integers(0, 255, shape).astype(dtype)
    else:
        x = rng.standard_normal(shape).astype(dtype)
    t = torch.from_numpy(x).cuda()
    comp = Transpose(t, axes=axes)
    ref = numpy.transpose(x, axes)
    out = torch.empty(ref.shape, dtype=t.dtype, device="cuda")
    comp.compile()(None, out, t)
    torch.cuda.synchronize()
    assert numpy.array_equal(out.cpu().numpy(), ref)


@pytest.mark.gpu
def test_transpose_abi_rejects_alias_and_misalignment():
    import torch

    from reikna_b200 import _native as N

    buf = torch.zeros(1024, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert N.lib().rk_transpose_execute(p, p, 8, 1, 16, 16, None) == N.ERR_INVALID
    assert N.lib().rk_transpose_execute(p + 4096, p + 4, 8, 1, 16, 16, None) == N.ERR_INVALID
    assert N.lib().rk_transpose_execute(p + 4096, p, 12, 1, 16, 16, None) == N.ERR_INVALID
