"""Tensor-core split-precision mode (RK_FLAG_SPLIT_TC) against numpy in FP64.

The mode runs 256- and 1024-point contiguous complex64 lines on the tensor cores. Its
error is reported separately from the FP32 path; the tests hold it to the same bound
as complex64 (rel-L2 <= 2e-6 log2 N), the full-size cases to 4e-7 as well, and print
both errors.
"""

import numpy
import pytest

from helpers import fft_bound, normal_array, rel_l2

pytestmark = pytest.mark.gpu


def _run(x, flags, inverse=0, inplace=False, fft=None):
    import torch

    from reikna_b200.fft import FFT

    t = torch.from_numpy(numpy.ascontiguousarray(x)).cuda()
    comp = fft if fft is not None else FFT(t, axes=(x.ndim - 1,))
    c = comp.compile(flags=flags)
    out = t if inplace else torch.empty_like(t)
    c(None, out, t, inverse)
    torch.cuda.synchronize()
    return out.cpu().numpy(), c._runner.plan.tc_passes


def _sixty_db(rng, shape):
    mag = 10 ** rng.uniform(-3, 0, (2,) + shape)
    sgn = rng.choice([-1.0, 1.0], (2,) + shape)
    return (sgn[0] * mag[0] + 1j * sgn[1] * mag[1]).astype(numpy.complex64)


@pytest.mark.parametrize("rows", [1, 3, 64, 16384])
def test_split_tc_matches_fp64(rows):
    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(7)
    x = normal_array(rng, (rows, 1024), numpy.complex64)
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    y, ntc = _run(x, N.FLAG_SPLIT_TC)
    assert ntc == 1
    err = rel_l2(y, ref)
    y32, _ = _run(x, 0)
    print(f"rows={rows}: split-TC rel-L2 {err:.3e}, FP32 {rel_l2(y32, ref):.3e}")
    assert err < fft_bound(numpy.complex64, 1024)
    if rows == 16384:
        assert err < 4e-7


@pytest.mark.parametrize("rows", [1, 7, 64, 65536])
def test_split_tc_256_matches_fp64(rows):
    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(70)
    x = normal_array(rng, (rows, 256), numpy.complex64)
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    y, ntc = _run(x, N.FLAG_SPLIT_TC)
    assert ntc == 1
    err = rel_l2(y, ref)
    print(f"256 rows={rows}: split-TC rel-L2 {err:.3e}")
    assert err < fft_bound(numpy.complex64, 256)
    if rows == 65536:
        assert err < 4e-7
    yi, _ = _run(x, N.FLAG_SPLIT_TC, inverse=1, inplace=True)
    assert rel_l2(yi, numpy.fft.ifft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 256)


@pytest.mark.parametrize("n", [256, 1024])
@pytest.mark.parametrize("conj_in,conj_out,inverse", [(1, 0, 0), (0, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 0)])
def test_split_tc_edge_conjugation(n, conj_in, conj_out, inverse):
    """Conjugating edges: one side alone conjugates data in the kernel, both sides of
    a forward transform (or neither of an inverse) take the conjugate tables."""
    import torch

    from reikna_b200 import _native as N

    rows = 9
    x = normal_array(numpy.random.default_rng(71 + n), (rows, n), numpy.complex64)
    d = N.desc(N.FMT_C64, (rows, n), (1,), N.FLAG_SPLIT_TC)
    d.input = N.edge(N.FMT_C64, (rows, n))
    d.output = N.edge(N.FMT_C64, (rows, n))
    d.input.conj = conj_in
    d.output.conj = conj_out
    plan = N.Plan(d)
    assert plan.tc_passes == 1
    a = torch.from_numpy(x).cuda()
    b = torch.empty_like(a)
    plan.execute([b.data_ptr()], [a.data_ptr()], inverse=inverse, stream=0)
    torch.cuda.synchronize()
    xr = x.astype(numpy.complex128)
    if conj_in:
        xr = numpy.conj(xr)
    ref = numpy.fft.ifft(xr, axis=1) if inverse else numpy.fft.fft(xr, axis=1)
    if conj_out:
        ref = numpy.conj(ref)
    assert rel_l2(b.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.parametrize("rows", [512, 16384])
def test_split_tc_sixty_db_and_inverse(rows):
    """The precision workload's 60 dB variant (components +-10^U(-3,0)), up to the
    full 16384 x 1024 configuration, forward and inverse."""
    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(8)
    x = _sixty_db(rng, (rows, 1024))
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    y, ntc = _run(x, N.FLAG_SPLIT_TC)
    assert ntc == 1
    err = rel_l2(y, ref)
    print(f"60 dB rows={rows}: split-TC rel-L2 {err:.3e}")
    assert err < fft_bound(numpy.complex64, 1024)
    # per-element check on the small components too: within the FP32 path's error
    y32, _ = _run(x, 0)
    assert numpy.abs(y - ref).max() < 8 * max(numpy.abs(y32 - ref).max(), 1e-6)
    yi, _ = _run(x, N.FLAG_SPLIT_TC, inverse=1, inplace=True)
    assert rel_l2(yi, numpy.fft.ifft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 1024)


def test_split_tc_with_scaling_transformation():
    import torch

    from reikna_b200 import _native as N
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(12)
    x = normal_array(rng, (100, 1024), numpy.complex64)
    t = torch.from_numpy(x).cuda()
    fft = FFT(t, axes=(1,))
    sc = tr.mul_const(t, 0.25 - 0.5j)
    fft.parameter.output.connect(sc, sc.input, scaled=sc.output)
    y, ntc = _run(x, N.FLAG_SPLIT_TC, fft=fft)
    assert ntc == 1
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1) * (0.25 - 0.5j)
    assert rel_l2(y, ref) < fft_bound(numpy.complex64, 1024)


def test_split_tc_request_falls_back_where_not_applicable():
    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(13)
    for shape, axis in (((64, 512), 1), ((1024, 8), 0), ((256, 64), 0)):
        x = normal_array(rng, shape, numpy.complex64)
        import torch

        from reikna_b200.fft import FFT

        t = torch.from_numpy(x).cuda()
        y, ntc = _run(x, N.FLAG_SPLIT_TC, fft=FFT(t, axes=(axis,)))
        assert ntc == 0
        ref = numpy.fft.fft(x.astype(numpy.complex128), axis=axis)
        assert rel_l2(y, ref) < fft_bound(numpy.complex64, shape[axis])


def test_split_tc_device_status_clean():
    from reikna_b200 import _native as N

    x = normal_array(numpy.random.default_rng(14), (256, 1024), numpy.complex64)
    _run(x, N.FLAG_SPLIT_TC)
    assert N.device_status(clear=True) == 0


def test_split_tc_view_off_the_16_byte_grid():
    # a view starting 8 bytes into its allocation takes 8-byte loads instead of 16-byte ones
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(15)
    x = normal_array(rng, (5, 1024), numpy.complex64)
    base = torch.zeros(5 * 1024 + 1, dtype=torch.complex64, device="cuda")
    view = base[1:].view(5, 1024)
    assert view.data_ptr() % 16 == 8
    view.copy_(torch.from_numpy(x))
    out = torch.empty_like(view)
    c = FFT(view, axes=(1,)).compile(flags=N.FLAG_SPLIT_TC)
    c(None, out, view)
    torch.cuda.synchronize()
    assert c._runner.plan.tc_passes == 1
    ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 1024)
