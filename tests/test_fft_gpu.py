"""GPU parity: the sm_100a kernels through the C ABI against numpy (FP64) and the oracle.

Shape lists follow reikna's own tests (tests/test_fft/test_fft.py:28-111); every case
runs in place, forward then inverse, like reikna's check_errors (:148-170), and is
checked with reikna's element-wise tolerances plus the stated rel-L2 bound
(complex64 2e-6 log2 N, complex128 1e-14 log2 N).
"""

import math

import numpy
import pytest

from helpers import FFT_ATOL, FFT_RTOL, diff_is_negligible, fft_bound, normal_array, rel_l2, uniform_array
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def to_dev(x):
    return _torch().from_numpy(numpy.ascontiguousarray(x)).cuda()


def run(x, axes, inverse=False, inplace=True, fft=None):
    from reikna_b200.fft import FFT

    torch = _torch()
    t = to_dev(x)
    comp = fft if fft is not None else FFT(t, axes=axes)
    c = comp.compile()
    out = t if inplace else torch.empty_like(t)
    c(None, out, t, int(inverse))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def check(x, axes, rtol=FFT_RTOL, oracle=False):
    n = math.prod(x.shape[a] for a in axes)
    for inverse in (False, True):
        y = run(x, axes, inverse)
        ref = O.numpy_ref(x, axes, inverse)
        err = rel_l2(y, ref)
        assert err < fft_bound(x.dtype, n), (inverse, err)
        if x.dtype == numpy.complex64:
            assert diff_is_negligible(y, ref.astype(x.dtype), FFT_ATOL, rtol)
        if oracle:
            # reikna's own FP64 Bluestein weights take exp of the unreduced angle
            # pi n^2 / N (reikna/fft/fft.py:224-225), so the oracle carries its own
            # error; the two results must agree within both errors plus the bound
            yo = O.fft(x, axes, inverse=inverse)
            own = rel_l2(yo, ref)
            assert rel_l2(y, yo) < 2 * fft_bound(x.dtype, n) + own + err


def _local_cases():
    vals = []
    for p in (3, 7, 8, 9, 10, 12):
        size = 2**p
        batch = 2**20 // size
        for s in (size, size // 2 - 1):
            for b in (1, batch - 1, batch):
                vals.append(((b, s), (1,)))
    return vals


def _global_cases():
    vals = []
    for p in (3, 7, 9, 10):
        size = 2**p
        batch = 2**22 // size // 64
        for s in (size, size // 2 - 1):
            for ib in (2, 3, 63, 64):
                for ob in (1, batch - 1, batch):
                    vals.append(((ob, s, ib), (1,)))
    big = 2**15
    batch = 2**22 // big // 8
    vals += [((1, big, 1), (1,)), ((1, big, 2), (1,)), ((1, big, 3), (1,)), ((batch, big, 3), (1,)), ((batch - 1, big, 3), (1,))]
    return vals


SEQUENCE = [((3, 255, 7), (2, 0)), ((17, 200, 131), (1, 0)), ((7, 1000, 11), (1, 2)), ((15, 900, 57), (2, 0, 1))]


@pytest.mark.parametrize("shape_axes", _local_cases(), ids=lambda v: f"{v[0][0]}x{v[0][1]}")
def test_local(rng, shape_axes):
    shape, axes = shape_axes
    check(uniform_array(rng, shape, numpy.complex64), axes)


@pytest.mark.parametrize("shape_axes", _global_cases(), ids=lambda v: "x".join(map(str, v[0])))
def test_global(rng, shape_axes):
    shape, axes = shape_axes
    check(uniform_array(rng, shape, numpy.complex64), axes)


@pytest.mark.parametrize("shape_axes", SEQUENCE, ids=lambda v: f"{v[0]}over{v[1]}")
def test_sequence(rng, shape_axes):
    shape, axes = shape_axes
    check(uniform_array(rng, shape, numpy.complex64), axes, rtol=1e-2, oracle=True)


@pytest.mark.parametrize(
    "shape_axes",
    [((64, 4096), (1,)), ((8, 3001), (1,)), ((4, 127, 64), (1,)), ((16, 16, 16), (0, 1, 2)), ((2, 2**15), (1,)), ((5, 90, 17), (2, 0, 1))],
    ids=str,
)
def test_complex128(rng, shape_axes):
    shape, axes = shape_axes
    check(uniform_array(rng, shape, numpy.complex128), axes, oracle=True)


@pytest.mark.parametrize("shape_axes", [((64, 4096), (1,)), ((3, 255, 7), (2, 0)), ((33, 1000), (1,))], ids=str)
def test_against_oracle(rng, shape_axes):
    shape, axes = shape_axes
    check(uniform_array(rng, shape, numpy.complex64), axes, oracle=True)


def test_out_of_place_keeps_input(rng):
    x = uniform_array(rng, (32, 1000), numpy.complex64)
    from reikna_b200.fft import FFT

    torch = _torch()
    t = to_dev(x)
    out = torch.empty_like(t)
    FFT(t, axes=(0, 1)).compile()(None, out, t)
    torch.cuda.synchronize()
    assert numpy.array_equal(t.cpu().numpy(), x)
    assert rel_l2(out.cpu().numpy(), numpy.fft.fft2(x)) < fft_bound(numpy.complex64, 32000)


def test_trivial(rng):
    # reikna tests/test_fft/test_fft.py:173: transformations run even for a trivial FFT
    from reikna_b200.fft import FFT
    from reikna_b200.transformations import mul_param

    torch = _torch()
    x = uniform_array(rng, (128, 1, 1, 128), numpy.complex64)
    t = to_dev(x)
    res = torch.empty_like(t)
    fft = FFT(t, axes=(1, 2))
    scale = mul_param(t, numpy.int32)
    fft.parameter.input.connect(scale, scale.output, input_prime=scale.input, param=scale.param)
    fft.compile()(None, res, t, 4)
    torch.cuda.synchronize()
    assert diff_is_negligible(res.cpu().numpy(), x * 4, 1e-8, 1e-5)


@pytest.mark.parametrize("shape,axes", [((65, 1024), (1,)), ((3, 257, 256, 16), (2,)), ((9, 64, 64), (1, 2))])
def test_misaligned_views(rng, shape, axes):
    # views starting 8 bytes into an allocation take the non-TMA path
    from reikna_b200.fft import FFT

    torch = _torch()
    x = uniform_array(rng, shape, numpy.complex64)
    base = to_dev(x)
    t = base[1:]
    out = torch.empty_like(t)
    c = FFT(t, axes=axes).compile()
    c(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fftn(x[1:].astype(numpy.complex128), axes=axes)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, math.prod(shape[a] for a in axes))


def test_device_status_clear():
    import ctypes

    from reikna_b200 import _native as N

    s = ctypes.c_int32(-1)
    N.check(N.lib().rk_device_status(ctypes.byref(s), 1))
    assert s.value == 0


def test_strided_input_view(rng):
    from reikna_b200.fft import FFT

    torch = _torch()
    x = uniform_array(rng, (256, 96), numpy.complex64)
    t = to_dev(x).t()  # (96, 256) with strides (1, 96)
    out = torch.empty_like(t)
    FFT(t, axes=(1,)).compile()(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fft(x.T, axis=1)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 256)


# --- benchmark configurations at full size -------------------------------------


def test_config_1d_64x4096_round_trip():
    rng = numpy.random.default_rng(1)
    x = normal_array(rng, (64, 4096), numpy.complex64)
    from reikna_b200.fft import FFT

    torch = _torch()
    t = to_dev(x)
    c = FFT(t, axes=(1,)).compile()
    y = torch.empty_like(t)
    z = torch.empty_like(t)
    c(None, y, t, 0)
    c(None, z, y, 1)
    torch.cuda.synchronize()
    assert rel_l2(y.cpu().numpy(), numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 4096)
    assert rel_l2(z.cpu().numpy(), x) < 2 * fft_bound(numpy.complex64, 4096)


def _shift_scale_3d(n, dtype, seed):
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    torch = _torch()
    rng = numpy.random.default_rng(seed)
    x = normal_array(rng, (n, n, n), dtype)
    t = to_dev(x)
    fft = FFT(t)
    sh = tr.fftshift(t)
    sc = tr.mul_const(t, 1.0 / n**3)
    fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
    fft.parameter.shifted.connect(sc, sc.input, result=sc.output)
    out = torch.empty_like(t)
    fft.compile()(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fftshift(numpy.fft.fftn(x.astype(numpy.complex128))) / n**3
    return rel_l2(out.cpu().numpy(), ref)


def test_config_3d_256_shift_scale():
    assert _shift_scale_3d(256, numpy.complex64, 2) < fft_bound(numpy.complex64, 256**3)


def test_config_3d_128_complex128():
    assert _shift_scale_3d(128, numpy.complex128, 3) < fft_bound(numpy.complex128, 128**3)


def test_config_bluestein_1000x3001():
    rng = numpy.random.default_rng(4)
    x = normal_array(rng, (1000, 3001), numpy.complex64)
    y = run(x, (1,), inplace=False)
    assert rel_l2(y, numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 3001)


def test_config_2d_1000x1000():
    rng = numpy.random.default_rng(5)
    x = normal_array(rng, (1000, 1000), numpy.complex64)
    y = run(x, (0, 1), inplace=False)
    assert rel_l2(y, numpy.fft.fft2(x.astype(numpy.complex128))) < fft_bound(numpy.complex64, 10**6)


def test_config_r2c_1000x1000():
    from reikna_b200 import transformations as tr
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import FFT

    torch = _torch()
    rng = numpy.random.default_rng(6)
    x = rng.uniform(-1, 1, (1000, 1000)).astype(numpy.float32)
    t = to_dev(x)
    r2c = tr.real_to_complex(t)
    fft = FFT(r2c.parameter.output)
    fft.parameter.input.connect(r2c, r2c.parameter.output, real_input=r2c.parameter.input)
    crop = tr.crop_frequencies(fft.parameter.output)
    fft.parameter.output.connect(crop, crop.parameter.input, half=crop.parameter.output)
    out = torch.empty((1000, 501), dtype=torch.complex64, device="cuda")
    fft.compile()(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft2(x.astype(numpy.float64))
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 10**6)
    del ArrayMetadata


def test_config_precision_16384x1024():
    for seed, sixty_db in ((7, False), (8, True)):
        rng = numpy.random.default_rng(seed)
        if sixty_db:
            mag = 10 ** rng.uniform(-3, 0, (2, 16384, 1024))
            sgn = rng.choice([-1.0, 1.0], (2, 16384, 1024))
            x = (sgn[0] * mag[0] + 1j * sgn[1] * mag[1]).astype(numpy.complex64)
        else:
            x = normal_array(rng, (16384, 1024), numpy.complex64)
        y = run(x, (1,), inplace=False)
        assert rel_l2(y, numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 1024)


@pytest.mark.parametrize("n", [2**20, 65521, 2**17 + 1])
def test_long_1d(n):
    rng = numpy.random.default_rng(n)
    x = normal_array(rng, (n,), numpy.complex64)
    check(x, (0,))


# --- transformations ------------------------------------------------------------


def test_real_to_complex_demo():
    # examples/demo_real_to_complex_fft.py: rel-L2 < 1e-6 at N = 3000
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    torch = _torch()
    arr = numpy.random.default_rng(11).normal(size=3000).astype(numpy.float32)
    t = to_dev(arr)
    trf = tr.real_to_complex(t)
    fft = FFT(trf.parameter.output)
    fft.parameter.input.connect(trf, trf.parameter.output, new_input=trf.parameter.input)
    res = torch.empty(3000, dtype=torch.complex64, device="cuda")
    fft.compile()(None, res, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fft(arr)
    assert numpy.linalg.norm(res.cpu().numpy() - ref) / numpy.linalg.norm(ref) < 1e-6


@pytest.mark.parametrize("shape,axes", [((60, 64), (0, 1)), ((61, 65), (0, 1)), ((10, 12, 9), (0, 2)), ((1001,), (0,))])
@pytest.mark.parametrize("inplace", [False, True])
def test_fftshift_output_transformation(rng, shape, axes, inplace):
    # examples/demo_fftshift_transformation.py:116-147
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    torch = _torch()
    x = normal_array(rng, shape, numpy.complex64)
    t = to_dev(x)
    fft = FFT(t, axes=axes)
    sh = tr.fftshift(t, axes=axes)
    fft.parameter.output.connect(sh, sh.parameter.input, new_output=sh.parameter.output)
    out = t if inplace else torch.empty_like(t)
    fft.compile()(None, out, t)
    torch.cuda.synchronize()
    ref = numpy.fft.fftshift(numpy.fft.fftn(x.astype(numpy.complex128), axes=axes), axes=axes)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, math.prod(shape[a] for a in axes))


def test_split_combine_norm(rng):
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    torch = _torch()
    x = normal_array(rng, (40, 300), numpy.complex64)
    re, im = to_dev(x.real.copy()), to_dev(x.imag.copy())
    arr = to_dev(x)
    fft = FFT(arr, axes=(1,))
    cc = tr.combine_complex(arr)
    sc = tr.split_complex(arr)
    fft.parameter.input.connect(cc, cc.output, in_re=cc.real, in_im=cc.imag)
    fft.parameter.output.connect(sc, sc.input, out_re=sc.real, out_im=sc.imag)
    ore, oim = torch.empty_like(re), torch.empty_like(im)
    fft.compile()(None, ore, oim, re, im, 1)
    torch.cuda.synchronize()
    ref = numpy.fft.ifft(x.astype(numpy.complex128), axis=1)
    got = ore.cpu().numpy() + 1j * oim.cpu().numpy()
    assert rel_l2(got, ref) < fft_bound(numpy.complex64, 300)

    fft2 = FFT(arr, axes=(1,))
    nrm = tr.norm_const(arr, 2)
    fft2.parameter.output.connect(nrm, nrm.input, power=nrm.output)
    pw = torch.empty(x.shape, dtype=torch.float32, device="cuda")
    fft2.compile()(None, pw, arr)
    torch.cuda.synchronize()
    ref2 = numpy.abs(numpy.fft.fft(x.astype(numpy.complex128), axis=1)) ** 2
    assert rel_l2(pw.cpu().numpy(), ref2) < 4 * fft_bound(numpy.complex64, 300)


def test_spectrogram_pipeline():
    # examples/demo_specgram.py:196-268, restated with numpy instead of matplotlib
    from reikna_b200 import transformations as tr
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import FFT

    torch = _torch()
    rng = numpy.random.default_rng(9)
    sig = rng.standard_normal(2**16).astype(numpy.float32)
    nfft, hop = 1024, 256
    frame = tr.rolling_frame(ArrayMetadata(sig.shape, numpy.float32), nfft, nfft - hop, None)
    shape = frame.parameter.output.shape
    fft_arr = ArrayMetadata(shape, numpy.complex64)
    real_arr = ArrayMetadata(shape, numpy.float32)
    win = tr.hanning_window(real_arr, nfft)
    zero = tr.broadcast_const(real_arr, 0)
    to_c = tr.combine_complex(fft_arr)
    amp = tr.norm_const(fft_arr, 1)
    crop = tr.crop_frequencies(amp.parameter.output)
    fft = FFT(fft_arr, axes=(1,))
    fft.parameter.input.connect(to_c, to_c.parameter.output, input_real=to_c.parameter.real, input_imag=to_c.parameter.imag)
    fft.parameter.input_imag.connect(zero, zero.parameter.output)
    fft.parameter.input_real.connect(win, win.parameter.output, unwindowed_input=win.parameter.input)
    fft.parameter.unwindowed_input.connect(frame, frame.parameter.output, flat_input=frame.parameter.input)
    fft.parameter.output.connect(amp, amp.parameter.input, amplitude=amp.parameter.output)
    fft.parameter.amplitude.connect(crop, crop.parameter.input, cropped=crop.parameter.output)
    out = torch.empty(crop.parameter.output.shape, dtype=torch.float32, device="cuda")
    fft.compile()(None, out, to_dev(sig))
    torch.cuda.synchronize()
    nfr = shape[0]
    idx = numpy.arange(nfr)[:, None] * hop + numpy.arange(nfft)[None, :]
    w = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(nfft) / (nfft - 1)))
    ref = numpy.abs(numpy.fft.rfft(sig.astype(numpy.float64)[idx] * w, axis=1))
    assert numpy.allclose(out.cpu().numpy(), ref, atol=1e-4 * ref.max(), rtol=1e-4)


# --- FFTShift computation ---------------------------------------------------------

SHIFT_CASES = [
    ((10,), (0,)),
    ((11,), (0,)),
    ((9000,), (0,)),
    ((9001,), (0,)),
    ((128, 60), (0, 1)),
    ((127, 60), (0, 1)),
    ((127, 61), (0, 1)),
    ((100, 80, 60), (0, 1, 2)),
    ((101, 80, 61), (0, 1, 2)),
    ((101, 80, 61), (0, 2)),
    ((20, 31, 80, 61), (0, 2)),
]


@pytest.mark.parametrize("shape_axes", SHIFT_CASES, ids=str)
@pytest.mark.parametrize("inverse", [False, True], ids=["forward", "inverse"])
def test_fftshift_computation(shape_axes, inverse):
    # reikna tests/test_fft/test_fftshift.py:81-102 (exact, in place)
    from reikna_b200.fft import FFTShift

    torch = _torch()
    shape, axes = shape_axes
    data = numpy.arange(math.prod(shape)).reshape(shape).astype(numpy.int32)
    t = to_dev(data)
    FFTShift(t, axes=axes).compile()(None, t, t, int(inverse))
    torch.cuda.synchronize()
    ref = (numpy.fft.ifftshift if inverse else numpy.fft.fftshift)(data, axes=axes)
    assert numpy.array_equal(t.cpu().numpy(), ref)


@pytest.mark.parametrize("shape_axes", [((256, 4096), (0, 1)), ((4096, 256), (0,)), ((64, 64, 64), (1, 2)),
                                        ((64, 62), (1,)), ((33, 64), (0, 1)), ((8, 1, 128), (0, 2))], ids=str)
@pytest.mark.parametrize("dtype", [numpy.complex64, numpy.complex128])
@pytest.mark.parametrize("mode", ["out", "inplace", "offset"])
def test_fftshift_computation_complex(shape_axes, dtype, mode):
    """Complex elements take the row form's vector accesses where rows, shifts and
    addresses allow; a view starting one element into its allocation does not."""
    from reikna_b200.fft import FFTShift

    torch = _torch()
    shape, axes = shape_axes
    rng = numpy.random.default_rng(math.prod(shape))
    data = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    if mode == "offset":
        base = torch.zeros(math.prod(shape) + 1, dtype=torch.complex64 if dtype == numpy.complex64 else torch.complex128,
                           device="cuda")
        t = base[1:].view(shape)
        t.copy_(torch.from_numpy(data))
    else:
        t = to_dev(data)
    out = t if mode == "inplace" else torch.empty_like(t)
    FFTShift(t, axes=axes).compile()(None, out, t)
    torch.cuda.synchronize()
    assert numpy.array_equal(out.cpu().numpy(), numpy.fft.fftshift(data, axes=axes))


def test_fftshift_unordered_and_no_axes():
    from reikna_b200.fft import FFTShift

    torch = _torch()
    data = numpy.arange(40 * 50 * 60).reshape(40, 50, 60).astype(numpy.int32)
    for axes in ((2, 0), None):
        t = to_dev(data)
        o = torch.empty_like(t)
        FFTShift(t, axes=axes).compile()(None, o, t)
        torch.cuda.synchronize()
        assert numpy.array_equal(o.cpu().numpy(), numpy.fft.fftshift(data, axes=axes))


def test_fftshift_trivial_with_transformation(rng):
    from reikna_b200.fft import FFTShift
    from reikna_b200.transformations import mul_param

    torch = _torch()
    x = uniform_array(rng, (128, 1, 1, 128), numpy.complex64)
    t = to_dev(x)
    res = torch.empty_like(t)
    s = FFTShift(t, axes=(1, 2))
    scale = mul_param(t, numpy.int32)
    s.parameter.input.connect(scale, scale.output, input_prime=scale.input, param=scale.param)
    s.compile()(None, res, t, 4)
    torch.cuda.synchronize()
    assert diff_is_negligible(res.cpu().numpy(), x * 4, 1e-8, 1e-5)
